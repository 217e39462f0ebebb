"""The persisted tuning table: save / load round trip and rejection of malformed
files (host side, no GPU), and on the GPU: a product tuned in one process, the
table saved, loaded by a fresh process and applied to the same pattern gives the
same plan, and refills bit-identical to the tuned product's."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_table_round_trip_and_malformed(sdl, tmp_path):
    from sparsediff_linalg_b200 import device as D
    D.tune_table_clear()
    assert D.tune_table_size() == 0
    src = tmp_path / "t.txt"
    src.write_text("# comment\n"
                   "m10.n9.t6.c4.h3:8, 512 8 256 512 512 768 4 0 256 41.5\n"       # first format
                   "m4.n4.t2.c4.h1:8, 128 16 256 512 512 512 0 512 128 2 3.25\n")  # with refill kind
    assert D.tune_table_load(src) == 2
    assert D.tune_table_size() == 2
    out = tmp_path / "u.txt"
    D.tune_table_save(out)
    lines = [ln for ln in out.read_text().splitlines() if not ln.startswith("#")]
    assert sorted(ln.split()[0] for ln in lines) == ["m10.n9.t6.c4.h3:8,", "m4.n4.t2.c4.h1:8,"]
    kinds = {ln.split()[0]: ln.split()[10] for ln in lines}
    assert kinds == {"m10.n9.t6.c4.h3:8,": "0", "m4.n4.t2.c4.h1:8,": "2"}
    D.tune_table_clear()
    assert D.tune_table_load(out) == 2
    for bad in ("key 512 8\n",                                        # too few fields
                "key 512 8 256 512 512 768 4 0 256 41.5 extra\n",     # too many
                "key 512 8 256 512 512 768 4 0 256 1 41.5 7\n",       # too many
                "key 333 8 256 512 512 768 4 0 256 41.5\n",           # invalid threshold
                "key 512 8 256 512 512 768 4 0 256 3 41.5\n",         # invalid refill kind
                "key 512 8 256 512 512 768 4 0 256 1.5 41.5\n",       # non-integer refill kind
                "key 512 8 256 512 512 768 4 0 64 41.5\n"):           # invalid refill threads
        f = tmp_path / "bad.txt"
        f.write_text(bad)
        with pytest.raises(Exception):
            D.tune_table_load(f)
    assert D.tune_table_size() == 2          # a rejected file adds nothing
    with pytest.raises(Exception):
        D.tune_table_load(tmp_path / "missing.txt")
    D.tune_table_clear()


_CHILD = r"""
import json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from sparsediff_linalg_b200 import device as D, workloads as wl
A, B, d = wl.btda(seed=21, m=20000, nA=9000, nB=7000, k=6)
T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
P, Tr = D.btda_product(T(A[0]), T(A[1]), A[4], T(B[0]), T(B[1]), B[4])
n = D.tune_table_load(sys.argv[2])
found = P.apply_tuned()
Cx = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
P.fill(T(B[2]), T(d), T(A[2]), Cx)
torch.cuda.synchronize()
np.save(sys.argv[3], Cx.cpu().numpy())
print(json.dumps({"loaded": n, "found": found, "key": P.pattern_key(), "tuning": P.tuning(),
                  "shape": P.refill_shape()}))
"""


@pytest.mark.gpu
def test_tuned_plan_survives_a_fresh_process(sdl, tmp_path):
    import torch
    from sparsediff_linalg_b200 import device as D, workloads as wl
    D.tune_table_clear()
    A, B, d = wl.btda(seed=21, m=20000, nA=9000, nB=7000, k=6)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    P, Tr = D.btda_product(T(A[0]), T(A[1]), A[4], T(B[0]), T(B[1]), B[4])
    assert not P.apply_tuned()                 # nothing recorded yet
    tuned = P.autotune(reps=3)
    key = P.pattern_key()
    assert D.tune_table_size() == 1
    Cx = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
    P.fill(T(B[2]), T(d), T(A[2]), Cx)
    torch.cuda.synchronize()
    path = tmp_path / "tuning.txt"
    D.tune_table_save(path)
    out = tmp_path / "cx.npy"
    r = subprocess.run([sys.executable, "-c", _CHILD, str(ROOT), str(path), str(out)], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    child = json.loads(r.stdout.strip().splitlines()[-1])
    assert child["loaded"] == 1 and child["found"] and child["key"] == key
    for k in ("warp_max_terms", "rows_per_cta_warp", "tile_budget", "refill_ctas_per_sm", "refill_threads",
              "tile_max_terms"):
        assert child["tuning"][k] == tuned[k], k
    assert np.array_equal(np.load(out).view(np.int64), Cx.cpu().numpy().view(np.int64))
    D.tune_table_clear()
