"""bench.py's multi-rank plumbing on the CPU: `--gpus N` starts N ranks itself (one
process each, torch.distributed.run on 127.0.0.1), every rank takes the same
barrier / timed region / max-over-ranks steps (gloo, no GPU: --stub), and rank 0
prints one JSON line whose n_gpus is the number of ranks that ran."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _run(args, env=None):
    e = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        e.pop(k, None)
    e.update(env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py")] + args, capture_output=True, text=True,
                          timeout=300, env=e, cwd=str(ROOT))


def test_launcher_starts_n_ranks_and_prints_one_line():
    r = _run(["--gpus", "2", "--stub", "--steps", "3", "--warmup", "1"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["ranks_seen"] == 2 and line["steps"] == 3


def test_world_size_must_match_gpus():
    r = _run(["--gpus", "2", "--stub"], env={"WORLD_SIZE": "1", "RANK": "0", "LOCAL_RANK": "0"})
    assert r.returncode != 0
    assert "--gpus 2" in (r.stderr + r.stdout)
