"""Known-answer cases restated from the upstream test suite (paths relative to the
upstream project). Each case gives the operands and the expected result that the
upstream test asserts; values are compared with upstream's default comparator
(|a - b| <= 1e-6 + 1e-6 |b|, tests/test_helpers.c:12-18) because the upstream
literals are rounded."""
import numpy as np


def csc_to_csr(p, i, x, m, n):
    """Plain-numpy CSC -> CSR (test helper; mirrors upstream tests' new_csr_of_csc)."""
    p = np.asarray(p); i = np.asarray(i); x = np.asarray(x, float)
    cols = np.repeat(np.arange(n), np.diff(p))
    order = np.lexsort((cols, i))
    rp = np.zeros(m + 1, np.int32)
    np.add.at(rp, i + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    return rp, cols[order].astype(np.int32), x[order], m, n


# tests/test_csc_matrix.h:177-236 (test_BTA_alloc_and_BTDA_fill): C = B^T D A
BTDA_SMALL = dict(
    A_csc=([0, 2, 4, 6], [0, 2, 1, 3, 0, 2], [1.0, 4.0, 3.0, 6.0, 2.0, 5.0], 4, 3),
    B_csc=([0, 2, 4], [0, 2, 1, 3], [1.0, 3.0, 2.0, 4.0], 4, 2),
    d=[1.0, 2.0, 3.0, 4.0],
    Cp=[0, 2, 3], Ci=[0, 2, 1], Cx=[37.0, 47.0, 108.0],
)

# tests/test_csc_matrix.h:95-134 (test_ATA_alloc_random): C = A^T D A
ATA_RANDOM = dict(
    A_csc=([0, 1, 1, 1, 1, 4, 5, 6, 7, 8, 9, 11, 11, 11, 13, 15],
           [5, 0, 6, 9, 0, 5, 1, 3, 6, 0, 6, 3, 6, 6, 8],
           [7, 4, 8, 5, 7, 3, 7, 8, 5, 4, 8, 8, 3, 6, 5], 10, 15),
    d=[2, 8, 6, 2, 5, 1, 6, 9, 1, 3],
    Cp=[0, 2, 2, 2, 2, 8, 11, 13, 14, 16, 21, 27, 27, 27, 33, 38],
    Ci=[0, 6, 4, 5, 9, 10, 13, 14, 4, 5, 10, 0, 6, 7, 8, 13, 4, 9, 10, 13, 14, 4, 5, 9, 10,
        13, 14, 4, 8, 9, 10, 13, 14, 4, 9, 10, 13, 14],
    Cx=[49., 21., 491., 56., 240., 416., 144., 288., 56., 98., 56., 21., 9., 392., 128.,
        128., 240., 150., 240., 90., 180., 416., 56., 240., 416., 144., 288., 144., 128., 90.,
        144., 182., 108., 288., 180., 288., 108., 241.],
)

# tests/test_csc_matrix.h:136-176 (test_ATA_alloc_random2)
ATA_RANDOM2 = dict(
    A_csc=([0, 2, 4, 6, 6, 9, 12, 12, 14, 14, 15],
           [9, 12, 3, 4, 1, 6, 4, 8, 13, 1, 3, 7, 5, 13, 6],
           [0.99, 0.9, 0.51, 0.64, 0.39, 0.29, 0.26, 0.91, 0.35, 0.18, 0.33, 0.73, 0.97,
            0.86, 1.03], 15, 10),
    d=[-0.6, -0.23, -0.29, -1.36, 0.4, 0.36, 0.11, -0.13, -1.32, -0.32, -0.24, -0.7, -0.06,
       0.5, 1.99],
    Cp=[0, 1, 4, 7, 7, 10, 13, 13, 15, 15, 17],
    Ci=[0, 1, 4, 5, 2, 5, 9, 1, 4, 7, 1, 2, 5, 4, 7, 2, 9],
    Cx=[-0.362232, -0.189896, 0.06656, -0.228888, -0.025732, -0.016146, 0.032857, 0.06656,
        -1.004802, 0.1505, -0.228888, -0.016146, -0.224833, 0.1505, 0.708524, 0.032857,
        0.116699],
)

# tests/test_csc_matrix.h:29-55 and :71-93: structure of A^T A only
ATA_SIMPLE = dict(A_csc=([0, 2, 3, 5], [0, 2, 1, 2, 3], [1.0] * 5, 4, 3),
                  Cp=[0, 2, 3, 5], Ci=[0, 2, 1, 0, 2])
ATA_DIAGONAL_LIKE = dict(A_csc=([0, 1, 2, 3, 4], [0, 1, 2, 0], [1, 1, 1, 2], 3, 4),
                         Cp=[0, 2, 3, 4, 6], Ci=[0, 3, 1, 2, 0, 3])

# tests/test_csr_csc_conversion.h:12-55 (CSR -> CSC), :58-135 (CSC -> CSR)
CSR_TO_CSC = dict(A_csr=([0, 2, 3, 4, 5], [0, 4, 2, 1, 3], [1.0, 1.0, 3.0, 2.0, 4.0], 4, 5),
                  Cp=[0, 1, 2, 3, 4, 5], Ci=[0, 2, 1, 3, 0], Cx=[1.0, 2.0, 3.0, 4.0, 1.0])
CSC_TO_CSR = dict(A_csc=([0, 1, 2, 3, 4, 5], [0, 2, 1, 3, 0], [1.0, 4.0, 3.0, 5.0, 2.0], 4, 5),
                  Cp=[0, 2, 3, 4, 5], Ci=[0, 4, 2, 1, 3], Cx=[1.0, 2.0, 3.0, 4.0, 5.0])
# tests/test_csr_csc_conversion.h:138-171: CSR -> CSC -> CSR round trip
ROUNDTRIP = dict(A_csr=([0, 3, 5, 8], [0, 1, 3, 1, 2, 0, 2, 3],
                        [1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0, 8.0], 3, 4))


def close(a, b):
    a = np.asarray(a, float); b = np.asarray(b, float)
    return a.shape == b.shape and bool(np.all(np.abs(a - b) <= 1e-6 + 1e-6 * np.abs(b)))
