"""Pins the oracle against the reference's own known-answer tests and the published
Philox4x32-10 answers.  The reference cases come from tests/golden/reference_kats.json,
extracted by tests/golden/make_golden.py from test_sparse_ops.cpp, sp_blas.hpp and
ma_operations.hpp of the reference; the CSR cases of the reference's generator
(gensparse.py) are restated in the test."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


def _csr(M, K, entries, rows_used=None):
    rows_used = M if rows_used is None else rows_used
    dense = np.zeros((M, K), np.complex128)
    for r, c, v in entries:
        dense[r, c] = v
    dense = dense[:rows_used]
    ri, ci, vals = [0], [], []
    for r in range(rows_used):
        nz = np.nonzero(dense[r])[0]
        ci += list(nz)
        vals += list(dense[r, nz])
        ri.append(len(ci))
    return (np.array(ri, np.int32), np.array(ci, np.int32), np.array(vals, np.complex128))


def _csrmm(trans, nrows, ncols, csr, B, ncolsB, alpha, beta, C):
    lib = O.load()
    ri, ci, v = csr
    a = np.array([alpha, 0.0])
    b = np.array([beta, 0.0])
    lib.orc_csrmm(trans.encode(), nrows, ncols, ri.ctypes.data, ci.ctypes.data, v.ctypes.data,
                  ncolsB, a.ctypes.data, B.ctypes.data, ncolsB, b.ctypes.data, C.ctypes.data, ncolsB)


@pytest.mark.parametrize("case", KATS["sparse_ops"], ids=lambda c: c["name"])
def test_sparse_ops_known_answers(case):
    """test_sparse_ops.cpp: C = alpha*op(A)*B + beta*C through the csrmm restatement."""
    M, K, ncolsB = case["M"], case["K"], case["ncolsB"]
    rows = case["rows_used"]
    csr = _csr(M, K, case["entries"], rows)
    nB = (K if case["op"] == "N" else M) * ncolsB
    nC = (M if case["op"] == "N" else K) * ncolsB
    B = np.zeros(max(nB, 1), np.complex128)
    for i, v in case["B"].items():
        B[int(i)] = v
    C = np.zeros(max(nC, 1), np.complex128)
    for i, v in case["C0"].items():
        C[int(i)] = v
    _csrmm(case["op"], rows, K, csr, B, ncolsB, case["alpha"], case["beta"], C)
    for i, v in case["expect"].items():
        assert C[int(i)].real == pytest.approx(v, rel=1e-12, abs=1e-12)
        assert C[int(i)].imag == 0.0


def test_sp_blas_known_answers():
    """sp_blas.hpp self-test: csrmm 'N' and 'T' on a 4x4 CSR."""
    c = KATS["sp_blas"]
    csr = _csr(c["M"], c["K"], c["entries"])
    B = np.array(c["B"], np.complex128)
    C = np.zeros(16, np.complex128)
    _csrmm("N", 4, 4, csr, B, 4, 1.0, 0.0, C)
    np.testing.assert_array_equal(C.real, c["C_N"])
    D = np.zeros(16, np.complex128)
    _csrmm("T", 4, 4, csr, B, 4, 1.0, 0.0, D)
    np.testing.assert_array_equal(D.real, c["C_T"])


def _rm_gemm(opA, opB, A, B):
    lib = O.load()
    A = np.ascontiguousarray(A, np.complex128)
    B = np.ascontiguousarray(B, np.complex128)
    Aop = A.T if opA == "T" else A
    Bop = B.T if opB == "T" else B
    M, K = Aop.shape
    Nc = Bop.shape[1]
    C = np.zeros((M, Nc), np.complex128)
    lib.orc_rm_gemm(opA.encode(), opB.encode(), M, Nc, K, A.ctypes.data, A.shape[1],
                    B.ctypes.data, B.shape[1], C.ctypes.data, Nc)
    return C


def test_ma_operations_gemm_known_answers():
    """ma_operations.hpp self-test: the row-major operand swap for all N/T combos."""
    g = KATS["ma_operations"]["gemm"]
    A = np.array(g["A"]).reshape(3, 3)
    B = np.array(g["B"]).reshape(3, 3)
    for (oa, ob), key in ((("N", "N"), "AB"), (("T", "N"), "AtB"), (("N", "T"), "ABt"),
                          (("T", "T"), "AtBt")):
        C = _rm_gemm(oa, ob, A, B)
        np.testing.assert_array_equal(C.real, np.array(g[key]).reshape(3, 3))


@pytest.mark.parametrize("i", range(4))
def test_ma_operations_gemv_known_answers(i):
    g = KATS["ma_operations"]["gemv"][i]
    M = np.array(g["M"]).reshape(g["rows"], g["cols"])
    x = np.array(g["x"]).reshape(-1, 1)
    y = _rm_gemm("T" if g["trans"] else "N", "N", M, x)
    np.testing.assert_array_equal(y.real.ravel(), g["y"])


def test_ma_operations_invert_known_answer():
    """ma::invert then A^-1 B == I to 1e-14 (ma_operations.hpp:491-505)."""
    inv = KATS["ma_operations"]["invert"]
    A = np.array(inv["A"], np.complex128).reshape(3, 3)
    Ai = A.copy()
    det = np.zeros(2)
    assert O.load().orc_invert(3, Ai.ctypes.data, det.ctypes.data) == 0
    np.testing.assert_allclose(Ai @ A, np.eye(3), atol=inv["tol"] * 1e3)
    assert det[0] == pytest.approx(np.linalg.det(A.real), rel=1e-12)


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors published with the Random123 library."""
    assert list(O.philox([0, 0, 0, 0], [0, 0])) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert list(O.philox([0xffffffff] * 4, [0xffffffff] * 2)) == \
        [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert list(O.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                         [0xa4093822, 0x299f31d0])) == [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_normals_moments():
    x = O.normals(0, 3, 400000)
    assert abs(x.mean()) < 0.01
    assert abs(x.var() - 1.0) < 0.01
    assert np.all(np.isfinite(x))


def _gensparse_cases():
    """The four C = alpha A X + beta Y cases of the reference's generator
    (src/Numerics/tests/gensparse.py:19-58: alpha 1, beta 2), restated.  The script itself
    no longer runs on current scipy (dok_matrix.iteritems), so its answer formula
    b = alpha*(A.dot(X)) + beta*Y (:65) is evaluated here in numpy."""
    cases = []
    A = np.eye(3)
    cases.append((A, np.ones((3, 1)), np.ones((3, 1))))
    A = np.eye(3)
    A[1, 2] = 2.0
    cases.append((A, np.arange(0, 6.0).reshape(3, 2), np.arange(0, 6.0).reshape(3, 2)))
    A = np.eye(3)
    A[1, 1] = 0.0
    A[1, 2] = 1.0
    cases.append((A, np.arange(0, 9.0).reshape(3, 3), np.arange(0, 9.0).reshape(3, 3)))
    A = np.eye(2)
    A[0, 1] = 1.0
    cases.append((A, np.arange(0, 6.0).reshape(2, 3), np.arange(0, 6.0).reshape(2, 3)))
    return cases


@pytest.mark.parametrize("i", range(4))
@pytest.mark.parametrize("cplx", [False, True])
def test_gensparse_known_answers(i, cplx):
    """The generator's cases through the csrmm restatement (its double and complex<double>
    cases hold the same real values); cplx adds imaginary parts to the same pattern."""
    A, X, Y = _gensparse_cases()[i]
    if cplx:
        A = A * (1.0 + 0.5j)
        X = X - 0.25j * X
        Y = Y + 1j
    M, K = A.shape
    ncolsB = X.shape[1]
    entries = [(r, c, A[r, c]) for r in range(M) for c in range(K) if A[r, c] != 0]
    csr = _csr(M, K, entries)
    B = np.ascontiguousarray(X, np.complex128).reshape(-1)
    C = np.ascontiguousarray(Y, np.complex128).reshape(-1).copy()
    _csrmm("N", M, K, csr, B, ncolsB, 1.0, 2.0, C)
    np.testing.assert_allclose(C.reshape(M, ncolsB), 1.0 * (A @ X) + 2.0 * Y, rtol=0,
                               atol=1e-14)
