"""Extracts the reference's own known-answer tests into tests/golden/reference_kats.json.

Run where the reference tree is mounted, with its path as the only argument
(`python tests/golden/make_golden.py <reference tree>`).  The numbers are parsed out of
the reference's test sources as text:

  src/Numerics/tests/test_sparse_ops.cpp   CSR x vector / CSR x matrix cases (alpha, beta)
  src/Numerics/sp_blas.hpp  (_TEST_SP_BLAS)        4x4 csrmm 'N' and 'T'
  src/Numerics/ma_operations.hpp (_TEST_MA_OPERATIONS)  gemv / gemm N,T combos, invert

Uninitialised buffer entries in test_sparse_ops.cpp (B[4..7], C[4..5] of the 3x4 real
case) are taken as zero, which is what the expected values imply.
"""
from __future__ import annotations

import json
import os
import re
import sys

if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
    sys.exit("usage: make_golden.py <path of the miniAFQMC reference tree>")
REF = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")

NUM = r"[-+]?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?"


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def sparse_ops_cases():
    src = read("src/Numerics/tests/test_sparse_ops.cpp")
    cases = []
    # the templated 1x1 case lives in a helper function, the rest in TEST_CASE bodies
    bodies = re.split(r"\n(?=TEST_CASE\(|template<typename T> void test_matrix_mult_1_1)", src)
    for body in bodies:
        m = re.match(r'TEST_CASE\("([^"]+)"', body)
        name = m.group(1) if m else ("sparse_matrix_mult_1x1"
                                     if "test_matrix_mult_1_1()" in body and "SparseMatrix<T> A(1,1)" in body else None)
        if name is None or name == "sparse_matrix_mult":
            continue
        dims = re.search(r"SparseMatrix<.*?>\s+A\((\w+),\s*(\w+)\)", body)
        consts = dict(re.findall(r"const int (\w) = (\d+);", body))
        M = int(consts.get(dims.group(1), dims.group(1)))
        K = int(consts.get(dims.group(2), dims.group(2)))
        entries = [(int(r), int(c), float(v)) for r, c, v in
                   re.findall(rf"s2D<.*?>\((\d+),\s*(\d+),\s*({NUM})\)", body)]
        entries += [(0, int(i), float(v)) for i, v in
                    re.findall(rf"s1D<.*?>\((\d+),\s*({NUM})\)", body)]
        B = {int(i): float(v) for i, v in re.findall(rf"\bB\[(\d+)\]\s*=\s*({NUM});", body)}
        C0 = {int(i): float(v) for i, v in re.findall(rf"\bC\[(\d+)\]\s*=\s*({NUM});", body)}
        alpha = re.search(rf"alpha\s*=\s*({NUM});", body)
        beta = re.search(rf"beta\s*=\s*({NUM});", body)
        nrows = re.search(r"int nrows = (\d+);", body)
        if "product_SpMatTV" in body:
            op, ncolsB = "T", 1
        elif "product_SpMatM" in body:
            op, ncolsB = "N", int(consts.get("N", nrows.group(1) if nrows else 1))
        else:
            op, ncolsB = "N", 1
        expect = {}
        for i, v in re.findall(rf"REQUIRE\((?:realPart\()?C\[(\d+)\](?:\.real\(\))?\)?\s*==\s*Approx\(({NUM})\)\)", body):
            expect[int(i)] = float(v)
        # the first axpy-style check of zaxpy_T_2x2 is repeated after re-initialising C
        cases.append({
            "name": name, "M": M, "K": K, "entries": entries, "op": op, "ncolsB": ncolsB,
            "rows_used": int(nrows.group(1)) if (nrows and op == "N" and ncolsB == 1) else M,
            "B": B, "C0": C0,
            "alpha": float(alpha.group(1)) if alpha else 1.0,
            "beta": float(beta.group(1)) if beta else 0.0,
            "expect": expect,
        })
    return cases


def vec(block, name):
    m = re.search(rf"std::vector<double>\s+{name}\s*=\s*\{{([^}}]*)\}}", block)
    body = re.sub(r"//[^\n]*", "", m.group(1))
    return [float(x) for x in re.findall(NUM, body)]


def spblas_case():
    src = read("src/Numerics/sp_blas.hpp")
    test = src[src.index("#ifdef _TEST_SP_BLAS"):]
    entries = [(int(r), int(c), float(v)) for r, c, v in
               re.findall(rf"\bA\((\d+),(\d+)\)\s*=\s*({NUM});", test)]
    return {"name": "sp_blas_csrmm_4x4", "M": 4, "K": 4, "entries": entries,
            "B": vec(test, "b"), "C_N": vec(test, "c2"), "C_T": vec(test, "d2")}


def ma_operations_cases():
    src = read("src/Numerics/ma_operations.hpp")
    test = src[src.index("#ifdef _TEST_MA_OPERATIONS"):]
    blocks = re.split(r"\n\t\{", test)
    gemv, gemm, inv = [], [], None
    for b in blocks:
        if "ma::product(M, X, Y)" in b or "ma::product(T(M), X, Y)" in b:
            shape = re.search(r"extents\[(\d+)\]\[(\d+)\]", b)
            gemv.append({"M": vec(b, "m"), "rows": int(shape.group(1)), "cols": int(shape.group(2)),
                         "x": vec(b, "x"), "trans": "ma::product(T(M), X, Y)" in b,
                         "y": vec(b, "mx") if "mx" in b else vec(b, "y2")})
        if "ma::product(A, B, C);" in b and "atb" in b:
            gemm = {"A": vec(b, "a"), "B": vec(b, "b"), "AB": vec(b, "ab"), "AtB": vec(b, "atb"),
                    "ABt": vec(b, "abt"), "AtBt": vec(b, "atbt")}
        if "ma::invert(A)" in b:
            inv = {"A": vec(b, "a"), "tol": 1e-14}
    return {"gemv": gemv, "gemm": gemm, "invert": inv}


def main():
    out = {
        "source": "QMCPACK miniAFQMC self-tests (test_sparse_ops.cpp, sp_blas.hpp, ma_operations.hpp)",
        "sparse_ops": sparse_ops_cases(),
        "sp_blas": spblas_case(),
        "ma_operations": ma_operations_cases(),
    }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {OUT}: {len(out['sparse_ops'])} sparse cases, "
          f"{len(out['ma_operations']['gemv'])} gemv cases")


if __name__ == "__main__":
    main()
