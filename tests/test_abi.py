"""The C-ABI library loads without a GPU and exports every entry point the header
declares (no compute calls here)."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "afqmc_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:afq_status|void|const char\*)\s+(afq_\w+)\s*\(", src, re.M)))


def test_header_declares_the_operation_set():
    names = declared_functions()
    for op in ("afq_mixed_density_matrix", "afq_overlaps", "afq_vbias", "afq_sigma", "afq_vhs",
               "afq_propagate", "afq_update_weights", "afq_orthogonalize", "afq_energy",
               "afq_substep", "afq_create", "afq_set_hamiltonian"):
        assert op in names


def test_library_exports_every_declared_symbol():
    from miniafqmc_b200 import build
    build.build()
    lib = ctypes.CDLL(build.LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from miniafqmc_b200.afqmc import EXPORTS
    assert set(declared_functions()) <= set(EXPORTS)


def test_status_strings_without_gpu():
    from miniafqmc_b200.afqmc import load_library
    lib = load_library()
    assert lib.afq_status_string(0) == b"ok"
    assert lib.afq_status_string(6) == b"singular overlap matrix"


def test_batch_rejects_bad_arguments_without_gpu():
    """The multi-system batch checks its arguments before touching the device."""
    import ctypes
    from miniafqmc_b200.afqmc import load_library
    lib = load_library()
    out = ctypes.c_void_p()
    assert lib.afq_batch_create(None, 1, ctypes.byref(out)) == 1      # AFQ_ERR_ARG
    arr = (ctypes.c_void_p * 1)(None)
    assert lib.afq_batch_create(arr, 1, ctypes.byref(out)) == 1
    assert lib.afq_batch_substep(None, None, 0, 5) == 1
    assert lib.afq_batch_synchronize(None) == 1


def test_control_variate_calls_reject_bad_arguments_without_gpu():
    """The control-variate set-up calls check their arguments before any device work."""
    from miniafqmc_b200.afqmc import load_library
    lib = load_library()
    assert lib.afq_cv_configure(None, 256, 1e-3, 1, 2000, 8) == 1      # AFQ_ERR_ARG
    assert lib.afq_cv_set_base(None, 1) == 1
    assert lib.afq_cv_stats(None, None) == 1


def test_halfrotate_rejects_bad_arguments_without_gpu():
    """The GPU half-rotation checks its arguments before selecting a device."""
    import ctypes
    import numpy as np
    from miniafqmc_b200.afqmc import load_library, CsrZ
    lib = load_library()
    nnz = ctypes.c_longlong()
    ri = np.zeros(5, np.int32)
    m = CsrZ(4, 3, ri.ctypes.data, None, None)        # nmo = 2, nchol = 3, no nonzeros
    tr = np.zeros(8)
    ok = (0, ctypes.byref(m), 2, 1, 3, tr.ctypes.data, 1e-6, 1.0, ctypes.byref(nnz))
    assert lib.afq_halfrotate(0, None, 2, 1, 3, tr.ctypes.data, 1e-6, 1.0, ctypes.byref(nnz),
                              None, None, None, None) == 1
    assert lib.afq_halfrotate(*ok[:2], 3, 1, 3, *ok[5:], None, None, None, None) == 1   # nrows
    assert lib.afq_halfrotate(*ok[:6], -1.0, 1.0, ctypes.byref(nnz), None, None, None,
                              None) == 1                                            # cutoff
    cols = np.zeros(1, np.int32)
    assert lib.afq_halfrotate(*ok, None, cols.ctypes.data, None, None) == 1        # no rowIndex



def _header_prototypes():
    """{name: (return type, [parameter types])} of the header's function declarations."""
    import re
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    out = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(afq_\w+)\s*\(([^()]*)\)\s*;", text):
        ret, name, params = " ".join(m.group(1).split()), m.group(2), m.group(3).strip()
        plist = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        types = []
        for p in plist:
            words = p.replace("*", " * ").split()
            if "*" in words:
                types.append("*")
            else:   # drop the parameter name
                types.append(" ".join(w for w in words[:-1] if w != "const"))
        out[name] = (ret.replace("typedef", "").strip(), types)
    return out


def test_python_signatures_match_header_prototypes():
    """Every ctypes declaration has the header prototype's arity and type classes
    (pointer / int or enum / uint64_t / long long / double / float)."""
    import ctypes
    from miniafqmc_b200.afqmc import signatures
    protos = _header_prototypes()
    enums = {"afq_status", "int", "afq_precision", "afq_energy_mode", "afq_buffer", "afq_stage"}

    def cls_of(c):
        if c in ("*",):
            return ctypes.c_void_p
        if c in enums:
            return ctypes.c_int
        return {"uint64_t": ctypes.c_uint64, "long long": ctypes.c_longlong,
                "double": ctypes.c_double, "float": ctypes.c_float}[c]

    sigs = signatures()
    assert set(sigs) == set(protos)
    for name, (args, res) in sigs.items():
        ret, params = protos[name]
        assert len(args) == len(params), name
        for a, p in zip(args, params):
            assert a == cls_of(p), (name, p, a)
        want = {"void": None, "const char *": ctypes.c_char_p, "const char*": ctypes.c_char_p,
                "afq_status": ctypes.c_int, "long long": ctypes.c_longlong}[ret]
        assert res == want, (name, ret, res)


def _header_enum_values():
    """{enumerator: value} of the header's enums (explicit values or running count)."""
    import re
    text = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    vals = {}
    for body in re.findall(r"typedef\s+enum\s*\{(.*?)\}", text, flags=re.S):
        nxt = 0
        for item in body.split(","):
            item = item.strip()
            if not item:
                continue
            name, _, v = item.partition("=")
            nxt = int(v.strip()) if v.strip() else nxt
            vals[name.strip()] = nxt
            nxt += 1
    return vals


def test_python_constants_match_header_enums():
    """Precision, energy-mode, buffer and stage numbering of the Python binding equal the
    header's enums."""
    from miniafqmc_b200 import afqmc as A
    e = _header_enum_values()
    assert (A.AFQ_PREC_FP64, A.AFQ_PREC_MIXED) == (e["AFQ_PREC_FP64"], e["AFQ_PREC_MIXED"])
    assert (A.AFQ_ENERGY_VAKBL, A.AFQ_ENERGY_CHOLESKY, A.AFQ_ENERGY_CV) == (
        e["AFQ_ENERGY_VAKBL"], e["AFQ_ENERGY_CHOLESKY"], e["AFQ_ENERGY_CV"])
    header_buf = {"Gc": "AFQ_BUF_GC", "vbias": "AFQ_BUF_VBIAS", "X": "AFQ_BUF_X",
                  "vHS": "AFQ_BUF_VHS", "hybridW": "AFQ_BUF_HYBRIDW", "xraw": "AFQ_BUF_XRAW",
                  "info": "AFQ_BUF_INFO", "energy_parts": "AFQ_BUF_ENERGY_PARTS",
                  "cv_pred": "AFQ_BUF_CV_PRED", "G_full": "AFQ_BUF_G_FULL"}
    assert set(A.BUFFERS) == set(header_buf)
    for k, v in A.BUFFERS.items():
        assert v == e[header_buf[k]], k
    stages = ["AFQ_STAGE_DM", "AFQ_STAGE_VBIAS", "AFQ_STAGE_SIGMA", "AFQ_STAGE_VHS",
              "AFQ_STAGE_PROPAGATE", "AFQ_STAGE_OVERLAP", "AFQ_STAGE_WEIGHTS",
              "AFQ_STAGE_ORTHO", "AFQ_STAGE_ENERGY"]
    assert [e[s] for s in stages] == list(range(len(A.STAGES))) and e["AFQ_NSTAGES"] == 9
