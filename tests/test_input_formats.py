"""The miniapp's input datasets (the HDF5 layout of `synthetic.System.hdf5_datasets`) read
back the way the reference's `afqmc::Initialize` reads them
(src/Matrix/initialize_serial.hpp:37-228), restated here in numpy, give exactly the
in-memory objects the library and the oracle are fed: haj, trial, Vakbl (compacted spin
indices), Propg1 and Spvn (scaled by sqrt(dt)).  No HDF5 library is present, so the
datasets are checked as arrays, not as a file."""
import math

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import system, tiny_system

WF = "/Wavefunctions/PureSingleDeterminant/"
PR = "/Propagators/phaseless_ImpSamp_ForceBias/"


def initialize(d: dict, dt: float) -> dict:
    """initialize_serial.hpp:37-224 on the datasets."""
    Idata = d[WF + "dims"]
    assert Idata[5] == Idata[6] and Idata[7] == 0              # :67-80
    NMO, NAEA = int(Idata[4]), int(Idata[5])
    assert Idata[2] == 2 * NMO * NMO and Idata[3] == 2 * NMO * NMO   # :81-86

    def compact(lin):                                          # :102-106, :147-151
        i, j = lin // NMO, lin % NMO
        a = np.where(i < NMO, i, i - NMO + NAEA)
        assert np.all(np.where(i < NMO, i < NAEA, i - NMO < NAEA))
        return a * NMO + j

    haj = np.zeros((2 * NAEA, NMO), np.complex128)             # :92-108
    ivec, vvec = d[WF + "hij_indx"], d[WF + "hij"]
    haj.reshape(-1)[compact(ivec.astype(np.int64))] = vvec
    wf = d[WF + "Wavefun"]                                     # :113-130
    assert wf.size == 2 * NMO * NAEA
    trial = np.conj(wf.reshape(2, NMO, NAEA))
    out = {"NMO": NMO, "NAEA": NAEA, "haj": haj, "trial": trial, "Vakbl": None}
    if Idata[1] > 0:                                           # :134-164
        ri = d[WF + "SpHijkl_rowIndex"].astype(np.int64)
        rows = np.repeat(np.arange(ri.shape[0] - 1), np.diff(ri))
        cols = d[WF + "SpHijkl_cols"].astype(np.int64)
        V = sp.csr_matrix((d[WF + "SpHijkl_vals"], (compact(rows), compact(cols))),
                          shape=(2 * NMO * NAEA, 2 * NMO * NAEA))
        V.sum_duplicates()
        V.sort_indices()
        out["Vakbl"] = V
    Ldims = d[PR + "Spvn_dims"]                                # :171-181
    ntot, nrows, nvecs, nblk = int(Ldims[0]), int(Ldims[1]), int(Ldims[2]), int(Ldims[4])
    assert nrows == NMO * NMO and int(Ldims[3]) == NMO
    P = d[PR + "Spvn_propg1"]                                  # :183-192
    assert P.size == NMO * NMO
    out["Propg1"] = P.reshape(NMO, NMO)
    counts = d[PR + "Spvn_block_sizes"]
    assert counts.shape[0] == nblk and int(np.sum(counts)) == ntot
    r, c, v = [], [], []
    for b in range(nblk):                                      # :201-216
        idx = d[PR + f"Spvn_index_{b}"].reshape(-1, 2)
        r.append(idx[:, 0])
        c.append(idx[:, 1])
        v.append(d[PR + f"Spvn_vals_{b}"])
    S = sp.csr_matrix((np.concatenate(v), (np.concatenate(r), np.concatenate(c))),
                      shape=(nrows, nvecs))
    S.sum_duplicates()
    S.sort_indices()
    out["Spvn"] = S * math.sqrt(dt)                            # :217-218
    return out


@pytest.mark.parametrize("make", [lambda: system("C1"), lambda: tiny_system()])
def test_datasets_initialize_to_the_in_memory_system(make):
    s = make()
    d = s.hdf5_datasets()
    got = initialize(d, s.cfg.dt)
    assert (got["NMO"], got["NAEA"]) == (s.N, s.n)
    assert np.array_equal(got["haj"], s.haj)
    assert np.array_equal(got["trial"], s.trial)
    assert np.array_equal(got["Propg1"], s.Propg1)
    Sp = got["Spvn"]
    assert np.array_equal(Sp.indptr, s.Spvn.rowIndex) and np.array_equal(Sp.indices, s.Spvn.cols)
    assert np.array_equal(Sp.data, s.Spvn.vals)
    if s.Vakbl is None:
        assert got["Vakbl"] is None
    else:
        V = got["Vakbl"]
        assert np.array_equal(V.indptr, s.Vakbl.rowIndex)
        assert np.array_equal(V.indices, s.Vakbl.cols) and np.array_equal(V.data, s.Vakbl.vals)
