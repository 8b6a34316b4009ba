"""The reference's transposed_Spvn == false path (CLI `-t no`, miniafqmc_base.cpp:265-273)
on the GPU against the oracle's restatement: the full density matrix G[2][N][N] of every
walker (mixed_density_matrix.hpp:96-99) and vbias = T(Spvn) G_alpha + T(Spvn) G_beta
(vbias.hpp:66-81), to 1e-10 relative, the FP64 bar; then a substep driven by that vbias
agrees as well."""
import numpy as np
import pytest

from conftest import system, tiny_system
from test_gpu_parity import engines, perturbed, rel, TOL

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make,nw", [
    (lambda: system("C1"), 16),
    (lambda: system("C1", complex_trial=True, complex_chol=True, nchol=96, seed=5), 8),
    (lambda: tiny_system(nmo=13, nel=5, nchol=21), 5),
])
def test_full_g_path_matches_oracle(make, nw):
    s = make()
    g, o = engines(s, nw, walkers=perturbed(s, nw))
    for e in (g, o):
        e.calculate_mixed_density_matrix_full()
    assert rel(g.copy_out("G_full"), o.copy_out("G_full")) < TOL
    assert rel(g.get_walker_data()[:, 2:4], o.get_walkers()[1][:, 2:4]) < TOL
    for e in (g, o):
        e.get_vbias_full()
    vb = g.copy_out("vbias")
    assert rel(vb, o.copy_out("vbias")) < TOL
    # the transposed path gives the same vbias up to its half-rotation cutoff (1e-6)
    g.calculate_mixed_density_matrix()
    g.get_vbias()
    assert np.max(np.abs(g.copy_out("vbias") - vb)) < 1e-6 * s.nchol
    # a substep on the full-G vbias: fields, vHS, propagation
    for e in (g, o):
        e.calculate_mixed_density_matrix_full()
        e.get_vbias_full()
        e.sigma(3, 0)
        e.get_vHS()
        e.propagate()
    assert rel(g.get_walkers()[0], o.get_walkers()[0]) < TOL
    g.close()


def test_full_g_path_rejects_calls_out_of_order():
    from miniafqmc_b200.afqmc import AfqmcSys, AfqmcError
    s = system("C1")
    e = AfqmcSys(s, 16)
    with pytest.raises(AfqmcError):      # vbias before the full density matrix
        e.get_vbias_full()
    e.close()


def test_full_g_path_mixed_form():
    """The mixed form's -t no branch: full G from its tensor-core compact Gc (the FP64
    full-G product and T(Spvn) gather on top), against the FP64 form's on the same walkers
    (1e-4 relative, the split-bf16 tolerance of Gc), and a substep driven by that vbias."""
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_FP64, AFQ_PREC_MIXED
    s = system("C1")
    nw = 16
    wk = perturbed(s, nw)
    d = AfqmcSys(s, nw, precision=AFQ_PREC_FP64, walkers=wk)
    m = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED, walkers=wk)
    for e in (d, m):
        e.calculate_mixed_density_matrix_full()
        e.get_vbias_full()
    assert rel(m.copy_out("G_full"), d.copy_out("G_full")) < 1e-4
    assert rel(m.copy_out("vbias"), d.copy_out("vbias")) < 1e-4
    for e in (d, m):
        e.sigma(3, 0)
        e.get_vHS()
        e.propagate()
    assert rel(m.get_walkers()[0], d.get_walkers()[0]) < 2e-2
    d.close()
    m.close()
