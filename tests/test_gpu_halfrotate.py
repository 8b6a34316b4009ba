"""GPU half-rotation of the Cholesky tensor (rotate.hpp:69-169, base::halfrotate_cholesky)
through the C ABI against the oracle's restatement of the reference's count-and-fill
passes: the same SpvnT sparsity (rowIndex and cols equal) with values within 1e-12
relative, and the dense factors Lh within 1e-12 of the host construction."""
import numpy as np
import pytest

from conftest import system, tiny_system
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("make", [
    lambda: system("C1"),
    lambda: system("C1", complex_trial=True, complex_chol=True, nchol=96, seed=5),
    lambda: tiny_system(nmo=13, nel=5, nchol=21),                    # ragged sizes
    lambda: system("C2", with_vakbl=False),
])
def test_halfrotate_matches_oracle(make):
    from miniafqmc_b200.afqmc import halfrotate
    s = make()
    ri, ci, v, Lh = halfrotate(s, cutoff=1e-6, dense=True)
    ri0, ci0, v0 = O.halfrotate(s, 1e-6)
    assert np.array_equal(ri, ri0) and np.array_equal(ci, ci0)
    assert rel(v, v0) < 1e-12
    assert rel(Lh, s.Lh) < 1e-12


def test_halfrotate_cutoff_and_empty_vectors():
    """A cutoff above every value leaves an empty CSR; a zero cutoff keeps every nonzero."""
    from miniafqmc_b200.afqmc import halfrotate
    s = tiny_system()
    ri, ci, v = halfrotate(s, cutoff=1e30)
    assert ri.shape == (s.nchol + 1,) and np.all(ri == 0) and ci.size == 0
    ri, ci, v = halfrotate(s, cutoff=0.0)
    ri0, ci0, v0 = O.halfrotate(s, 0.0)
    assert np.array_equal(ri, ri0) and np.array_equal(ci, ci0) and rel(v, v0) < 1e-12
