"""The driver program (`miniafqmc_b200/miniafqmc`) on a GPU, against the Python driver
on the same library.  Collected last: it runs a second process on the GPU."""
import os
import subprocess

import pytest

from conftest import system
from test_driver_program import product_binary, step_energies

pytestmark = pytest.mark.gpu


def test_program_on_the_gpu_matches_the_python_driver(tmp_path):
    """The product binary (FP64 form, op by op and graph substeps) against the Python
    driver: the same calls in the same order, with SpvnT half-rotated on the GPU by the
    program instead of in numpy, so the last digits differ (1e-10 relative)."""
    from miniafqmc_b200 import driver
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_FP64
    exe = product_binary()
    s = system("C1")
    path = str(tmp_path / "c1.bin")
    s.write_input(path)
    nwalk, nsteps, nsub, northo, seed = 8, 3, 4, 5, 11
    e = AfqmcSys(s, nwalk, precision=AFQ_PREC_FP64)
    want = driver.run(e, nsteps, nsub, northo, seed, energy_mode="vakbl",
                      graph=False).energies[1:]
    e.close()
    for flags in ([], ["-g"]):
        r = subprocess.run([exe, "-f", path, "-w", str(nwalk), "-i", str(nsteps), "-s",
                            str(nsub), "-o", str(northo), "-r", str(seed), "-P", "17",
                            *flags], capture_output=True, text=True, timeout=600,
                           env=dict(os.environ))
        assert r.returncode == 0, r.stderr
        got = step_energies(r.stdout)
        assert len(got) == nsteps
        for (_, g), w in zip(got, want):
            assert abs(g - w) <= 1e-10 * abs(w), (flags, g, w)
