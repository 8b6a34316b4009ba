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


def test_program_two_level_control_variate_on_the_gpu(tmp_path):
    """`-p mixed -e cv2` (the two-level control variate) against `-p mixed -e chol` (exact
    exchange) on the same walkers: the estimator does not touch the walkers, so the two
    runs print energies of the same ensemble, equal once the estimator is active up to its
    subset-sampling noise (about 2e-3 Ha per measurement at C1; bound 5e-2 Ha).  With the
    FP64 form the option is refused with an error exit."""
    exe = product_binary()
    s = system("C1")
    path = str(tmp_path / "c1.bin")
    s.write_input(path)
    base = [exe, "-f", path, "-w", "64", "-i", "40", "-s", "2", "-o", "5", "-r", "11", "-P",
            "17"]
    runs = {}
    for mode in ("chol", "cv2"):
        r = subprocess.run(base + ["-p", "mixed", "-e", mode], capture_output=True, text=True,
                           timeout=600, env=dict(os.environ))
        assert r.returncode == 0, r.stderr
        runs[mode] = step_energies(r.stdout)
        assert len(runs[mode]) == 40
    # 64 walkers x 32 measurements fill the network's first 2000 exact samples
    for (_, a), (_, b) in list(zip(runs["chol"], runs["cv2"]))[-6:]:
        assert abs(a - b) < 5e-2, (a, b)
    r = subprocess.run(base + ["-p", "fp64", "-e", "cv2"], capture_output=True, text=True,
                       timeout=600, env=dict(os.environ))
    assert r.returncode != 0
