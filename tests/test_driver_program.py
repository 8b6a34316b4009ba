"""The miniapp's driver program (`miniafqmc_b200/miniafqmc`, a C++ restatement of
src/miniapps/miniafqmc_base.cpp:93-360 over the C ABI).

On the host: the program built against the FP64 oracle behind the same ABI
(`oracle/abi_shim.cpp`) prints, step by step, the energies of the Python driver
(`miniafqmc_b200.driver.run`) on the oracle, to 1e-10 relative (the program half-rotates
Spvn itself, as the miniapp's main does, so SpvnT and the Cholesky factors are formed in a
different order than the Python system's: the last digits differ).  Covered: the
transposed path with the two-body energy, the Cholesky energy, the `-t no` full-G path,
checkpoint and exact resume, population control, and the input and option errors of the
product binary.  The product binary on a GPU:
`test_zzz_driver_program_gpu.py`."""
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, system

INCLUDE = os.path.join(ROOT, "include")


def scipy_openblas():
    import scipy
    libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs",
                                  "libscipy_openblas*.so"))
    return os.path.realpath(libs[0]) if libs else None


@pytest.fixture(scope="module")
def oracle_driver(tmp_path_factory):
    """The driver program linked against the oracle behind the C ABI."""
    if scipy_openblas() is None:
        pytest.skip("no scipy OpenBLAS library to resolve the oracle's LAPACK calls")
    d = tmp_path_factory.mktemp("oracle_driver")
    lib = str(d / "libafqmc_b200.so")
    subprocess.check_call(["g++", "-O2", "-fopenmp", "-std=c++17", "-fPIC", "-shared",
                           "-I", INCLUDE, os.path.join(ROOT, "oracle", "afqmc_oracle.cpp"),
                           os.path.join(ROOT, "oracle", "abi_shim.cpp"), "-ldl", "-o", lib])
    from miniafqmc_b200 import build
    exe = str(d / "miniafqmc")
    subprocess.check_call(build.driver_command(str(d), exe))
    return exe


@pytest.fixture(scope="module")
def c1_input(tmp_path_factory):
    s = system("C1")
    path = str(tmp_path_factory.mktemp("c1") / "c1.bin")
    s.write_input(path)
    return s, path


def run_program(exe, args, **kw):
    env = dict(os.environ, AFQ_ORACLE_LAPACK=scipy_openblas() or "",
               AFQ_ORACLE_LAPACK_PREFIX="scipy_", OMP_NUM_THREADS="4",
               OPENBLAS_NUM_THREADS="1")
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=900, env=env,
                          **kw)


def step_energies(stdout):
    """The `step   Eav` lines after the `# Step   Energy` header."""
    out, on = [], False
    for ln in stdout.splitlines():
        if ln.startswith("# Step"):
            on = True
            continue
        m = re.match(r"^(\d+)\s+(\S+)$", ln.strip()) if on else None
        if m:
            out.append((int(m.group(1)), float(m.group(2))))
        elif on and ln.strip() == "":
            if out:
                break
    return out


def python_energies(s, nwalk, nsteps, nsub, northo, seed, mode, full_g=False):
    from oracle import oracle as O
    o = O.Oracle(s, nwalk)
    if not full_g:
        from miniafqmc_b200 import driver
        return driver.run(o, nsteps, nsub, northo, seed, energy_mode=mode,
                          graph=False).energies[1:]
    o.calculate_mixed_density_matrix()
    energies, step_tot = [], 0
    for _ in range(nsteps):
        for _ in range(nsub):
            o.calculate_mixed_density_matrix_full()
            o.get_vbias_full()
            o.sigma(seed, step_tot)
            o.get_vHS()
            o.propagate()
            o.calculate_overlaps(save_old=True)
            o.update_weights()
            if step_tot > 0 and step_tot % northo == 0:
                o.orthogonalize()
                o.calculate_overlaps(save_old=False)
            step_tot += 1
        o.calculate_mixed_density_matrix()
        energies.append(o.calculate_energy(mode))
    return energies


@pytest.mark.parametrize("flags,mode,full_g", [
    ([], "vakbl", False),
    (["-e", "chol", "-g"], "chol", False),
    (["-t", "no"], "vakbl", True),
])
def test_program_on_the_oracle_matches_the_python_driver(oracle_driver, c1_input, flags,
                                                         mode, full_g):
    s, path = c1_input
    nwalk, nsteps, nsub, northo, seed = 4, 3, 4, 5, 11
    out = run_program(oracle_driver, ["-f", path, "-w", str(nwalk), "-i", str(nsteps), "-s",
                                      str(nsub), "-o", str(northo), "-r", str(seed),
                                      "-P", "17", *flags])
    assert out.returncode == 0, out.stderr
    got = step_energies(out.stdout)
    assert [k for k, _ in got] == list(range(nsteps))
    want = python_energies(s, nwalk, nsteps, nsub, northo, seed, mode, full_g)
    for (_, e), w in zip(got, want):
        assert abs(e - w) <= 1e-10 * abs(w), (e, w)
    assert "    NMO: 64" in out.stdout and "    nwalk: 4" in out.stdout
    assert f"({nsteps * nsub} substeps of {nwalk} walkers in" in out.stdout


@pytest.mark.parametrize("flags", [[], ["-g"]])
def test_checkpoint_resume_repeats_the_uninterrupted_run(oracle_driver, c1_input, tmp_path,
                                                         flags):
    """-c after two of four steps, then -R: the resumed steps print the energies of the
    run that was never interrupted, to the last digit (the fields are counter-based)."""
    s, path = c1_input
    base = ["-f", path, "-w", "4", "-s", "3", "-o", "4", "-r", "5", "-P", "17", *flags]
    full = run_program(oracle_driver, base + ["-i", "4"])
    assert full.returncode == 0, full.stderr
    ck = str(tmp_path / "ck.bin")
    first = run_program(oracle_driver, base + ["-i", "2", "-c", ck])
    assert first.returncode == 0, first.stderr
    # a different -r is ignored on resume: the checkpoint's seed continues the stream
    rest = run_program(oracle_driver, base[:-4] + ["-r", "99", "-P", "17", *flags,
                                                   "-i", "4", "-R", ck])
    assert rest.returncode == 0, rest.stderr
    want = step_energies(full.stdout)
    assert step_energies(first.stdout) == want[:2]
    assert step_energies(rest.stdout) == want[2:]
    assert "resumed after step 1 (substep 6)" in rest.stdout
    # the checkpoint must match the run
    bad = run_program(oracle_driver, base + ["-i", "4", "-w", "8", "-R", ck])
    assert bad.returncode == 1 and "the checkpoint holds 4 walkers" in bad.stderr
    junk = tmp_path / "junk.bin"
    junk.write_bytes(b"AFQCKP01" + b"\0" * 12)
    bad = run_program(oracle_driver, base + ["-i", "4", "-R", str(junk)])
    assert bad.returncode == 1 and "truncated header" in bad.stderr


def test_program_on_a_complex_system_without_the_two_body_matrix(oracle_driver, tmp_path):
    """Complex trial and Cholesky vectors, no Vakbl in the input: the program defaults to
    the Cholesky energy and passes only the half-rotated factors."""
    import dataclasses
    from conftest import tiny_system
    s = dataclasses.replace(tiny_system(), Vakbl=None)
    path = str(tmp_path / "tiny.bin")
    s.write_input(path)
    out = run_program(oracle_driver, ["-f", path, "-w", "3", "-i", "3", "-s", "3", "-o", "2",
                                      "-r", "7", "-P", "17"])
    assert out.returncode == 0, out.stderr
    assert "    energy: chol" in out.stdout
    got = step_energies(out.stdout)
    want = python_energies(s, 3, 3, 3, 2, 7, "chol")
    assert len(got) == 3
    for (_, e), w in zip(got, want):
        assert abs(e - w) <= 1e-10 * abs(w), (e, w)


def test_population_control_in_both_drivers(oracle_driver, c1_input):
    """-b 1 / branch_every=1: the comb after every step's energy, in the program (through
    afq_population_control) and in the Python driver on the oracle, gives the same energies;
    the combed run differs from the uncombed one."""
    from miniafqmc_b200 import driver
    from oracle import oracle as O
    s, path = c1_input
    nwalk, nsteps, nsub, northo, seed = 6, 4, 3, 4, 13
    out = run_program(oracle_driver, ["-f", path, "-w", str(nwalk), "-i", str(nsteps), "-s",
                                      str(nsub), "-o", str(northo), "-r", str(seed), "-P", "17",
                                      "-b", "1"])
    assert out.returncode == 0, out.stderr
    got = [e for _, e in step_energies(out.stdout)]
    want = driver.run(O.Oracle(s, nwalk), nsteps, nsub, northo, seed, "vakbl", graph=False,
                      branch_every=1).energies[1:]
    plain = driver.run(O.Oracle(s, nwalk), nsteps, nsub, northo, seed, "vakbl",
                       graph=False).energies[1:]
    assert len(got) == nsteps
    for e, w in zip(got, want):
        assert abs(e - w) <= 1e-10 * abs(w), (e, w)
    assert got[0] == pytest.approx(plain[0], rel=1e-10)   # the first comb follows step 0
    assert any(abs(a - b) > 1e-9 * abs(b) for a, b in zip(want[1:], plain[1:]))


def test_python_driver_resume_and_checkpoints_shared_with_the_program(oracle_driver, c1_input,
                                                                      tmp_path):
    """driver.run writes and resumes the program's checkpoint layout: its own resumed steps
    repeat its uninterrupted run exactly, and a checkpoint of either driver continues in
    the other with the other's uninterrupted energies (1e-10: the two half-rotate Spvn in
    different orders)."""
    from miniafqmc_b200 import driver
    from oracle import oracle as O
    s, path = c1_input
    nwalk, nsub, northo, seed = 4, 3, 4, 5
    full = driver.run(O.Oracle(s, nwalk), 4, nsub, northo, seed, "vakbl", graph=False).energies
    ck = str(tmp_path / "py.bin")
    driver.run(O.Oracle(s, nwalk), 2, nsub, northo, seed, "vakbl", graph=False, checkpoint=ck)
    r = driver.read_checkpoint(ck)
    assert (r["steps"], r["step_tot"], r["seed"], r["nwalk"]) == (2, 2 * nsub, seed, nwalk)
    rest = driver.run(O.Oracle(s, nwalk), 4, nsub, northo, 999, "vakbl", graph=False,
                      resume=r).energies
    assert rest[1:] == full[3:]
    # the Python checkpoint continued by the program
    base = ["-f", path, "-w", str(nwalk), "-s", str(nsub), "-o", str(northo), "-P", "17"]
    out = run_program(oracle_driver, base + ["-i", "4", "-R", ck])
    assert out.returncode == 0, out.stderr
    got = step_energies(out.stdout)
    assert [k for k, _ in got] == [2, 3]
    for (_, e), w in zip(got, full[3:]):
        assert abs(e - w) <= 1e-10 * abs(w)
    # the program's checkpoint continued by the Python driver
    ckc = str(tmp_path / "cpp.bin")
    prog_full = run_program(oracle_driver, base + ["-r", str(seed), "-i", "4"])
    first = run_program(oracle_driver, base + ["-r", str(seed), "-i", "2", "-c", ckc])
    assert prog_full.returncode == 0 and first.returncode == 0
    cont = driver.run(O.Oracle(s, nwalk), 4, nsub, northo, 0, "vakbl", graph=False,
                      resume=driver.read_checkpoint(ckc)).energies[1:]
    for (_, w), e in zip(step_energies(prog_full.stdout)[2:], cont):
        assert abs(e - w) <= 1e-10 * abs(w)


def test_input_file_round_trip(c1_input):
    from miniafqmc_b200.synthetic import read_input
    s, path = c1_input
    d = read_input(path)
    assert (d["nmo"], d["naea"], d["naeb"], d["nchol"], d["dt"]) == (s.N, s.n, s.n, s.nchol,
                                                                      s.cfg.dt)
    for k in ("rowIndex", "cols", "vals"):
        assert np.array_equal(getattr(d["Spvn"], k), getattr(s.Spvn, k))
        assert np.array_equal(getattr(d["Vakbl"], k), getattr(s.Vakbl, k))
    for k in ("Propg1", "haj", "trial"):
        assert np.array_equal(d[k], getattr(s, k))


def product_binary():
    """The driver program linked against the in-tree library (relinked when stale)."""
    from miniafqmc_b200 import build
    if os.path.exists(build.LIB):
        return build.build_driver()
    build.build()
    return build.DRIVER


def test_program_help_and_option_errors():
    exe = product_binary()
    h = subprocess.run([exe, "-h"], capture_output=True, text=True, timeout=60)
    assert h.returncode == 1 and "-t                If set to no" in h.stdout
    for bad in (["-p", "half"], ["-e", "none"], ["-w", "0"],
                ["-t", "no", "-g"], ["-b", "-1"], ["-x"]):
        r = subprocess.run([exe, *bad], capture_output=True, text=True, timeout=60)
        assert r.returncode == 1 and "bad option" in r.stderr, bad


def test_program_input_errors(tmp_path, c1_input):
    exe = product_binary()
    s, path = c1_input
    blob = open(path, "rb").read()
    cases = {
        "missing": (str(tmp_path / "none.bin"), "cannot open"),
        "magic": (b"NOTAFILE" + blob[8:], "not a driver input file"),
        "truncated": (blob[: len(blob) // 2], "truncated"),
        "trailing": (blob + b"\0" * 8, "trailing bytes"),
        # NAEB != NAEA: the reference reads closed shells only (initialize_serial.hpp:67-71)
        "open_shell": (blob[:16] + np.array([s.n + 1], "<i4").tobytes() + blob[20:],
                       "NAEA != NAEB"),
        "bad_sizes": (blob[:8] + np.array([0], "<i4").tobytes() + blob[12:],
                      "bad sizes in the header"),
    }
    for name, (content, msg) in cases.items():
        if isinstance(content, bytes):
            p = tmp_path / f"{name}.bin"
            p.write_bytes(content)
            content = str(p)
        r = subprocess.run([exe, "-f", content], capture_output=True, text=True, timeout=60)
        assert r.returncode == 1 and msg in r.stderr, (name, r.stderr)
    # the two-body energy needs the two-body matrix
    s2 = system("C2", with_vakbl=False)
    p2 = str(tmp_path / "c2.bin")
    s2.write_input(p2)
    r = subprocess.run([exe, "-f", p2, "-e", "vakbl"], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 1 and "needs the two-body matrix" in r.stderr
