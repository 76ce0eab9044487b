"""The PETSc-path GMRES control flow (doublyexcited_b200/csrc/gmres.h, the
code the solver's device instance runs) compiled with host vector
operations (tests/gmres_host_check.cpp) and compared on the CPU with the
oracle's restatement (oracle.petsc_gmres): same iterate to 1e-12 relative,
same iteration count.  It covers the fixed-count, rtol-stop and restart paths
and a zero right-hand side."""
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "doublyexcited_b200", "csrc")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("gmres") / "gmres_host_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-I", CSRC, os.path.join(HERE, "gmres_host_check.cpp"),
                    "-o", exe], check=True)
    return exe


def _run(driver, tmp_path, a, b, max_it, rtol, restart):
    n = b.size
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(src, "wb") as f:
        np.array([n, max_it, restart], np.int32).tofile(f)
        np.array([rtol], np.float64).tofile(f)
        np.asfortranarray(a, dtype=np.complex128).ravel(order="F").tofile(f)
        np.asarray(b, np.complex128).tofile(f)
    subprocess.run([driver, str(src), str(dst)], check=True, timeout=60)
    raw = np.fromfile(dst, np.uint8)
    status, its = np.frombuffer(raw[:8].tobytes(), np.int32)
    return int(status), int(its), np.frombuffer(raw[8:].tobytes(), np.complex128)


def _system(seed, n=70):
    rng = np.random.default_rng(seed)
    a = np.diag(np.linspace(1.0, 2.5, n) + 0.25j) + 0.08 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return a, b


@pytest.mark.parametrize("max_it,restart", [(1, 30), (5, 30), (9, 30), (7, 3), (11, 4)])
def test_fixed_iterations_match_oracle(oracle, driver, tmp_path, max_it, restart):
    a, b = _system(max_it * 10 + restart)
    status, its, x = _run(driver, tmp_path, a, b, max_it, 1e-300, restart)
    ref = oracle.petsc_gmres(lambda v: a @ v, b, max_it=max_it, rtol=1e-300, restart=restart)
    assert status == 0 and its == ref.its == max_it
    assert np.linalg.norm(x - ref.x) < 1e-12 * np.linalg.norm(ref.x)


@pytest.mark.parametrize("rtol", [1e-1, 1e-3, 1e-6])
def test_rtol_stop_matches_oracle(oracle, driver, tmp_path, rtol):
    a, b = _system(3)
    status, its, x = _run(driver, tmp_path, a, b, 30, rtol, 30)
    ref = oracle.petsc_gmres(lambda v: a @ v, b, max_it=30, rtol=rtol)
    assert ref.reason == "converged_rtol"
    assert status == 0 and its == ref.its
    assert np.linalg.norm(x - ref.x) < 1e-12 * np.linalg.norm(ref.x)


def test_zero_right_hand_side(oracle, driver, tmp_path):
    a, _ = _system(4)
    status, its, x = _run(driver, tmp_path, a, np.zeros(70, np.complex128), 5, 1e-3, 30)
    assert status == 0 and its == 0 and not np.any(x)
