"""de_run (PROGRAM ATOM, doublyexcited.F90:60-262) on the GPU: an Input.Inp
run equals the same steps made one by one through the C ABI.  The steps
are the initial guess, GET_EXPECTS, the shift as the real part of the mean
expectation value, GPLMR_EIG, and WRITEVECS.  Bars: guess and expectation
values to 1e-12, the eigenvalue after a fixed 8 iterations to 1e-10, the
written file equal to the returned vectors.  (The file name sorts last: the
suite stops at its first failure and this test is the newest.)"""
import numpy as np
import pytest

from conftest import load_json

pytestmark = pytest.mark.gpu


def test_run_replays_the_program_step_by_step(de, tmp_path):
    inp = tmp_path / "Input.Inp"
    out = tmp_path / "eigvecs.out"
    inp.write_text("&main\n WRITEVECS=.TRUE.\n/\n"
                   "&grid\n AUTODELTA=.false.\n DELTA=2d0\n N=3\n/\n"
                   "&orbitals\n NUMORBS=5\n SINGLET=T\n/\n"
                   "&gplmr\n GPLMR_SHIFT=(-0.78d0,0d0)\n GPLMR_MAXIT=8\n GPLMR_TOL=1D-14\n GPLMR_NEV=1\n/\n")
    # a list-directed read ends an unquoted value at '/': paths are quoted
    r = de.run([f"Inp={inp}", "Theta=0.3", f"Outfile='{out}'"])
    assert r.totget == 6  # min(MAXGET = 15, NEV + NUMSKIP + 5)
    with de.Problem(n=3, delta=2.0, theta=0.3) as h:
        e0, x0 = h.subspace_guess(5, True, False, -0.78, 6)
        ex = h.get_expects(x0)
        sigma = complex(ex[0].real, 0.0)
        g = h.gplmr_eig(x0[:, :1], sigma, ns=5, maxit=8, tol=1e-14, max_inner_iter=5)
    assert np.max(np.abs(r.e0 - e0)) < 1e-12
    assert np.max(np.abs(r.expects - ex)) < 1e-12
    assert abs(r.shift - sigma) < 1e-12
    assert r.iterations == g.iterations == 8
    assert abs(r.e[0] - g.e[0]) < 1e-10
    back = de.read_vectors(str(out), 7 ** 3, 1)
    assert np.array_equal(back[:, 0], r.x[:, 0])


def test_run_replays_the_reference_n5_program(de, tmp_path):
    """The reference's logged N=5 run (Out.S.N5) through de_run with its
    settings: 14 orbitals, singlet, NEV 1, the shift's imaginary part kept,
    gm_usepetscflag = 0 (the PETSc GMRES path), tol 1e-7.  Against the
    oracle's replay of the same program (pipeline_n5_petsc.json): the shift
    to 1e-9, the iteration count to one (the last residual sits near the
    tolerance), the resonance to 2e-8 Hartree; and the logged resonance to
    3e-8 (its start came from Lanczos orbitals)."""
    g = load_json("pipeline_n5_petsc.json")
    inp = tmp_path / "Input.Inp"
    inp.write_text("&grid\n AUTODELTA=.false.\n DELTA=2d0\n N=5\n/\n"
                   "&orbitals\n NUMORBS=14\n SINGLET=T\n/\n"
                   "&gmres\n gm_usepetscflag=0\n/\n"
                   "&gplmr\n GPLMR_SHIFT=(-0.7131541429d0,0d0)\n GPLMR_MAXIT=40\n GPLMR_TOL=1D-7\n"
                   " GPLMR_NEV=1\n TAKEREALPART=.FALSE.\n/\n")
    r = de.run([f"Inp={inp}", "Theta=0.2"])
    assert r.totget == 6
    assert abs(r.shift - complex(*g["shift"])) < 1e-9
    assert r.converged and abs(r.iterations - g["iterations"]) <= 1
    assert abs(r.e[0] - complex(*g["e"][0])) < 2e-8
    assert abs(r.e[0] - complex(*g["reference_log"]["final"]["e"])) < 3e-8


def test_run_warm_starts_n6_from_the_n5_eigenvector(de, tmp_path):
    """The reference's warm start along N (Out.S.N5 then
    Out.S.D2d0.T0.2d0.N6.petsc): the N=5 program writes its eigenvector, the
    N=6 program reads it onto the bigger grid (SIXD_FIX), takes the real part
    of its expectation value as the shift and solves on the BASIC path
    (gm_usepetscflag = 1).  Against the oracle's replay
    (pipeline_n6_readvecs.json) and the logged resonance."""
    g = load_json("pipeline_n6_readvecs.json")
    vec = tmp_path / "eigvecs.S.N5"
    inp5 = tmp_path / "Input.N5"
    inp5.write_text("&main\n WRITEVECS=.TRUE.\n/\n&grid\n AUTODELTA=.false.\n DELTA=2d0\n N=5\n/\n"
                    "&orbitals\n NUMORBS=14\n SINGLET=T\n/\n&gmres\n gm_usepetscflag=0\n/\n"
                    "&gplmr\n GPLMR_SHIFT=(-0.7131541429d0,0d0)\n GPLMR_MAXIT=40\n GPLMR_TOL=1D-7\n"
                    " GPLMR_NEV=1\n TAKEREALPART=.FALSE.\n/\n")
    r5 = de.run([f"Inp={inp5}", "Theta=0.2", f"Outfile='{vec}'"])
    assert r5.converged
    inp6 = tmp_path / "Input.N6"
    inp6.write_text("&grid\n AUTODELTA=.false.\n DELTA=2d0\n/\n&gmres\n gm_usepetscflag=1\n/\n"
                    "&gplmr\n GPLMR_MAXIT=40\n GPLMR_TOL=1D-7\n GPLMR_NEV=1\n/\n")
    r6 = de.run([f"Inp={inp6}", "Read", "N=6", "Theta=0.2", f"Infile='{vec}'"])
    run, log = g["runs_by_usepetscflag"]["1"], g["reference_log"]
    assert r6.totget == 1
    assert abs(r6.expects[0] - complex(*g["expects"])) < 3e-8
    assert r6.converged and abs(r6.iterations - run["iterations"]) <= 1
    assert abs(r6.e[0] - complex(*run["e"][0])) < 3e-8
    assert abs(r6.e[0] - complex(*log["1"]["final"]["e"])) < 4e-8


@pytest.mark.parametrize("flag,log_it,log_e", [
    (1, 17, (-0.713160218513, 0.035265673069)),   # Out.S.D2d0.T0.2d0.N9.petsc:92-98 (BASIC)
    (0, 22, (-0.713160220730, 0.035265681394)),   # Out.S.D2d0.T0.2d0.N9.nopetsc:92-98 (GMRES)
])
def test_run_warm_start_n9_against_the_reference_logs(de, tmp_path, flag, log_it, log_e):
    """The reference's N=9 runs read the N=5 eigenvector straight onto the
    19^6 grid.  Their ICALLED counters show 72 products per iteration in
    the .petsc run (BASIC) and 36 in the .nopetsc run (GMRES).  The same
    program through de_run, from the N=5 program's eigenvector, against the
    logs: iteration count within one, resonance within 3e-8 Hartree (both
    starts are converged only to 1e-7)."""
    vec = tmp_path / "eigvecs.S.N5"
    inp5 = tmp_path / "Input.N5"
    inp5.write_text("&main\n WRITEVECS=.TRUE.\n/\n&grid\n AUTODELTA=.false.\n DELTA=2d0\n N=5\n/\n"
                    "&orbitals\n NUMORBS=14\n SINGLET=T\n/\n&gmres\n gm_usepetscflag=0\n/\n"
                    "&gplmr\n GPLMR_SHIFT=(-0.7131541429d0,0d0)\n GPLMR_MAXIT=40\n GPLMR_TOL=1D-7\n"
                    " GPLMR_NEV=1\n TAKEREALPART=.FALSE.\n/\n")
    assert de.run([f"Inp={inp5}", "Theta=0.2", f"Outfile='{vec}'"]).converged
    inp9 = tmp_path / "Input.N9"
    inp9.write_text(f"&grid\n AUTODELTA=.false.\n DELTA=2d0\n/\n&gmres\n gm_usepetscflag={flag}\n/\n"
                    "&gplmr\n GPLMR_MAXIT=40\n GPLMR_TOL=1D-7\n GPLMR_NEV=1\n/\n")
    r = de.run([f"Inp={inp9}", "Read", "N=9", "Theta=0.2", f"Infile='{vec}'"])
    assert abs(r.expects[0] - complex(-0.71315414287425, 0.03522745948576)) < 3e-8  # Out.S.D2d0.T0.2d0.N9.*:68
    assert r.converged and abs(r.iterations - log_it) <= 1
    assert abs(r.e[0] - complex(*log_e)) < 3e-8


def test_run_warm_start_at_inner_order_20(de, tmp_path):
    """Out.S.D2d0.T0.2d0.N6.petsc.20_inner_iter: the same warm start with
    BASIC at inner order 20 (Iter=20), which also takes the inner solve's
    Gram-Schmidt past 16 earlier vectors.  Against the oracle's replay
    (pipeline_n6_readvecs_order20.json) and the logged resonance.  Kept last:
    it is the one GPU test of an inner order above 16."""
    g = load_json("pipeline_n6_readvecs_order20.json")
    vec = tmp_path / "eigvecs.S.N5"
    inp5 = tmp_path / "Input.N5"
    inp5.write_text("&main\n WRITEVECS=.TRUE.\n/\n&grid\n AUTODELTA=.false.\n DELTA=2d0\n N=5\n/\n"
                    "&orbitals\n NUMORBS=14\n SINGLET=T\n/\n&gmres\n gm_usepetscflag=0\n/\n"
                    "&gplmr\n GPLMR_SHIFT=(-0.7131541429d0,0d0)\n GPLMR_MAXIT=40\n GPLMR_TOL=1D-7\n"
                    " GPLMR_NEV=1\n TAKEREALPART=.FALSE.\n/\n")
    assert de.run([f"Inp={inp5}", "Theta=0.2", f"Outfile='{vec}'"]).converged
    inp6 = tmp_path / "Input.N6"
    inp6.write_text("&grid\n AUTODELTA=.false.\n DELTA=2d0\n/\n&gmres\n gm_usepetscflag=1\n/\n"
                    "&gplmr\n GPLMR_MAXIT=40\n GPLMR_TOL=1D-7\n GPLMR_NEV=1\n/\n")
    r = de.run([f"Inp={inp6}", "Read", "N=6", "Theta=0.2", f"Infile='{vec}'", "Iter=20"])
    assert r.converged and abs(r.iterations - g["iterations"]) <= 1
    assert abs(r.e[0] - complex(*g["e"][0])) < 3e-8
    assert abs(r.e[0] - complex(*g["reference_log"]["final"]["e"])) < 3e-8


def test_run_warm_start_n9_at_inner_order_20(de, tmp_path):
    """Out.S.D2d0.T0.2d0.N9.petsc.120core.20_inner_iter: the N=5 eigenvector
    read onto N=9, BASIC at inner order 20.  Against the log: converged at
    iteration 6 (within one), resonance within 3e-8 Hartree (lines 90-96)."""
    vec = tmp_path / "eigvecs.S.N5"
    inp5 = tmp_path / "Input.N5"
    inp5.write_text("&main\n WRITEVECS=.TRUE.\n/\n&grid\n AUTODELTA=.false.\n DELTA=2d0\n N=5\n/\n"
                    "&orbitals\n NUMORBS=14\n SINGLET=T\n/\n&gmres\n gm_usepetscflag=0\n/\n"
                    "&gplmr\n GPLMR_SHIFT=(-0.7131541429d0,0d0)\n GPLMR_MAXIT=40\n GPLMR_TOL=1D-7\n"
                    " GPLMR_NEV=1\n TAKEREALPART=.FALSE.\n/\n")
    assert de.run([f"Inp={inp5}", "Theta=0.2", f"Outfile='{vec}'"]).converged
    inp9 = tmp_path / "Input.N9"
    inp9.write_text("&grid\n AUTODELTA=.false.\n DELTA=2d0\n/\n&gmres\n gm_usepetscflag=1\n/\n"
                    "&gplmr\n GPLMR_MAXIT=40\n GPLMR_TOL=1D-7\n GPLMR_NEV=1\n/\n")
    r = de.run([f"Inp={inp9}", "Read", "N=9", "Theta=0.2", f"Infile='{vec}'", "Iter=20"])
    assert r.converged and abs(r.iterations - 6) <= 1
    assert abs(r.e[0] - complex(-0.713160212291, 0.035265678863)) < 3e-8
