"""GPU parity of the PETSc-style GMRES inner solve (usepetscflag = 0:
PRECBLOCK_PETSC gplmr.F90:507-563 with KSPGMRES as PETSCSOLVE
petscsolve.F90:142-279 configures it) through the C ABI, against the
oracle's runs from the same seeded start.  PETSc itself is absent; the
oracle's GMRES is pinned to the Krylov least-squares definition on the CPU.
Bars: resonance energies within 1e-10 Hartree of the oracle; the
reference's matvec count within 2 % (a GMRES column whose residual
estimate lands within rounding of GM_TOL may stop one iteration apart).
(The file name sorts last: the suite stops at its first failure and these
tests are the newest.)"""
import numpy as np
import pytest

from conftest import load_json

pytestmark = pytest.mark.gpu


def _run(de, oracle, g, maxit=None):
    p, s, st = g["params"], g["solver"], g["start"]
    op = oracle.Params(n=p["n"], delta=p["delta"], theta=p["theta"])
    x0 = oracle.seeded_start(op, st["nev"], st["seed"], st["spin"])
    with de.Problem(n=p["n"], delta=p["delta"], theta=p["theta"]) as h:
        return h.gplmr_eig(x0, complex(*s["sigma"]), ns=s["ns"], maxit=maxit or s["maxit"], tol=s["tol"],
                           max_inner_iter=s["order"], usepetscflag=s["usepetscflag"])


def test_gmres_inner_solve_converges_like_the_oracle(de, oracle):
    g = load_json("gplmr_n3_nev1_petsc.json")
    assert g["solver"]["usepetscflag"] == 0
    r = _run(de, oracle, g)
    assert r.converged and abs(r.iterations - g["iterations"]) <= 1
    assert abs(r.e[0] - complex(*g["e"][0])) < 1e-10
    assert abs(r.matvecs_reference - g["matvecs_reference"]) <= 0.02 * g["matvecs_reference"]


def test_gmres_inner_solve_block_history(de, oracle):
    """NEV = 2: each column gets its own GMRES; the Ritz values after 6
    iterations agree with the oracle's."""
    g = load_json("gplmr_n3_nev2_petsc.json")
    k = 6
    r = _run(de, oracle, g, maxit=k)
    assert r.iterations == k
    e = np.array([complex(*z) for z in g["history"][k - 1]["e"]])
    assert np.max(np.abs(np.sort_complex(r.e) - np.sort_complex(e))) < 1e-10
