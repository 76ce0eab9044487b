"""The initial guess's He+ orbital step (de_heplus_orbitals: DIAGONALIZE +
HELIUM_ORBITALGATHER, doublyexcited.F90:135-137, hammod.F90:1084-1113) on
the host, against the oracle's dense ZGEEV of the same operator.  The
library splits the eigenproblem into the cube's 8 reflection-parity
sectors; inside a degenerate level the basis is free, so orbitals are
compared by span.  Bars: energies within 1e-12 Hartree, spans to 1e-10."""
import numpy as np
import pytest


def _span_residual(x, basis):
    coef, *_ = np.linalg.lstsq(basis, x, rcond=None)
    return np.linalg.norm(basis @ coef - x, axis=0).max()


@pytest.mark.parametrize("n,theta,numorbs,hermopt", [(3, 0.3, 5, False), (3, 0.3, 10, True), (2, 0.0, 5, False),
                                                     (4, 0.2, 14, False)])
def test_heplus_orbitals_match_oracle(de, oracle, n, theta, numorbs, hermopt):
    p = oracle.Params(n=n, delta=2.0, theta=theta)
    h1 = oracle.init_hamiltonian(p, nelec=1)
    a = oracle.dense_one_electron(h1)
    w_or, v_or = oracle.heplus_orbitals(h1, numorbs)
    w, orb = de.heplus_orbitals(n, a, numorbs, hermopt)
    assert np.max(np.abs(w - w_or)) < 1e-12
    assert _span_residual(orb, v_or) < 1e-10
    # orthonormal under the product the Gram-Schmidt used
    g = (orb.conj().T @ orb) if hermopt else (orb.T @ orb)
    assert np.max(np.abs(g - np.eye(numorbs))) < 1e-12
    # eigenvectors: H maps the span into itself
    assert _span_residual(a @ orb, orb) < 1e-10


def test_heplus_orbitals_feed_the_reference_subspace_n5(de, oracle):
    """N=5, 14 orbitals: the oracle's DIAGSUBSPACE on the library's orbitals
    gives the six subspace eigenvalues the reference printed
    (Out.S.N5:100-107) to the accuracy of its Lanczos orbitals."""
    p = oracle.Params(n=5, delta=2.0, theta=0.2)
    h1 = oracle.init_hamiltonian(p, nelec=1)
    h2 = oracle.init_hamiltonian(p, nelec=2)
    _, orb = de.heplus_orbitals(5, oracle.dense_one_electron(h1), 14, False)
    e0, _, _ = oracle.diagsubspace(h2, orb, True, False, -0.7131541429, 6)
    log = [(-0.70668286560422, 0.03676471730071), (-0.63390932605588, 0.02889602525833),
           (-0.63390456155722, 0.02890205309617), (-0.63390250056812, 0.02890988095510),
           (-0.63028124855576, 0.02597489130175), (-0.63027701879070, 0.02598683463795)]
    log = np.array([complex(a, b) for a, b in log])
    assert abs(e0[0] - log[0]) < 5e-6
    assert np.max(np.abs(e0 - log)) < 2e-5


def test_heplus_orbitals_rejects_bad_arguments(de):
    a = np.eye(27, dtype=np.complex128)
    with pytest.raises(de.DeError) as e:
        de.heplus_orbitals(1, a, 28)
    assert e.value.status == de.DE_E_INVALID
    with pytest.raises(ValueError):
        de.heplus_orbitals(2, a, 1)
