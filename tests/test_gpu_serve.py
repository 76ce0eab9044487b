"""Batched and served solves (de_server_*): every result is the same alone
and in the mix, admission respects the device budget in arrival order, and
oversized requests are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (N, theta, nev, spin, precision, seed): uneven sizes, shifts, precisions
MIX = [
    (3, 0.20, 1, "singlet", "fp64", 0),
    (4, 0.30, 2, "singlet", "fp64", 1),
    (3, 0.35, 2, "triplet", "mixed", 2),
    (4, 0.25, 1, "singlet", "mixed", 3),
    (2, 0.40, 1, "singlet", "fp64", 4),
    (4, 0.20, 4, "singlet", "fp64", 5),
]
SIGMA = -0.78


def _start(oracle, n, nev, seed, spin):
    p = oracle.Params(n=n, delta=2.0, theta=0.2)
    return oracle.seeded_start(p, nev, seed, spin)


def _alone(de, oracle, case, maxit):
    n, theta, nev, spin, prec, seed = case
    x0 = _start(oracle, n, nev, seed, spin)
    with de.Problem(n=n, delta=2.0, theta=theta, precision=prec) as h:
        r = h.gplmr_eig(x0, SIGMA, ns=5, maxit=maxit, tol=1e-9, max_inner_iter=5)
    return r.e, r.iterations


def test_results_alone_and_in_the_mix_agree(de, oracle):
    """Each solve is deterministic and shares nothing with the others but
    the GPU, so a solve run among others gives the bits it gives alone."""
    maxit = 12
    alone = [_alone(de, oracle, c, maxit) for c in MIX]
    with de.Server(workers=3) as srv:
        ids = []
        for k, c in enumerate(MIX):
            n, theta, nev, spin, prec, seed = c
            req = srv.request(n, _start(oracle, n, nev, seed, spin), SIGMA, theta=theta, precision=prec, ns=5,
                              maxit=maxit, tol=1e-9)
            ids.append(srv.submit(req, tag=k))
        got = {}
        for _ in ids:
            r = srv.wait_any()
            assert r.status == de.DE_OK
            got[r.tag] = r
        workers = {r.worker for r in got.values()}
    assert len(workers) > 1  # they did run side by side
    for k, (e, iters) in enumerate(alone):
        r = got[k]
        assert r.iterations == iters
        assert np.max(np.abs(r.e - e)) <= 1e-12, (k, r.e, e)


def test_admission_in_arrival_order_within_budget(de, oracle):
    """With a budget that holds one request at a time, solves run one after
    another in submission order whatever the number of workers."""
    cases = [(3, 0.2, 1, "singlet", "fp64", s) for s in range(4)]
    reqs = []
    for c in cases:
        n, theta, nev, spin, prec, seed = c
        reqs.append(de.Server.request(n, _start(oracle, n, nev, seed, spin), SIGMA, theta=theta, maxit=4, tol=1e-12))
    fp = de.Server.footprint(reqs[0])
    with de.Server(workers=3, max_bytes=int(1.5 * fp)) as srv:
        ids = [srv.submit(r) for r in reqs]
        res = [srv.wait(i) for i in ids]
    for a, b in zip(res, res[1:]):
        assert b.t_start_s >= a.t_end_s - 1e-6  # never two at once
        assert b.t_start_s >= a.t_start_s       # first come, first served
    assert all(r.status == de.DE_OK for r in res)


def test_oversized_request_is_refused(de, oracle):
    x0 = _start(oracle, 3, 1, 0, "singlet")
    req = de.Server.request(3, x0, SIGMA)
    with de.Server(workers=1, max_bytes=de.Server.footprint(req) // 2) as srv:
        with pytest.raises(de.DeError) as e:
            srv.submit(req)
        assert e.value.status == de.DE_E_BUSY
