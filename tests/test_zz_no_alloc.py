"""The allocation-free dot products (de_dots_noalloc_d), for callers that
cannot call cudaMalloc (a host application that owns all device memory
through its own pool or a fixed reservation).

Checked through the C ABI against the allocating entry point de_dots_d and
against numpy's products of the same host blocks, twice in a row (the calls
share one static scratch array, so the second call also checks that the
first left it reusable).  Same tolerance as the other dot-product checks
here: 1e-12 relative."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()  # columns contiguous


@pytest.mark.parametrize("nbra,nket,herm", [(5, 1, 1), (32, 1, 0), (4, 8, 1), (8, 3, 0)])
def test_noalloc_dots_match_allocating_dots(de, nbra, nket, herm):
    import torch

    L = de.lib()
    rng = np.random.default_rng(100 + nbra * 10 + nket)
    size = 1_000_003
    a = rng.standard_normal((size, nbra)) + 1j * rng.standard_normal((size, nbra))
    b = rng.standard_normal((size, nket)) + 1j * rng.standard_normal((size, nket))
    ad, bd = _dev(torch, a), _dev(torch, b)
    want = (a.conj().T if herm else a.T) @ b  # numpy, independent of the library's kernels
    ref = np.empty((nbra, nket), np.complex128, order="F")
    with de.Problem(n=1, delta=2.0, theta=0.3) as g:
        torch.cuda.synchronize()
        s = L.de_dots_d(g.handle, ctypes.c_void_p(ad.data_ptr()), ctypes.c_void_p(bd.data_ptr()), size, nbra,
                        nket, ctypes.c_void_p(ref.ctypes.data), herm)
        assert s == de.DE_OK
    out = torch.empty((nket, nbra), dtype=torch.complex128, device="cuda")  # nbra x nket column-major
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out.fill_(float("nan"))
        s = L.de_dots_noalloc_d(ctypes.c_void_p(ad.data_ptr()), ctypes.c_void_p(bd.data_ptr()), size, nbra, nket,
                                ctypes.c_void_p(out.data_ptr()), herm, ctypes.c_void_p(stream))
        assert s == de.DE_OK, L.de_last_error()
        got = out.cpu().numpy().T
        assert np.linalg.norm(got - ref) <= TOL * np.linalg.norm(ref)
        assert np.linalg.norm(got - want) <= TOL * np.linalg.norm(want)


def test_noalloc_dots_reject_shapes_beyond_the_scratch(de):
    import torch

    L = de.lib()
    x = torch.zeros(64 * 16, dtype=torch.complex128, device="cuda")
    o = torch.zeros(64 * 16, dtype=torch.complex128, device="cuda")
    for nbra, nket in [(33, 1), (8, 8), (5, 5)]:
        s = L.de_dots_noalloc_d(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()), 16, nbra, nket,
                                ctypes.c_void_p(o.data_ptr()), 1, None)
        assert s == de.DE_E_INVALID
        assert b"allocation-free maximum" in L.de_last_error()
