"""GPU parity of the matvec (HAMMULT / MATBLOCK) through the C ABI against
the CPU oracle and the golden fixtures.  Bar: relative 2-norm error <= 1e-12
(the plain FP64 form must match the reference's matvec to 1e-12)."""
import numpy as np
import pytest

from conftest import load_npz, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("n,theta", [(1, 0.3), (2, 0.0), (2, 0.35), (3, 0.2), (4, 0.3), (5, 0.2), (6, 0.2)])
def test_hammult_matches_oracle(de, oracle, n, theta):
    p = oracle.Params(n=n, delta=2.0, theta=theta)
    h = oracle.init_hamiltonian(p, nelec=2)
    x = oracle.seeded_vectors(p.m ** 2, 1, 100 + n)[:, 0]
    with de.Problem(n=n, delta=2.0, theta=theta) as g:
        y = g.hammult(x)
    assert rel_err(y, h.matvec(x)) < TOL


@pytest.mark.parametrize("n", [7, 8])
def test_hammult_matches_oracle_large(de, oracle, n):
    """N=7,8 (NN=15,17): the shared-memory tilings of the larger grids."""
    p = oracle.Params(n=n, delta=2.0, theta=0.35)
    h = oracle.init_hamiltonian(p, nelec=2)
    x = oracle.seeded_vectors(p.m ** 2, 1, 7)[:, 0]
    with de.Problem(n=n, delta=2.0, theta=0.35) as g:
        y = g.hammult(x)
    assert rel_err(y, h.matvec(x)) < TOL


@pytest.mark.parametrize("kind", ["fma", "tensor"])
@pytest.mark.parametrize("n", [3, 4, 5, 6, 7])
def test_both_matvec_kernels_match_oracle(de, oracle, n, kind):
    """The CUDA-core kernels and the FP64 tensor-core (DMMA) kernels each
    match the oracle (N=4..9 have both; other grids use the CUDA-core ones)
    on a block of two vectors with a fused shift."""
    import torch

    p = oracle.Params(n=n, delta=2.0, theta=0.3)
    h = oracle.init_hamiltonian(p, nelec=2)
    x = oracle.seeded_vectors(p.m ** 2, 2, 40 + n)
    with de.Problem(n=n, delta=2.0, theta=0.3) as g:
        g.set_matvec_kernel(kind)
        y = g.matblock(x)
    for j in range(2):
        assert rel_err(y[:, j], h.matvec(x[:, j])) < TOL


@pytest.mark.parametrize("name", ["hammult_n1.npz", "hammult_n2.npz"])
def test_hammult_full_golden(de, name):
    meta, a = load_npz(name)
    with de.Problem(n=meta["n"], delta=meta["delta"], theta=meta["theta"]) as g:
        assert rel_err(g.hammult(a["x"]), a["y"]) < TOL


@pytest.mark.parametrize("name", ["hammult_n3.npz", "hammult_n4.npz", "hammult_n5.npz", "hammult_n6.npz"])
def test_hammult_sampled_golden(de, oracle, name):
    meta, a = load_npz(name)
    p = oracle.Params(n=meta["n"], delta=meta["delta"], theta=meta["theta"])
    x = oracle.seeded_vectors(p.m ** 2, 1, meta["seed"])[:, 0]
    with de.Problem(n=meta["n"], delta=meta["delta"], theta=meta["theta"]) as g:
        y = g.hammult(x)
    assert rel_err(y[a["idx"]], a["y_idx"]) < TOL
    assert abs(np.linalg.norm(y) - a["y_norm"][0]) < TOL * a["y_norm"][0]


def test_one_electron_golden(de):
    """NELEC=1 (KEMULT1 + POTENTIAL1), the operator of the He+ pin."""
    meta, a = load_npz("hammult1_n5.npz")
    with de.Problem(n=meta["n"], delta=meta["delta"], theta=meta["theta"], nelec=1) as g:
        y = g.matblock(a["x"])
    assert rel_err(y, a["y"]) < TOL


def test_heplus_ground_state_by_power_free_check(de, oracle):
    """The GPU one-electron operator reproduces the reference's He+ level:
    for the oracle's dense eigenvector v of E0, ||H v - E0 v|| is tiny."""
    p = oracle.Params(n=5, delta=2.0, theta=0.2)
    h = oracle.init_hamiltonian(p, nelec=1)
    w, v = np.linalg.eig(oracle.dense_one_electron(h))
    i = int(np.argmin(w.real))
    with de.Problem(n=5, delta=2.0, theta=0.2, nelec=1) as g:
        hv = g.hammult(v[:, i])
    e_log = complex(-1.474195629488970, 0.148077368771954)
    assert abs(w[i] - e_log) < 1e-12
    assert np.linalg.norm(hv - e_log * v[:, i]) < 1e-11


def test_matblock_is_columnwise_hammult(de, oracle):
    p = oracle.Params(n=3, delta=2.0, theta=0.3)
    x = oracle.seeded_vectors(p.m ** 2, 3, 21)
    with de.Problem(n=3, delta=2.0, theta=0.3) as g:
        ax = g.matblock(x)
        for j in range(3):
            assert np.array_equal(ax[:, j], g.hammult(x[:, j]))  # deterministic, bitwise


def test_size_mismatch_is_an_error(de):
    import ctypes

    with de.Problem(n=2, delta=2.0, theta=0.3) as g:
        x = np.zeros(g.dim + 1, np.complex128)
        y = np.zeros_like(x)
        s = de.lib().de_hammult(g.handle, ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(y.ctypes.data), g.dim + 1)
        assert s == de.DE_E_SIZE
        s = de.lib().de_matblock(g.handle, ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(y.ctypes.data),
                                 g.m, g.m + 1, 1)
        assert s == de.DE_E_SIZE


def test_device_pointer_api(de, oracle):
    import torch

    p = oracle.Params(n=4, delta=2.0, theta=0.3)
    x = oracle.seeded_vectors(p.m ** 2, 2, 9)
    with de.Problem(n=4, delta=2.0, theta=0.3) as g:
        ref = g.matblock(x)
        g.set_stream(torch.cuda.current_stream().cuda_stream)
        xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
        yd = torch.empty_like(xd)
        g.matblock_d(xd.data_ptr(), yd.data_ptr(), 2)
        y = yd.cpu().numpy().T  # ordered after the kernels on the same stream
    assert np.array_equal(y, ref)


@pytest.mark.parametrize("kind", ["fma", "tensor", "tf32"])
@pytest.mark.parametrize("n,theta", [(3, 0.2), (5, 0.35), (6, 0.2)])
def test_fp32_matvec_relative_error(de, oracle, n, theta, kind):
    """The mixed form's FP32 matvec on complex64 inputs, per call, against
    the FP64 oracle's H x: relative 2-norm error within 1e-6 (FP32 unit
    roundoff 6e-8 times the contraction length and the conditioning of T).
    The first column is sampled at N=6 to keep the oracle fast."""
    import torch

    p = oracle.Params(n=n, delta=2.0, theta=theta)
    h = oracle.init_hamiltonian(p, nelec=2)
    x = oracle.seeded_vectors(p.m ** 2, 2, 21)
    x32 = x.astype(np.complex64)
    with de.Problem(n=n, delta=2.0, theta=theta, precision="mixed") as g:
        g.set_matvec_kernel(kind)
        g.set_stream(torch.cuda.current_stream().cuda_stream)
        xd = torch.from_numpy(np.ascontiguousarray(x32.T)).cuda()
        yd = torch.empty_like(xd)
        g.matblock32_d(xd.data_ptr(), yd.data_ptr(), 2)
        y = yd.cpu().numpy().T
    for j in range(2 if n < 6 else 1):
        ref = h.matvec(x32[:, j].astype(np.complex128))
        rel = np.linalg.norm(y[:, j] - ref) / np.linalg.norm(ref)
        assert rel < 1e-6, rel


@pytest.mark.parametrize("n", [9, 10])
def test_full_size_properties(de, n):
    """At the benchmark sizes (N=9: 753 MB per vector) the oracle is too
    slow, so check size-independent properties on the device: linearity,
    complex symmetry x^T H y = y^T H x and electron exchange
    H(X^T) = (H X)^T."""
    import torch

    with de.Problem(n=n, delta=2.0, theta=0.35) as g:
        g.set_stream(torch.cuda.current_stream().cuda_stream)
        m, dim = g.m, g.dim
        gen = torch.Generator(device="cuda").manual_seed(5)
        x = torch.randn(dim, dtype=torch.complex128, device="cuda", generator=gen)
        y = torch.randn(dim, dtype=torch.complex128, device="cuda", generator=gen)
        hx = torch.empty_like(x)
        hy = torch.empty_like(x)
        g.matblock_d(x.data_ptr(), hx.data_ptr(), 1)
        g.matblock_d(y.data_ptr(), hy.data_ptr(), 1)
        a = torch.dot(x, hy)
        b = torch.dot(y, hx)
        assert abs(a - b).item() < 1e-12 * abs(a).item()
        z = 2 * x + 1j * y
        hz = torch.empty_like(z)
        g.matblock_d(z.data_ptr(), hz.data_ptr(), 1)
        err = torch.linalg.norm(hz - (2 * hx + 1j * hy)) / torch.linalg.norm(hz)
        assert err.item() < 1e-14
        del y, hy, z, hz
        xt = x.view(m, m).t().contiguous().view(-1)  # X^T in the reference layout
        hxt = torch.empty_like(xt)
        g.matblock_d(xt.data_ptr(), hxt.data_ptr(), 1)
        err = torch.linalg.norm(hxt - hx.view(m, m).t().contiguous().view(-1)) / torch.linalg.norm(hx)
        assert err.item() < 1e-13
        torch.cuda.synchronize()


@pytest.mark.parametrize("n", [9])
def test_tensor_and_fma_kernels_agree_at_full_size(de, n):
    """N=9 (NN=19, 753 MB per vector): the DMMA kernels and the CUDA-core
    kernels give the same H x to FP64 rounding."""
    import torch

    with de.Problem(n=n, delta=2.0, theta=0.35) as g:
        g.set_stream(torch.cuda.current_stream().cuda_stream)
        gen = torch.Generator(device="cuda").manual_seed(9)
        x = torch.randn(g.dim, dtype=torch.complex128, device="cuda", generator=gen)
        y1 = torch.empty_like(x)
        y2 = torch.empty_like(x)
        g.set_matvec_kernel("fma")
        g.matblock_d(x.data_ptr(), y1.data_ptr(), 1)
        g.set_matvec_kernel("tensor")
        g.matblock_d(x.data_ptr(), y2.data_ptr(), 1)
        err = (torch.linalg.norm(y1 - y2) / torch.linalg.norm(y1)).item()
    assert err < 1e-13


@pytest.mark.parametrize("n", [8, 9])
def test_block_matvec_config_matches_oracle(de, oracle, n):
    """The block-matvec configuration (N=9 and N=8, theta=0.35, seed 1): the
    FP64 matvec within 1e-12 and the mixed form's FP32 matvec within 1e-6
    of the oracle's HAMMULT, on one full-size vector of the block (753 MB at
    N=9)."""
    import torch

    p = oracle.Params(n=n, delta=2.0, theta=0.35)
    h = oracle.init_hamiltonian(p, nelec=2)
    x = oracle.seeded_vectors(p.m ** 2, 1, 1)[:, 0]
    ref = h.matvec(x)
    with de.Problem(n=n, delta=2.0, theta=0.35) as g64, \
            de.Problem(n=n, delta=2.0, theta=0.35, precision="mixed") as g32:
        st = torch.cuda.current_stream()
        g64.set_stream(st.cuda_stream)
        g32.set_stream(st.cuda_stream)
        xd = torch.from_numpy(x).to("cuda")
        yd = torch.empty_like(xd)
        g64.matblock_d(xd.data_ptr(), yd.data_ptr(), 1)
        y64 = yd.cpu().numpy()
        x32 = xd.to(torch.complex64)
        y32 = torch.empty_like(x32)
        g32.matblock32_d(x32.data_ptr(), y32.data_ptr(), 1)
        y32h = y32.cpu().numpy().astype(np.complex128)
        torch.cuda.synchronize()
    assert rel_err(y64, ref) < TOL
    assert rel_err(y32h, ref) < 1e-6


@pytest.mark.parametrize("n", [4, 5, 6, 7, 8, 9, 10])
def test_even_odd_kernels_match_streaming_kernels(de, n):
    """The default kernels (even/odd-split where they are faster) against
    the streaming / cube kernels on a block of two vectors with a fused
    shift, FP64 within 1e-13 and FP32 within 1e-6 relative; N=4..10 covers
    every grid the even/odd kernels serve and both passes' partial last
    units."""
    import torch

    with de.Problem(n=n, delta=2.0, theta=0.3) as g64, \
            de.Problem(n=n, delta=2.0, theta=0.3, precision="mixed") as g32:
        st = torch.cuda.current_stream()
        g64.set_stream(st.cuda_stream)
        g32.set_stream(st.cuda_stream)
        gen = torch.Generator(device="cuda").manual_seed(50 + n)
        x = torch.randn(2, g64.dim, dtype=torch.complex128, device="cuda", generator=gen)
        ys = {}
        for kind in ("fma", "stream"):
            g64.set_matvec_kernel(kind)
            g32.set_matvec_kernel(kind)
            y = torch.empty_like(x)
            g64.matblock_d(x.data_ptr(), y.data_ptr(), 2)
            x32 = x.to(torch.complex64)
            y32 = torch.empty_like(x32)
            g32.matblock32_d(x32.data_ptr(), y32.data_ptr(), 2)
            ys[kind] = (y, y32.to(torch.complex128))
        torch.cuda.synchronize()
    for j in range(2):
        ref = ys["stream"][0][j]
        assert (torch.linalg.norm(ys["fma"][0][j] - ref) / torch.linalg.norm(ref)).item() < 1e-13
        assert (torch.linalg.norm(ys["fma"][1][j] - ref) / torch.linalg.norm(ref)).item() < 1e-6


@pytest.mark.parametrize("n", [4, 5, 6, 7])
def test_tf32_tensor_core_matvec(de, n):
    """The complex64 matvec with its kinetic contractions on the TF32 tensor
    cores (tcgen05, head/tail-split operands) against the FP64 matvec, on a
    block of two vectors: within 1e-6 relative, the FP32 bar; N=4..7 are the
    grids it serves (NN 9..15), both passes' partial last batches
    included."""
    import torch

    with de.Problem(n=n, delta=2.0, theta=0.3) as g64, \
            de.Problem(n=n, delta=2.0, theta=0.3, precision="mixed") as g32:
        st = torch.cuda.current_stream()
        g64.set_stream(st.cuda_stream)
        g32.set_stream(st.cuda_stream)
        gen = torch.Generator(device="cuda").manual_seed(70 + n)
        x = torch.randn(2, g64.dim, dtype=torch.complex128, device="cuda", generator=gen)
        y = torch.empty_like(x)
        g64.matblock_d(x.data_ptr(), y.data_ptr(), 2)
        g32.set_matvec_kernel("tf32")
        x32 = x.to(torch.complex64)
        y32 = torch.empty_like(x32)
        g32.matblock32_d(x32.data_ptr(), y32.data_ptr(), 2)
        torch.cuda.synchronize()
    for j in range(2):
        err = (torch.linalg.norm(y32[j].to(torch.complex128) - y[j]) / torch.linalg.norm(y[j])).item()
        assert err < 1e-6, err


def test_handle_reads_the_tuning_table(de):
    """A handle starts from the committed tuning table's entries."""
    import os

    path = os.path.join(os.path.dirname(de.lib_path()), "matvec_tuning.txt")
    with de.Problem(n=6, delta=2.0, theta=0.3, precision="mixed") as g:
        for storage in ("c128", "c64"):
            for pass_ in (0, 1):
                assert g.get_matvec_launch(storage, pass_) == de.tuning_lookup(path, storage, 13, pass_)


@pytest.mark.parametrize("n", [4, 6, 7])
def test_every_tuning_candidate_gives_the_same_matvec(de, n):
    """Each launch choice the autotuner may pick, on either pass, against the
    built-in kernels: complex128 within 1e-13, complex64 within 1e-6 of the
    complex128 result."""
    import torch

    from doublyexcited_b200.tune import FAMILY_CODE, candidates

    with de.Problem(n=n, delta=2.0, theta=0.3) as g64, \
            de.Problem(n=n, delta=2.0, theta=0.3, precision="mixed") as g32:
        st = torch.cuda.current_stream()
        g64.set_stream(st.cuda_stream)
        g32.set_stream(st.cuda_stream)
        gen = torch.Generator(device="cuda").manual_seed(90 + n)
        x = torch.randn(2, g64.dim, dtype=torch.complex128, device="cuda", generator=gen)
        ref = torch.empty_like(x)
        g64.set_matvec_kernel("fma")
        g64.matblock_d(x.data_ptr(), ref.data_ptr(), 2)
        x32 = x.to(torch.complex64)
        for storage, g, xx, tol in (("c128", g64, x, 1e-13), ("c64", g32, x32, 1e-6)):
            for pass_ in (0, 1):
                for fam, ctas in candidates(storage, 2 * n + 1):
                    g.set_matvec_kernel("fma")
                    g.set_matvec_launch(storage, pass_, FAMILY_CODE[fam], ctas)
                    y = torch.empty_like(xx)
                    (g.matblock32_d if storage == "c64" else g.matblock_d)(xx.data_ptr(), y.data_ptr(), 2)
                    torch.cuda.synchronize()
                    err = (torch.linalg.norm(y.to(torch.complex128) - ref) / torch.linalg.norm(ref)).item()
                    assert err < tol, (storage, pass_, fam, ctas, err)
