// guess.cu -- the reference's initial guess for GPLMR: He+ orbitals,
// symmetrised two-electron products of them, and H diagonalised in their
// span (doublyexcited.F90:135-190; HELIUM_ORBITALGATHER, HELIUM_ORBITAL,
// DIAGSUBSPACE and mysort hammod.F90:1041-1256,1658-1690).
//
// The reference converges the He+ orbitals with block Lanczos (lanmod.F90).
// Here they are exact eigenvectors of the one-electron operator: the GPU
// builds it column by column (M <= 12167 points) and the host runs a ZGEEV
// per parity sector.  The products, H times the products and the subspace
// matrix are formed on the device; the k x k eigenproblem runs on the host.
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "de_internal.h"
#include "de_kernels.h"

using namespace de;

namespace {

// psi_k(p, q) = f (a(p) b(q) + s b(p) a(q)) for the k-th orbital pair
__global__ void products_kernel(const double2 *__restrict__ orb, const int2 *__restrict__ pairs, int npairs,
                                int64_t m, double sign, double2 *__restrict__ psi)
{
    const int64_t d = m * m;
    const int k = blockIdx.y;
    if (k >= npairs) return;
    const int2 ij = pairs[k];
    const double f = ij.x == ij.y ? 0.5 : 1.0 / sqrt(2.0);
    const double2 *a = orb + (int64_t)ij.x * m, *b = orb + (int64_t)ij.y * m;
    double2 *out = psi + (int64_t)k * d;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < d; e += stride) {
        const int64_t p = e % m, q = e / m;
        const double2 ap = a[p], aq = a[q], bp = b[p], bq = b[q];
        const double xr = ap.x * bq.x - ap.y * bq.y + sign * (bp.x * aq.x - bp.y * aq.y);
        const double xi = ap.x * bq.y + ap.y * bq.x + sign * (bp.x * aq.y + bp.y * aq.x);
        out[e] = make_double2(f * xr, f * xi);
    }
}

__global__ void identity_kernel(double2 *x, int64_t m)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
        x[i + m * i] = make_double2(1.0, 0.0);
}

// general complex eigenproblem (ZGEEV, right vectors); a is destroyed
int zgeev_right(int n, std::vector<cplx> &a, std::vector<cplx> &w, std::vector<cplx> &vr)
{
    const Lapack &L = lapack();
    if (!L.ok || !L.zgeev) return set_error(DE_E_LAPACK, "host LAPACK (zgeev) not found (set DE_LAPACK_LIB)");
    w.assign(n, 0.0);
    vr.assign((size_t)n * n, 0.0);
    std::vector<cplx> vl(1);
    std::vector<double> rwork(2 * (size_t)n);
    int info = 0, one = 1, lwork = -1;
    cplx wq;
    L.zgeev("N", "V", &n, a.data(), &n, w.data(), vl.data(), &one, vr.data(), &n, &wq, &lwork, rwork.data(), &info,
            1, 1);
    lwork = std::max(2 * n, (int)wq.real());
    std::vector<cplx> work(lwork);
    L.zgeev("N", "V", &n, a.data(), &n, w.data(), vl.data(), &one, vr.data(), &n, work.data(), &lwork, rwork.data(),
            &info, 1, 1);
    if (info != 0) return set_error(DE_E_GEVP, "zgeev failed (info=%d)", info);
    return DE_OK;
}

struct DevBuf {
    void *p = nullptr;
    cudaStream_t st = nullptr;
    ~DevBuf()
    {
        if (p) cudaFreeAsync(p, st);
    }
    int alloc(size_t bytes, cudaStream_t s)
    {
        st = s;
        DE_CUDA(cudaMallocAsync(&p, bytes, s));
        return DE_OK;
    }
    double2 *d() const { return static_cast<double2 *>(p); }
};

struct Handle1 {
    de_problem *h = nullptr;
    ~Handle1()
    {
        if (h) de_problem_destroy(h);
    }
};

// One axis's parity functions about the centre c = (nn-1)/2: even ones are
// e_c and (e_{c+a} + e_{c-a})/sqrt(2), odd ones (e_{c+a} - e_{c-a})/sqrt(2),
// a = 1..c.  (i1 < 0: a single point.)
struct AxisFn {
    int i0, i1;
    double w0, w1;
};

std::vector<AxisFn> axis_basis(int nn, int odd)
{
    const int c = (nn - 1) / 2;
    const double r = 1.0 / std::sqrt(2.0);
    std::vector<AxisFn> b;
    if (!odd) b.push_back({c, -1, 1.0, 0.0});
    for (int a = 1; a <= c; ++a) b.push_back({c + a, c - a, r, odd ? -r : r});
    return b;
}

}  // namespace

namespace de {

// The numorbs He+ levels of lowest real part and their right eigenvectors,
// Gram-Schmidt orthonormalised as HELIUM_ORBITALGATHER hammod.F90:1084-1113
// does (c-products, or Hermitian products with hermopt), from the dense
// one-electron operator h1 (M x M, column-major, M = nn^3).
//
// The reference converges these levels with block Lanczos (lanmod.F90).
// Here they are exact eigenvectors.  The operator on the cube commutes with
// the reflections of each axis about the nucleus, so it is block diagonal in
// the 8 parity sectors (even/odd along x, y, z), each about M/8 wide; one
// ZGEEV per sector replaces a ZGEEV of the whole operator (about 64 times
// fewer flops).  Levels of equal real part keep sector order.
int heplus_orbitals(int nn, const cplx *h1, int numorbs, int hermopt, std::vector<cplx> &energy,
                    std::vector<cplx> &orb)
{
    const int64_t m = (int64_t)nn * nn * nn;
    if (nn < 1 || nn % 2 == 0) return set_error(DE_E_INVALID, "grid width %d is not 2N+1", nn);
    if (numorbs < 1 || numorbs > m)
        return set_error(DE_E_INVALID, "numorbs %d is not in 1..%lld", numorbs, (long long)m);
    struct Level {
        cplx w;
        int sector, col;
    };
    std::vector<Level> levels;
    std::vector<std::vector<cplx>> vecs(8);
    std::vector<std::vector<int>> sup_idx(8);
    std::vector<std::vector<double>> sup_w(8);
    std::vector<int> dims(8);
    for (int sec = 0; sec < 8; ++sec) {
        const auto bx = axis_basis(nn, sec & 1), by = axis_basis(nn, (sec >> 1) & 1), bz = axis_basis(nn, (sec >> 2) & 1);
        const int ds = (int)(bx.size() * by.size() * bz.size());
        dims[sec] = ds;
        if (ds == 0) continue;
        // support of each sector function: up to 8 grid points and weights
        std::vector<int> &si = sup_idx[sec];
        std::vector<double> &sw = sup_w[sec];
        si.assign((size_t)ds * 8, -1);
        sw.assign((size_t)ds * 8, 0.0);
        int k = 0;
        for (const auto &fz : bz)
            for (const auto &fy : by)
                for (const auto &fx : bx) {
                    int t = 0;
                    for (int cz = 0; cz < 2; ++cz) {
                        const int iz = cz ? fz.i1 : fz.i0;
                        if (iz < 0) continue;
                        for (int cy = 0; cy < 2; ++cy) {
                            const int iy = cy ? fy.i1 : fy.i0;
                            if (iy < 0) continue;
                            for (int cx = 0; cx < 2; ++cx) {
                                const int ix = cx ? fx.i1 : fx.i0;
                                if (ix < 0) continue;
                                si[(size_t)k * 8 + t] = ix + nn * (iy + nn * iz);
                                sw[(size_t)k * 8 + t] = (cx ? fx.w1 : fx.w0) * (cy ? fy.w1 : fy.w0) *
                                                        (cz ? fz.w1 : fz.w0);
                                ++t;
                            }
                        }
                    }
                    ++k;
                }
        // H_s = B_s^T H B_s
        std::vector<cplx> hs((size_t)ds * ds);
#pragma omp parallel for schedule(static)
        for (int b = 0; b < ds; ++b)
            for (int a = 0; a < ds; ++a) {
                cplx acc = 0.0;
                for (int u = 0; u < 8; ++u) {
                    const int q = si[(size_t)b * 8 + u];
                    if (q < 0) break;
                    const cplx *col = h1 + (size_t)q * m;
                    cplx part = 0.0;
                    for (int t = 0; t < 8; ++t) {
                        const int pidx = si[(size_t)a * 8 + t];
                        if (pidx < 0) break;
                        part += sw[(size_t)a * 8 + t] * col[pidx];
                    }
                    acc += sw[(size_t)b * 8 + u] * part;
                }
                hs[a + (size_t)ds * b] = acc;
            }
        std::vector<cplx> w;
        DE_TRY(zgeev_right(ds, hs, w, vecs[sec]));
        for (int c = 0; c < ds; ++c) levels.push_back({w[c], sec, c});
    }
    std::stable_sort(levels.begin(), levels.end(),
                     [](const Level &x, const Level &y) { return x.w.real() < y.w.real(); });
    energy.resize(numorbs);
    orb.assign((size_t)m * numorbs, 0.0);
    for (int k = 0; k < numorbs; ++k) {
        const Level &L = levels[k];
        energy[k] = L.w;
        const int ds = dims[L.sector];
        const cplx *y = vecs[L.sector].data() + (size_t)ds * L.col;
        cplx *out = orb.data() + (size_t)m * k;
        for (int a = 0; a < ds; ++a)
            for (int t = 0; t < 8; ++t) {
                const int pidx = sup_idx[L.sector][(size_t)a * 8 + t];
                if (pidx < 0) break;
                out[pidx] += sup_w[L.sector][(size_t)a * 8 + t] * y[a];
            }
    }
    // HELIUM_ORBITALGATHER: modified Gram-Schmidt in level order
    auto dotp = [&](const cplx *x, const cplx *y) {
        cplx s = 0.0;
        for (int64_t r = 0; r < m; ++r) s += (hermopt ? std::conj(x[r]) : x[r]) * y[r];
        return s;
    };
    for (int i = 0; i < numorbs; ++i) {
        cplx *xi = orb.data() + (size_t)i * m;
        for (int j = 0; j < i; ++j) {
            const cplx *xj = orb.data() + (size_t)j * m;
            const cplx c = dotp(xj, xi);
            for (int64_t r = 0; r < m; ++r) xi[r] -= xj[r] * c;
        }
        const cplx nrm = std::sqrt(dotp(xi, xi));
        if (std::abs(nrm) == 0.0) return set_error(DE_E_INVALID, "orbital %d has zero norm after Gram-Schmidt", i);
        for (int64_t r = 0; r < m; ++r) xi[r] /= nrm;
    }
    return DE_OK;
}

}  // namespace de

extern "C" DE_API int de_subspace_guess_d(de_problem *h, int numorbs, int singlet, int hermopt, de_complex etarget,
                                         int numout, de_complex *x_d, de_complex *e0)
{
    if (!h || !x_d || !e0) return set_error(DE_E_INVALID, "null argument");
    if (h->p.nelec != 2) return set_error(DE_E_INVALID, "the initial guess is for the two-electron operator");
    if (numorbs < 1) return set_error(DE_E_INVALID, "numorbs must be >= 1");
    const int totbas = singlet ? numorbs * (numorbs + 1) / 2 : numorbs * (numorbs - 1) / 2;
    if (numout < 1 || numout > totbas)
        return set_error(DE_E_INVALID, "Reset NUMOUT to be less than tot orbital basis size (%d > %d)", numout, totbas);
    if (numout > 16 || totbas > 128)
        return set_error(DE_E_INVALID, "subspace of %d products / %d outputs exceeds 128 / 16", totbas, numout);
    std::lock_guard<std::mutex> lk(h->mu);
    cudaSetDevice(h->p.device);
    cudaStream_t st = h->stream;
    const int64_t m = h->m, d = h->dim;

    // He+ orbitals from the dense one-electron H, column j = H e_j
    if (numorbs > m)
        return set_error(DE_E_INVALID, "numorbs %d exceeds the %lld one-electron levels", numorbs, (long long)m);
    Handle1 h1;
    de_params p1 = h->p;
    p1.nelec = 1;
    p1.precision = DE_PREC_FP64;
    DE_TRY(de_problem_create(&p1, &h1.h));
    std::vector<cplx> a1((size_t)m * m);
    {
        const cudaStream_t s1 = h1.h->stream;
        DevBuf eye, h1d;
        DE_TRY(eye.alloc((size_t)m * m * sizeof(double2), s1));
        DE_TRY(h1d.alloc((size_t)m * m * sizeof(double2), s1));
        DE_CUDA(cudaMemsetAsync(eye.p, 0, (size_t)m * m * sizeof(double2), s1));
        identity_kernel<<<(unsigned)std::min<int64_t>((m + 255) / 256, 1024), 256, 0, s1>>>(eye.d(), m);
        count_launch();
        DE_CUDA(cudaGetLastError());
        DE_TRY(h1.h->matblock(eye.d(), h1d.d(), (int)m));
        DE_CUDA(cudaMemcpyAsync(a1.data(), h1d.p, a1.size() * sizeof(cplx), cudaMemcpyDeviceToHost, s1));
        DE_CUDA(cudaStreamSynchronize(s1));
    }
    std::vector<cplx> energy, orb;
    DE_TRY(heplus_orbitals(h->nn, a1.data(), numorbs, hermopt, energy, orb));

    // HELIUM_ORBITAL products (i <= j singlet, i < j triplet) and H times them
    std::vector<int2> pairs;
    for (int i = 0; i < numorbs; ++i)
        for (int j = i + (singlet ? 0 : 1); j < numorbs; ++j) pairs.push_back(make_int2(i, j));
    DevBuf orbd, pairsd, psi, hpsi, amat;
    DE_TRY(orbd.alloc(orb.size() * sizeof(double2), st));
    DE_TRY(pairsd.alloc(pairs.size() * sizeof(int2), st));
    DE_TRY(psi.alloc((size_t)totbas * d * sizeof(double2), st));
    DE_TRY(hpsi.alloc((size_t)totbas * d * sizeof(double2), st));
    DE_TRY(amat.alloc((size_t)totbas * totbas * sizeof(double2), st));
    DE_CUDA(cudaMemcpyAsync(orbd.p, orb.data(), orb.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
    DE_CUDA(cudaMemcpyAsync(pairsd.p, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    products_kernel<<<dim3(592, totbas), 256, 0, st>>>(orbd.d(), static_cast<const int2 *>(pairsd.p), totbas, m,
                                                        singlet ? 1.0 : -1.0, psi.d());
    count_launch();
    DE_CUDA(cudaGetLastError());
    DE_TRY(h->matblock(psi.d(), hpsi.d(), totbas));

    // A(I, J) = psi_I . (H psi_J) (c-product, Hermitian with hermopt), in
    // blocks of at most 64 x 128
    DE_TRY(h->ensure_work(gram_work_elems(64, 128, d)));
    for (int i0 = 0; i0 < totbas; i0 += 64) {
        ColList L{}, R{};
        L.n = std::min(64, totbas - i0);
        for (int i = 0; i < L.n; ++i) L.a[i] = psi.d() + (int64_t)(i0 + i) * d;
        R.n = totbas;
        for (int j = 0; j < totbas; ++j) R.a[j] = hpsi.d() + (int64_t)j * d;
        cudaError_t e = gram_launch(L, R, d, hermopt ? 1 : 0, amat.d() + i0, totbas, h->d_work, st);
        if (e != cudaSuccess) return cuda_error(e, "gram");
    }
    std::vector<cplx> a((size_t)totbas * totbas);
    DE_CUDA(cudaMemcpyAsync(a.data(), amat.p, a.size() * sizeof(cplx), cudaMemcpyDeviceToHost, st));
    DE_CUDA(cudaStreamSynchronize(st));
    std::vector<cplx> e0all, vs;
    DE_TRY(zgeev_right(totbas, a, e0all, vs));
    // mysort hammod.F90:1658-1690: nearest to etarget first, later index on ties
    const cplx tgt(etarget.re, etarget.im);
    std::vector<int> order;
    std::vector<char> taken(totbas, 0);
    for (int k = 0; k < totbas; ++k) {
        int best = -1;
        double low = 0.0;
        for (int i = 0; i < totbas; ++i)
            if (!taken[i]) {
                const double dd = std::abs(e0all[i] - tgt);
                if (best < 0 || dd <= low) {
                    best = i;
                    low = dd;
                }
            }
        taken[best] = 1;
        order.push_back(best);
    }
    // X = Psi VR(:, order[0..numout)), then unit Hermitian norm
    std::vector<double2> c((size_t)totbas * numout);
    for (int j = 0; j < numout; ++j) {
        e0[j] = de_complex{e0all[order[j]].real(), e0all[order[j]].imag()};
        for (int i = 0; i < totbas; ++i) {
            const cplx v = vs[i + (size_t)totbas * order[j]];
            c[i + (size_t)totbas * j] = make_double2(v.real(), v.imag());
        }
    }
    DevBuf cd;
    DE_TRY(cd.alloc(c.size() * sizeof(double2), st));
    DE_CUDA(cudaMemcpyAsync(cd.p, c.data(), c.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
    double2 *x = reinterpret_cast<double2 *>(x_d);
    UpdList U{};
    U.nin = totbas;
    U.nout = numout;
    for (int i = 0; i < totbas; ++i) U.x[i] = psi.d() + (int64_t)i * d;
    for (int j = 0; j < numout; ++j) {
        U.y[j] = x + (int64_t)j * d;
        U.beta[j] = make_double2(0.0, 0.0);
    }
    U.alpha = make_double2(1.0, 0.0);
    cudaError_t e = update_launch(U, cd.d(), totbas, d, st);
    if (e != cudaSuccess) return cuda_error(e, "update");
    std::vector<const double2 *> cols(numout);
    std::vector<double2 *> wcols(numout);
    for (int j = 0; j < numout; ++j) cols[j] = wcols[j] = x + (int64_t)j * d;
    DE_TRY(h->ensure_work(dotdiag_work_elems(numout, d)));
    if ((e = dotdiag_launch(cols.data(), cols.data(), numout, d, 1, h->d_small, h->d_work, st)) != cudaSuccess)
        return cuda_error(e, "dotdiag");
    if ((e = inv_sqrt_abs_launch(h->d_small, h->d_small + 64, numout, st)) != cudaSuccess)
        return cuda_error(e, "inv_sqrt");
    if ((e = scale_cols_launch(wcols.data(), numout, h->d_small + 64, d, st)) != cudaSuccess)
        return cuda_error(e, "scale");
    DE_CUDA(cudaStreamSynchronize(st));
    return DE_OK;
}

extern "C" DE_API int de_subspace_guess(de_problem *h, int numorbs, int singlet, int hermopt, de_complex etarget,
                                       int numout, de_complex *x, de_complex *e0)
{
    if (!h || !x || !e0) return set_error(DE_E_INVALID, "null argument");
    if (numout < 1 || numout > 16) return set_error(DE_E_INVALID, "numout must be in 1..16");
    cudaSetDevice(h->p.device);
    const size_t bytes = (size_t)h->dim * numout * sizeof(double2);
    DevBuf xd;
    DE_TRY(xd.alloc(bytes, h->stream));
    DE_TRY(de_subspace_guess_d(h, numorbs, singlet, hermopt, etarget, numout, static_cast<de_complex *>(xd.p), e0));
    DE_CUDA(cudaMemcpyAsync(x, xd.p, bytes, cudaMemcpyDeviceToHost, xd.st));
    DE_CUDA(cudaStreamSynchronize(xd.st));
    return DE_OK;
}

extern "C" DE_API int de_heplus_orbitals(int n, const de_complex *h1, int numorbs, int hermopt, de_complex *energies,
                                        de_complex *orbitals)
{
    if (!h1 || !energies || !orbitals) return set_error(DE_E_INVALID, "null argument");
    if (n < 0 || n > 11) return set_error(DE_E_INVALID, "N = %d is not in 0..11", n);
    std::vector<cplx> energy, orb;
    DE_TRY(heplus_orbitals(2 * n + 1, reinterpret_cast<const cplx *>(h1), numorbs, hermopt, energy, orb));
    for (int k = 0; k < numorbs; ++k) energies[k] = de_complex{energy[k].real(), energy[k].imag()};
    std::copy(orb.begin(), orb.end(), reinterpret_cast<cplx *>(orbitals));
    return DE_OK;
}
