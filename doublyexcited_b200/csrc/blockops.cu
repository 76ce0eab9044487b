// blockops.cu -- tall-skinny FP64 complex block operations of the GPLMR
// eigensolver and its inner solve, for sm_100a.
//
// Reference: crossmult / crossmult_diag / colnorms / normalize / cholQR
// lamod.f90:21-180, the K/M projection ZGEMMs gplmr.F90:201-277, the
// 'N','N' ZGEMM updates gplmr.F90:101-103,298-320 and the inner-solve
// products harmonic_ritz_small.F90:28-75,145,313-316.  The MPI_ALLREDUCE
// of every k x k result becomes a deterministic two-stage on-device
// reduction (per-CTA partials, then a fixed-order sum), so repeated runs
// are bitwise identical.
//
// Every kernel here streams its vectors once; they are HBM-bound except the
// 64 x 64 projection Gram, which is FP64-FMA bound (8 flops per complex MAC).
#include "de_kernels.h"

#include <algorithm>

namespace de {
namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// ---------------------------------------------------------------- Gram

constexpr int kGramRT = 32;  // rows per smem tile
constexpr int kGramTX = 16;  // thread grid 16 x 16

__device__ __forceinline__ double2 col_elem(const ColList &L, int c, int64_t r)
{
    double2 v = __ldg(L.a[c] + r);
    if (L.b[c] != nullptr) {
        const double2 w = __ldg(L.b[c] + r);
        v.x -= L.sigma.x * w.x - L.sigma.y * w.y;
        v.y -= L.sigma.x * w.y + L.sigma.y * w.x;
    }
    return v;
}

template <int TA, int TB>
__global__ void __launch_bounds__(256)
    gram_partial(const __grid_constant__ ColList L, const __grid_constant__ ColList R, int64_t len,
                 int64_t chunk, int herm, double2 *__restrict__ work)
{
    extern __shared__ double2 gsm[];
    const int nl = L.n, nr = R.n;
    double2 *ls = gsm;                  // [RT][nl]
    double2 *rs = gsm + kGramRT * nl;   // [RT][nr]
    const int tx = threadIdx.x % kGramTX, ty = threadIdx.x / kGramTX;
    double ar[TA][TB], ai[TA][TB];
#pragma unroll
    for (int a = 0; a < TA; ++a)
#pragma unroll
        for (int b = 0; b < TB; ++b) ar[a][b] = ai[a][b] = 0.0;
    const int64_t r0 = (int64_t)blockIdx.x * chunk;
    const int64_t r1 = min(len, r0 + chunk);
    const double sg = herm ? -1.0 : 1.0;  // conj(L) flips the sign of L.im
    for (int64_t rt = r0; rt < r1; rt += kGramRT) {
        const int rows = (int)min((int64_t)kGramRT, r1 - rt);
        for (int idx = threadIdx.x; idx < kGramRT * nl; idx += blockDim.x) {
            const int r = idx % kGramRT, c = idx / kGramRT;
            double2 v = make_double2(0.0, 0.0);
            if (r < rows) v = col_elem(L, c, rt + r);
            v.y *= sg;
            ls[r * nl + c] = v;
        }
        for (int idx = threadIdx.x; idx < kGramRT * nr; idx += blockDim.x) {
            const int r = idx % kGramRT, c = idx / kGramRT;
            double2 v = make_double2(0.0, 0.0);
            if (r < rows) v = col_elem(R, c, rt + r);
            rs[r * nr + c] = v;
        }
        __syncthreads();
#pragma unroll 4
        for (int r = 0; r < kGramRT; ++r) {
            double2 lv[TA], rv[TB];
#pragma unroll
            for (int a = 0; a < TA; ++a) {
                const int i = tx + kGramTX * a;
                lv[a] = (i < nl) ? ls[r * nl + i] : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int b = 0; b < TB; ++b) {
                const int j = ty + kGramTX * b;
                rv[b] = (j < nr) ? rs[r * nr + j] : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int a = 0; a < TA; ++a)
#pragma unroll
                for (int b = 0; b < TB; ++b) {
                    ar[a][b] = fma(lv[a].x, rv[b].x, ar[a][b]);
                    ar[a][b] = fma(-lv[a].y, rv[b].y, ar[a][b]);
                    ai[a][b] = fma(lv[a].x, rv[b].y, ai[a][b]);
                    ai[a][b] = fma(lv[a].y, rv[b].x, ai[a][b]);
                }
        }
        __syncthreads();
    }
    double2 *out = work + (int64_t)blockIdx.x * nl * nr;
#pragma unroll
    for (int a = 0; a < TA; ++a)
#pragma unroll
        for (int b = 0; b < TB; ++b) {
            const int i = tx + kGramTX * a, j = ty + kGramTX * b;
            if (i < nl && j < nr) out[i + nl * j] = make_double2(ar[a][b], ai[a][b]);
        }
}

__global__ void gram_reduce(const double2 *__restrict__ work, int nblk, int nl, int nr,
                            double2 *__restrict__ out, int ldo)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nl * nr) return;
    double sr = 0.0, si = 0.0;
    const int64_t stride = (int64_t)nl * nr;
    for (int b = 0; b < nblk; ++b) {
        const double2 v = work[b * stride + o];
        sr += v.x;
        si += v.y;
    }
    const int i = o % nl, j = o / nl;
    out[i + (int64_t)ldo * j] = make_double2(sr, si);
}

int gram_blocks(int nl, int nr, int64_t len)
{
    const int64_t tiles = (len + kGramRT - 1) / kGramRT;
    const int64_t cap = (int64_t)nl * nr > 1024 ? 296 : 592;
    return (int)std::max<int64_t>(1, std::min(tiles, cap));
}

template <int TA, int TB>
cudaError_t gram_go(const ColList &L, const ColList &R, int64_t len, int herm, double2 *work,
                    int nblk, int64_t chunk, cudaStream_t st)
{
    const size_t smem = (size_t)kGramRT * (L.n + R.n) * sizeof(double2);
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        cudaError_t e = cudaFuncSetAttribute(gram_partial<TA, TB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)(kGramRT * (64 + 128) * sizeof(double2)));
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    gram_partial<TA, TB><<<nblk, 256, smem, st>>>(L, R, len, chunk, herm, work);
    return cudaGetLastError();
}

int round_t(int n)
{
    const int t = (n + kGramTX - 1) / kGramTX;
    return t <= 1 ? 1 : t <= 2 ? 2 : t <= 4 ? 4 : 8;
}

// ---------------------------------------------------------------- update

template <int NOUT>
__global__ void __launch_bounds__(256)
    update_kernel(const __grid_constant__ UpdList U, const double2 *__restrict__ C, int ldc,
                  int64_t len)
{
    extern __shared__ double2 cs[];  // [nin][NOUT]
    const int nin = U.nin, nout = U.nout;
    for (int idx = threadIdx.x; idx < nin * NOUT; idx += blockDim.x) {
        const int i = idx / NOUT, j = idx % NOUT;
        cs[idx] = (j < nout) ? C[i + (int64_t)ldc * j] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < len; r += stride) {
        double2 acc[NOUT], yb[NOUT];
#pragma unroll
        for (int j = 0; j < NOUT; ++j) {
            acc[j] = make_double2(0.0, 0.0);
            yb[j] = make_double2(0.0, 0.0);
            if (j < nout && (U.beta[j].x != 0.0 || U.beta[j].y != 0.0)) yb[j] = cmul(U.beta[j], U.y[j][r]);
        }
        for (int i = 0; i < nin; ++i) {
            const double2 xv = U.x[i][r];
#pragma unroll
            for (int j = 0; j < NOUT; ++j) {
                const double2 c = cs[i * NOUT + j];
                acc[j].x = fma(xv.x, c.x, acc[j].x);
                acc[j].x = fma(-xv.y, c.y, acc[j].x);
                acc[j].y = fma(xv.x, c.y, acc[j].y);
                acc[j].y = fma(xv.y, c.x, acc[j].y);
            }
        }
#pragma unroll
        for (int j = 0; j < NOUT; ++j) {
            const double2 s = cmul(U.alpha, acc[j]);
            if (j < nout) U.y[j][r] = make_double2(yb[j].x + s.x, yb[j].y + s.y);
        }
    }
}

template <int NOUT>
cudaError_t update_go(const UpdList &U, const double2 *c, int ldc, int64_t len, cudaStream_t st)
{
    const size_t smem = (size_t)U.nin * NOUT * sizeof(double2);
    const int64_t want = (len + 255) / 256;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, 148 * 8));
    update_kernel<NOUT><<<blocks, 256, smem, st>>>(U, c, ldc, len);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- small

struct PtrPack {
    double2 *out[64];
    const double2 *a[64];
    const double2 *b[64];
};

__global__ void axpc_kernel(const __grid_constant__ PtrPack P, double2 s, const double2 *c_dev,
                            int64_t len)
{
    const int j = blockIdx.y;
    double2 c = c_dev ? c_dev[j] : make_double2(1.0, 0.0);
    const double2 sc = cmul(s, c);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < len; r += stride) {
        const double2 av = P.a[j][r], bv = P.b[j][r];
        P.out[j][r] = make_double2(av.x + sc.x * bv.x - sc.y * bv.y, av.y + sc.x * bv.y + sc.y * bv.x);
    }
}

__global__ void scale_kernel(const __grid_constant__ PtrPack P, const double2 *c_dev, int64_t len)
{
    const int j = blockIdx.y;
    const double2 c = c_dev[j];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < len; r += stride)
        P.out[j][r] = cmul(P.out[j][r], c);
}

__global__ void dotdiag_partial(const __grid_constant__ PtrPack P, int64_t len, int herm,
                                double2 *__restrict__ work)
{
    const int j = blockIdx.y;
    double sr = 0.0, si = 0.0;
    const double sg = herm ? -1.0 : 1.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < len; r += stride) {
        const double2 a = P.a[j][r], b = P.b[j][r];
        const double ay = sg * a.y;
        sr = fma(a.x, b.x, sr);
        sr = fma(-ay, b.y, sr);
        si = fma(a.x, b.y, si);
        si = fma(ay, b.x, si);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        sr += __shfl_down_sync(0xffffffffu, sr, off);
        si += __shfl_down_sync(0xffffffffu, si, off);
    }
    __shared__ double red[2][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        red[0][w] = sr;
        red[1][w] = si;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tr = 0.0, ti = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            tr += red[0][k];
            ti += red[1][k];
        }
        work[(int64_t)j * gridDim.x + blockIdx.x] = make_double2(tr, ti);
    }
}

__global__ void dotdiag_reduce(const double2 *__restrict__ work, int nblk, int n,
                               double2 *__restrict__ out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double sr = 0.0, si = 0.0;
    for (int b = 0; b < nblk; ++b) {
        const double2 v = work[(int64_t)j * nblk + b];
        sr += v.x;
        si += v.y;
    }
    out[j] = make_double2(sr, si);
}

__global__ void inv_sqrt_abs_kernel(const double2 *d, double2 *c, int n)
{
    const int j = threadIdx.x;
    if (j < n) {
        const double a = sqrt(hypot(d[j].x, d[j].y));
        c[j] = make_double2(1.0 / a, 0.0);
    }
}

__global__ void tables_kernel(int nn, int n, double charge, double delta,
                              const double *__restrict__ tinv, int nbd, double *__restrict__ t1a,
                              double *__restrict__ v12)
{
    const int nb = nn;  // TINV is (-NB..NB)^3 with NB = 2N+1 (initmod.F90:39)
    const double d3 = delta * delta * delta;
    const double a = -charge / d3;
    const int64_t m = (int64_t)nn * nn * nn;
    const int w = 2 * nn - 1;
    const int64_t nv = (int64_t)w * w * w;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < m + nv; idx += stride) {
        if (idx < m) {
            const int i = (int)(idx % nn) - n, j = (int)((idx / nn) % nn) - n, k = (int)(idx / ((int64_t)nn * nn)) - n;
            t1a[idx] = a * tinv[(i + nb) + (int64_t)nbd * ((j + nb) + (int64_t)nbd * (k + nb))];
        } else {
            const int64_t v = idx - m;
            const int di = (int)(v % w) - (nn - 1), dj = (int)((v / w) % w) - (nn - 1),
                      dk = (int)(v / ((int64_t)w * w)) - (nn - 1);
            v12[v] = tinv[(di + nb) + (int64_t)nbd * ((dj + nb) + (int64_t)nbd * (dk + nb))] / d3;
        }
    }
}

int stream_blocks(int64_t len)
{
    return (int)std::max<int64_t>(1, std::min<int64_t>((len + 255) / 256, 148 * 4));
}

}  // namespace

int64_t gram_work_elems(int nl, int nr, int64_t len)
{
    return (int64_t)gram_blocks(nl, nr, len) * nl * nr;
}

cudaError_t gram_launch(const ColList &L, const ColList &R, int64_t len, int herm, double2 *out,
                        int ldo, double2 *work, cudaStream_t st)
{
    if (L.n < 1 || L.n > 64 || R.n < 1 || R.n > 128 || len < 1) return cudaErrorInvalidValue;
    const int nblk = gram_blocks(L.n, R.n, len);
    int64_t chunk = (len + nblk - 1) / nblk;
    chunk = (chunk + kGramRT - 1) / kGramRT * kGramRT;
    const int ta = round_t(L.n), tb = round_t(R.n);
    cudaError_t e;
    if (ta > 4) return cudaErrorInvalidValue;
#define GRAM_CASE(A, B) \
    if (ta == A && tb == B) e = gram_go<A, B>(L, R, len, herm, work, nblk, chunk, st); else
    GRAM_CASE(1, 1) GRAM_CASE(1, 2) GRAM_CASE(1, 4) GRAM_CASE(1, 8)
    GRAM_CASE(2, 1) GRAM_CASE(2, 2) GRAM_CASE(2, 4) GRAM_CASE(2, 8)
    GRAM_CASE(4, 1) GRAM_CASE(4, 2) GRAM_CASE(4, 4) GRAM_CASE(4, 8)
    return cudaErrorInvalidValue;
#undef GRAM_CASE
    if (e != cudaSuccess) return e;
    const int nout = L.n * R.n;
    gram_reduce<<<(nout + 255) / 256, 256, 0, st>>>(work, nblk, L.n, R.n, out, ldo);
    return cudaGetLastError();
}

cudaError_t update_launch(const UpdList &U, const double2 *c_dev, int ldc, int64_t len,
                          cudaStream_t st)
{
    if (U.nin < 1 || U.nin > kMaxCols || U.nout < 1 || U.nout > 16 || len < 1)
        return cudaErrorInvalidValue;
    if (U.nout <= 1) return update_go<1>(U, c_dev, ldc, len, st);
    if (U.nout <= 2) return update_go<2>(U, c_dev, ldc, len, st);
    if (U.nout <= 4) return update_go<4>(U, c_dev, ldc, len, st);
    if (U.nout <= 8) return update_go<8>(U, c_dev, ldc, len, st);
    return update_go<16>(U, c_dev, ldc, len, st);
}

cudaError_t axpc_launch(double2 *const *out, const double2 *const *a, const double2 *const *b,
                        int n, double2 s, const double2 *c_dev, int64_t len, cudaStream_t st)
{
    if (n < 1 || n > 64) return cudaErrorInvalidValue;
    PtrPack P{};
    for (int j = 0; j < n; ++j) {
        P.out[j] = out[j];
        P.a[j] = a[j];
        P.b[j] = b[j];
    }
    axpc_kernel<<<dim3(stream_blocks(len) / n + 1, n), 256, 0, st>>>(P, s, c_dev, len);
    return cudaGetLastError();
}

cudaError_t scale_cols_launch(double2 *const *x, int n, const double2 *c_dev, int64_t len,
                              cudaStream_t st)
{
    if (n < 1 || n > 64) return cudaErrorInvalidValue;
    PtrPack P{};
    for (int j = 0; j < n; ++j) P.out[j] = x[j];
    scale_kernel<<<dim3(stream_blocks(len) / n + 1, n), 256, 0, st>>>(P, c_dev, len);
    return cudaGetLastError();
}

int64_t dotdiag_work_elems(int n, int64_t len)
{
    (void)len;
    return (int64_t)n * 296;
}

cudaError_t dotdiag_launch(const double2 *const *a, const double2 *const *b, int n, int64_t len,
                           int herm, double2 *out, double2 *work, cudaStream_t st)
{
    if (n < 1 || n > 64) return cudaErrorInvalidValue;
    PtrPack P{};
    for (int j = 0; j < n; ++j) {
        P.a[j] = a[j];
        P.b[j] = b[j];
    }
    const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>((len + 255) / 256, std::max(1, 296 / n)));
    dotdiag_partial<<<dim3(nblk, n), 256, 0, st>>>(P, len, herm, work);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dotdiag_reduce<<<1, 64, 0, st>>>(work, nblk, n, out);
    return cudaGetLastError();
}

cudaError_t inv_sqrt_abs_launch(const double2 *d, double2 *c, int n, cudaStream_t st)
{
    if (n < 1 || n > 64) return cudaErrorInvalidValue;
    inv_sqrt_abs_kernel<<<1, 64, 0, st>>>(d, c, n);
    return cudaGetLastError();
}

cudaError_t build_tables_launch(int nn, int n, double charge, double delta, const double *tinv,
                                int nbd, double *t1a, double *v12, cudaStream_t st)
{
    tables_kernel<<<148, 256, 0, st>>>(nn, n, charge, delta, tinv, nbd, t1a, v12);
    return cudaGetLastError();
}

}  // namespace de
