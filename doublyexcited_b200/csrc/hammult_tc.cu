// hammult_tc.cu -- the two-electron matvec on the FP64 tensor cores (DMMA,
// mma.sync m8n8k4 f64) for sm_100a.
//
// Reference: HAMMULT hammod.F90:19-67 -> KEMULT2 :138-187 -> KEMULTS
// :264-286, plus Y = Y + V*X (:58-59) with V from POTENTIAL2 :502-582.
//
// The same two passes as the CUDA-core kernels in hammult.cu (pass A: row
// cubes X(p, :), electron-2 axes + potential, writes Y; pass B: column cubes
// X(:, q), electron-1 axes, Y +=), but each axis contraction of a cube is a
// small real GEMM on the tensor cores:
//
//   U_a[o][(pq, c)] = sum_l T[o][l] X[l along axis a, pq][c]
//
// with T (NN x NN, zero-padded to 8*MT x 4*KS) as the A operand held in
// registers for the whole kernel, the cube's (re, im) components as the
// columns of B (4 (p,q) pairs x 2 components per n-tile), and the FP64
// accumulators of one n-tile in registers.  A CTA stages one cube in shared
// memory (cp.async, double-buffered when three cubes fit), runs the three
// axis GEMMs into a shared output cube (axis k writes, axes i and j add;
// every output element has one owner per phase), then an elementwise
// epilogue adds the potential (pass A), scales by 1/SCALE^2 and writes or
// accumulates the result in HBM.
//
// Storage R is double (complex128) or float (complex64, the mixed form's
// inner solve): FP32 inputs are widened to FP64 for the tensor cores, so
// the FP32 path only loses accuracy in its loads and stores.
#include "de_kernels.h"

#include <algorithm>

namespace de {
namespace {

template <class R>
struct TcC2;
template <>
struct TcC2<double> {
    using C = double2;
};
template <>
struct TcC2<float> {
    using C = float2;
};
template <class R>
using TC2 = typename TcC2<R>::C;

template <int NN, class R>
struct TcCfg {
    static constexpr int M = NN * NN * NN;
    static constexpr int P2 = NN * NN;
    // slab stride padded so that consecutive slabs start 64 bytes apart
    // modulo 128 (complex128): the four l-rows of a B fragment along the k
    // axis then fall in two bank-disjoint pairs
    static constexpr int P2P = P2 + ((4 - P2 % 8) + 8) % 8;
    static constexpr int CUBE = NN * P2P;
    static constexpr int MT = (NN + 7) / 8;  // m-tiles of outputs o
    static constexpr int KS = (NN + 3) / 4;  // k-steps over l
    static constexpr int NTILE = (P2 + 3) / 4;
    static constexpr int THREADS = 256;
    static constexpr size_t CUBE_BYTES = (size_t)CUBE * sizeof(TC2<R>);
    // double-buffered input only while three CTAs still fit on an SM;
    // otherwise more resident CTAs hide the load latency better
    static constexpr bool DB = 3 * 3 * CUBE_BYTES <= 227 * 1024;
    static constexpr size_t SMEM = (DB ? 3 : 2) * CUBE_BYTES;
};

enum TcMode { kTcRowsPot = 0, kTcColsAcc = 1 };

template <class R>
struct TcArgs {
    const TC2<R> *x;
    TC2<R> *y;
    int64_t vstride;
    double2 shs;  // shift * SCALE^2
};

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_8(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit_tc() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all_tc() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Copy cube `cube` into shared buffer xs (padded slab stride).
template <int NN, class R, int MODE>
__device__ __forceinline__ void load_cube(const TcArgs<R> &a, int64_t cube, TC2<R> *xs)
{
    using C = TcCfg<NN, R>;
    const int64_t vec = cube / C::M, cc = cube - vec * C::M;
    const TC2<R> *xv = a.x + vec * a.vstride;
    for (int g = threadIdx.x; g < C::M; g += C::THREADS) {
        const int k = g / C::P2, r = g - k * C::P2;
        const TC2<R> *src = (MODE == kTcRowsPot) ? xv + cc + (int64_t)C::M * g : xv + cc * (int64_t)C::M + g;
        TC2<R> *dst = xs + r + C::P2P * k;
        if constexpr (sizeof(R) == 8) cp_async_16(dst, src);
        else cp_async_8(dst, src);
    }
}

// Copy cube `cube` into shared buffer xs in its natural order (slab stride
// NN^2), `nthreads` threads.
template <int NN, class R, int MODE>
__device__ __forceinline__ void load_cube_flat(const TcArgs<R> &a, int64_t cube, TC2<R> *xs, int nthreads)
{
    constexpr int M = NN * NN * NN;
    const int64_t vec = cube / M, cc = cube - vec * M;
    const TC2<R> *xv = a.x + vec * a.vstride;
    for (int g = threadIdx.x; g < M; g += nthreads) {
        const TC2<R> *src = (MODE == kTcRowsPot) ? xv + cc + (int64_t)M * g : xv + cc * (int64_t)M + g;
        if constexpr (sizeof(R) == 8) cp_async_16(xs + g, src);
        else cp_async_8(xs + g, src);
    }
}

// Element offset of (l along axis A, pair pq of the other two coordinates).
template <int NN, int P2P, int A>
__device__ __forceinline__ int tc_base(int pq)
{
    if constexpr (A == 0) return NN * (pq % NN) + P2P * (pq / NN);  // (l, j, k)
    else if constexpr (A == 1) return (pq % NN) + P2P * (pq / NN);  // (i, l, k)
    else return pq;                                                 // (i, j, l)
}
template <int NN, int P2P, int A>
__device__ __forceinline__ constexpr int tc_stride()
{
    return A == 0 ? 1 : A == 1 ? NN : P2P;
}

// One axis of the cube: ys (=, or += when ADD) T x along axis A.  A warp
// takes two n-tiles per step (2*MT independent accumulator chains; all B
// loads issued before the first MMA).
template <int NN, class R, int A, bool ADD>
__device__ __forceinline__ void axis_gemm(const double (&ta)[TcCfg<NN, R>::MT][TcCfg<NN, R>::KS], const TC2<R> *xs,
                                          TC2<R> *ys)
{
    using C = TcCfg<NN, R>;
    constexpr int P2P = C::P2P, MT = C::MT, KS = C::KS;
    constexpr int S = tc_stride<NN, P2P, A>();
    constexpr int NW = C::THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const R *xr = reinterpret_cast<const R *>(xs);
    // B fragment: row (l) = lane % 4, column = lane / 4 -> pair (lane/4)/2, component (lane/4)%2
    const int bl = lane & 3, bpq = (lane >> 2) >> 1, bc = (lane >> 2) & 1;
    // C fragment: row (o) = lane / 4, columns 2*(lane%4) + {0,1} -> pair lane%4, (re, im)
    const int co = lane >> 2, cpq = lane & 3;
    for (int nt0 = warp; nt0 < C::NTILE; nt0 += 2 * NW) {
        double b[2][KS];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int pqb = 4 * (nt0 + u * NW) + bpq;
            const bool ok = pqb < C::P2;
            const int boff = ok ? tc_base<NN, P2P, A>(pqb) : 0;
#pragma unroll
            for (int ks = 0; ks < KS; ++ks) {
                const int l = 4 * ks + bl;
                b[u][ks] = (ok && l < NN) ? (double)xr[2 * (boff + S * l) + bc] : 0.0;
            }
        }
        double acc[2][MT][2];
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) acc[u][mt][0] = acc[u][mt][1] = 0.0;
#pragma unroll
        for (int ks = 0; ks < KS; ++ks)
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
#pragma unroll
                for (int u = 0; u < 2; ++u) dmma(acc[u][mt][0], acc[u][mt][1], ta[mt][ks], b[u][ks]);
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int pqc = 4 * (nt0 + u * NW) + cpq;
            if (pqc < C::P2) {
                const int coff = tc_base<NN, P2P, A>(pqc);
#pragma unroll
                for (int mt = 0; mt < MT; ++mt) {
                    const int o = 8 * mt + co;
                    if (o < NN) {
                        TC2<R> &dst = ys[coff + S * o];
                        if constexpr (ADD) {
                            dst.x = (R)((double)dst.x + acc[u][mt][0]);
                            dst.y = (R)((double)dst.y + acc[u][mt][1]);
                        } else {
                            dst.x = (R)acc[u][mt][0];
                            dst.y = (R)acc[u][mt][1];
                        }
                    }
                }
            }
        }
    }
}

template <int NN, class R, int MODE>
__global__ void __launch_bounds__(256) tc_kernel(const __grid_constant__ HamDev h, const __grid_constant__ TcArgs<R> a,
                                                 int64_t ncubes)
{
    using C = TcCfg<NN, R>;
    constexpr int M = C::M, P2 = C::P2, P2P = C::P2P, MT = C::MT, KS = C::KS;
    extern __shared__ __align__(16) unsigned char tc_smem[];
    TC2<R> *buf0 = reinterpret_cast<TC2<R> *>(tc_smem);
    TC2<R> *ys = buf0 + C::CUBE;
    TC2<R> *buf1 = C::DB ? ys + C::CUBE : buf0;
    // T as the A operand: row o = 8 mt + lane/4, column l = 4 ks + lane%4
    double ta[MT][KS];
    {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int mt = 0; mt < MT; ++mt)
#pragma unroll
            for (int ks = 0; ks < KS; ++ks) {
                const int o = 8 * mt + (lane >> 2), l = 4 * ks + (lane & 3);
                ta[mt][ks] = (o < NN && l < NN) ? h.t[o > l ? o - l : l - o] : 0.0;
            }
    }
    int64_t cube = blockIdx.x;
    int cur = 0;
    if (cube < ncubes) load_cube<NN, R, MODE>(a, cube, buf0);
    cp_commit_tc();
    for (; cube < ncubes; cube += gridDim.x) {
        TC2<R> *xs = cur ? buf1 : buf0;
        cp_wait_all_tc();
        __syncthreads();
        if constexpr (C::DB) {  // prefetch the next cube into the other buffer
            const int64_t nc = cube + gridDim.x;
            if (nc < ncubes) load_cube<NN, R, MODE>(a, nc, cur ? buf0 : buf1);
            cp_commit_tc();
        }
        axis_gemm<NN, R, 2, false>(ta, xs, ys);
        __syncthreads();
        axis_gemm<NN, R, 0, true>(ta, xs, ys);
        __syncthreads();
        axis_gemm<NN, R, 1, true>(ta, xs, ys);
        __syncthreads();
        // epilogue: potential (pass A), 1/SCALE^2, store
        const int64_t vec = cube / M, cc = cube - vec * M;
        TC2<R> *yv = a.y + vec * a.vstride;
        const double s2r = h.s2re, s2i = h.s2im;
        int ip = 0, jp = 0, kp = 0;
        double t1p = 0.0;
        if constexpr (MODE == kTcRowsPot) {
            ip = (int)(cc % NN);
            jp = (int)((cc / NN) % NN);
            kp = (int)(cc / P2);
            t1p = h.t1a[cc];
        }
        constexpr int EU = 4;  // elements per thread per step, loads first
        for (int g0 = threadIdx.x; g0 < M; g0 += EU * C::THREADS) {
            double ar[EU], ai[EU], xr[EU], xi[EU], vr[EU], orr[EU], oi[EU];
            int gs[EU];
#pragma unroll
            for (int u = 0; u < EU; ++u) {
                const int g = g0 + u * C::THREADS;
                gs[u] = g;
                ar[u] = ai[u] = xr[u] = xi[u] = vr[u] = orr[u] = oi[u] = 0.0;
                if (g < M) {
                    const int k = g / P2, r = g - k * P2;
                    const int s = r + P2P * k;
                    const TC2<R> uu = ys[s];
                    ar[u] = (double)uu.x;
                    ai[u] = (double)uu.y;
                    if constexpr (MODE == kTcRowsPot) {
                        constexpr int W = 2 * NN - 1;
                        const int i = r % NN, j = r / NN;
                        vr[u] = (h.t1a[g] + t1p) +
                                h.v12[(i - ip + NN - 1) + W * ((j - jp + NN - 1) + W * (k - kp + NN - 1))];
                        const TC2<R> xe = xs[s];
                        xr[u] = (double)xe.x;
                        xi[u] = (double)xe.y;
                    } else {
                        const TC2<R> o = yv[cc * (int64_t)M + g];
                        orr[u] = (double)o.x;
                        oi[u] = (double)o.y;
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < EU; ++u) {
                const int g = gs[u];
                if (g >= M) continue;
                if constexpr (MODE == kTcRowsPot) {
                    // V(p,q) (hammod.F90:576-578) times SCALE; the factor
                    // 1/SCALE^2 below leaves V/SCALE (initmod.F90:224).
                    const double pr = vr[u] * h.sre + a.shs.x, pi = vr[u] * h.sim + a.shs.y;
                    ar[u] += pr * xr[u] - pi * xi[u];
                    ai[u] += pr * xi[u] + pi * xr[u];
                }
                const double yr = s2r * ar[u] - s2i * ai[u];
                const double yi = s2r * ai[u] + s2i * ar[u];
                TC2<R> o;
                if constexpr (MODE == kTcRowsPot) {
                    o.x = (R)yr;
                    o.y = (R)yi;
                    yv[cc + (int64_t)M * g] = o;
                } else {
                    o.x = (R)(orr[u] + yr);
                    o.y = (R)(oi[u] + yi);
                    yv[cc * (int64_t)M + g] = o;
                }
            }
        }
        if constexpr (!C::DB) {  // single buffer: load the next cube after everyone is done with this one
            __syncthreads();
            const int64_t nc = cube + gridDim.x;
            if (nc < ncubes) load_cube<NN, R, MODE>(a, nc, buf0);
            cp_commit_tc();
        } else {
            cur ^= 1;
        }
    }
    cp_wait_all_tc();
}

int tc_sm_count()
{
    static int cnt[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    if (!cnt[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        cnt[dev] = v > 0 ? v : 148;
    }
    return cnt[dev];
}

// ---------------------------------------------------------------------------
// Register-tile form (NN = 13, 15).  A warp owns the output tile
// i in [8a, 8a+8), j in [8b, 8b+8) for every k, with FP64 accumulators in
// registers for all NN slabs and both components, so the three axis
// contractions sum in registers and the result leaves the SM once:
//   axes i and j of slab k:  C_k += T X_k + X_k T      (DMMA: T as A, X_k as
//                            B; then X_k as A, T as B -- the same C layout)
//   axis k:                  C_k += sum_l T(k,l) X_l  (FP64 FMA on the
//                            lane's own two (i, j) positions)
// The real and imaginary parts are separate real GEMMs (T is real).

template <int NN>
struct Tc2Cfg {
    static constexpr int M = NN * NN * NN;
    static constexpr int P2 = NN * NN;
    static constexpr int TI = (NN + 7) / 8;  // tiles per axis
    static constexpr int WARPS = TI * TI;
    static constexpr int THREADS = 32 * WARPS;
    static constexpr int KS = (NN + 3) / 4;  // k-steps of 4 over the contracted index
};

template <int NN, class R, int MODE>
__global__ void __launch_bounds__(Tc2Cfg<NN>::THREADS, 3)
    tc2_kernel(const __grid_constant__ HamDev h, const __grid_constant__ TcArgs<R> a, int64_t ncubes)
{
    using C = Tc2Cfg<NN>;
    constexpr int M = C::M, P2 = C::P2, KS = C::KS, TI = C::TI;
    extern __shared__ __align__(16) unsigned char tc2_smem[];
    TC2<R> *buf[2] = {reinterpret_cast<TC2<R> *>(tc2_smem), reinterpret_cast<TC2<R> *>(tc2_smem) + M};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ta_ = warp % TI, tb_ = warp / TI;
    const int q4 = lane & 3, r8 = lane >> 2;
    // output positions of this lane: i = 8a + lane/4, j = 8b + 2(lane%4) + {0,1}
    const int oi = 8 * ta_ + r8, oj0 = 8 * tb_ + 2 * q4;
    // T fragments: TA[ks] = T(i = 8a + lane/4, i' = 4ks + lane%4) (A operand);
    // TB[ks] = T(j' = 4ks + lane%4, j = 8b + lane/4) (B operand)
    double TA[KS], TB[KS];
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
        const int kk = 4 * ks + q4;
        const int ri = 8 * ta_ + r8, cj = 8 * tb_ + r8;
        TA[ks] = (ri < NN && kk < NN) ? h.t[ri > kk ? ri - kk : kk - ri] : 0.0;
        TB[ks] = (cj < NN && kk < NN) ? h.t[cj > kk ? cj - kk : kk - cj] : 0.0;
    }
    // B loads of T X_k: X(i' = 4ks + lane%4, j = 8b + lane/4); A loads of X_k T:
    // X(i = 8a + lane/4, j' = 4ks + lane%4); own positions (oi, oj0 + {0,1})
    const int bj = 8 * tb_ + r8, ai_ = 8 * ta_ + r8;
    const bool own0 = oi < NN && oj0 < NN, own1 = oi < NN && oj0 + 1 < NN;
    int64_t cube = blockIdx.x;
    int cur = 0;
    if (cube < ncubes) load_cube_flat<NN, R, MODE>(a, cube, buf[0], C::THREADS);
    cp_commit_tc();
    for (; cube < ncubes; cube += gridDim.x) {
        const TC2<R> *xs = buf[cur];
        cp_wait_all_tc();
        __syncthreads();
        {  // prefetch the next cube
            const int64_t nc = cube + gridDim.x;
            if (nc < ncubes) load_cube_flat<NN, R, MODE>(a, nc, buf[cur ^ 1], C::THREADS);
            cp_commit_tc();
        }
        const R *xr = reinterpret_cast<const R *>(xs);
        double acc[NN][2][2];  // [k][component][position]
#pragma unroll
        for (int k = 0; k < NN; ++k)
#pragma unroll
            for (int c = 0; c < 2; ++c) acc[k][c][0] = acc[k][c][1] = 0.0;
        // axes i and j: k-step by k-step over all slabs, so that the 2*NN
        // accumulator chains of a step are independent (DMMA latency hidden)
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
            const int kk = 4 * ks + q4;
            const bool okb = kk < NN && bj < NN, oka = ai_ < NN && kk < NN;
#pragma unroll
            for (int l = 0; l < NN; ++l)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const double xb = okb ? (double)xr[2 * (kk + NN * bj + P2 * l) + c] : 0.0;
                    dmma(acc[l][c][0], acc[l][c][1], TA[ks], xb);
                }
#pragma unroll
            for (int l = 0; l < NN; ++l)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const double xa = oka ? (double)xr[2 * (ai_ + NN * kk + P2 * l) + c] : 0.0;
                    dmma(acc[l][c][0], acc[l][c][1], xa, TB[ks]);
                }
        }
        // axis k on the lane's own positions
#pragma unroll
        for (int l = 0; l < NN; ++l) {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const double p0 = own0 ? (double)xr[2 * (oi + NN * oj0 + P2 * l) + c] : 0.0;
                const double p1 = own1 ? (double)xr[2 * (oi + NN * (oj0 + 1) + P2 * l) + c] : 0.0;
#pragma unroll
                for (int k = 0; k < NN; ++k) {
                    const double t = h.t[k > l ? k - l : l - k];
                    acc[k][c][0] = fma(t, p0, acc[k][c][0]);
                    acc[k][c][1] = fma(t, p1, acc[k][c][1]);
                }
            }
        }
        // epilogue: potential (pass A), 1/SCALE^2, store; lane positions only
        const int64_t vec = cube / M, cc = cube - vec * M;
        TC2<R> *yv = a.y + vec * a.vstride;
        const double s2r = h.s2re, s2i = h.s2im;
        int ip = 0, jp = 0, kp = 0;
        double t1p = 0.0;
        if constexpr (MODE == kTcRowsPot) {
            ip = (int)(cc % NN);
            jp = (int)((cc / NN) % NN);
            kp = (int)(cc / P2);
            t1p = h.t1a[cc];
        }
#pragma unroll
        for (int pos = 0; pos < 2; ++pos) {
            const bool own = pos ? own1 : own0;
            if (!own) continue;
            const int oj = oj0 + pos;
#pragma unroll
            for (int k = 0; k < NN; ++k) {
                const int g = oi + NN * oj + P2 * k;
                double ar = acc[k][0][pos], ai = acc[k][1][pos];
                if constexpr (MODE == kTcRowsPot) {
                    // V(p,q) (hammod.F90:576-578) times SCALE; the factor
                    // 1/SCALE^2 below leaves V/SCALE (initmod.F90:224).
                    constexpr int W = 2 * NN - 1;
                    const double vr =
                        (h.t1a[g] + t1p) + h.v12[(oi - ip + NN - 1) + W * ((oj - jp + NN - 1) + W * (k - kp + NN - 1))];
                    const double pr = vr * h.sre + a.shs.x, pi = vr * h.sim + a.shs.y;
                    const TC2<R> xe = xs[g];
                    const double xre = (double)xe.x, xim = (double)xe.y;
                    ar += pr * xre - pi * xim;
                    ai += pr * xim + pi * xre;
                }
                const double yr = s2r * ar - s2i * ai;
                const double yi = s2r * ai + s2i * ar;
                TC2<R> o;
                if constexpr (MODE == kTcRowsPot) {
                    o.x = (R)yr;
                    o.y = (R)yi;
                    yv[cc + (int64_t)M * g] = o;
                } else {
                    TC2<R> &dst = yv[cc * (int64_t)M + g];
                    const TC2<R> old = dst;
                    o.x = (R)((double)old.x + yr);
                    o.y = (R)((double)old.y + yi);
                    dst = o;
                }
            }
        }
        cur ^= 1;
    }
    cp_wait_all_tc();
}

template <int NN, class R, int MODE>
cudaError_t tc2_launch(const HamDev &h, const TcArgs<R> &a, int64_t ncubes, cudaStream_t st)
{
    using C = Tc2Cfg<NN>;
    const size_t smem = 2 * (size_t)C::M * sizeof(TC2<R>);
    static int per_sm[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!per_sm[dev]) {
        cudaError_t e = cudaFuncSetAttribute(tc2_kernel<NN, R, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        int per = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, tc2_kernel<NN, R, MODE>, C::THREADS, smem);
        if (e != cudaSuccess) return e;
        per_sm[dev] = std::max(1, per);
    }
    const int64_t grid = std::min<int64_t>(ncubes, (int64_t)tc_sm_count() * per_sm[dev]);
    tc2_kernel<NN, R, MODE><<<(unsigned)grid, C::THREADS, smem, st>>>(h, a, ncubes);
    count_launch();
    return cudaGetLastError();
}


template <int NN, class R, int MODE>
cudaError_t tc_launch(const HamDev &h, const TcArgs<R> &a, int64_t ncubes, cudaStream_t st)
{
    using C = TcCfg<NN, R>;
    static int per_sm[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!per_sm[dev]) {
        cudaError_t e = cudaFuncSetAttribute(tc_kernel<NN, R, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)C::SMEM);
        if (e != cudaSuccess) return e;
        int per = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, tc_kernel<NN, R, MODE>, C::THREADS, C::SMEM);
        if (e != cudaSuccess) return e;
        per_sm[dev] = std::max(1, per);
    }
    const int64_t grid = std::min<int64_t>(ncubes, (int64_t)tc_sm_count() * per_sm[dev]);
    tc_kernel<NN, R, MODE><<<(unsigned)grid, C::THREADS, C::SMEM, st>>>(h, a, ncubes);
    count_launch();
    return cudaGetLastError();
}

template <class R, int MODE>
cudaError_t tc_dispatch(const HamDev &h, const TcArgs<R> &a, int64_t ncubes, cudaStream_t st)
{
    switch (h.nn) {
    case 9: return tc_launch<9, R, MODE>(h, a, ncubes, st);
    case 11: return tc_launch<11, R, MODE>(h, a, ncubes, st);
    case 13: return tc2_launch<13, R, MODE>(h, a, ncubes, st);
    case 15: return tc2_launch<15, R, MODE>(h, a, ncubes, st);
    case 17: return tc_launch<17, R, MODE>(h, a, ncubes, st);
    case 19: return tc_launch<19, R, MODE>(h, a, ncubes, st);
    default: return cudaErrorInvalidValue;
    }
}

template <class R>
cudaError_t tc_pass(const HamDev &h, const TC2<R> *x, TC2<R> *y, int nvec, int64_t vstride, int pass, cudaStream_t st,
                    double2 shift)
{
    if (h.nelec != 2 || nvec <= 0) return cudaErrorInvalidValue;
    TcArgs<R> a{x, y, vstride, make_double2(0.0, 0.0)};
    const double s2r = h.sre * h.sre - h.sim * h.sim, s2i = 2.0 * h.sre * h.sim;  // SCALE^2
    a.shs = make_double2(shift.x * s2r - shift.y * s2i, shift.x * s2i + shift.y * s2r);
    const int64_t ncubes = h.m * (int64_t)nvec;
    if (ncubes > 0x7fffffffLL) return cudaErrorInvalidValue;
    return pass == 0 ? tc_dispatch<R, kTcRowsPot>(h, a, ncubes, st) : tc_dispatch<R, kTcColsAcc>(h, a, ncubes, st);
}

}  // namespace

bool hammult_tc_supported(int nn) { return nn == 9 || nn == 11 || nn == 13 || nn == 15 || nn == 17 || nn == 19; }

cudaError_t hammult_tc_pass_launch(const HamDev &h, const double2 *x, double2 *y, int nvec, int64_t vstride, int pass,
                                   cudaStream_t st, double2 shift)
{
    return tc_pass<double>(h, x, y, nvec, vstride, pass, st, shift);
}

cudaError_t hammult_tc_pass_launch(const HamDev &h, const float2 *x, float2 *y, int nvec, int64_t vstride, int pass,
                                   cudaStream_t st, double2 shift)
{
    return tc_pass<float>(h, x, y, nvec, vstride, pass, st, shift);
}

}  // namespace de
