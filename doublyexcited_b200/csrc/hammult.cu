// hammult.cu -- FP64 two-electron Hamiltonian matvec for sm_100a.
//
// Reference: HAMMULT hammod.F90:19-67 -> KEMULT2 :138-187 -> KEMULTS
// :264-286, plus Y = Y + V*X (:58-59) with V from POTENTIAL2 :502-582 scaled
// by 1/SCALE (initmod.F90:224) and T = KEMATRIX/SCALE^2 (initmod.F90:208).
//
// The reference applies T along the three electron-1 axes of every column
// (contiguous NN^3 "cube"), transposes X with MPI_ALLTOALL, applies T along
// the electron-1 axes again and transposes back.  Here the transposes are
// gone: the electron-2 contraction works on "row cubes" X(p, :) (elements
// M apart) in place, so one matvec is two passes over HBM:
//
//   pass A  (row cubes, q axes)    Y  = S2 * (T(x)1(x)1 + ...)_q X + V o X
//   pass B  (column cubes, p axes) Y += S2 * (T(x)1(x)1 + ...)_p X
//
// with S2 = 1/SCALE^2 and T the REAL kinetic matrix (T is real times a
// scalar, so the contraction runs in real*complex arithmetic: 24 NN^7 flops
// per vector instead of the reference's 48 NN^7).  V is never stored: it is
// rebuilt per element from two L2-resident tables (A*TINV(r) and
// TINV(r_q - r_p)/delta^3), three loads instead of a 16-byte stream.
//
// One CTA contracts one cube held in shared memory.  The cube is processed
// in groups of G k-slabs: first the i-lines and j-lines of the group's slabs
// (full reuse of every loaded element: each line thread produces CS outputs
// per load), then the "owner" threads (one per (i,j) column of the cube)
// add the k-axis contraction for the group's outputs and write them.  All
// T indices are compile-time, so T lives in the constant bank.
//
// Every kernel is templated on the arithmetic type R: double (the plain
// FP64 form, complex128 storage) or float (the mixed form's inner solve:
// complex64 storage, FP32 arithmetic with FP32 copies of T and of the
// potential tables).
#include "de_kernels.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>

namespace de {
namespace {

constexpr int kThreads = 384;

template <class R>
struct CT;
template <>
struct CT<double> {
    using C = double2;
};
template <>
struct CT<float> {
    using C = float2;
};
template <class R>
using C2 = typename CT<R>::C;

template <class R>
__device__ __forceinline__ C2<R> mk(R a, R b)
{
    C2<R> v;
    v.x = a;
    v.y = b;
    return v;
}
// T_real(0, d) and the potential tables in the arithmetic type
template <class R>
__device__ __forceinline__ R tval(const HamDev &h, int d)
{
    if constexpr (sizeof(R) == 8) return h.t[d];
    else return h.tf[d];
}
template <class R>
__device__ __forceinline__ const R *t1a_tab(const HamDev &h)
{
    if constexpr (sizeof(R) == 8) return h.t1a;
    else return h.t1af;
}
template <class R>
__device__ __forceinline__ const R *v12_tab(const HamDev &h)
{
    if constexpr (sizeof(R) == 8) return h.v12;
    else return h.v12f;
}

template <int NN>
struct CubeCfg {
    static constexpr int M = NN * NN * NN;
    static constexpr int P2 = NN * NN;
    // k-slabs per group (smem budget: cube + 2 group buffers).
    static constexpr int G = NN == 23 ? 1
                           : NN == 21 ? 5
                           : NN == 19 ? 10
                           : NN == 17 ? 3
                           : NN == 15 ? 5
                           : NN == 13 ? 7
                                      : NN;
    // output chunks per line (parallelism of the line phase).
    static constexpr int CH = (4 * 2 * NN * G >= 3 * kThreads) ? 1 : 2;
    static constexpr int CS = (NN + CH - 1) / CH;
    static constexpr int GMAX = G < NN ? G : NN;
    template <class R>
    static constexpr size_t smem()
    {
        return (size_t)(M + 2 * GMAX * P2) * sizeof(C2<R>);
    }
};

__device__ __forceinline__ constexpr int iabs(int v) { return v < 0 ? -v : v; }

// Outputs [C*CS, min(NN,(C+1)*CS)) of one line: u[ub + o*us] =
// sum_l T(|o-l|) xs[xb + l*xsd].
template <class R, int NN, int C>
__device__ __forceinline__ void line_chunk(const HamDev &h, const C2<R> *__restrict__ xs, int xb, int xsd,
                                           C2<R> *__restrict__ u, int ub, int us)
{
    constexpr int CS = CubeCfg<NN>::CS;
    constexpr int O0 = C * CS;
    constexpr int O1 = (O0 + CS < NN) ? O0 + CS : NN;
    R ar[CS], ai[CS];
#pragma unroll
    for (int o = 0; o < CS; ++o) {
        ar[o] = R(0);
        ai[o] = R(0);
    }
#pragma unroll
    for (int l = 0; l < NN; ++l) {
        const C2<R> v = xs[xb + l * xsd];
#pragma unroll
        for (int o = O0; o < O1; ++o) {
            const R t = tval<R>(h, iabs(o - l));
            ar[o - O0] = fma(t, v.x, ar[o - O0]);
            ai[o - O0] = fma(t, v.y, ai[o - O0]);
        }
    }
#pragma unroll
    for (int o = O0; o < O1; ++o) u[ub + o * us] = mk<R>(ar[o - O0], ai[o - O0]);
}

template <class R, int NN, int C>
__device__ __forceinline__ void line_dispatch(int c, const HamDev &h, const C2<R> *xs, int xb, int xsd, C2<R> *u,
                                              int ub, int us)
{
    if constexpr (C < CubeCfg<NN>::CH) {
        if (c == C) {
            line_chunk<R, NN, C>(h, xs, xb, xsd, u, ub, us);
            return;
        }
        line_dispatch<R, NN, C + 1>(c, h, xs, xb, xsd, u, ub, us);
    }
}

// i-lines and j-lines of slabs k0..k0+gk-1 into ui / uj ([gk][P2]).
template <class R, int NN>
__device__ __forceinline__ void line_phase(const HamDev &h, const C2<R> *xs, C2<R> *ui, C2<R> *uj, int k0, int gk)
{
    constexpr int P2 = CubeCfg<NN>::P2, CH = CubeCfg<NN>::CH;
    const int nlines = NN * gk;
    const int wpt = (nlines + 31) >> 5;
    const int ntasks = 2 * CH * wpt;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int task = warp; task < ntasks; task += nwarps) {
        const int dc = task / wpt;
        const int L = (task - dc * wpt) * 32 + lane;
        if (L >= nlines) continue;
        const int dir = dc / CH, c = dc - dir * CH;
        const int a = L % NN, kk = L / NN;
        const int kof = P2 * (k0 + kk);
        if (dir == 0)  // i-line through (., a, k): outputs ui[kk][o + NN a]
            line_dispatch<R, NN, 0>(c, h, xs, NN * a + kof, 1, ui, kk * P2 + NN * a, 1);
        else  // j-line through (a, ., k): outputs uj[kk][a + NN o]
            line_dispatch<R, NN, 0>(c, h, xs, a + kof, NN, uj, kk * P2 + a, NN);
    }
}

enum Mode { kRowsPot = 0, kColsAcc = 1, kOneElec = 2 };

template <class R>
struct CubeArgs {
    const C2<R> *x;
    C2<R> *y;
    int64_t vstride;
    const double *vfull;  // kOneElec: real V (length M)
    double2 shd;          // diagonal shift added to V (cube kernel)
    double2 shs;          // the same shift times SCALE^2 (streaming kernel)
};

// Owner phase of the group starting at slab K0: k-axis contraction for the
// group's outputs + epilogue.
template <class R, int NN, int K0, int MODE>
__device__ __forceinline__ void owner_group(const HamDev &h, const CubeArgs<R> &a, const C2<R> *xs, const C2<R> *ui,
                                            const C2<R> *uj, int64_t cube, const C2<R> *__restrict__ xv,
                                            C2<R> *__restrict__ yv)
{
    constexpr int P2 = CubeCfg<NN>::P2, M = CubeCfg<NN>::M, G = CubeCfg<NN>::G;
    constexpr int GK = (K0 + G <= NN) ? G : NN - K0;
    const R s2r = (R)h.s2re, s2i = (R)h.s2im, vsr = (R)h.vsre, vsi = (R)h.vsim;
    const R shr = (R)a.shd.x, shi = (R)a.shd.y;
    for (int t = threadIdx.x; t < P2; t += blockDim.x) {
        R ar[GK], ai[GK];
#pragma unroll
        for (int kk = 0; kk < GK; ++kk) {
            const C2<R> p = ui[kk * P2 + t], q = uj[kk * P2 + t];
            ar[kk] = p.x + q.x;
            ai[kk] = p.y + q.y;
        }
#pragma unroll
        for (int l = 0; l < NN; ++l) {
            const C2<R> v = xs[t + P2 * l];
#pragma unroll
            for (int kk = 0; kk < GK; ++kk) {
                const R tt = tval<R>(h, iabs(K0 + kk - l));
                ar[kk] = fma(tt, v.x, ar[kk]);
                ai[kk] = fma(tt, v.y, ai[kk]);
            }
        }
        const int i = t % NN, j = t / NN;
#pragma unroll
        for (int kk = 0; kk < GK; ++kk) {
            const int k = K0 + kk;
            const int e = t + P2 * k;
            // kinetic part times 1/SCALE^2
            R yr = s2r * ar[kk] - s2i * ai[kk];
            R yi = s2r * ai[kk] + s2i * ar[kk];
            if constexpr (MODE == kRowsPot) {
                // cube = row p (electron-1 point), element e = q (electron 2).
                const int c = (int)(cube % M);
                const int ip = c % NN, jp = (c / NN) % NN, kp = c / P2;
                constexpr int W = 2 * NN - 1;
                const R *t1a = t1a_tab<R>(h);
                const R vr = (t1a[e] + t1a[c]) +
                             v12_tab<R>(h)[(i - ip + NN - 1) + W * ((j - jp + NN - 1) + W * (k - kp + NN - 1))];
                const R pr = vr * vsr + shr, pi = vr * vsi + shi;
                const C2<R> xe = xs[e];
                yr += pr * xe.x - pi * xe.y;
                yi += pr * xe.y + pi * xe.x;
                yv[c + (int64_t)M * e] = mk<R>(yr, yi);
            } else if constexpr (MODE == kColsAcc) {
                const int64_t c = cube % M;
                C2<R> &dst = yv[c * M + e];
                const C2<R> old = dst;
                dst = mk<R>(old.x + yr, old.y + yi);
            } else {
                const R vr = (R)a.vfull[e];
                const R pr = vr * vsr + shr, pi = vr * vsi + shi;
                const C2<R> xe = xs[e];
                yr += pr * xe.x - pi * xe.y;
                yi += pr * xe.y + pi * xe.x;
                yv[e] = mk<R>(yr, yi);
            }
        }
    }
}

template <class R, int NN, int K0, int MODE>
__device__ __forceinline__ void groups(const HamDev &h, const CubeArgs<R> &a, const C2<R> *xs, C2<R> *ui, C2<R> *uj,
                                       int64_t cube, const C2<R> *xv, C2<R> *yv)
{
    if constexpr (K0 < NN) {
        constexpr int G = CubeCfg<NN>::G;
        constexpr int GK = (K0 + G <= NN) ? G : NN - K0;
        line_phase<R, NN>(h, xs, ui, uj, K0, GK);
        __syncthreads();
        owner_group<R, NN, K0, MODE>(h, a, xs, ui, uj, cube, xv, yv);
        __syncthreads();
        groups<R, NN, K0 + G, MODE>(h, a, xs, ui, uj, cube, xv, yv);
    }
}

template <class R, int NN, int MODE>
__global__ void __launch_bounds__(kThreads)
    cube_kernel(const __grid_constant__ HamDev h, const __grid_constant__ CubeArgs<R> a)
{
    constexpr int M = CubeCfg<NN>::M, P2 = CubeCfg<NN>::P2, GMAX = CubeCfg<NN>::GMAX;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C2<R> *xs = reinterpret_cast<C2<R> *>(smem_raw);
    C2<R> *ui = xs + M;
    C2<R> *uj = ui + GMAX * P2;
    const int64_t cube = blockIdx.x;
    const int64_t vec = (MODE == kOneElec) ? cube : cube / M;
    const C2<R> *__restrict__ xv = a.x + vec * a.vstride;
    C2<R> *__restrict__ yv = a.y + vec * a.vstride;
    if constexpr (MODE == kRowsPot) {
        const int64_t c = cube % M;
        for (int e = threadIdx.x; e < M; e += blockDim.x) xs[e] = __ldg(xv + c + (int64_t)M * e);
    } else if constexpr (MODE == kColsAcc) {
        const C2<R> *src = xv + (cube % M) * M;
        for (int e = threadIdx.x; e < M; e += blockDim.x) xs[e] = __ldg(src + e);
    } else {
        for (int e = threadIdx.x; e < M; e += blockDim.x) xs[e] = __ldg(xv + e);
    }
    __syncthreads();
    groups<R, NN, 0, MODE>(h, a, xs, ui, uj, cube, xv, yv);
}

template <class R, int NN, int MODE>
cudaError_t launch_cube(const HamDev &h, const CubeArgs<R> &a, int64_t ncubes, cudaStream_t st)
{
    const size_t smem = CubeCfg<NN>::template smem<R>();
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        cudaError_t e = cudaFuncSetAttribute(cube_kernel<R, NN, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    cube_kernel<R, NN, MODE><<<(unsigned)ncubes, kThreads, smem, st>>>(h, a);
    count_launch();
    return cudaGetLastError();
}

// ------------------------------------------------------------------ streaming form
//
// Persistent kernel, one CTA per SM.  Thread t < NN^2 "owns" the k-line
// (i,j) = (t % NN, t / NN) of the current cube and keeps its NN outputs in
// registers.  The cube's k-slabs (NN^2 elements each) stream through shared
// memory in groups of G slabs, double-buffered with cp.async; the copy of the
// next group (which may belong to the CTA's next cube) overlaps the compute of
// the current one.  Per group:
//   * line work: every (dir, slab, line) of the group's i-lines and j-lines
//     is split into two output chunks; a warp handles one chunk of 32 lines,
//     so the chunk - and with it every T index - is a compile-time constant
//     and T comes from the constant bank.  Each loaded element feeds CSZ
//     outputs (re and im: 2*CSZ independent FMA chains);
//   * owner work: each owner adds T(k,l) x(i,j,l) to all NN of its outputs
//     for every slab l of the group (2*NN independent chains), plus the
//     potential term of element (i,j,l) in pass A;
//   * after a barrier the owner adds the group's line outputs to its outputs.
// Two barriers per group of G slabs.

template <int NN, class R = double>
struct SCfg {
    static constexpr int M = NN * NN * NN;
    static constexpr int P2 = NN * NN;
    // slabs per group; complex64 at NN=13 takes larger groups (fewer
    // barriers per cube; shared memory is no limit there)
    static constexpr int G = (NN == 13 && sizeof(R) == 4) ? 5 : NN == 13 ? 3 : NN == 15 ? 4 : NN == 17 ? 4 : 5;
    static constexpr int CSZ = (NN + 1) / 2;                                   // outputs per chunk
    static constexpr int WPC = (2 * NN * G + 31) / 32;                         // warps per chunk
    static constexpr int NT_LINES = 2 * WPC * 32;
    static constexpr int NT_OWN = ((P2 + 31) / 32) * 32;
    static constexpr int NT = NT_LINES > NT_OWN ? NT_LINES : NT_OWN;
    static constexpr int NG = (NN + G - 1) / G;  // groups per cube
    static constexpr int MINB = NT <= 256 ? 2 : 1;
};
// resident CTAs per SM the launch bounds ask for: complex64 storage needs
// fewer registers, so one more CTA (a fourth at NN=13 fits without spills
// but measured no faster), and two of the 320-thread complex64 NN=13 CTAs
template <int NN, class R>
constexpr int smin_blocks()
{
    using C = SCfg<NN, R>;
    if constexpr (sizeof(R) == 4) return C::NT <= 256 ? C::MINB + 1 : NN == 13 ? 2 : C::MINB;
    return C::MINB;
}

// Asynchronous global -> shared copy of one complex element (16 bytes for
// complex128, 8 for complex64).
template <class R>
__device__ __forceinline__ void cp_async_elem(C2<R> *smem, const C2<R> *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(R) == 8)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Issue the copies of slabs [g*G, g*G+gk) of cube `cube` into ring half `half`.
template <class R, int NN, int MODE>
__device__ __forceinline__ void issue_group(const CubeArgs<R> &a, int64_t cube, int g, C2<R> *ring, int half)
{
    using C = SCfg<NN, R>;
    constexpr int P2 = C::P2, M = C::M, G = C::G;
    const int64_t vec = cube / M, c = cube - vec * M;
    const C2<R> *xv = a.x + vec * a.vstride;
    const int l0 = g * G;
    const int gk = (l0 + G <= NN) ? G : NN - l0;
    C2<R> *dst = ring + (size_t)half * G * P2;
    for (int idx = threadIdx.x; idx < gk * P2; idx += blockDim.x) {
        const int64_t e = (int64_t)l0 * P2 + idx;
        const C2<R> *src = (MODE == kRowsPot) ? xv + c + (int64_t)M * e : xv + c * (int64_t)M + e;
        cp_async_elem<R>(dst + idx, src);
    }
}

// One output chunk (outputs [C*CSZ, min(NN,(C+1)*CSZ))) of one line.
template <class R, int NN, int CK>
__device__ __forceinline__ void line_chunk2(const HamDev &h, const C2<R> *xs, int xs_stride, C2<R> *u, int u_stride)
{
    constexpr int CSZ = SCfg<NN, R>::CSZ;
    constexpr int O0 = CK * CSZ;
    constexpr int O1 = (O0 + CSZ < NN) ? O0 + CSZ : NN;
    constexpr int NO = O1 - O0;
    R ar[NO], ai[NO];
#pragma unroll
    for (int o = 0; o < NO; ++o) ar[o] = ai[o] = R(0);
#pragma unroll
    for (int l = 0; l < NN; ++l) {
        const C2<R> v = xs[l * xs_stride];
#pragma unroll
        for (int o = 0; o < NO; ++o) {
            const R tt = tval<R>(h, iabs(O0 + o - l));
            ar[o] = fma(tt, v.x, ar[o]);
            ai[o] = fma(tt, v.y, ai[o]);
        }
    }
#pragma unroll
    for (int o = 0; o < NO; ++o) u[(O0 + o) * u_stride] = mk<R>(ar[o], ai[o]);
}

template <class R, int NN, int GI, int MODE>
__device__ __forceinline__ void stream_groups(const HamDev &h, const CubeArgs<R> &a, int64_t cube, int64_t ncubes,
                                              C2<R> *ring, C2<R> *ub, int &half, R (&ar)[NN], R (&ai)[NN], int ip,
                                              int jp, int kp, R t1p)
{
    using C = SCfg<NN, R>;
    constexpr int P2 = C::P2, G = C::G, NG = C::NG, WPC = C::WPC;
    if constexpr (GI < NG) {
        constexpr int L0 = GI * G;
        constexpr int GK = (L0 + G <= NN) ? G : NN - L0;
        const int t = threadIdx.x;
        {  // prefetch the next group (this cube's, else the next cube's first)
            const int nh = half ^ 1;
            if (GI + 1 < NG) {
                issue_group<R, NN, MODE>(a, cube, GI + 1, ring, nh);
            } else {
                const int64_t nc = cube + gridDim.x;
                if (nc < ncubes) issue_group<R, NN, MODE>(a, nc, 0, ring, nh);
            }
            cp_commit();
        }
        // pass A: this group's potential values, loaded now so that the
        // table latency hides behind the line work
        R vpre[GK];
        if constexpr (MODE == kRowsPot) {
            if (t < P2) {
                constexpr int W = 2 * NN - 1;
                const int oi = t % NN, oj = t / NN;
#pragma unroll
                for (int s = 0; s < GK; ++s) {
                    const int l = L0 + s;
                    vpre[s] = (t1a_tab<R>(h)[t + P2 * l] + t1p) +
                              v12_tab<R>(h)[(oi - ip + NN - 1) + W * ((oj - jp + NN - 1) + W * (l - kp + NN - 1))];
                }
            }
        }
        cp_wait<1>();
        __syncthreads();
        const C2<R> *slabs = ring + (size_t)half * G * P2;
        // line work
        {
            const int warp = t >> 5, lane = t & 31;
            const int ck = warp / WPC;
            const int L = (warp - ck * WPC) * 32 + lane;
            if (ck < 2 && L < 2 * NN * GK) {
                const int dir = L / (NN * GK);
                const int rem = L - dir * NN * GK;
                const int s = rem / NN, la = rem - s * NN;
                const C2<R> *xs = slabs + (size_t)s * P2;
                C2<R> *u = ub + ((size_t)s * 2 + dir) * P2;
                if (dir == 0) {  // i-line through (., la, L0+s): outputs u[o + NN la]
                    if (ck == 0) line_chunk2<R, NN, 0>(h, xs + NN * la, 1, u + NN * la, 1);
                    else line_chunk2<R, NN, 1>(h, xs + NN * la, 1, u + NN * la, 1);
                } else {  // j-line through (la, ., L0+s): outputs u[la + NN o]
                    if (ck == 0) line_chunk2<R, NN, 0>(h, xs + la, NN, u + la, NN);
                    else line_chunk2<R, NN, 1>(h, xs + la, NN, u + la, NN);
                }
            }
        }
        // owner work: k-axis contraction (+ potential in pass A)
        if (t < P2) {
#pragma unroll
            for (int s = 0; s < GK; ++s) {
                const int l = L0 + s;
                const C2<R> v = slabs[(size_t)s * P2 + t];
#pragma unroll
                for (int k = 0; k < NN; ++k) {
                    const R tt = tval<R>(h, iabs(k - l));
                    ar[k] = fma(tt, v.x, ar[k]);
                    ai[k] = fma(tt, v.y, ai[k]);
                }
                if constexpr (MODE == kRowsPot) {
                    // V(p,q) (hammod.F90:576-578) times SCALE: the final factor
                    // 1/SCALE^2 leaves V/SCALE (initmod.F90:224).
                    const R vr = vpre[s];
                    const R pr = vr * (R)h.sre + (R)a.shs.x, pi = vr * (R)h.sim + (R)a.shs.y;
                    ar[l] += pr * v.x - pi * v.y;
                    ai[l] += pr * v.y + pi * v.x;
                }
            }
        }
        __syncthreads();
        if (t < P2) {
#pragma unroll
            for (int s = 0; s < GK; ++s) {
                const C2<R> u0 = ub[((size_t)s * 2) * P2 + t], u1 = ub[((size_t)s * 2 + 1) * P2 + t];
                ar[L0 + s] += u0.x + u1.x;
                ai[L0 + s] += u0.y + u1.y;
            }
        }
        half ^= 1;
        stream_groups<R, NN, GI + 1, MODE>(h, a, cube, ncubes, ring, ub, half, ar, ai, ip, jp, kp, t1p);
    }
}

template <class R, int NN, int MODE>
__global__ void __launch_bounds__(SCfg<NN, R>::NT, (smin_blocks<NN, R>()))
    stream_kernel(const __grid_constant__ HamDev h, const __grid_constant__ CubeArgs<R> a, int64_t ncubes)
{
    using C = SCfg<NN, R>;
    constexpr int P2 = C::P2, M = C::M;
    extern __shared__ __align__(16) unsigned char ssm_raw[];
    C2<R> *ring = reinterpret_cast<C2<R> *>(ssm_raw);  // [2][G][P2]
    C2<R> *ub = ring + (size_t)2 * C::G * P2;          // [G][2][P2]
    const int t = threadIdx.x;
    int64_t cube = blockIdx.x;
    int half = 0;
    if (cube < ncubes) issue_group<R, NN, MODE>(a, cube, 0, ring, 0);
    cp_commit();
    const R s2r = (R)h.s2re, s2i = (R)h.s2im;
    for (; cube < ncubes; cube += gridDim.x) {
        const int64_t vec = cube / M, cc = cube - vec * M;
        R ar[NN], ai[NN];
#pragma unroll
        for (int k = 0; k < NN; ++k) ar[k] = ai[k] = R(0);
        int ip = 0, jp = 0, kp = 0;
        R t1p = R(0);
        if constexpr (MODE == kRowsPot) {
            ip = (int)(cc % NN);
            jp = (int)((cc / NN) % NN);
            kp = (int)(cc / P2);
            t1p = t1a_tab<R>(h)[cc];
        }
        stream_groups<R, NN, 0, MODE>(h, a, cube, ncubes, ring, ub, half, ar, ai, ip, jp, kp, t1p);
        if (t < P2) {
            C2<R> *yv = a.y + vec * a.vstride;
#pragma unroll
            for (int k = 0; k < NN; ++k) {
                const R yr = s2r * ar[k] - s2i * ai[k];
                const R yi = s2r * ai[k] + s2i * ar[k];
                const int64_t e = t + (int64_t)P2 * k;
                if constexpr (MODE == kRowsPot) {
                    yv[cc + (int64_t)M * e] = mk<R>(yr, yi);
                } else {
                    C2<R> &dst = yv[cc * M + e];
                    const C2<R> old = dst;
                    dst = mk<R>(old.x + yr, old.y + yi);
                }
            }
        }
    }
    cp_wait<0>();
}

int sm_count()
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

template <class R, int NN, int MODE>
cudaError_t launch_stream(const HamDev &h, const CubeArgs<R> &a, int64_t ncubes, cudaStream_t st, int ctas)
{
    using C = SCfg<NN, R>;
    const size_t smem = (size_t)4 * C::G * C::P2 * sizeof(C2<R>);
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        cudaError_t e = cudaFuncSetAttribute(stream_kernel<R, NN, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    const int per_sm = ctas > 0 ? std::min(ctas, smin_blocks<NN, R>()) : smin_blocks<NN, R>();
    const int64_t grid = std::min<int64_t>(ncubes, (int64_t)sm_count() * per_sm);
    stream_kernel<R, NN, MODE><<<(unsigned)grid, C::NT, smem, st>>>(h, a, ncubes);
    count_launch();
    return cudaGetLastError();
}

template <class R, int MODE>
cudaError_t dispatch(const HamDev &h, const CubeArgs<R> &a, int64_t ncubes, cudaStream_t st, int ctas = 0)
{
    if constexpr (MODE != kOneElec) {
        switch (h.nn) {
        case 13: return launch_stream<R, 13, MODE>(h, a, ncubes, st, ctas);
        case 15: return launch_stream<R, 15, MODE>(h, a, ncubes, st, ctas);
        case 17: return launch_stream<R, 17, MODE>(h, a, ncubes, st, ctas);
        case 19: return launch_stream<R, 19, MODE>(h, a, ncubes, st, ctas);
        default: break;
        }
    }
    switch (h.nn) {
    case 3: return launch_cube<R, 3, MODE>(h, a, ncubes, st);
    case 5: return launch_cube<R, 5, MODE>(h, a, ncubes, st);
    case 7: return launch_cube<R, 7, MODE>(h, a, ncubes, st);
    case 9: return launch_cube<R, 9, MODE>(h, a, ncubes, st);
    case 11: return launch_cube<R, 11, MODE>(h, a, ncubes, st);
    case 13: return launch_cube<R, 13, MODE>(h, a, ncubes, st);
    case 15: return launch_cube<R, 15, MODE>(h, a, ncubes, st);
    case 17: return launch_cube<R, 17, MODE>(h, a, ncubes, st);
    case 19: return launch_cube<R, 19, MODE>(h, a, ncubes, st);
    case 21: return launch_cube<R, 21, MODE>(h, a, ncubes, st);
    case 23: return launch_cube<R, 23, MODE>(h, a, ncubes, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

void fill_ev_coefficients(HamDev &h)
{
    const int nn = h.nn, n = nn / 2;
    for (int i = 0; i < kEvCoef; ++i) h.ev_ce[i] = h.ev_co[i] = 0.0;
    if (n + 1 > 12) return;
    auto t = [&](int d) { return d < nn ? h.t[d] : 0.0; };
    for (int a = 0; a <= n; ++a)
        for (int b = 0; b <= n; ++b) {
            const int idx = a * (n + 1) + b;
            h.ev_ce[idx] = b == 0 ? t(a) : 0.5 * (t(std::abs(a - b)) + t(a + b));
            h.ev_co[idx] = (a >= 1 && b >= 1) ? 0.5 * (t(std::abs(a - b)) - t(a + b)) : 0.0;
        }
    for (int i = 0; i < kEvCoef; ++i) {
        h.ev_cef[i] = (float)h.ev_ce[i];
        h.ev_cof[i] = (float)h.ev_co[i];
    }
}

template <class R>
static CubeArgs<R> make_args(const HamDev &h, const C2<R> *x, C2<R> *y, int64_t vstride, double2 shift)
{
    CubeArgs<R> a{x, y, vstride, nullptr, shift, make_double2(0.0, 0.0)};
    // shift * SCALE^2 = shift / (1/SCALE^2)
    const double s2r = h.sre * h.sre - h.sim * h.sim, s2i = 2.0 * h.sre * h.sim;
    a.shs = make_double2(shift.x * s2r - shift.y * s2i, shift.x * s2i + shift.y * s2r);
    return a;
}

template <class R>
static cudaError_t pass_go(const HamDev &h, const C2<R> *x, C2<R> *y, int nvec, int64_t vstride, int pass,
                           cudaStream_t st, double2 shift)
{
    if (h.nelec != 2 || nvec <= 0) return cudaErrorInvalidValue;
    if (sizeof(R) == 4 && (!h.t1af || !h.v12f)) return cudaErrorInvalidValue;
    if (pass != 0 && pass != 1) return cudaErrorInvalidValue;
    const int sto = sizeof(R) == 4 ? 1 : 0;
    const int fam = h.fam[sto][pass], ctas = h.ctas[sto][pass];
    if (fam == 1 && hammult_tc_supported(h.nn)) return hammult_tc_pass_launch(h, x, y, nvec, vstride, pass, st, shift);
    const CubeArgs<R> a = make_args<R>(h, x, y, vstride, shift);
    if constexpr (sizeof(R) == 4) {
        if (fam == 3 && hammult_tc32_supported(h.nn))
            return hammult_tc32_pass_launch(h, x, y, nvec, vstride, pass, st, a.shs, ctas);
    }
    // even/odd kernels where they are built (hammult_ev_supported)
    if ((fam == 0 || fam == 1 || fam == 3) && hammult_ev_supported(h.nn, sizeof(R) == 8))
        return hammult_ev_pass_launch(h, x, y, nvec, vstride, pass, st, a.shs, ctas);
    const int64_t ncubes = h.m * (int64_t)nvec;
    if (ncubes > 0x7fffffffLL) return cudaErrorInvalidValue;
    return pass == 0 ? dispatch<R, kRowsPot>(h, a, ncubes, st, ctas) : dispatch<R, kColsAcc>(h, a, ncubes, st, ctas);
}

cudaError_t hammult_launch(const HamDev &h, const double2 *x, double2 *y, int nvec, int64_t vstride,
                           cudaStream_t st, double2 shift)
{
    cudaError_t e = pass_go<double>(h, x, y, nvec, vstride, 0, st, shift);
    if (e != cudaSuccess) return e;
    return pass_go<double>(h, x, y, nvec, vstride, 1, st, shift);
}

cudaError_t hammult_pass_launch(const HamDev &h, const double2 *x, double2 *y, int nvec, int64_t vstride,
                                int pass, cudaStream_t st, double2 shift)
{
    return pass_go<double>(h, x, y, nvec, vstride, pass, st, shift);
}

cudaError_t hammult_pass_launch(const HamDev &h, const float2 *x, float2 *y, int nvec, int64_t vstride, int pass,
                                cudaStream_t st, double2 shift)
{
    return pass_go<float>(h, x, y, nvec, vstride, pass, st, shift);
}

cudaError_t hammult1_launch(const HamDev &h, const double *vfull, const double2 *x, double2 *y,
                            int nvec, int64_t vstride, cudaStream_t st)
{
    if (h.nelec != 1 || nvec <= 0) return cudaErrorInvalidValue;
    CubeArgs<double> a{x, y, vstride, vfull, make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    return dispatch<double, kOneElec>(h, a, nvec, st);
}

}  // namespace de
