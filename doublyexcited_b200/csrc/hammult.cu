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
#include "de_kernels.h"

#include <algorithm>
#include <cstdio>

namespace de {
namespace {

constexpr int kThreads = 384;

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
    static constexpr size_t smem = (size_t)(M + 2 * GMAX * P2) * sizeof(double2);
};

__device__ __forceinline__ constexpr int iabs(int v) { return v < 0 ? -v : v; }

// Outputs [C*CS, min(NN,(C+1)*CS)) of one line: u[ub + o*us] =
// sum_l T(|o-l|) xs[xb + l*xsd].
template <int NN, int C>
__device__ __forceinline__ void line_chunk(const HamDev &h, const double2 *__restrict__ xs, int xb,
                                           int xsd, double2 *__restrict__ u, int ub, int us)
{
    constexpr int CS = CubeCfg<NN>::CS;
    constexpr int O0 = C * CS;
    constexpr int O1 = (O0 + CS < NN) ? O0 + CS : NN;
    double ar[CS], ai[CS];
#pragma unroll
    for (int o = 0; o < CS; ++o) {
        ar[o] = 0.0;
        ai[o] = 0.0;
    }
#pragma unroll
    for (int l = 0; l < NN; ++l) {
        const double2 v = xs[xb + l * xsd];
#pragma unroll
        for (int o = O0; o < O1; ++o) {
            const double t = h.t[iabs(o - l)];
            ar[o - O0] = fma(t, v.x, ar[o - O0]);
            ai[o - O0] = fma(t, v.y, ai[o - O0]);
        }
    }
#pragma unroll
    for (int o = O0; o < O1; ++o) u[ub + o * us] = make_double2(ar[o - O0], ai[o - O0]);
}

template <int NN, int C>
__device__ __forceinline__ void line_dispatch(int c, const HamDev &h, const double2 *xs, int xb,
                                              int xsd, double2 *u, int ub, int us)
{
    if constexpr (C < CubeCfg<NN>::CH) {
        if (c == C) {
            line_chunk<NN, C>(h, xs, xb, xsd, u, ub, us);
            return;
        }
        line_dispatch<NN, C + 1>(c, h, xs, xb, xsd, u, ub, us);
    }
}

// i-lines and j-lines of slabs k0..k0+gk-1 into ui / uj ([gk][P2]).
template <int NN>
__device__ __forceinline__ void line_phase(const HamDev &h, const double2 *xs, double2 *ui,
                                           double2 *uj, int k0, int gk)
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
            line_dispatch<NN, 0>(c, h, xs, NN * a + kof, 1, ui, kk * P2 + NN * a, 1);
        else  // j-line through (a, ., k): outputs uj[kk][a + NN o]
            line_dispatch<NN, 0>(c, h, xs, a + kof, NN, uj, kk * P2 + a, NN);
    }
}

enum Mode { kRowsPot = 0, kColsAcc = 1, kOneElec = 2 };

struct CubeArgs {
    const double2 *x;
    double2 *y;
    int64_t vstride;
    const double *vfull;  // kOneElec: real V (length M)
    double2 shd;          // diagonal shift added to V (cube kernel)
    double2 shs;          // the same shift times SCALE^2 (streaming kernel)
};

// Owner phase of the group starting at slab K0: k-axis contraction for the
// group's outputs + epilogue.
template <int NN, int K0, int MODE>
__device__ __forceinline__ void owner_group(const HamDev &h, const CubeArgs &a, const double2 *xs,
                                            const double2 *ui, const double2 *uj, int64_t cube,
                                            const double2 *__restrict__ xv, double2 *__restrict__ yv)
{
    constexpr int P2 = CubeCfg<NN>::P2, M = CubeCfg<NN>::M, G = CubeCfg<NN>::G;
    constexpr int GK = (K0 + G <= NN) ? G : NN - K0;
    for (int t = threadIdx.x; t < P2; t += blockDim.x) {
        double ar[GK], ai[GK];
#pragma unroll
        for (int kk = 0; kk < GK; ++kk) {
            const double2 p = ui[kk * P2 + t], q = uj[kk * P2 + t];
            ar[kk] = p.x + q.x;
            ai[kk] = p.y + q.y;
        }
#pragma unroll
        for (int l = 0; l < NN; ++l) {
            const double2 v = xs[t + P2 * l];
#pragma unroll
            for (int kk = 0; kk < GK; ++kk) {
                const double tt = h.t[iabs(K0 + kk - l)];
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
            double yr = h.s2re * ar[kk] - h.s2im * ai[kk];
            double yi = h.s2re * ai[kk] + h.s2im * ar[kk];
            if constexpr (MODE == kRowsPot) {
                // cube = row p (electron-1 point), element e = q (electron 2).
                const int c = (int)(cube % M);
                const int ip = c % NN, jp = (c / NN) % NN, kp = c / P2;
                constexpr int W = 2 * NN - 1;
                const double vr = (h.t1a[e] + h.t1a[c]) +
                                  h.v12[(i - ip + NN - 1) + W * ((j - jp + NN - 1) + W * (k - kp + NN - 1))];
                const double pr = vr * h.vsre + a.shd.x, pi = vr * h.vsim + a.shd.y;
                const double2 xe = xs[e];
                yr += pr * xe.x - pi * xe.y;
                yi += pr * xe.y + pi * xe.x;
                yv[c + (int64_t)M * e] = make_double2(yr, yi);
            } else if constexpr (MODE == kColsAcc) {
                const int64_t c = cube % M;
                double2 &dst = yv[c * M + e];
                const double2 old = dst;
                dst = make_double2(old.x + yr, old.y + yi);
            } else {
                const double vr = a.vfull[e];
                const double pr = vr * h.vsre + a.shd.x, pi = vr * h.vsim + a.shd.y;
                const double2 xe = xs[e];
                yr += pr * xe.x - pi * xe.y;
                yi += pr * xe.y + pi * xe.x;
                yv[e] = make_double2(yr, yi);
            }
        }
    }
}

template <int NN, int K0, int MODE>
__device__ __forceinline__ void groups(const HamDev &h, const CubeArgs &a, const double2 *xs,
                                       double2 *ui, double2 *uj, int64_t cube,
                                       const double2 *xv, double2 *yv)
{
    if constexpr (K0 < NN) {
        constexpr int G = CubeCfg<NN>::G;
        constexpr int GK = (K0 + G <= NN) ? G : NN - K0;
        line_phase<NN>(h, xs, ui, uj, K0, GK);
        __syncthreads();
        owner_group<NN, K0, MODE>(h, a, xs, ui, uj, cube, xv, yv);
        __syncthreads();
        groups<NN, K0 + G, MODE>(h, a, xs, ui, uj, cube, xv, yv);
    }
}

template <int NN, int MODE>
__global__ void __launch_bounds__(kThreads)
    cube_kernel(const __grid_constant__ HamDev h, const __grid_constant__ CubeArgs a)
{
    constexpr int M = CubeCfg<NN>::M, P2 = CubeCfg<NN>::P2, GMAX = CubeCfg<NN>::GMAX;
    extern __shared__ double2 smem[];
    double2 *xs = smem;
    double2 *ui = smem + M;
    double2 *uj = ui + GMAX * P2;
    const int64_t cube = blockIdx.x;
    const int64_t vec = (MODE == kOneElec) ? cube : cube / M;
    const double2 *__restrict__ xv = a.x + vec * a.vstride;
    double2 *__restrict__ yv = a.y + vec * a.vstride;
    if constexpr (MODE == kRowsPot) {
        const int64_t c = cube % M;
        for (int e = threadIdx.x; e < M; e += blockDim.x) xs[e] = __ldg(xv + c + (int64_t)M * e);
    } else if constexpr (MODE == kColsAcc) {
        const double2 *src = xv + (cube % M) * M;
        for (int e = threadIdx.x; e < M; e += blockDim.x) xs[e] = __ldg(src + e);
    } else {
        for (int e = threadIdx.x; e < M; e += blockDim.x) xs[e] = __ldg(xv + e);
    }
    __syncthreads();
    groups<NN, 0, MODE>(h, a, xs, ui, uj, cube, xv, yv);
}

template <int NN, int MODE>
cudaError_t launch_cube(const HamDev &h, const CubeArgs &a, int64_t ncubes, cudaStream_t st)
{
    const size_t smem = CubeCfg<NN>::smem;
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        cudaError_t e = cudaFuncSetAttribute(cube_kernel<NN, MODE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    cube_kernel<NN, MODE><<<(unsigned)ncubes, kThreads, smem, st>>>(h, a);
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

template <int NN>
struct SCfg {
    static constexpr int M = NN * NN * NN;
    static constexpr int P2 = NN * NN;
    static constexpr int G = NN == 13 ? 3 : NN == 15 ? 4 : NN == 17 ? 4 : 5;  // slabs per group
    static constexpr int CSZ = (NN + 1) / 2;                                   // outputs per chunk
    static constexpr int WPC = (2 * NN * G + 31) / 32;                         // warps per chunk
    static constexpr int NT_LINES = 2 * WPC * 32;
    static constexpr int NT_OWN = ((P2 + 31) / 32) * 32;
    static constexpr int NT = NT_LINES > NT_OWN ? NT_LINES : NT_OWN;
    static constexpr int NG = (NN + G - 1) / G;  // groups per cube
    static constexpr int MINB = NT <= 256 ? 2 : 1;
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Issue the copies of slabs [g*G, g*G+gk) of cube `cube` into ring half `half`.
template <int NN, int MODE>
__device__ __forceinline__ void issue_group(const CubeArgs &a, int64_t cube, int g, double2 *ring, int half)
{
    using C = SCfg<NN>;
    constexpr int P2 = C::P2, M = C::M, G = C::G;
    const int64_t vec = cube / M, c = cube - vec * M;
    const double2 *xv = a.x + vec * a.vstride;
    const int l0 = g * G;
    const int gk = (l0 + G <= NN) ? G : NN - l0;
    double2 *dst = ring + (size_t)half * G * P2;
    for (int idx = threadIdx.x; idx < gk * P2; idx += blockDim.x) {
        const int64_t e = (int64_t)l0 * P2 + idx;
        const double2 *src = (MODE == kRowsPot) ? xv + c + (int64_t)M * e : xv + c * (int64_t)M + e;
        cp_async16(dst + idx, src);
    }
}

// One output chunk (outputs [C*CSZ, min(NN,(C+1)*CSZ))) of one line.
template <int NN, int CK>
__device__ __forceinline__ void line_chunk2(const HamDev &h, const double2 *xs, int xs_stride,
                                            double2 *u, int u_stride)
{
    constexpr int CSZ = SCfg<NN>::CSZ;
    constexpr int O0 = CK * CSZ;
    constexpr int O1 = (O0 + CSZ < NN) ? O0 + CSZ : NN;
    constexpr int NO = O1 - O0;
    double ar[NO], ai[NO];
#pragma unroll
    for (int o = 0; o < NO; ++o) ar[o] = ai[o] = 0.0;
#pragma unroll
    for (int l = 0; l < NN; ++l) {
        const double2 v = xs[l * xs_stride];
#pragma unroll
        for (int o = 0; o < NO; ++o) {
            const double tt = h.t[iabs(O0 + o - l)];
            ar[o] = fma(tt, v.x, ar[o]);
            ai[o] = fma(tt, v.y, ai[o]);
        }
    }
#pragma unroll
    for (int o = 0; o < NO; ++o) u[(O0 + o) * u_stride] = make_double2(ar[o], ai[o]);
}

template <int NN, int GI, int MODE>
__device__ __forceinline__ void stream_groups(const HamDev &h, const CubeArgs &a, int64_t cube, int64_t ncubes,
                                              double2 *ring, double2 *ub, int &half, double (&ar)[NN],
                                              double (&ai)[NN], int ip, int jp, int kp, double t1p)
{
    using C = SCfg<NN>;
    constexpr int P2 = C::P2, G = C::G, NG = C::NG, WPC = C::WPC;
    if constexpr (GI < NG) {
        constexpr int L0 = GI * G;
        constexpr int GK = (L0 + G <= NN) ? G : NN - L0;
        const int t = threadIdx.x;
        {  // prefetch the next group (this cube's, else the next cube's first)
            const int nh = half ^ 1;
            if (GI + 1 < NG) {
                issue_group<NN, MODE>(a, cube, GI + 1, ring, nh);
            } else {
                const int64_t nc = cube + gridDim.x;
                if (nc < ncubes) issue_group<NN, MODE>(a, nc, 0, ring, nh);
            }
            cp_commit();
        }
        cp_wait<1>();
        __syncthreads();
        const double2 *slabs = ring + (size_t)half * G * P2;
        // line work
        {
            const int warp = t >> 5, lane = t & 31;
            const int ck = warp / WPC;
            const int L = (warp - ck * WPC) * 32 + lane;
            if (ck < 2 && L < 2 * NN * GK) {
                const int dir = L / (NN * GK);
                const int rem = L - dir * NN * GK;
                const int s = rem / NN, la = rem - s * NN;
                const double2 *xs = slabs + (size_t)s * P2;
                double2 *u = ub + ((size_t)s * 2 + dir) * P2;
                if (dir == 0) {  // i-line through (., la, L0+s): outputs u[o + NN la]
                    if (ck == 0) line_chunk2<NN, 0>(h, xs + NN * la, 1, u + NN * la, 1);
                    else line_chunk2<NN, 1>(h, xs + NN * la, 1, u + NN * la, 1);
                } else {  // j-line through (la, ., L0+s): outputs u[la + NN o]
                    if (ck == 0) line_chunk2<NN, 0>(h, xs + la, NN, u + la, NN);
                    else line_chunk2<NN, 1>(h, xs + la, NN, u + la, NN);
                }
            }
        }
        // owner work: k-axis contraction (+ potential in pass A)
        if (t < P2) {
#pragma unroll
            for (int s = 0; s < GK; ++s) {
                constexpr int dummy = 0;
                (void)dummy;
                const int l = L0 + s;
                const double2 v = slabs[(size_t)s * P2 + t];
#pragma unroll
                for (int k = 0; k < NN; ++k) {
                    const double tt = h.t[iabs(k - l)];
                    ar[k] = fma(tt, v.x, ar[k]);
                    ai[k] = fma(tt, v.y, ai[k]);
                }
                if constexpr (MODE == kRowsPot) {
                    // V(p,q) (hammod.F90:576-578) times SCALE: the final factor
                    // 1/SCALE^2 leaves V/SCALE (initmod.F90:224).
                    constexpr int W = 2 * NN - 1;
                    const int oi = t % NN, oj = t / NN;
                    const int e = t + P2 * l;
                    const double vr = (h.t1a[e] + t1p) +
                                      h.v12[(oi - ip + NN - 1) + W * ((oj - jp + NN - 1) + W * (l - kp + NN - 1))];
                    const double pr = vr * h.sre + a.shs.x, pi = vr * h.sim + a.shs.y;
                    ar[l] += pr * v.x - pi * v.y;
                    ai[l] += pr * v.y + pi * v.x;
                }
            }
        }
        __syncthreads();
        if (t < P2) {
#pragma unroll
            for (int s = 0; s < GK; ++s) {
                const double2 u0 = ub[((size_t)s * 2) * P2 + t], u1 = ub[((size_t)s * 2 + 1) * P2 + t];
                ar[L0 + s] += u0.x + u1.x;
                ai[L0 + s] += u0.y + u1.y;
            }
        }
        half ^= 1;
        stream_groups<NN, GI + 1, MODE>(h, a, cube, ncubes, ring, ub, half, ar, ai, ip, jp, kp, t1p);
    }
}

template <int NN, int MODE>
__global__ void __launch_bounds__(SCfg<NN>::NT, SCfg<NN>::MINB)
    stream_kernel(const __grid_constant__ HamDev h, const __grid_constant__ CubeArgs a, int64_t ncubes)
{
    using C = SCfg<NN>;
    constexpr int P2 = C::P2, M = C::M;
    extern __shared__ __align__(16) double2 ssm[];
    double2 *ring = ssm;                         // [2][G][P2]
    double2 *ub = ssm + (size_t)2 * C::G * P2;   // [G][2][P2]
    const int t = threadIdx.x;
    int64_t cube = blockIdx.x;
    int half = 0;
    if (cube < ncubes) issue_group<NN, MODE>(a, cube, 0, ring, 0);
    cp_commit();
    for (; cube < ncubes; cube += gridDim.x) {
        const int64_t vec = cube / M, cc = cube - vec * M;
        double ar[NN], ai[NN];
#pragma unroll
        for (int k = 0; k < NN; ++k) ar[k] = ai[k] = 0.0;
        int ip = 0, jp = 0, kp = 0;
        double t1p = 0.0;
        if constexpr (MODE == kRowsPot) {
            ip = (int)(cc % NN);
            jp = (int)((cc / NN) % NN);
            kp = (int)(cc / P2);
            t1p = h.t1a[cc];
        }
        stream_groups<NN, 0, MODE>(h, a, cube, ncubes, ring, ub, half, ar, ai, ip, jp, kp, t1p);
        if (t < P2) {
            double2 *yv = a.y + vec * a.vstride;
#pragma unroll
            for (int k = 0; k < NN; ++k) {
                const double yr = h.s2re * ar[k] - h.s2im * ai[k];
                const double yi = h.s2re * ai[k] + h.s2im * ar[k];
                const int64_t e = t + (int64_t)P2 * k;
                if constexpr (MODE == kRowsPot) {
                    yv[cc + (int64_t)M * e] = make_double2(yr, yi);
                } else {
                    double2 &dst = yv[cc * M + e];
                    const double2 old = dst;
                    dst = make_double2(old.x + yr, old.y + yi);
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

template <int NN, int MODE>
cudaError_t launch_stream(const HamDev &h, const CubeArgs &a, int64_t ncubes, cudaStream_t st)
{
    using C = SCfg<NN>;
    const size_t smem = (size_t)4 * C::G * C::P2 * sizeof(double2);
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        cudaError_t e = cudaFuncSetAttribute(stream_kernel<NN, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    const int64_t grid = std::min<int64_t>(ncubes, (int64_t)sm_count() * C::MINB);
    stream_kernel<NN, MODE><<<(unsigned)grid, C::NT, smem, st>>>(h, a, ncubes);
    count_launch();
    return cudaGetLastError();
}

template <int MODE>
cudaError_t dispatch(const HamDev &h, const CubeArgs &a, int64_t ncubes, cudaStream_t st)
{
    if constexpr (MODE != kOneElec) {
        switch (h.nn) {
        case 13: return launch_stream<13, MODE>(h, a, ncubes, st);
        case 15: return launch_stream<15, MODE>(h, a, ncubes, st);
        case 17: return launch_stream<17, MODE>(h, a, ncubes, st);
        case 19: return launch_stream<19, MODE>(h, a, ncubes, st);
        default: break;
        }
    }
    switch (h.nn) {
    case 3: return launch_cube<3, MODE>(h, a, ncubes, st);
    case 5: return launch_cube<5, MODE>(h, a, ncubes, st);
    case 7: return launch_cube<7, MODE>(h, a, ncubes, st);
    case 9: return launch_cube<9, MODE>(h, a, ncubes, st);
    case 11: return launch_cube<11, MODE>(h, a, ncubes, st);
    case 13: return launch_cube<13, MODE>(h, a, ncubes, st);
    case 15: return launch_cube<15, MODE>(h, a, ncubes, st);
    case 17: return launch_cube<17, MODE>(h, a, ncubes, st);
    case 19: return launch_cube<19, MODE>(h, a, ncubes, st);
    case 21: return launch_cube<21, MODE>(h, a, ncubes, st);
    case 23: return launch_cube<23, MODE>(h, a, ncubes, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

static CubeArgs make_args(const HamDev &h, const double2 *x, double2 *y, int64_t vstride, double2 shift)
{
    CubeArgs a{x, y, vstride, nullptr, shift, make_double2(0.0, 0.0)};
    // shift * SCALE^2 = shift / (1/SCALE^2)
    const double s2r = h.sre * h.sre - h.sim * h.sim, s2i = 2.0 * h.sre * h.sim;
    a.shs = make_double2(shift.x * s2r - shift.y * s2i, shift.x * s2i + shift.y * s2r);
    return a;
}

cudaError_t hammult_launch(const HamDev &h, const double2 *x, double2 *y, int nvec, int64_t vstride,
                           cudaStream_t st, double2 shift)
{
    if (h.nelec != 2 || nvec <= 0) return cudaErrorInvalidValue;
    const CubeArgs a = make_args(h, x, y, vstride, shift);
    const int64_t ncubes = h.m * (int64_t)nvec;
    if (ncubes > 0x7fffffffLL) return cudaErrorInvalidValue;
    cudaError_t e = dispatch<kRowsPot>(h, a, ncubes, st);
    if (e != cudaSuccess) return e;
    return dispatch<kColsAcc>(h, a, ncubes, st);
}

cudaError_t hammult_pass_launch(const HamDev &h, const double2 *x, double2 *y, int nvec, int64_t vstride,
                                int pass, cudaStream_t st, double2 shift)
{
    if (h.nelec != 2 || nvec <= 0) return cudaErrorInvalidValue;
    const CubeArgs a = make_args(h, x, y, vstride, shift);
    const int64_t ncubes = h.m * (int64_t)nvec;
    if (ncubes > 0x7fffffffLL) return cudaErrorInvalidValue;
    return pass == 0 ? dispatch<kRowsPot>(h, a, ncubes, st) : dispatch<kColsAcc>(h, a, ncubes, st);
}

cudaError_t hammult1_launch(const HamDev &h, const double *vfull, const double2 *x, double2 *y,
                            int nvec, int64_t vstride, cudaStream_t st)
{
    if (h.nelec != 1 || nvec <= 0) return cudaErrorInvalidValue;
    CubeArgs a{x, y, vstride, vfull, make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    return dispatch<kOneElec>(h, a, nvec, st);
}

}  // namespace de
