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
                const double pr = vr * h.vsre, pi = vr * h.vsim;
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
                const double pr = vr * h.vsre, pi = vr * h.vsim;
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
    return cudaGetLastError();
}

template <int MODE>
cudaError_t dispatch(const HamDev &h, const CubeArgs &a, int64_t ncubes, cudaStream_t st)
{
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

cudaError_t hammult_launch(const HamDev &h, const double2 *x, double2 *y, int nvec, int64_t vstride,
                           cudaStream_t st)
{
    if (h.nelec != 2 || nvec <= 0) return cudaErrorInvalidValue;
    CubeArgs a{x, y, vstride, nullptr};
    const int64_t ncubes = h.m * (int64_t)nvec;
    if (ncubes > 0x7fffffffLL) return cudaErrorInvalidValue;
    cudaError_t e = dispatch<kRowsPot>(h, a, ncubes, st);
    if (e != cudaSuccess) return e;
    return dispatch<kColsAcc>(h, a, ncubes, st);
}

cudaError_t hammult1_launch(const HamDev &h, const double *vfull, const double2 *x, double2 *y,
                            int nvec, int64_t vstride, cudaStream_t st)
{
    if (h.nelec != 1 || nvec <= 0) return cudaErrorInvalidValue;
    CubeArgs a{x, y, vstride, vfull};
    return dispatch<kOneElec>(h, a, nvec, st);
}

}  // namespace de
