// kinpc.cu -- the kinetic-eigenbasis preconditioner MSOLVECPLX22
// (littlesolver.F90:372-436), the PETSc inner solve's shell preconditioner
// option 2 ("spectral decomposition").
//
// With W the eigenvectors of the real kinetic matrix and lam its eigenvalues
// (KINETIC_EIGS littlesolver.F90:709-740), the 3D operator
//     P = W D^-1 W^T,   D(i,j,k) = (lam_i + lam_j + lam_k) / SCALE^2 - shift,
// is the inverse of (T3 / SCALE^2 - shift) on one electron's cube
// (EIGMULT hammod.F90:764-799 with WT, the division, EIGMULT with W).  For
// two electrons the preconditioner is P on every row cube X(p, :) (electron
// 2, reached in the reference through MPITRANSPOSE) plus P on every column
// cube X(:, q) (electron 1), which is this file's pass 0 (writes Y) and
// pass 1 (adds to Y).
//
// One CTA transforms one cube in shared memory: the three axes by W^T, the
// division by D, the three axes by W, each axis a dense NN-long contraction
// into the other buffer.
#include "de_kernels.h"

#include <algorithm>
#include <atomic>

namespace de {
namespace {

struct KpArgs {
    const double2 *x;
    double2 *y;
    int64_t vstride;
    const double *w;      // W, column-major NN x NN: W(a, i) at a + NN i
    const double2 *dinv;  // 1 / D on the cube, i fastest
    int64_t ncubes;       // cubes of all vectors
};

// dst(..., c, ...) = sum_l op(W)(c, l) src(..., l, ...) along axis AX; op(W)
// = W^T when TRANS (sum_l W(l, c)), else W.
template <int NN, int AX, bool TRANS>
__device__ __forceinline__ void axis_transform(const double2 *__restrict__ src, double2 *__restrict__ dst,
                                               const double *__restrict__ w)
{
    constexpr int M = NN * NN * NN;
    constexpr int S = AX == 0 ? 1 : AX == 1 ? NN : NN * NN;
    for (int e = threadIdx.x; e < M; e += blockDim.x) {
        const int c = (e / S) % NN;
        const int base = e - c * S;
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int l = 0; l < NN; ++l) {
            const double wv = TRANS ? w[l + NN * c] : w[c + NN * l];
            const double2 v = src[base + l * S];
            re = fma(wv, v.x, re);
            im = fma(wv, v.y, im);
        }
        dst[e] = make_double2(re, im);
    }
    __syncthreads();
}

template <int NN, int MODE>
__global__ void __launch_bounds__(256) kinpc_kernel(const __grid_constant__ KpArgs a)
{
    constexpr int M = NN * NN * NN;
    extern __shared__ double2 kp_sm[];
    double2 *A = kp_sm, *B = kp_sm + M;
    double *w = reinterpret_cast<double *>(kp_sm + 2 * M);
    for (int e = threadIdx.x; e < NN * NN; e += blockDim.x) w[e] = a.w[e];
    __syncthreads();
    for (int64_t u = blockIdx.x; u < a.ncubes; u += gridDim.x) {
        const int64_t vec = u / M, c = u - vec * M;  // c: p (pass 0) or q (pass 1)
        const double2 *xv = a.x + vec * a.vstride;
        double2 *yv = a.y + vec * a.vstride;
        for (int e = threadIdx.x; e < M; e += blockDim.x)
            A[e] = MODE == 0 ? xv[c + (int64_t)M * e] : xv[(int64_t)M * c + e];
        __syncthreads();
        axis_transform<NN, 0, true>(A, B, w);
        axis_transform<NN, 1, true>(B, A, w);
        axis_transform<NN, 2, true>(A, B, w);
        for (int e = threadIdx.x; e < M; e += blockDim.x) {
            const double2 v = B[e], d = a.dinv[e];
            B[e] = make_double2(v.x * d.x - v.y * d.y, v.x * d.y + v.y * d.x);
        }
        __syncthreads();
        axis_transform<NN, 0, false>(B, A, w);
        axis_transform<NN, 1, false>(A, B, w);
        axis_transform<NN, 2, false>(B, A, w);
        for (int e = threadIdx.x; e < M; e += blockDim.x) {
            if (MODE == 0) {
                yv[c + (int64_t)M * e] = A[e];
            } else {
                double2 &t = yv[(int64_t)M * c + e];
                t = make_double2(t.x + A[e].x, t.y + A[e].y);
            }
        }
        __syncthreads();
    }
}

int kp_sm_count()
{
    static std::atomic<int> cnt[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    int v = cnt[dev].load(std::memory_order_relaxed);
    if (!v) {
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        if (v <= 0) v = 148;
        cnt[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

template <int NN, int MODE>
cudaError_t kp_launch(const KpArgs &a, cudaStream_t st)
{
    constexpr int M = NN * NN * NN;
    const size_t smem = (size_t)2 * M * sizeof(double2) + (size_t)NN * NN * sizeof(double);
    static_assert((size_t)2 * M * sizeof(double2) + (size_t)NN * NN * sizeof(double) <= 227 * 1024,
                  "two cubes and W in shared memory");
    static std::atomic<int> done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev].load(std::memory_order_acquire)) {
        cudaError_t e = cudaFuncSetAttribute(kinpc_kernel<NN, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        done[dev].store(1, std::memory_order_release);
    }
    int per = 1;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kinpc_kernel<NN, MODE>, 256, smem);
    if (e != cudaSuccess) return e;
    const int64_t grid = std::min<int64_t>(a.ncubes, (int64_t)kp_sm_count() * std::max(1, per));
    kinpc_kernel<NN, MODE><<<(unsigned)grid, 256, smem, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace

bool kinetic_pc_supported(int nn) { return nn >= 3 && nn <= 19 && (nn & 1); }

cudaError_t kinetic_pc_launch(int nn, const double2 *x, double2 *y, int nvec, int64_t vstride, const double *w_dev,
                              const double2 *dinv_dev, int pass, cudaStream_t st)
{
    if (!kinetic_pc_supported(nn) || nvec < 1 || pass < 0 || pass > 1) return cudaErrorInvalidValue;
    KpArgs a{x, y, vstride, w_dev, dinv_dev, (int64_t)nn * nn * nn * nvec};
#define KP_CASE(NNV)                                                     \
    case NNV:                                                            \
        return pass == 0 ? kp_launch<NNV, 0>(a, st) : kp_launch<NNV, 1>(a, st);
    switch (nn) {
        KP_CASE(3)
        KP_CASE(5)
        KP_CASE(7)
        KP_CASE(9)
        KP_CASE(11)
        KP_CASE(13)
        KP_CASE(15)
        KP_CASE(17)
        KP_CASE(19)
    default: return cudaErrorInvalidValue;
    }
#undef KP_CASE
}

}  // namespace de
