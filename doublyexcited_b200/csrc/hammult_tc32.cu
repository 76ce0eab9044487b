// hammult_tc32.cu -- the mixed form's FP32 matvec with the kinetic
// contractions on the 5th-generation tensor cores (tcgen05, kind::tf32).
//
// Reference: KEMULTS hammod.F90:264-286 inside KEMULT2 :138-187, and the
// potential term Y = Y + V*X (:58-59).  The two passes are the CUDA-core
// kernels' (hammult.cu, hammult_ev.cu): pass A contracts the electron-2
// axes of row cubes X(p, :) and adds the potential, writing Y; pass B
// contracts the electron-1 axes of column cubes X(:, q) and folds pass A's
// Y in.
//
// A CTA stages a batch of PB adjacent cubes in shared memory (pass A: PB
// adjacent p, so every strided request carries PB consecutive elements).
// Each axis contraction of the batch is one GEMM,
//     D[line][o] = sum_k line[k] T(k, o),
// with the batch's lines along the axis as the M rows (real and imaginary
// parts as separate lines: T is real), the line's NN points as K (padded
// to 16) and T as the K x N operand (N padded to 16).  The rows go through
// the tensor cores 128 at a time (GCH chunks per commit), the accumulators
// live in tensor memory and come back with tcgen05.ld.
//
// FP32 accuracy from TF32 products: both operands are split into a TF32
// head and an FP32 tail, x = xh + xl, and D = Xh Th + Xl Th + Xh Tl (the
// Xl Tl term is ~2^-22 of the product and dropped).
//
// The operands are written to shared memory by the threads in the
// canonical K-major layout without swizzle: 8-row x 16-byte core matrices,
// 128 bytes each, the two core matrices of an 8-wide K step 128 bytes
// apart (leading byte offset) and consecutive 8-row groups 256 bytes
// apart (stride byte offset).  One elected thread issues the MMAs and
// commits them to an mbarrier that every thread waits on (bounded: on
// timeout the kernel records an error and stops).
#include "de_kernels.h"

#include <algorithm>
#include <atomic>
#include <cstdint>

namespace de {
namespace {

__device__ int g_tc32_error;  // set when an mbarrier wait gave up

template <int NN>
struct TcCfg {
    static constexpr int PB = NN <= 9 ? 4 : NN <= 13 ? 2 : 1;  // cubes per batch (two CTAs per SM)
    static constexpr int P2 = NN * NN, M = NN * NN * NN;
    static constexpr int KP = 16, KST = KP / 8;  // K (and N) padded; 8-wide K steps
    static constexpr int LINES = 2 * PB * P2;     // GEMM rows per axis
    static constexpr int CHUNKS = (LINES + 127) / 128;
    static constexpr int GCH = 2;                 // 128-row chunks per commit
    static constexpr int GROUPS = (CHUNKS + GCH - 1) / GCH;
    static constexpr int NT = GCH * 128;          // one GEMM row per thread per group
    static constexpr int STEP_BYTES = 4096;       // one 128 x 8 TF32 operand block
    static constexpr int A_BYTES = GCH * 2 * KST * STEP_BYTES;
    static constexpr int B_OFF = A_BYTES, B_BYTES = 2 * KST * 512;
    static constexpr int X_OFF = B_OFF + B_BYTES, X_BYTES = PB * M * 8;
    static constexpr int Y_OFF = X_OFF + X_BYTES;
    static constexpr int BAR_OFF = Y_OFF + X_BYTES;
    static constexpr int SMEM = BAR_OFF + 16;
    static constexpr int TCOLS = 32;  // GCH x 16 fp32 accumulator columns
    static_assert(NN <= 16, "K and N are padded to 16");
    static_assert(GCH * 16 <= TCOLS, "tensor-memory columns");
    static_assert(SMEM <= 113 * 1024, "shared memory: two CTAs per SM");
    static_assert(BAR_OFF % 8 == 0, "mbarrier alignment");
};

// Element of cube c at (i, j, k) in the staged batch.  Pass A keeps the PB
// cubes interleaved (adjacent p adjacent in memory), pass B cube by cube.
template <int NN, int MODE>
__device__ __forceinline__ int eidx(int c, int i, int j, int k)
{
    using C = TcCfg<NN>;
    if constexpr (MODE == 0) return c + C::PB * (i + NN * (j + NN * k));
    else return i + NN * (j + NN * (k + NN * c));
}

template <int NN, int MODE>
__device__ __forceinline__ int axis_stride(int a)
{
    using C = TcCfg<NN>;
    const int s = a == 0 ? 1 : a == 1 ? NN : NN * NN;
    return MODE == 0 ? C::PB * s : s;
}

// GEMM row -> first element of its line along axis a, and which part.
template <int NN, int MODE>
__device__ __forceinline__ bool row_line(int row, int a, int &base, int &part)
{
    using C = TcCfg<NN>;
    const int L = row >> 1;
    part = row & 1;
    if (L >= C::PB * C::P2) return false;
    int c, u, v;
    if constexpr (MODE == 0) {
        c = L % C::PB;
        const int r2 = L / C::PB;
        u = r2 % NN;
        v = r2 / NN;
    } else {
        u = L % NN;
        v = (L / NN) % NN;
        c = L / C::P2;
    }
    base = a == 0 ? eidx<NN, MODE>(c, 0, u, v) : a == 1 ? eidx<NN, MODE>(c, u, 0, v) : eidx<NN, MODE>(c, u, v, 0);
    return true;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// 8-byte asynchronous copy global -> shared, zero-filled when !ok.
__device__ __forceinline__ void cpa8(void *dst, const void *src, bool ok)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(ok ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cpa_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ float tf32_head(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Shared-memory operand descriptor: K-major, no swizzle, LBO 128 B, SBO 256 B.
__device__ __forceinline__ uint64_t op_desc(uint32_t saddr)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)(128u >> 4) << 16;
    d |= (uint64_t)(256u >> 4) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;
}

// Instruction descriptor: D f32, A and B tf32, both K-major, M = 128, N = 16.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t acc)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(dtmem), "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

// Waits for the mbarrier phase with the given parity; gives up after about
// a second of SM clock (the MMAs it waits for take microseconds).
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity)
{
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > 2000000000LL) return false;
    }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

struct TcArgs {
    const float2 *x;
    float2 *y;
    int64_t vstride;
    double2 shs;  // diagonal shift times SCALE^2 (pass A)
    int64_t nunits;
    int upv;  // batches per vector
};

template <int NN, int MODE>
__global__ void __launch_bounds__(TcCfg<NN>::NT, 2) tc32_kernel(const __grid_constant__ HamDev h, const TcArgs a)
{
    using C = TcCfg<NN>;
    extern __shared__ __align__(1024) unsigned char smem[];
    float2 *xs = reinterpret_cast<float2 *>(smem + C::X_OFF);
    float2 *ys = reinterpret_cast<float2 *>(smem + C::Y_OFF);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + C::BAR_OFF);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + C::BAR_OFF + 8);
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t sbase = smem_u32(smem), bar_s = smem_u32(bar);

    // T^T as the B operand, head and tail: row o (N), column k (K)
    for (int e = tid; e < 2 * C::KST * 16 * 8; e += C::NT) {
        const int kk = e & 7, o = (e >> 3) & 15, ks = (e >> 7) % C::KST, hl = (e >> 7) / C::KST;
        const int k = ks * 8 + kk;
        const double t = (k < NN && o < NN) ? h.t[k > o ? k - o : o - k] : 0.0;
        const float th = tf32_head((float)t);
        const float v = hl == 0 ? th : (float)(t - (double)th);
        const int off = C::B_OFF + (hl * C::KST + ks) * 512 + (o >> 3) * 256 + (kk >> 2) * 128 + (o & 7) * 16 +
                        (kk & 3) * 4;
        *reinterpret_cast<float *>(smem + off) = v;
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_s) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"(C::TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tbase = *tslot;

    const float s2r = (float)h.s2re, s2i = (float)h.s2im;
    const float sre = (float)h.sre, sim = (float)h.sim;
    const float shr = (float)a.shs.x, shi = (float)a.shs.y;
    const float sc2r = (float)(h.sre * h.sre - h.sim * h.sim), sc2i = (float)(2.0 * h.sre * h.sim);
    uint32_t phase = 0, waited = 0;
    bool failed = false;

    for (int64_t u = blockIdx.x; u < a.nunits && !failed; u += gridDim.x) {
        const int64_t vec = u / a.upv;
        const int c0 = (int)(u - vec * a.upv) * C::PB;  // first p (pass A) or q (pass B) of the batch
        const float2 *xv = a.x + vec * a.vstride;
        float2 *yv = a.y + vec * a.vstride;
        // stage the batch: every copy in flight at once
#pragma unroll 4
        for (int e = tid; e < C::PB * C::M; e += C::NT) {
            int c, rest;
            if constexpr (MODE == 0) {
                c = e % C::PB;
                rest = e / C::PB;
            } else {
                c = e / C::M;
                rest = e - c * C::M;
            }
            const bool ok = c0 + c < C::M;
            const int64_t g = MODE == 0 ? (int64_t)(c0 + c) + (int64_t)C::M * rest : (int64_t)C::M * (c0 + c) + rest;
            cpa8(xs + e, xv + (ok ? g : 0), ok);
        }
        cpa_wait_all();
        __syncthreads();
        for (int ax = 0; ax < 3 && !failed; ++ax) {
            const int st = axis_stride<NN, MODE>(ax);
            for (int grp = 0; grp < C::GROUPS; ++grp) {
                const int ch0 = grp * C::GCH, nch = min(C::GCH, C::CHUNKS - ch0);
                // thread tid owns GEMM row r of chunk ch: it writes the row's
                // operands and later reads the row's accumulators back
                const int ch = tid >> 7, r = tid & 127;
                int base = 0, part = 0;
                const bool mine = ch < nch && row_line<NN, MODE>((ch0 + ch) * 128 + r, ax, base, part);
                const float *xl = reinterpret_cast<const float *>(xs + base) + part;
                if (ch < nch) {
                    float hv[C::KP], lv[C::KP];
#pragma unroll
                    for (int q = 0; q < C::KP; ++q) {
                        const float xval = (mine && q < NN) ? xl[2 * q * st] : 0.f;
                        hv[q] = tf32_head(xval);
                        lv[q] = xval - hv[q];
                    }
#pragma unroll
                    for (int ks = 0; ks < C::KST; ++ks) {
                        unsigned char *blk = smem + ((ch * 2) * C::KST + ks) * C::STEP_BYTES + (r >> 3) * 256 + (r & 7) * 16;
                        unsigned char *blkl = blk + C::KST * C::STEP_BYTES;
                        const int q0 = ks * 8;
                        *reinterpret_cast<float4 *>(blk) = make_float4(hv[q0], hv[q0 + 1], hv[q0 + 2], hv[q0 + 3]);
                        *reinterpret_cast<float4 *>(blk + 128) = make_float4(hv[q0 + 4], hv[q0 + 5], hv[q0 + 6], hv[q0 + 7]);
                        *reinterpret_cast<float4 *>(blkl) = make_float4(lv[q0], lv[q0 + 1], lv[q0 + 2], lv[q0 + 3]);
                        *reinterpret_cast<float4 *>(blkl + 128) = make_float4(lv[q0 + 4], lv[q0 + 5], lv[q0 + 6], lv[q0 + 7]);
                    }
                }
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
                __syncthreads();
                if (MODE == 1 && ax == 2 && grp == C::GROUPS - 1) {
                    // the batch is no longer read: pass A's Y comes into its place under the last MMAs
#pragma unroll 4
                    for (int e = tid; e < C::PB * C::M; e += C::NT) {
                        const int c = e / C::M, rest = e - c * C::M;
                        const bool ok = c0 + c < C::M;
                        cpa8(xs + e, yv + (ok ? (int64_t)C::M * (c0 + c) + rest : 0), ok);
                    }
                    asm volatile("cp.async.commit_group;\n" ::: "memory");
                }
                bool ok = true;
                if (tid == 0) {
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    // consecutive MMAs go to different accumulators, so the
                    // dependent chains of the chunks interleave
#pragma unroll
                    for (int ks = 0; ks < C::KST; ++ks)
#pragma unroll
                        for (int sp = 0; sp < 3; ++sp)
                            for (int cc = 0; cc < nch; ++cc) {
                                const uint32_t ah = sbase + ((cc * 2) * C::KST + ks) * C::STEP_BYTES;
                                const uint32_t al = ah + C::KST * C::STEP_BYTES;
                                const uint32_t bh = sbase + C::B_OFF + ks * 512;
                                const uint32_t bl = bh + C::KST * 512;
                                mma_tf32(tbase + cc * 16, op_desc(sp == 1 ? al : ah), op_desc(sp == 2 ? bl : bh),
                                         (ks > 0 || sp > 0) ? 1u : 0u);
                            }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                                     bar_s)
                                 : "memory");
                    // one thread waits; the others sleep in the barrier below
                    ok = bar_wait(bar_s, phase);
                }
                waited = phase;
                phase ^= 1u;
                if (__syncthreads_or(!ok)) {
                    failed = true;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                // accumulators back: warp w reads lanes 32 (w % 4) .. + 31 of chunk w / 4,
                // which is row r of chunk ch for this thread
                if (ch < nch) {
                    float v[16];
                    tmem_ld16(tbase + ((uint32_t)((warp & 3) * 32) << 16) + ch * 16, v);
                    if (mine) {
                        float *yp = reinterpret_cast<float *>(ys + base) + part;
#pragma unroll
                        for (int o = 0; o < NN; ++o) {
                            if (ax == 0) yp[2 * o * st] = v[o];
                            else yp[2 * o * st] += v[o];
                        }
                    }
                }
                asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
                __syncthreads();
            }
        }
        if (failed) break;
        if constexpr (MODE == 1) {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            __syncthreads();
        }
        // epilogue: potential (pass A) or pass A's Y (pass B, staged in xs), then 1/SCALE^2
#pragma unroll 4
        for (int e = tid; e < C::PB * C::M; e += C::NT) {
            int c, rest;
            if constexpr (MODE == 0) {
                c = e % C::PB;
                rest = e / C::PB;
            } else {
                c = e / C::M;
                rest = e - c * C::M;
            }
            if (c0 + c >= C::M) continue;
            const float2 kin = ys[e], xv2 = xs[e];
            float zr, zi;
            int64_t g;
            if constexpr (MODE == 0) {
                const int p = c0 + c, q = rest;
                g = (int64_t)p + (int64_t)C::M * q;
                const int ip = p % NN, jp = (p / NN) % NN, kp = p / C::P2;
                const int iq = q % NN, jq = (q / NN) % NN, kq = q / C::P2;
                constexpr int W = 2 * NN - 1;
                const float v = (__ldg(h.t1af + p) + __ldg(h.t1af + q)) +
                                __ldg(h.v12f + (iq - ip + NN - 1) + W * ((jq - jp + NN - 1) + W * (kq - kp + NN - 1)));
                const float pr = fmaf(v, sre, shr), pi = fmaf(v, sim, shi);
                zr = kin.x + (pr * xv2.x - pi * xv2.y);
                zi = kin.y + (pr * xv2.y + pi * xv2.x);
            } else {
                g = (int64_t)C::M * (c0 + c) + rest;
                const float2 yo = xv2;
                zr = kin.x + (sc2r * yo.x - sc2i * yo.y);
                zi = kin.y + (sc2r * yo.y + sc2i * yo.x);
            }
            yv[g] = make_float2(s2r * zr - s2i * zi, s2r * zi + s2i * zr);
        }
        __syncthreads();
    }
    if (failed && tid == 0) atomicExch(&g_tc32_error, 1);
    if (failed) bar_wait(bar_s, waited);  // let a late commit land before the memory goes
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tbase), "r"(C::TCOLS) : "memory");
    }
}

int tc32_sm_count()
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
cudaError_t tc32_launch(const HamDev &h, const float2 *x, float2 *y, int nvec, int64_t vstride, double2 shs,
                        cudaStream_t st, int ctas)
{
    using C = TcCfg<NN>;
    static std::atomic<int> attr_done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_done[dev].load(std::memory_order_acquire)) {
        cudaError_t e =
            cudaFuncSetAttribute(tc32_kernel<NN, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
        if (e != cudaSuccess) return e;
        attr_done[dev].store(1, std::memory_order_release);
    }
    TcArgs a{};
    a.x = x;
    a.y = y;
    a.vstride = vstride;
    a.shs = shs;
    a.upv = (C::M + C::PB - 1) / C::PB;
    a.nunits = (int64_t)a.upv * nvec;
    const int per_sm = ctas == 1 ? 1 : 2;  // two fit (launch bounds, shared memory)
    const int64_t grid = std::min<int64_t>(a.nunits, per_sm * (int64_t)tc32_sm_count());
    tc32_kernel<NN, MODE><<<(unsigned)grid, C::NT, C::SMEM, st>>>(h, a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace

bool hammult_tc32_supported(int nn) { return nn == 9 || nn == 11 || nn == 13 || nn == 15; }

cudaError_t hammult_tc32_pass_launch(const HamDev &h, const float2 *x, float2 *y, int nvec, int64_t vstride,
                                     int pass, cudaStream_t st, double2 shs, int ctas)
{
    if (!h.t1af || !h.v12f) return cudaErrorInvalidValue;
#define TC32_CASE(NNV)                                                        \
    case NNV:                                                                 \
        return pass == 0 ? tc32_launch<NNV, 0>(h, x, y, nvec, vstride, shs, st, ctas) \
                         : tc32_launch<NNV, 1>(h, x, y, nvec, vstride, shs, st, ctas);
    switch (h.nn) {
        TC32_CASE(9)
        TC32_CASE(11)
        TC32_CASE(13)
        TC32_CASE(15)
    default: return cudaErrorInvalidValue;
    }
#undef TC32_CASE
}

int hammult_tc32_error(cudaStream_t st)
{
    int v = 0, z = 0;
    if (cudaMemcpyFromSymbolAsync(&v, g_tc32_error, sizeof v, 0, cudaMemcpyDeviceToHost, st) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(st) != cudaSuccess) return -1;
    if (v) cudaMemcpyToSymbolAsync(g_tc32_error, &z, sizeof z, 0, cudaMemcpyHostToDevice, st);
    return v;
}

}  // namespace de
