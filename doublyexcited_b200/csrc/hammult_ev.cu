// hammult_ev.cu -- the two-electron matvec on even/odd-split contractions.
//
// Reference: HAMMULT hammod.F90:19-67 -> KEMULT2 :138-187 -> KEMULTS
// :264-286, plus Y = Y + V*X (:58-59) with V from POTENTIAL2 :502-582.
//
// Same two passes as the streaming kernels of hammult.cu (pass A: the three
// electron-2 axes of the row cubes X(p, :) plus the potential, writes Y;
// pass B: the three electron-1 axes of the column cubes X(:, q), Y += ...),
// with three changes that aim each pass at the HBM bound instead of latency:
//
// * Even/odd split.  The sinc-DVR kinetic matrix T(a,b) = t(|a-b|) is
//   symmetric Toeplitz, so it commutes with the reflection a -> 2N - a of
//   a line of NN = 2N+1 points.  With u_b = v(N+b) + v(N-b), w_b = v(N+b) -
//   v(N-b) (u_0 = v(N)) a line transform is two small products,
//       E(a) = sum_b ce(a,b) u_b  (a = 0..N),   O(a) = sum_b co(a,b) w_b
//       (a = 1..N),   out(N +- a) = E(a) +- O(a),   out(N) = E(0),
//   ce(a,0) = t(a), ce(a,b) = (t(|a-b|) + t(a+b))/2, co(a,b) = (t(|a-b|) -
//   t(a+b))/2: (N+1)^2 + N^2 multiply-adds per line instead of NN^2.
// * Slab pairs.  The slowest cube axis k streams through shared memory in
//   the order k = N, then the pairs (N-b, N+b).  A pair's even and odd
//   combinations u = x(N+b) + x(N-b), w = x(N+b) - x(N-b) feed all three
//   axes: the k axis through the same ce/co products (each owner thread
//   keeps the accumulators e(a), o(a) of its k-line, y(N +- a) = e(a) +-
//   o(a)), and the i and j axes because a line transform of u (of w) is the
//   sum (difference) of the two slabs' line transforms, which is what e(b)
//   (o(b)) receives.
// * Adjacent row cubes.  Pass A loads PB row cubes X(p0..p0+PB-1, :) at
//   once with adjacent p in adjacent lanes, so each request of its strided
//   gather carries PB elements instead of one.  Copies are cp.async into two
//   ring slots of GP slab steps each, at compile-time offsets from a
//   per-unit base; pass B streams pass A's partial Y through the same ring
//   and folds it into its accumulators (times SCALE^2, undone by the final
//   1/SCALE^2), so its read-modify-write never waits on a load.  Pass A
//   keeps A*TINV(r_q) in shared memory.
//
// Per stage: [barrier] issue the next stage's copies; line transforms of
// the stage's u and w planes along i and j (the "line tasks", outputs to
// shared memory) and the owners' k-axis products and potential term;
// [barrier] the owners add the line outputs.  After a unit's last stage each
// owner writes its k-line.
//
// Work per vector-matvec is still counted as 24 NN^7 + 8 NN^6 flops (the
// algorithmic numerator); these kernels execute about 0.55 of the kinetic
// part.
#include "de_kernels.h"

#include <algorithm>
#include <atomic>

namespace de {
namespace {

template <class R>
struct EvT;
template <>
struct EvT<double> {
    using C = double2;
};
template <>
struct EvT<float> {
    using C = float2;
};
template <class R>
using CX = typename EvT<R>::C;

template <class R>
__device__ __forceinline__ CX<R> mkc(R a, R b)
{
    CX<R> v;
    v.x = a;
    v.y = b;
    return v;
}

// Even/odd coefficients ce(a,b), co(a,b) of the handle's grid.  Every call
// site sits in fully unrolled loops, so the index is a compile-time constant
// and the value a constant-bank operand (the tables are kernel parameters).
template <class R, int NN>
__device__ __forceinline__ R cev(const HamDev &h, int a, int b)
{
    if constexpr (sizeof(R) == 8) return h.ev_ce[a * (NN / 2 + 1) + b];
    else return h.ev_cef[a * (NN / 2 + 1) + b];
}
template <class R, int NN>
__device__ __forceinline__ R cov(const HamDev &h, int a, int b)
{
    if constexpr (sizeof(R) == 8) return h.ev_co[a * (NN / 2 + 1) + b];
    else return h.ev_cof[a * (NN / 2 + 1) + b];
}
template <class R>
__device__ __forceinline__ const R *t1a_of(const HamDev &h)
{
    if constexpr (sizeof(R) == 8) return h.t1a;
    else return h.t1af;
}
template <class R>
__device__ __forceinline__ const R *v12_of(const HamDev &h)
{
    if constexpr (sizeof(R) == 8) return h.v12;
    else return h.v12f;
}

template <class R>
struct EvArgs {
    const CX<R> *x;
    CX<R> *y;
    int64_t vstride;
    double2 shs;  // diagonal shift times SCALE^2 (added to V * SCALE)
    int64_t nunits;
    int upv;  // units per vector
};

// Launch shape of one (precision, grid, pass): PB adjacent cubes per unit
// (pass A: p0..p0+PB-1; pass B: 1), GP slab steps per pipeline stage (two
// ring slots: the next stage's copies run under the current stage's work),
// LCH chunks per line transform (2 halves the line accumulators), MINB
// resident CTAs per SM asked of the compiler, LT line threads: 0 = every
// thread owns a k-line or takes a line task (threads added until no thread
// has two tasks in a stage); -1 = owners only, looping over the line tasks;
// LT > 0 = LT extra threads take all line tasks while the owners keep only
// their accumulators.
template <class R, int NN, int MODE>
struct EvShape;

#define EV_SHAPE(RT, NNV, MODEV, PBV, GPV, LCHV, MINB, LTV) \
    template <>                                              \
    struct EvShape<RT, NNV, MODEV> {                         \
        static constexpr int PB = PBV, GP = GPV;             \
        static constexpr int LCH = LCHV, MINBLK = MINB;      \
        static constexpr int LT = LTV;                       \
    };
// FP32 (complex64, the mixed form's inner solve)
EV_SHAPE(float, 9, 0, 4, 2, 1, 1, 0)
EV_SHAPE(float, 9, 1, 1, 5, 1, 3, 0)
EV_SHAPE(float, 11, 0, 4, 2, 1, 1, 0)
EV_SHAPE(float, 11, 1, 1, 3, 1, 3, 0)
EV_SHAPE(float, 13, 0, 4, 2, 1, 1, 0)
EV_SHAPE(float, 13, 1, 1, 4, 1, 2, 0)
EV_SHAPE(float, 15, 0, 2, 4, 1, 1, 0)
EV_SHAPE(float, 15, 1, 1, 4, 1, 2, 0)
EV_SHAPE(float, 17, 0, 2, 3, 1, 1, 0)
EV_SHAPE(float, 17, 1, 1, 3, 1, 1, 0)
// FP64 (complex128); larger grids run on the streaming kernels (hammult.cu)
EV_SHAPE(double, 9, 0, 2, 2, 1, 1, 0)
EV_SHAPE(double, 9, 1, 1, 5, 1, 2, 0)
EV_SHAPE(double, 11, 0, 2, 2, 1, 1, 0)
EV_SHAPE(double, 11, 1, 1, 3, 1, 2, 0)
EV_SHAPE(double, 13, 0, 1, 4, 1, 1, 0)
EV_SHAPE(double, 13, 1, 1, 4, 1, 1, 0)
#undef EV_SHAPE

template <class R, int NN, int MODE>
struct EvCfg {
    using S = EvShape<R, NN, MODE>;
    static constexpr int N = NN / 2, STEPS = N + 1;
    static constexpr int P2 = NN * NN, M = NN * NN * NN;
    static constexpr int PB = S::PB, GP = S::GP, LCH = S::LCH;
    static constexpr int UNIT = PB * P2;               // elements per slab plane
    static constexpr int TO = (UNIT + 31) / 32 * 32;   // owner threads (one k-line each)
    static constexpr int LT = S::LT;                   // dedicated line threads (0: owners take line tasks)
    // line tasks of a full stage: steps x (i, j) x (u, w) x chunks x lines
    static constexpr int TASKS = GP * 2 * 2 * LCH * PB * NN;
    // threads: LT > 0: owners + LT line threads; else enough that every
    // thread takes at most one line task per stage (the slowest thread of a
    // stage sets its time)
    // (LT < 0: owners only, looping over the line tasks)
    static constexpr int T = LT > 0 ? TO + LT : (LT == 0 && TASKS > UNIT ? (TASKS + 31) / 32 * 32 : TO);
    static constexpr int NST = (STEPS + GP - 1) / GP;  // stages per unit
    // planes per step: x+, x-, then pass A: V12(q+ - p), V12(q- - p) (in the
    // real part) and pass B: pass A's partial y+, y-
    static constexpr int XPL = 4;
    static constexpr int SLOT = GP * XPL;              // planes per ring slot
    static constexpr int DPL = GP * 4;                 // line-output planes [GP][u,w][i,j]
    static constexpr int T1A = MODE == 0 ? M : 0;      // A*TINV(r_q) copy (pass A)
    static constexpr size_t SMEM = (size_t)(2 * SLOT + DPL) * UNIT * sizeof(CX<R>) + (size_t)T1A * sizeof(R);
    static_assert(SMEM <= 227 * 1024, "launch shape needs more shared memory than a CTA may have");
    static constexpr int LINES = PB * NN;              // lines per (step, dir, u/w, chunk)
    static constexpr int CHW = (N + 1 + LCH - 1) / LCH;  // outputs a per chunk
    // element offset of slab k from a thread's base (pass A: rows M apart)
    static constexpr int64_t KS = MODE == 0 ? (int64_t)M * P2 : P2;
    // line strides in a plane: i-lines, j-lines
    static constexpr int SI = MODE == 0 ? PB : 1;
    static constexpr int SJ = MODE == 0 ? NN * PB : NN;
};

__device__ __forceinline__ void cpa16(void *s, const void *g)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa8(void *s, const void *g)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <class R>
__device__ __forceinline__ void cpa(CX<R> *s, const CX<R> *g)
{
    if constexpr (sizeof(R) == 8) cpa16(s, g);
    else cpa8(s, g);
}
// one real (into the real part of a complex slot)
template <class R>
__device__ __forceinline__ void cpa_real(CX<R> *s, const R *g)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
    if constexpr (sizeof(R) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(g) : "memory");
}

// Owner index o -> (p_sub, ij).  Pass A keeps adjacent p in adjacent lanes
// (coalesced strided gathers), pass B adjacent ij (contiguous cubes).
template <int NN, int MODE, int PB>
__device__ __forceinline__ void owner_coords(int o, int &psub, int &ij)
{
    if constexpr (MODE == 0) {
        psub = o % PB;
        ij = o / PB;
    } else {
        ij = o % (NN * NN);
        psub = o / (NN * NN);
    }
}

// A thread's view of one unit: element (ij, k) of its cube at xb + k*KS.
template <class R>
struct UnitView {
    const CX<R> *xb;
    CX<R> *yb;
    const R *v12b;  // pass A: V12 entry of (ij, k = 0) relative to p; + k*W*W
    R t1p;          // pass A: A*TINV(r_p)
    bool valid;
};

template <class R, int NN, int MODE>
__device__ __forceinline__ UnitView<R> unit_view(const HamDev &h, const EvArgs<R> &a, int64_t u, int psub, int ij,
                                                 bool owner)
{
    using C = EvCfg<R, NN, MODE>;
    UnitView<R> v;
    const int64_t vec = u / a.upv;
    const int r = (int)(u - vec * a.upv);
    const int c = (MODE == 0 ? r * C::PB : r) + psub;
    v.valid = owner && (MODE != 0 || c < C::M);
    const int cc = v.valid ? c : 0;
    if constexpr (MODE == 0) {
        v.xb = a.x + vec * a.vstride + cc + (int64_t)C::M * ij;
        v.yb = a.y + vec * a.vstride + cc + (int64_t)C::M * ij;
        const int ip = cc % NN, jp = (cc / NN) % NN, kp = cc / C::P2;
        const int oi = ij % NN, oj = ij / NN;
        constexpr int W = 2 * NN - 1;  // edge of the V12 table
        v.v12b = v12_of<R>(h) + (oi - ip + NN - 1) + W * ((oj - jp + NN - 1) + W * (NN - 1 - kp));
        v.t1p = v.valid ? __ldg(t1a_of<R>(h) + cc) : R(0);
    } else {
        v.xb = a.x + vec * a.vstride + (int64_t)cc * C::M + ij;
        v.yb = a.y + vec * a.vstride + (int64_t)cc * C::M + ij;
        v.v12b = nullptr;
        v.t1p = R(0);
    }
    return v;
}

// Copies of compile-time stage ST of a unit into a ring slot.
template <class R, int NN, int MODE, int ST>
__device__ __forceinline__ void issue_stage(const UnitView<R> &v, CX<R> *slot)
{
    using C = EvCfg<R, NN, MODE>;
    constexpr int B0 = ST * C::GP;
    constexpr int GN = (B0 + C::GP <= C::STEPS) ? C::GP : C::STEPS - B0;
    if (!v.valid) return;
    const int o = threadIdx.x;
#pragma unroll
    for (int g = 0; g < GN; ++g) {
        const int b = B0 + g;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            if (s == 1 && b == 0) continue;
            const int k = s == 0 ? C::N + b : C::N - b;
            cpa<R>(slot + (g * C::XPL + s) * C::UNIT + o, v.xb + k * C::KS);
            if constexpr (MODE == 1) cpa<R>(slot + (g * C::XPL + 2 + s) * C::UNIT + o, v.yb + k * C::KS);
            else cpa_real<R>(slot + (g * C::XPL + 2 + s) * C::UNIT + o, v.v12b + (2 * NN - 1) * (2 * NN - 1) * k);
        }
    }
}

// One line-transform chunk: outputs out(N +- a), a in [A0, A1), of the
// line val(l) = xp[l*S] + sgn * xm[l*S] (xp alone when single).
template <class R, int NN, int S, int A0, int A1>
__device__ __forceinline__ void line_chunk(const HamDev &h, const CX<R> *__restrict__ xp,
                                           const CX<R> *__restrict__ xm, R sgn, bool single,
                                           CX<R> *__restrict__ out)
{
    constexpr int N = NN / 2;
    constexpr int NA = A1 - A0;
    R er[NA], ei[NA], orr[NA], oi[NA];
#pragma unroll
    for (int q = 0; q < NA; ++q) er[q] = ei[q] = orr[q] = oi[q] = R(0);
#pragma unroll
    for (int b = 0; b <= N; ++b) {
        // complex128 lines: keep each step's loads next to their use, so
        // the compiler does not hoist all NN line values into registers
        if constexpr (sizeof(R) == 8) asm volatile("" ::: "memory");
        CX<R> vp = xp[(N + b) * S], vm = xp[(N - b) * S];
        if (!single) {
            const CX<R> mp = xm[(N + b) * S], mm = xm[(N - b) * S];
            vp.x = fma(sgn, mp.x, vp.x);
            vp.y = fma(sgn, mp.y, vp.y);
            vm.x = fma(sgn, mm.x, vm.x);
            vm.y = fma(sgn, mm.y, vm.y);
        }
        if (b == 0) {
#pragma unroll
            for (int q = 0; q < NA; ++q) {
                const R c = cev<R, NN>(h, A0 + q, 0);
                er[q] = fma(c, vp.x, er[q]);
                ei[q] = fma(c, vp.y, ei[q]);
            }
        } else {
            const R uer = vp.x + vm.x, uei = vp.y + vm.y, uor = vp.x - vm.x, uoi = vp.y - vm.y;
#pragma unroll
            for (int q = 0; q < NA; ++q) {
                const R c = cev<R, NN>(h, A0 + q, b);
                er[q] = fma(c, uer, er[q]);
                ei[q] = fma(c, uei, ei[q]);
                if (A0 + q >= 1) {
                    const R d = cov<R, NN>(h, A0 + q, b);
                    orr[q] = fma(d, uor, orr[q]);
                    oi[q] = fma(d, uoi, oi[q]);
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < NA; ++q) {
        if (A0 + q == 0) {
            out[N * S] = mkc<R>(er[q], ei[q]);
        } else {
            out[(N + A0 + q) * S] = mkc<R>(er[q] + orr[q], ei[q] + oi[q]);
            out[(N - A0 - q) * S] = mkc<R>(er[q] - orr[q], ei[q] - oi[q]);
        }
    }
}

template <class R, int NN, int MODE, int S, int CH>
__device__ __forceinline__ void line_chunk_sel(int ch, const HamDev &h, const CX<R> *xp, const CX<R> *xm, R sgn,
                                               bool single, CX<R> *out)
{
    using C = EvCfg<R, NN, MODE>;
    if constexpr (CH < C::LCH) {
        constexpr int A0 = CH * C::CHW;
        constexpr int A1 = (A0 + C::CHW < C::N + 1) ? A0 + C::CHW : C::N + 1;
        if (ch == CH) {
            line_chunk<R, NN, S, A0, A1>(h, xp, xm, sgn, single, out);
            return;
        }
        line_chunk_sel<R, NN, MODE, S, CH + 1>(ch, h, xp, xm, sgn, single, out);
    }
}

// Line tasks of a stage of GN steps starting at step B0 (ring slot `slot`):
// i- and j-line transforms of the u and w planes into the output planes.
template <class R, int NN, int MODE, int B0, int GN>
__device__ __forceinline__ void line_tasks(const HamDev &h, const CX<R> *slot, CX<R> *dpl)
{
    using C = EvCfg<R, NN, MODE>;
    constexpr int NT = GN * 2 * 2 * C::LCH * C::LINES;
    constexpr int T0 = C::LT > 0 ? C::TO : 0;
    constexpr int TS = C::LT > 0 ? C::LT : C::T;
    if ((int)threadIdx.x < T0) return;
    // task order (dir, chunk, step, u/w, line): the direction and chunk pick
    // different compiled code, so they change only between long runs of
    // tasks and few warps straddle two of them
#pragma unroll 1
    for (int tau = threadIdx.x - T0; tau < NT; tau += TS) {
        const int la = tau % C::LINES;
        int r = tau / C::LINES;
        const int uw = r & 1;
        r >>= 1;
        const int g = r % GN;
        r /= GN;
        const int ch = r % C::LCH;
        const int dir = r / C::LCH;
        const bool single = B0 + g == 0;
        if (single && uw == 1) continue;  // the single middle slab has no odd part
        int a, psub;
        if constexpr (MODE == 0) {
            psub = la % C::PB;
            a = la / C::PB;
        } else {
            a = la % NN;
            psub = la / NN;
        }
        const int base = dir == 0 ? NN * a * C::SI + (MODE == 0 ? psub : C::P2 * psub)
                                  : a * C::SI + (MODE == 0 ? psub : C::P2 * psub);
        const CX<R> *xp = slot + (g * C::XPL) * C::UNIT + base;
        const CX<R> *xm = xp + C::UNIT;
        CX<R> *out = dpl + ((g * 2 + uw) * 2 + dir) * C::UNIT + base;
        const R sgn = uw ? R(-1) : R(1);
        if (dir == 0) line_chunk_sel<R, NN, MODE, C::SI, 0>(ch, h, xp, xm, sgn, single, out);
        else line_chunk_sel<R, NN, MODE, C::SJ, 0>(ch, h, xp, xm, sgn, single, out);
    }
}

// Owner accumulators of one k-line: e(a), a = 0..N and o(a), a = 1..N.
template <class R, int NN>
struct Acc {
    R er[NN / 2 + 1], ei[NN / 2 + 1], orr[NN / 2 + 1], oi[NN / 2 + 1];
};

// Adds d+ (at slab N+B) and d- (at slab N-B) to the k-line: e(B) += (d+ +
// d-)/2, o(B) += (d+ - d-)/2 (B = 0: e(0) += d+).
template <class R, int NN, int B>
__device__ __forceinline__ void acc_pair(Acc<R, NN> &A, R pr, R pi, R mr, R mi)
{
    if constexpr (B == 0) {
        A.er[0] += pr;
        A.ei[0] += pi;
    } else {
        A.er[B] = fma(R(0.5), pr + mr, A.er[B]);
        A.ei[B] = fma(R(0.5), pi + mi, A.ei[B]);
        A.orr[B] = fma(R(0.5), pr - mr, A.orr[B]);
        A.oi[B] = fma(R(0.5), pi - mi, A.oi[B]);
    }
}

// Owner phase 1 of step B: k-axis products, the potential term (pass A) and
// the previous partial result brought to the accumulators' scale (pass B).
template <class R, int NN, int MODE, int B>
__device__ __forceinline__ void owner_k(const HamDev &h, Acc<R, NN> &A, const CX<R> *step, int o, const R *t1as,
                                        int ij, R t1p, R shr, R shi, R sc2r, R sc2i)
{
    using C = EvCfg<R, NN, MODE>;
    constexpr int N = NN / 2;
    const CX<R> xp = step[o];
    CX<R> xm = mkc<R>(R(0), R(0));
    if constexpr (B > 0) xm = step[C::UNIT + o];
    const R ur = xp.x + xm.x, ui = xp.y + xm.y;
#pragma unroll
    for (int a = 0; a <= N; ++a) {
        const R c = cev<R, NN>(h, a, B);
        A.er[a] = fma(c, ur, A.er[a]);
        A.ei[a] = fma(c, ui, A.ei[a]);
    }
    if constexpr (B > 0) {
        const R wr = xp.x - xm.x, wi = xp.y - xm.y;
#pragma unroll
        for (int a = 1; a <= N; ++a) {
            const R d = cov<R, NN>(h, a, B);
            A.orr[a] = fma(d, wr, A.orr[a]);
            A.oi[a] = fma(d, wi, A.oi[a]);
        }
    }
    if constexpr (MODE == 0) {
        // V(p,q) (hammod.F90:576-578) times SCALE (the final 1/SCALE^2 leaves
        // V/SCALE, initmod.F90:224) plus the shift times SCALE^2
        const R vp = (t1as[ij + C::P2 * (N + B)] + t1p) + step[2 * C::UNIT + o].x;
        const R vm = B > 0 ? (t1as[ij + C::P2 * (N - B)] + t1p) + step[3 * C::UNIT + o].x : R(0);
        const R sre = (R)h.sre, sim = (R)h.sim;
        const R pr = fma(vp, sre, shr), pi = fma(vp, sim, shi);
        const R qr = fma(vm, sre, shr), qi = fma(vm, sim, shi);
        acc_pair<R, NN, B>(A, pr * xp.x - pi * xp.y, pr * xp.y + pi * xp.x, qr * xm.x - qi * xm.y,
                           qr * xm.y + qi * xm.x);
    } else {
        // Y(N +- B) of pass A times SCALE^2: the final 1/SCALE^2 restores it
        const CX<R> yp = step[2 * C::UNIT + o];
        CX<R> ym = mkc<R>(R(0), R(0));
        if constexpr (B > 0) ym = step[3 * C::UNIT + o];
        acc_pair<R, NN, B>(A, sc2r * yp.x - sc2i * yp.y, sc2r * yp.y + sc2i * yp.x, sc2r * ym.x - sc2i * ym.y,
                           sc2r * ym.y + sc2i * ym.x);
    }
}

// Owner phase 2: the step's line outputs at the owner's position.
template <class R, int NN, int MODE, int B>
__device__ __forceinline__ void owner_lines(Acc<R, NN> &A, const CX<R> *dstep, int o)
{
    using C = EvCfg<R, NN, MODE>;
    const CX<R> ui = dstep[o], uj = dstep[C::UNIT + o];
    const R f = B == 0 ? R(1) : R(0.5);
    A.er[B] = fma(f, ui.x + uj.x, A.er[B]);
    A.ei[B] = fma(f, ui.y + uj.y, A.ei[B]);
    if constexpr (B > 0) {
        const CX<R> wi = dstep[2 * C::UNIT + o], wj = dstep[3 * C::UNIT + o];
        A.orr[B] = fma(R(0.5), wi.x + wj.x, A.orr[B]);
        A.oi[B] = fma(R(0.5), wi.y + wj.y, A.oi[B]);
    }
}

template <class R, int NN, int MODE, int B0, int G, int GN>
__device__ __forceinline__ void owner_k_all(const HamDev &h, Acc<R, NN> &A, const CX<R> *slot, int o, const R *t1as,
                                            int ij, R t1p, R shr, R shi, R sc2r, R sc2i)
{
    using C = EvCfg<R, NN, MODE>;
    if constexpr (G < GN) {
        owner_k<R, NN, MODE, B0 + G>(h, A, slot + G * C::XPL * C::UNIT, o, t1as, ij, t1p, shr, shi, sc2r, sc2i);
        owner_k_all<R, NN, MODE, B0, G + 1, GN>(h, A, slot, o, t1as, ij, t1p, shr, shi, sc2r, sc2i);
    }
}

template <class R, int NN, int MODE, int B0, int G, int GN>
__device__ __forceinline__ void owner_lines_all(Acc<R, NN> &A, const CX<R> *dpl, int o)
{
    using C = EvCfg<R, NN, MODE>;
    if constexpr (G < GN) {
        owner_lines<R, NN, MODE, B0 + G>(A, dpl + G * 4 * C::UNIT, o);
        owner_lines_all<R, NN, MODE, B0, G + 1, GN>(A, dpl, o);
    }
}

template <class R, int NN, int MODE, int ST>
__device__ __forceinline__ void stages(const HamDev &h, const EvArgs<R> &a, CX<R> *ring, CX<R> *dpl, const R *t1as,
                                       Acc<R, NN> &A, const UnitView<R> &cur, int64_t unext, int64_t sbase, int o,
                                       int psub, int ij, R shr, R shi, R sc2r, R sc2i)
{
    using C = EvCfg<R, NN, MODE>;
    if constexpr (ST < C::NST) {
        constexpr int B0 = ST * C::GP;
        constexpr int GN = (B0 + C::GP <= C::STEPS) ? C::GP : C::STEPS - B0;
        const int par = (int)((sbase + ST) & 1);
        CX<R> *slot = ring + (size_t)par * C::SLOT * C::UNIT;
        CX<R> *other = ring + (size_t)(par ^ 1) * C::SLOT * C::UNIT;
        cpa_wait_all();
        __syncthreads();
        // the next stage's copies run under this stage's work
        if constexpr (ST + 1 < C::NST) {
            issue_stage<R, NN, MODE, ST + 1>(cur, other);
        } else if (unext >= 0) {
            issue_stage<R, NN, MODE, 0>(unit_view<R, NN, MODE>(h, a, unext, psub, ij, o < C::UNIT), other);
        }
        cpa_commit();
        line_tasks<R, NN, MODE, B0, GN>(h, slot, dpl);
        if (o < C::UNIT) owner_k_all<R, NN, MODE, B0, 0, GN>(h, A, slot, o, t1as, ij, cur.t1p, shr, shi, sc2r, sc2i);
        __syncthreads();
        if (o < C::UNIT) owner_lines_all<R, NN, MODE, B0, 0, GN>(A, dpl, o);
        stages<R, NN, MODE, ST + 1>(h, a, ring, dpl, t1as, A, cur, unext, sbase, o, psub, ij, shr, shi, sc2r, sc2i);
    }
}

template <class R, int NN, int MODE>
__global__ void __launch_bounds__(EvCfg<R, NN, MODE>::T, EvShape<R, NN, MODE>::MINBLK)
    ev_kernel(const __grid_constant__ HamDev h, const __grid_constant__ EvArgs<R> a)
{
    using C = EvCfg<R, NN, MODE>;
    constexpr int N = C::N;
    extern __shared__ __align__(16) unsigned char ev_smem[];
    CX<R> *ring = reinterpret_cast<CX<R> *>(ev_smem);
    CX<R> *dpl = ring + (size_t)2 * C::SLOT * C::UNIT;
    R *t1as = reinterpret_cast<R *>(dpl + (size_t)C::DPL * C::UNIT);
    const int64_t nloc = a.nunits > blockIdx.x ? (a.nunits - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const int o = threadIdx.x;
    const bool owner = o < C::UNIT;
    int psub = 0, ij = 0;
    if (owner) owner_coords<NN, MODE, C::PB>(o, psub, ij);
    if constexpr (MODE == 0) {
        const R *t1a = t1a_of<R>(h);
        for (int e = o; e < C::M; e += C::T) t1as[e] = __ldg(t1a + e);
    }
    // Programmatic dependent launch: everything above reads only the
    // operator's tables, written once at set-up.  X and Y are touched after
    // the stream's previous kernel has completed and its writes are visible
    // (a no-op when the launch carries no programmatic attribute).  Every CTA
    // waits, so this grid never completes before its predecessor.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    UnitView<R> cur;
    cur.valid = false;
    if (nloc > 0) {
        cur = unit_view<R, NN, MODE>(h, a, blockIdx.x, psub, ij, owner);
        issue_stage<R, NN, MODE, 0>(cur, ring);
    }
    cpa_commit();
    const R s2r = (R)h.s2re, s2i = (R)h.s2im;
    const R shr = (R)a.shs.x, shi = (R)a.shs.y;
    // SCALE^2 (pass B folds pass A's partial result into its accumulators)
    const R sc2r = (R)(h.sre * h.sre - h.sim * h.sim), sc2i = (R)(2.0 * h.sre * h.sim);
    for (int64_t ul = 0; ul < nloc; ++ul) {
        const int64_t unext = ul + 1 < nloc ? blockIdx.x + (ul + 1) * gridDim.x : -1;
        // the last unit: let the stream's next programmatic launch be
        // scheduled (it waits for this grid's completion before reading)
        if (unext < 0) asm volatile("griddepcontrol.launch_dependents;");
        Acc<R, NN> A;
#pragma unroll
        for (int q = 0; q <= N; ++q) A.er[q] = A.ei[q] = A.orr[q] = A.oi[q] = R(0);
        stages<R, NN, MODE, 0>(h, a, ring, dpl, t1as, A, cur, unext, ul * C::NST, o, psub, ij, shr, shi, sc2r, sc2i);
        if (cur.valid) {
#pragma unroll
            for (int k = 0; k < NN; ++k) {
                const int al = k >= N ? k - N : N - k;
                R zr = A.er[al], zi = A.ei[al];
                if (k > N) {
                    zr += A.orr[al];
                    zi += A.oi[al];
                } else if (k < N) {
                    zr -= A.orr[al];
                    zi -= A.oi[al];
                }
                cur.yb[k * C::KS] = mkc<R>(s2r * zr - s2i * zi, s2r * zi + s2i * zr);
            }
        }
        if (unext >= 0) cur = unit_view<R, NN, MODE>(h, a, unext, psub, ij, owner);
    }
    cpa_wait_all();
}

int ev_sm_count()
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

// Resident CTAs per SM of one instance (queried once per device).
template <class R, int NN, int MODE>
cudaError_t ev_prepare(int &per_sm)
{
    using C = EvCfg<R, NN, MODE>;
    static std::atomic<int> occ[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    int v = occ[dev].load(std::memory_order_relaxed);
    if (!v) {
        cudaError_t e = cudaFuncSetAttribute(ev_kernel<R, NN, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)C::SMEM);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, ev_kernel<R, NN, MODE>, C::T, C::SMEM);
        if (e != cudaSuccess) return e;
        if (v < 1) return cudaErrorInvalidConfiguration;
        occ[dev].store(v, std::memory_order_relaxed);
    }
    per_sm = v;
    return cudaSuccess;
}

template <class R, int NN, int MODE>
cudaError_t ev_launch(const HamDev &h, const CX<R> *x, CX<R> *y, int nvec, int64_t vstride, double2 shs,
                      cudaStream_t st, int ctas)
{
    using C = EvCfg<R, NN, MODE>;
    int per_sm = 1;
    cudaError_t e = ev_prepare<R, NN, MODE>(per_sm);
    if (e != cudaSuccess) return e;
    if (ctas > 0) per_sm = std::min(per_sm, ctas);
    EvArgs<R> a{};
    a.x = x;
    a.y = y;
    a.vstride = vstride;
    a.shs = shs;
    a.upv = MODE == 0 ? (C::M + C::PB - 1) / C::PB : C::M;
    a.nunits = (int64_t)a.upv * nvec;
    const int64_t grid = std::min<int64_t>(a.nunits, (int64_t)ev_sm_count() * per_sm);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(C::T);
    cfg.dynamicSmemBytes = C::SMEM;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = programmatic_launch() ? 1 : 0;
    e = cudaLaunchKernelEx(&cfg, ev_kernel<R, NN, MODE>, h, a);
    count_launch();
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

template <class R>
cudaError_t ev_dispatch(const HamDev &h, const CX<R> *x, CX<R> *y, int nvec, int64_t vstride, int pass,
                        double2 shs, cudaStream_t st, int ctas)
{
#define EV_CASE(NNV)                                                                       \
    case NNV:                                                                              \
        if constexpr (NNV > (sizeof(R) == 8 ? 13 : 17)) return cudaErrorInvalidValue;      \
        else                                                                               \
            return pass == 0 ? ev_launch<R, NNV, 0>(h, x, y, nvec, vstride, shs, st, ctas) \
                             : ev_launch<R, NNV, 1>(h, x, y, nvec, vstride, shs, st, ctas);
    switch (h.nn) {
#ifdef EV_ONLY_NN
        EV_CASE(EV_ONLY_NN)
#else
        EV_CASE(9)
        EV_CASE(11)
        EV_CASE(13)
        EV_CASE(15)
        EV_CASE(17)
#endif
    default: return cudaErrorInvalidValue;
    }
#undef EV_CASE
}

}  // namespace

// Grids where these kernels beat the streaming / cube kernels on B200 (block
// matvec timings at N = 4..10): complex64 NN = 9..17, complex128 NN = 9..13.
bool hammult_ev_supported(int nn, bool fp64) { return nn >= 9 && nn <= (fp64 ? 13 : 17); }

cudaError_t hammult_ev_pass_launch(const HamDev &h, const double2 *x, double2 *y, int nvec, int64_t vstride,
                                   int pass, cudaStream_t st, double2 shs, int ctas)
{
    return ev_dispatch<double>(h, x, y, nvec, vstride, pass, shs, st, ctas);
}

cudaError_t hammult_ev_pass_launch(const HamDev &h, const float2 *x, float2 *y, int nvec, int64_t vstride, int pass,
                                   cudaStream_t st, double2 shs, int ctas)
{
    return ev_dispatch<float>(h, x, y, nvec, vstride, pass, shs, st, ctas);
}

}  // namespace de
