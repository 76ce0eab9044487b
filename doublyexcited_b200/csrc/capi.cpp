// capi.cpp -- C-ABI entry points: handle life cycle, HAMMULT / MATBLOCK /
// dot products / expectations.  The eigensolver lives in gplmr.cpp, the
// Input.Inp reader in input.cpp and the eigenvector files in vecio.cpp.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>

#include "de_internal.h"

namespace de {
const char *last_error_str();
}

using namespace de;

extern "C" {

DE_API int64_t de_kernel_launches(void) { return launch_count(); }

DE_API const char *de_version(void) { return "doublyexcited-b200 0.1 (sm_100a, FP64)"; }

DE_API const char *de_last_error(void) { return last_error_str(); }

DE_API const char *de_strerror(int s)
{
    switch (s) {
    case DE_OK: return "ok";
    case DE_E_INVALID: return "invalid argument";
    case DE_E_SIZE: return "size mismatch";
    case DE_E_CUDA: return "CUDA error";
    case DE_E_NOMEM: return "out of memory";
    case DE_E_UNSUPPORTED: return "unsupported option";
    case DE_E_CHOLESKY: return "Cholesky breakdown";
    case DE_E_GEVP: return "projected eigenproblem failed";
    case DE_E_SVD: return "SVD failed";
    case DE_E_ORTHO: return "inner-solve orthonormality check failed";
    case DE_E_NOT_CONVERGED: return "not converged";
    case DE_E_IO: return "I/O error";
    case DE_E_PARSE: return "parse error";
    case DE_E_LAPACK: return "host LAPACK not found";
    case DE_E_NAN: return "non-finite value";
    case DE_E_BUSY: return "admission refused";
    default: return "unknown status";
    }
}

DE_API void de_params_default(de_params *p)
{
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->n = 2;
    p->delta = 0.5;
    p->radius = 7.0;
    p->autodelta = 1;
    p->theta = 0.0;
    p->charge = 2.0;
    p->nelec = 2;
    p->nsmall = 22;
    p->tfactor = 4;
    p->precision = DE_PREC_FP64;
    p->device = 0;
}

}  // extern "C"

// ---------------------------------------------------------------- tables

namespace {

struct TinvKey {
    int nout, nbig, nsmall;
    double delta;
    bool operator<(const TinvKey &o) const
    {
        return std::tie(nout, nbig, nsmall, delta) < std::tie(o.nout, o.nbig, o.nsmall, o.delta);
    }
};

std::mutex g_tinv_mu;
std::map<TinvKey, std::shared_ptr<std::vector<double>>> g_tinv;

std::shared_ptr<std::vector<double>> cached_tinv(int nout, int nbig, int nsmall, double delta)
{
    std::lock_guard<std::mutex> lk(g_tinv_mu);
    TinvKey k{nout, nbig, nsmall, delta};
    auto it = g_tinv.find(k);
    if (it != g_tinv.end()) return it->second;
    auto v = std::make_shared<std::vector<double>>(getinverse(nout, nbig, nsmall, delta));
    g_tinv[k] = v;
    return v;
}

}  // namespace

// Device buffers of a handle come from the stream-ordered allocator
// (cudaMallocAsync / cudaFreeAsync on the handle's stream), so handles that
// run side by side on one GPU never force a device-wide synchronisation
// when they grow or release their workspace.
int de_problem::ensure_stage(int64_t elems)
{
    if (elems <= stage_elems) return DE_OK;
    if (d_x) cudaFreeAsync(d_x, stream);
    if (d_y) cudaFreeAsync(d_y, stream);
    d_x = d_y = nullptr;
    stage_elems = 0;
    DE_CUDA(cudaMallocAsync(&d_x, elems * sizeof(double2), stream));
    DE_CUDA(cudaMallocAsync(&d_y, elems * sizeof(double2), stream));
    stage_elems = elems;
    return DE_OK;
}

// MSOLVECPLX22 littlesolver.F90:372-436: W and lam from the real kinetic
// matrix (KINETIC_EIGS :709-740, here by Jacobi on the host), 1/D for the
// shift, then the two passes (kinpc.cu).
int de_problem::kinetic_pc(const double2 *x, double2 *y, int nvec, cplx shift)
{
    if (p.nelec != 2) return set_error(DE_E_UNSUPPORTED, "the kinetic preconditioner is built for two electrons");
    if (!de::kinetic_pc_supported(nn)) return set_error(DE_E_UNSUPPORTED, "kinetic preconditioner: NN %d not built", nn);
    if (x == y) return set_error(DE_E_INVALID, "kinetic preconditioner: output aliases input");
    std::vector<double> e, v;
    if (!d_kw) {
        de::jacobi_eigen(nn, de::kematrix(nn, delta), e, v);
        DE_CUDA(cudaMallocAsync(&d_kw, (size_t)nn * nn * sizeof(double), stream));
        DE_CUDA(cudaMallocAsync(&d_kdinv, (size_t)m * sizeof(double2), stream));
        DE_CUDA(cudaMemcpyAsync(d_kw, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        DE_CUDA(cudaStreamSynchronize(stream));  // v leaves scope
        kdinv_ok = false;
    }
    if (!kdinv_ok || kdinv_shift != shift) {
        if (e.empty()) de::jacobi_eigen(nn, de::kematrix(nn, delta), e, v);
        const cplx scale(ham.sre, ham.sim), s2 = scale * scale;
        std::vector<double2> d(m);
        for (int k = 0; k < nn; ++k)
            for (int j = 0; j < nn; ++j)
                for (int i = 0; i < nn; ++i) {
                    const cplx di = 1.0 / ((e[i] + e[j] + e[k]) / s2 - shift);
                    d[i + (size_t)nn * (j + (size_t)nn * k)] = make_double2(di.real(), di.imag());
                }
        DE_CUDA(cudaMemcpyAsync(d_kdinv, d.data(), d.size() * sizeof(double2), cudaMemcpyHostToDevice, stream));
        DE_CUDA(cudaStreamSynchronize(stream));  // d leaves scope
        kdinv_shift = shift;
        kdinv_ok = true;
    }
    for (int pass = 0; pass < 2; ++pass) {
        cudaError_t ce = de::kinetic_pc_launch(nn, x, y, nvec, dim, d_kw, d_kdinv, pass, stream);
        if (ce != cudaSuccess) return cuda_error(ce, "kinetic preconditioner");
    }
    return DE_OK;
}

int de_problem::ensure_work(int64_t elems)
{
    if (elems <= work_elems) return DE_OK;
    if (d_work) cudaFreeAsync(d_work, stream);
    d_work = nullptr;
    work_elems = 0;
    DE_CUDA(cudaMallocAsync(&d_work, elems * sizeof(double2), stream));
    DE_CUDA(cudaMemsetAsync(d_work, 0, sizeof(double2), stream));  // reduction ticket
    work_elems = elems;
    return DE_OK;
}

void de_problem::trim()
{
    for (auto it = cache.begin(); it != cache.end();) {
        if (!it->used) {
            cudaFreeAsync(it->p, stream);
            it = cache.erase(it);
        } else {
            ++it;
        }
    }
    if (d_x) cudaFreeAsync(d_x, stream);
    if (d_y) cudaFreeAsync(d_y, stream);
    d_x = d_y = nullptr;
    stage_elems = 0;
}

int64_t de_problem::cached_bytes() const
{
    int64_t b = 0;
    for (auto &c : cache) b += (int64_t)c.bytes;
    return b + 2 * stage_elems * (int64_t)sizeof(double2) + work_elems * (int64_t)sizeof(double2);
}

void *de_problem::cache_get(size_t bytes)
{
    Blk *best = nullptr;
    for (auto &b : cache)
        if (!b.used && b.bytes >= bytes && b.bytes <= 2 * bytes + (1 << 20) && (!best || b.bytes < best->bytes)) best = &b;
    if (best) {
        best->used = true;
        return best->p;
    }
    void *p = nullptr;
    if (cudaMallocAsync(&p, bytes, stream) != cudaSuccess) {
        cudaGetLastError();
        // release idle blocks and retry once
        for (auto it = cache.begin(); it != cache.end();) {
            if (!it->used) {
                cudaFreeAsync(it->p, stream);
                it = cache.erase(it);
            } else {
                ++it;
            }
        }
        if (cudaMallocAsync(&p, bytes, stream) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
    }
    cache.push_back(Blk{p, bytes, true});
    return p;
}

void de_problem::cache_put(void *p)
{
    for (auto &b : cache)
        if (b.p == p) b.used = false;
}

cudaEvent_t de_problem::take_event()
{
    if (!ev_free.empty()) {
        cudaEvent_t e = ev_free.back();
        ev_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

int de_problem::harvest()
{
    for (auto &r : ev_pending) {
        DE_CUDA(cudaEventSynchronize(r.e[2]));
        float a = 0.f, b = 0.f;
        DE_CUDA(cudaEventElapsedTime(&a, r.e[0], r.e[1]));
        DE_CUDA(cudaEventElapsedTime(&b, r.e[1], r.e[2]));
        prof_ms[r.f32][0] += a;
        prof_ms[r.f32][1] += b;
        prof_calls[r.f32] += 1;
        prof_vectors[r.f32] += r.nvec;
        for (auto ev : r.e) ev_free.push_back(ev);
    }
    ev_pending.clear();
    return DE_OK;
}

int de_problem::matblock(const double2 *x, double2 *y, int nvec, double2 shift)
{
    if (p.nelec != 2) {
        cudaError_t e = hammult1_launch(ham, d_t1a, x, y, nvec, dim, stream);
        if (e != cudaSuccess) return cuda_error(e, "hammult1");
        return DE_OK;
    }
    Rec r{{nullptr, nullptr, nullptr}, nvec, 0};
    DE_TRY(prof_begin(r));
    cudaError_t e = hammult_pass_launch(ham, x, y, nvec, dim, 0, stream, shift);
    if (e != cudaSuccess) return cuda_error(e, "hammult pass A");
    DE_TRY(prof_mid(r));
    e = hammult_pass_launch(ham, x, y, nvec, dim, 1, stream);
    if (e != cudaSuccess) return cuda_error(e, "hammult pass B");
    return prof_end(r);
}

int de_problem::prof_begin(Rec &r)
{
    if (!prof) return DE_OK;
    if (prof_seq[r.f32]++ % prof_every != 0) return DE_OK;  // not sampled: r.e stay null
    for (auto &ev : r.e)
        if (!(ev = take_event())) return set_error(DE_E_CUDA, "cudaEventCreate failed");
    DE_CUDA(cudaEventRecord(r.e[0], stream));
    return DE_OK;
}

int de_problem::prof_mid(Rec &r)
{
    if (prof && r.e[1]) DE_CUDA(cudaEventRecord(r.e[1], stream));
    return DE_OK;
}

int de_problem::prof_end(Rec &r)
{
    if (!prof || !r.e[2]) return DE_OK;
    DE_CUDA(cudaEventRecord(r.e[2], stream));
    ev_pending.push_back(r);
    if (ev_pending.size() > 4096) DE_TRY(harvest());
    return DE_OK;
}

int de_problem::matblock32(const float2 *x, float2 *y, int nvec, double2 shift)
{
    if (p.nelec != 2) return set_error(DE_E_INVALID, "the FP32 matvec is built for the two-electron operator");
    Rec r{{nullptr, nullptr, nullptr}, nvec, 1};
    DE_TRY(prof_begin(r));
    cudaError_t e = hammult_pass_launch(ham, x, y, nvec, dim, 0, stream, shift);
    if (e != cudaSuccess) return cuda_error(e, "hammult FP32 pass A");
    DE_TRY(prof_mid(r));
    e = hammult_pass_launch(ham, x, y, nvec, dim, 1, stream);
    if (e != cudaSuccess) return cuda_error(e, "hammult FP32 pass B");
    return prof_end(r);
}

extern "C" {

DE_API int de_problem_create(const de_params *pin, de_problem **out)
{
    if (!pin || !out) return set_error(DE_E_INVALID, "null argument");
    *out = nullptr;
    de_params p = *pin;
    if (p.nelec != 1 && p.nelec != 2) return set_error(DE_E_INVALID, "nelec must be 1 or 2 (got %d)", p.nelec);
    if (p.n < 1) return set_error(DE_E_INVALID, "N must be >= 1 (got %d)", p.n);
    const int nn = 2 * p.n + 1;
    if (nn > 23)
        return set_error(DE_E_UNSUPPORTED, "N=%d: grids above NN=23 are not built in this version", p.n);
    if (p.nsmall < 1 || p.tfactor < 1) return set_error(DE_E_INVALID, "nsmall/tfactor must be positive");
    if (p.precision != DE_PREC_FP64 && p.precision != DE_PREC_MIXED)
        return set_error(DE_E_INVALID, "precision must be DE_PREC_FP64 or DE_PREC_MIXED (got %d)", p.precision);
    double delta = p.autodelta ? p.radius / p.n : p.delta;  // INIT_STRUCTS input.F90:384
    if (!(delta > 0.0)) return set_error(DE_E_INVALID, "grid spacing must be positive");
    const int nbig_alloc = nn;  // PARAMS%NBIG = 2N+1 (initmod.F90:39)
    const int nbig_solve = p.nsmall * p.tfactor;
    if (nbig_solve < nbig_alloc) return set_error(DE_E_INVALID, "nbig lt nout (%d < %d)", nbig_solve, nbig_alloc);

    cudaError_t ce = cudaSetDevice(p.device);
    if (ce != cudaSuccess) return cuda_error(ce, "cudaSetDevice");

    std::unique_ptr<de_problem> h(new de_problem());
    h->p = p;
    h->n = p.n;
    h->nn = nn;
    h->m = (int64_t)nn * nn * nn;
    h->dim = (p.nelec == 2) ? h->m * h->m : h->m;
    h->delta = delta;
    DE_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    h->stream = h->own_stream;

    // T = KEMATRIX / SCALE^2; V scaled by 1/SCALE (initmod.F90:48,208,224)
    const cplx scale(std::cos(p.theta), std::sin(p.theta));
    const cplx s2 = 1.0 / (scale * scale), vs = 1.0 / scale;
    HamDev &hd = h->ham;
    hd.nn = nn;
    hd.nelec = p.nelec;
    hd.m = h->m;
    std::vector<double> t = kematrix(nn, delta);
    for (int d = 0; d < nn; ++d) hd.t[d] = t[d];  // T(d,0) = T(0,d)
    hd.s2re = s2.real();
    hd.s2im = s2.imag();
    hd.vsre = vs.real();
    hd.vsim = vs.imag();
    hd.sre = scale.real();
    hd.sim = scale.imag();
    apply_tuning(hd);  // kernel family and CTAs per SM of each pass (de_set_matvec_kernel overrides)

    auto tinv = cached_tinv(nbig_alloc, nbig_solve, p.nsmall, delta);
    const int nbd = 2 * nbig_alloc + 1;
    double *d_tinv = nullptr;
    DE_CUDA(cudaMallocAsync(&d_tinv, tinv->size() * sizeof(double), h->stream));
    const int64_t w = 2 * nn - 1;
    DE_CUDA(cudaMallocAsync(&h->d_t1a, h->m * sizeof(double), h->stream));
    DE_CUDA(cudaMallocAsync(&h->d_v12, w * w * w * sizeof(double), h->stream));
    DE_CUDA(cudaMemcpyAsync(d_tinv, tinv->data(), tinv->size() * sizeof(double), cudaMemcpyHostToDevice,
                            h->stream));
    ce = build_tables_launch(nn, p.n, p.charge, delta, d_tinv, nbd, h->d_t1a, h->d_v12, h->stream);
    if (ce != cudaSuccess) return cuda_error(ce, "build_tables");
    DE_CUDA(cudaStreamSynchronize(h->stream));
    cudaFreeAsync(d_tinv, h->stream);
    hd.t1a = h->d_t1a;
    hd.v12 = h->d_v12;
    // FP32 copies of T and of the potential tables for the mixed form
    for (int d = 0; d < nn; ++d) hd.tf[d] = (float)t[d];
    fill_ev_coefficients(hd);
    DE_CUDA(cudaMallocAsync(&h->d_t1af, h->m * sizeof(float), h->stream));
    DE_CUDA(cudaMallocAsync(&h->d_v12f, w * w * w * sizeof(float), h->stream));
    ce = to_f32_launch(h->d_t1a, h->d_t1af, h->m, h->stream);
    if (ce == cudaSuccess) ce = to_f32_launch(h->d_v12, h->d_v12f, w * w * w, h->stream);
    if (ce != cudaSuccess) return cuda_error(ce, "FP32 tables");
    DE_CUDA(cudaStreamSynchronize(h->stream));
    hd.t1af = h->d_t1af;
    hd.v12f = h->d_v12f;

    DE_CUDA(cudaMallocAsync(&h->d_small, 64 * 256 * sizeof(double2), h->stream));
    DE_CUDA(cudaMallocHost(&h->h_small, 64 * 256 * sizeof(double2)));
    *out = h.release();
    return DE_OK;
}

DE_API int de_problem_trim(de_problem *h)
{
    if (!h) return set_error(DE_E_INVALID, "null handle");
    std::lock_guard<std::mutex> lk(h->mu);
    cudaSetDevice(h->p.device);
    h->trim();
    return DE_OK;
}

DE_API int de_problem_destroy(de_problem *h)
{
    if (!h) return DE_OK;
    cudaSetDevice(h->p.device);
    if (h->own_stream) cudaStreamSynchronize(h->own_stream);
    // everything the handle allocated goes back through its own stream
    cudaStream_t st = h->own_stream ? h->own_stream : h->stream;
    if (h->stream && h->stream != st) cudaStreamSynchronize(h->stream);
    for (void *p : {(void *)h->d_t1a, (void *)h->d_v12, (void *)h->d_t1af, (void *)h->d_v12f, (void *)h->d_x,
                    (void *)h->d_y, (void *)h->d_small, (void *)h->d_work, (void *)h->d_kw, (void *)h->d_kdinv})
        if (p) cudaFreeAsync(p, st);
    for (auto &b : h->cache) cudaFreeAsync(b.p, st);
    cudaStreamSynchronize(st);
    if (h->h_small) cudaFreeHost(h->h_small);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    for (auto &r : h->ev_pending)
        for (auto ev : r.e) cudaEventDestroy(ev);
    for (auto ev : h->ev_free) cudaEventDestroy(ev);
    delete h;
    return DE_OK;
}

DE_API int de_problem_dims(const de_problem *h, int *nn, int64_t *m, int64_t *dim)
{
    if (!h) return set_error(DE_E_INVALID, "null handle");
    if (nn) *nn = h->nn;
    if (m) *m = h->m;
    if (dim) *dim = h->dim;
    return DE_OK;
}

DE_API int de_set_stream(de_problem *h, void *s)
{
    if (!h) return set_error(DE_E_INVALID, "null handle");
    h->stream = s ? (cudaStream_t)s : cudaStreamLegacy;
    return DE_OK;
}

DE_API int de_set_matvec_kernel(de_problem *h, int kind)
{
    if (!h) return set_error(DE_E_INVALID, "null handle");
    if (kind != DE_MATVEC_FMA && kind != DE_MATVEC_TENSOR && kind != DE_MATVEC_STREAM && kind != DE_MATVEC_TF32)
        return set_error(DE_E_INVALID,
                         "matvec kernel must be DE_MATVEC_FMA, DE_MATVEC_TENSOR, DE_MATVEC_STREAM or DE_MATVEC_TF32 "
                         "(got %d)",
                         kind);
    std::lock_guard<std::mutex> lk(h->mu);
    for (int s = 0; s < 2; ++s)
        for (int p = 0; p < 2; ++p) {
            // DE_MATVEC_TF32 is a complex64 form; complex128 passes keep the FMA kernels
            h->ham.fam[s][p] = (signed char)(kind == DE_MATVEC_TF32 && s == 0 ? DE_MATVEC_FMA : kind);
            h->ham.ctas[s][p] = 0;
        }
    return DE_OK;
}

DE_API int de_set_matvec_launch(de_problem *h, int storage, int pass, int family, int ctas_per_sm)
{
    if (!h) return set_error(DE_E_INVALID, "null handle");
    if (storage < 0 || storage > 1 || pass < 0 || pass > 1)
        return set_error(DE_E_INVALID, "storage must be 0 or 1 and pass 0 or 1 (got %d, %d)", storage, pass);
    if (family < DE_MATVEC_FMA || family > DE_MATVEC_TF32 || ctas_per_sm < 0 || ctas_per_sm > 32)
        return set_error(DE_E_INVALID, "family must be a DE_MATVEC_* kind and ctas_per_sm 0..32 (got %d, %d)", family,
                         ctas_per_sm);
    std::lock_guard<std::mutex> lk(h->mu);
    h->ham.fam[storage][pass] = (signed char)family;
    h->ham.ctas[storage][pass] = (signed char)ctas_per_sm;
    return DE_OK;
}

DE_API int de_get_matvec_launch(de_problem *h, int storage, int pass, int *family, int *ctas_per_sm)
{
    if (!h || !family || !ctas_per_sm) return set_error(DE_E_INVALID, "null argument");
    if (storage < 0 || storage > 1 || pass < 0 || pass > 1)
        return set_error(DE_E_INVALID, "storage must be 0 or 1 and pass 0 or 1 (got %d, %d)", storage, pass);
    std::lock_guard<std::mutex> lk(h->mu);
    *family = h->ham.fam[storage][pass];
    *ctas_per_sm = h->ham.ctas[storage][pass];
    return DE_OK;
}

DE_API int de_tuning_lookup(const char *path, int storage, int nn, int pass, int *family, int *ctas_per_sm)
{
    if (!path || !family || !ctas_per_sm) return set_error(DE_E_INVALID, "null argument");
    int f = 0, c = 0;
    if (!de::tuning_lookup(path, storage, nn, pass, f, c))
        return set_error(DE_E_INVALID, "no tuning entry for storage %d, NN %d, pass %d in %s", storage, nn, pass, path);
    *family = f;
    *ctas_per_sm = c;
    return DE_OK;
}

DE_API int de_kinetic_precond_d(de_problem *h, const de_complex *x_d, de_complex *y_d, int nvec, de_complex shift)
{
    if (!h || !x_d || !y_d) return set_error(DE_E_INVALID, "null argument");
    if (nvec < 1) return set_error(DE_E_INVALID, "nvec must be >= 1 (got %d)", nvec);
    std::lock_guard<std::mutex> lk(h->mu);
    cudaSetDevice(h->p.device);
    return h->kinetic_pc(reinterpret_cast<const double2 *>(x_d), reinterpret_cast<double2 *>(y_d), nvec,
                         cplx(shift.re, shift.im));
}

DE_API int de_set_gmres_pc(de_problem *h, int pcopt)
{
    if (!h) return set_error(DE_E_INVALID, "null handle");
    if (pcopt != 0 && pcopt != 2)
        return set_error(DE_E_INVALID, "GMRES preconditioner must be 0 (none) or 2 (kinetic eigenbasis), got %d",
                         pcopt);
    if (pcopt == 2 && (h->p.nelec != 2 || !de::kinetic_pc_supported(h->nn)))
        return set_error(DE_E_UNSUPPORTED, "the kinetic preconditioner is built for two electrons at NN 3..19");
    std::lock_guard<std::mutex> lk(h->mu);
    h->gm_pcopt = pcopt;
    return DE_OK;
}

DE_API int de_set_profiling(de_problem *h, int on)
{
    if (!h) return set_error(DE_E_INVALID, "null handle");
    if (on < 0) return set_error(DE_E_INVALID, "profiling must be 0 (off) or a sampling interval >= 1 (got %d)", on);
    h->prof = on != 0;
    h->prof_every = on > 1 ? on : 1;
    h->prof_seq[0] = h->prof_seq[1] = 0;
    return DE_OK;
}

DE_API int de_profile_read(de_problem *h, double *pass_a_ms, double *pass_b_ms, int64_t *calls, int64_t *vectors)
{
    if (!h) return set_error(DE_E_INVALID, "null handle");
    cudaSetDevice(h->p.device);
    DE_TRY(h->harvest());
    if (pass_a_ms) *pass_a_ms = h->prof_ms[0][0];
    if (pass_b_ms) *pass_b_ms = h->prof_ms[0][1];
    if (calls) *calls = h->prof_calls[0];
    if (vectors) *vectors = h->prof_vectors[0];
    h->prof_ms[0][0] = h->prof_ms[0][1] = 0.0;
    h->prof_calls[0] = h->prof_vectors[0] = 0;
    return DE_OK;
}

DE_API int de_profile_read32(de_problem *h, double *pass_a_ms, double *pass_b_ms, int64_t *calls, int64_t *vectors)
{
    if (!h) return set_error(DE_E_INVALID, "null handle");
    cudaSetDevice(h->p.device);
    DE_TRY(h->harvest());
    if (pass_a_ms) *pass_a_ms = h->prof_ms[1][0];
    if (pass_b_ms) *pass_b_ms = h->prof_ms[1][1];
    if (calls) *calls = h->prof_calls[1];
    if (vectors) *vectors = h->prof_vectors[1];
    h->prof_ms[1][0] = h->prof_ms[1][1] = 0.0;
    h->prof_calls[1] = h->prof_vectors[1] = 0;
    return DE_OK;
}

DE_API int de_hammult_d(de_problem *h, const de_complex *x, de_complex *y, int64_t mm)
{
    if (!h || !x || !y) return set_error(DE_E_INVALID, "null argument");
    if (mm != h->dim) return set_error(DE_E_SIZE, "SIZE ERRORRRR 66: %lld != %lld", (long long)mm, (long long)h->dim);
    if ((const void *)x == (const void *)y) return set_error(DE_E_INVALID, "x and y must not alias");
    cudaSetDevice(h->p.device);
    return h->matblock((const double2 *)x, (double2 *)y, 1);
}

DE_API int de_matblock_d(de_problem *h, const de_complex *x, de_complex *ax, int64_t m, int64_t mb, int nev)
{
    if (!h || !x || !ax) return set_error(DE_E_INVALID, "null argument");
    if (nev < 1) return set_error(DE_E_INVALID, "nev must be >= 1");
    if (m * mb != h->dim) return set_error(DE_E_SIZE, "SIZE ERRORRRR 66: %lld != %lld", (long long)(m * mb), (long long)h->dim);
    if ((const void *)x == (const void *)ax) return set_error(DE_E_INVALID, "x and ax must not alias");
    cudaSetDevice(h->p.device);
    return h->matblock((const double2 *)x, (double2 *)ax, nev);
}

DE_API int de_matblock32_d(de_problem *h, const void *x, void *ax, int64_t m, int64_t mb, int nev)
{
    if (!h || !x || !ax) return set_error(DE_E_INVALID, "null argument");
    if (nev < 1) return set_error(DE_E_INVALID, "nev must be >= 1");
    if (m * mb != h->dim) return set_error(DE_E_SIZE, "SIZE ERRORRRR 66: %lld != %lld", (long long)(m * mb), (long long)h->dim);
    if (x == (const void *)ax) return set_error(DE_E_INVALID, "x and ax must not alias");
    cudaSetDevice(h->p.device);
    return h->matblock32((const float2 *)x, (float2 *)ax, nev);
}

DE_API int de_matblock(de_problem *h, const de_complex *x, de_complex *ax, int64_t m, int64_t mb, int nev)
{
    if (!h || !x || !ax) return set_error(DE_E_INVALID, "null argument");
    if (nev < 1) return set_error(DE_E_INVALID, "nev must be >= 1");
    if (m * mb != h->dim) return set_error(DE_E_SIZE, "SIZE ERRORRRR 66: %lld != %lld", (long long)(m * mb), (long long)h->dim);
    std::lock_guard<std::mutex> lk(h->mu);
    cudaSetDevice(h->p.device);
    const int64_t n = h->dim * nev;
    DE_TRY(h->ensure_stage(n));
    DE_CUDA(cudaMemcpyAsync(h->d_x, x, n * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    DE_TRY(h->matblock(h->d_x, h->d_y, nev));
    DE_CUDA(cudaMemcpyAsync(ax, h->d_y, n * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    DE_CUDA(cudaStreamSynchronize(h->stream));
    return DE_OK;
}

DE_API int de_hammult(de_problem *h, const de_complex *x, de_complex *y, int64_t mm)
{
    if (!h) return set_error(DE_E_INVALID, "null handle");
    if (mm != h->dim) return set_error(DE_E_SIZE, "SIZE ERRORRRR 66: %lld != %lld", (long long)mm, (long long)h->dim);
    return de_matblock(h, x, y, h->dim, 1, 1);
}

DE_API int de_dots_d(de_problem *h, const de_complex *bras, const de_complex *kets, int64_t size, int nbra,
                     int nket, de_complex *out, int hermitian)
{
    if (!h || !bras || !kets || !out) return set_error(DE_E_INVALID, "null argument");
    if (size < 1 || nbra < 1 || nket < 1) return set_error(DE_E_INVALID, "empty dot");
    cudaSetDevice(h->p.device);
    for (int j0 = 0; j0 < nket; j0 += 128)
        for (int i0 = 0; i0 < nbra; i0 += 64) {
            ColList L{}, R{};
            L.n = std::min(64, nbra - i0);
            R.n = std::min(128, nket - j0);
            for (int i = 0; i < L.n; ++i) L.a[i] = (const double2 *)bras + (int64_t)(i0 + i) * size;
            for (int j = 0; j < R.n; ++j) R.a[j] = (const double2 *)kets + (int64_t)(j0 + j) * size;
            DE_TRY(h->ensure_work(gram_work_elems(L.n, R.n, size)));
            cudaError_t e = gram_launch(L, R, size, hermitian ? 1 : 0, h->d_small, L.n, h->d_work, h->stream);
            if (e != cudaSuccess) return cuda_error(e, "gram");
            DE_CUDA(cudaMemcpyAsync(h->h_small, h->d_small, (size_t)L.n * R.n * sizeof(double2),
                                    cudaMemcpyDeviceToHost, h->stream));
            DE_CUDA(cudaStreamSynchronize(h->stream));
            for (int j = 0; j < R.n; ++j)
                for (int i = 0; i < L.n; ++i) {
                    const double2 v = h->h_small[i + L.n * j];
                    out[(i0 + i) + (int64_t)nbra * (j0 + j)] = de_complex{v.x, v.y};
                }
        }
    return DE_OK;
}

DE_API int de_dots(de_problem *h, const de_complex *bras, const de_complex *kets, int64_t size, int nbra,
                   int nket, de_complex *out, int hermitian)
{
    if (!h || !bras || !kets || !out) return set_error(DE_E_INVALID, "null argument");
    if (size < 1 || nbra < 1 || nket < 1) return set_error(DE_E_INVALID, "empty dot");
    std::lock_guard<std::mutex> lk(h->mu);
    cudaSetDevice(h->p.device);
    double2 *db = nullptr, *dk = nullptr;
    DE_CUDA(cudaMalloc(&db, (size_t)size * nbra * sizeof(double2)));
    cudaError_t e = cudaMalloc(&dk, (size_t)size * nket * sizeof(double2));
    if (e != cudaSuccess) {
        cudaFree(db);
        return cuda_error(e, "cudaMalloc");
    }
    int s = DE_OK;
    if ((e = cudaMemcpyAsync(db, bras, (size_t)size * nbra * sizeof(double2), cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dk, kets, (size_t)size * nket * sizeof(double2), cudaMemcpyHostToDevice, h->stream)) != cudaSuccess)
        s = cuda_error(e, "cudaMemcpyAsync");
    if (s == DE_OK) s = de_dots_d(h, (const de_complex *)db, (const de_complex *)dk, size, nbra, nket, out, hermitian);
    cudaStreamSynchronize(h->stream);
    cudaFree(db);
    cudaFree(dk);
    return s;
}

DE_API int de_get_expects(de_problem *h, const de_complex *psi, int nvec, int cshiftopt, de_complex *expects)
{
    if (!h || !psi || !expects || nvec < 1) return set_error(DE_E_INVALID, "bad argument");
    std::lock_guard<std::mutex> lk(h->mu);
    cudaSetDevice(h->p.device);
    DE_TRY(h->ensure_stage(h->dim));
    DE_TRY(h->ensure_work(dotdiag_work_elems(2, h->dim)));
    for (int j = 0; j < nvec; ++j) {
        DE_CUDA(cudaMemcpyAsync(h->d_x, psi + (int64_t)j * h->dim, h->dim * sizeof(double2),
                                cudaMemcpyHostToDevice, h->stream));
        DE_TRY(h->matblock(h->d_x, h->d_y, 1));
        const double2 *a[2] = {h->d_x, h->d_x}, *b[2] = {h->d_y, h->d_x};
        cudaError_t e = dotdiag_launch(a, b, 2, h->dim, cshiftopt ? 0 : 1, h->d_small, h->d_work, h->stream);
        if (e != cudaSuccess) return cuda_error(e, "dotdiag");
        DE_CUDA(cudaMemcpyAsync(h->h_small, h->d_small, 2 * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
        DE_CUDA(cudaStreamSynchronize(h->stream));
        const cplx num(h->h_small[0].x, h->h_small[0].y), den(h->h_small[1].x, h->h_small[1].y);
        const cplx q = num / den;
        expects[j] = de_complex{q.real(), q.imag()};
    }
    return DE_OK;
}

}  // extern "C"
