// de_internal.h -- host-side internals shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <cstdarg>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/doublyexcited.h"
#include "de_kernels.h"

namespace de {

using cplx = std::complex<double>;

// ---- errors -----------------------------------------------------------
int set_error(int code, const char *fmt, ...);
int cuda_error(cudaError_t e, const char *what);

#define DE_CUDA(call)                                          \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return ::de::cuda_error(_e, #call); \
    } while (0)
#define DE_TRY(call)               \
    do {                           \
        int _s = (call);           \
        if (_s != DE_OK) return _s; \
    } while (0)

// ---- dense host LAPACK (loaded at run time) ----------------------------
struct Lapack {
    bool ok = false;
    std::string path;
    void (*zggev)(const char *, const char *, const int *, cplx *, const int *, cplx *, const int *,
                  cplx *, cplx *, cplx *, const int *, cplx *, const int *, cplx *, const int *,
                  double *, int *, size_t, size_t) = nullptr;
    void (*zpotrf)(const char *, const int *, cplx *, const int *, int *, size_t) = nullptr;
    void (*zgesdd)(const char *, const int *, const int *, cplx *, const int *, double *, cplx *,
                   const int *, cplx *, const int *, cplx *, const int *, double *, int *, int *,
                   size_t) = nullptr;
    void (*zgeev)(const char *, const char *, const int *, cplx *, const int *, cplx *, cplx *, const int *,
                  cplx *, const int *, cplx *, const int *, double *, int *, size_t, size_t) = nullptr;
};
const Lapack &lapack();  // loads once; check .ok

// ---- operator set-up (host) --------------------------------------------
// GETINVERSE tooth.f90:14-101 on (-nout..nout)^3 (column-major).
std::vector<double> getinverse(int nout, int nbig, int nsmall, double delta);
// KEMATRIX hammod.F90:235-260 (real), column-major nn x nn.
std::vector<double> kematrix(int nn, double delta);
// Symmetric eigen-decomposition (cyclic Jacobi): a = V diag(e) V^T.
void jacobi_eigen(int n, std::vector<double> a, std::vector<double> &e, std::vector<double> &v);

// ---- small dense helpers (host) -----------------------------------------
// gen_cmatsub flag=2 (hr_eigen.f90:223-291): returns DE status.
int herm_sqrt_pair(int k, const std::vector<cplx> &g, std::vector<cplx> &ginvsqrt,
                   std::vector<cplx> &gsqrt);
// SOLVE_GEVP gplmr.F90:395-439 (zggev, |alpha/beta| ascending): vr is
// kdim x nev column-major.
int solve_gevp(int kdim, int nev, std::vector<cplx> kp, std::vector<cplx> mp,
               std::vector<cplx> &vr, std::vector<cplx> *eigs = nullptr);

}  // namespace de

// ---- the handle -----------------------------------------------------------
struct de_problem {
    de_params p{};
    int n = 0, nn = 0;
    int64_t m = 0, dim = 0;
    double delta = 0.0;
    de::HamDev ham{};
    double *d_t1a = nullptr, *d_v12 = nullptr;
    float *d_t1af = nullptr, *d_v12f = nullptr;  // FP32 copies (mixed form)
    cudaStream_t own_stream = nullptr, stream = nullptr;
    // staging buffers for host-pointer calls
    double2 *d_x = nullptr, *d_y = nullptr;
    int64_t stage_elems = 0;
    // small scratch
    double2 *d_small = nullptr;   // 64 x 256 complex
    double2 *d_work = nullptr;    // reduction partials
    int64_t work_elems = 0;
    double2 *h_small = nullptr;   // pinned mirror of d_small
    std::mutex mu;
    // matvec device-time accounting (de_set_profiling): every prof_every-th
    // MATBLOCK call of each storage is timed
    bool prof = false;
    int prof_every = 1;
    int64_t prof_seq[2] = {0, 0};
    std::vector<cudaEvent_t> ev_free;
    struct Rec {
        cudaEvent_t e[3];
        int nvec;
        int f32;  // an FP32 (mixed-form) matvec
    };
    std::vector<Rec> ev_pending;
    double prof_ms[2][2] = {{0.0, 0.0}, {0.0, 0.0}};  // [fp64/fp32][pass]
    int64_t prof_calls[2] = {0, 0}, prof_vectors[2] = {0, 0};
    int prof_begin(Rec &r);
    int prof_mid(Rec &r);
    int prof_end(Rec &r);
    int harvest();
    cudaEvent_t take_event();

    // device workspace cache reused across solves (best fit)
    struct Blk {
        void *p;
        size_t bytes;
        bool used;
    };
    std::vector<Blk> cache;
    void *cache_get(size_t bytes);
    void cache_put(void *p);
    void trim();                   // release idle cached blocks and staging
    int64_t cached_bytes() const;  // device bytes the handle holds beyond its tables

    int ensure_stage(int64_t elems);
    int ensure_work(int64_t elems);
    // device pointers; y = (H + shift) x
    int matblock(const double2 *x, double2 *y, int nvec, double2 shift = double2{0.0, 0.0});
    // the same in FP32 on complex64 vectors (the mixed form's inner solve)
    int matblock32(const float2 *x, float2 *y, int nvec, double2 shift = double2{0.0, 0.0});
    // the kinetic-eigenbasis preconditioner MSOLVECPLX22 (kinpc.cu), y = P x
    // on device vectors (y must not alias x); W and 1/D are built on first
    // use and for each new shift
    int kinetic_pc(const double2 *x, double2 *y, int nvec, de::cplx shift);
    int gm_pcopt = 0;  // GMRES inner solve preconditioner: 0 none, 2 kinetic eigenbasis
    double *d_kw = nullptr;
    double2 *d_kdinv = nullptr;
    de::cplx kdinv_shift{0.0, 0.0};
    bool kdinv_ok = false;
};
