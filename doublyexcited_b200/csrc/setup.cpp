// setup.cpp -- host-side operator set-up, small dense linear algebra and
// the run-time LAPACK loader.
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "de_internal.h"

namespace de {

// ---------------------------------------------------------------- errors

static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

const char *last_error_str() { return g_last_error.c_str(); }

int cuda_error(cudaError_t e, const char *what)
{
    if (e == cudaErrorMemoryAllocation)
        return set_error(DE_E_NOMEM, "%s: %s", what, cudaGetErrorString(e));
    return set_error(DE_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// ---------------------------------------------------------------- LAPACK

#ifndef DE_LAPACK_DEFAULT
#define DE_LAPACK_DEFAULT ""
#endif

static Lapack load_lapack()
{
    Lapack L;
    std::vector<std::string> cands;
    if (const char *env = getenv("DE_LAPACK_LIB")) cands.push_back(env);
    if (DE_LAPACK_DEFAULT[0]) cands.push_back(DE_LAPACK_DEFAULT);
    cands.push_back("liblapack.so.3");
    cands.push_back("libopenblas.so.0");
    for (const auto &c : cands) {
        void *hd = dlopen(c.c_str(), RTLD_NOW | RTLD_LOCAL);
        if (!hd) continue;
        for (const char *pre : {"scipy_", ""}) {
            auto sym = [&](const char *name) {
                std::string s = std::string(pre) + name;
                return dlsym(hd, s.c_str());
            };
            void *a = sym("zggev_"), *b = sym("zpotrf_"), *d = sym("zgesdd_"), *g = sym("zgeev_");
            if (a && b && d && g) {
                L.zggev = reinterpret_cast<decltype(L.zggev)>(a);
                L.zpotrf = reinterpret_cast<decltype(L.zpotrf)>(b);
                L.zgesdd = reinterpret_cast<decltype(L.zgesdd)>(d);
                L.zgeev = reinterpret_cast<decltype(L.zgeev)>(g);
                L.ok = true;
                L.path = c;
                return L;
            }
        }
        dlclose(hd);
    }
    return L;
}

const Lapack &lapack()
{
    static Lapack L = load_lapack();
    return L;
}

// ---------------------------------------------------------------- set-up

std::vector<double> kematrix(int nn, double delta)
{
    const double pi = 4.0 * std::atan(1.0);
    std::vector<double> t((size_t)nn * nn);
    for (int j = 0; j < nn; ++j)
        for (int i = 0; i < nn; ++i) {
            if (i == j) {
                t[i + (size_t)nn * j] = (pi / delta) * (pi / delta) / 6.0;
            } else {
                const int d = i - j;
                const double sgn = (d % 2 == 0) ? 1.0 : -1.0;
                t[i + (size_t)nn * j] = sgn / (delta * delta * (double)(d * d));
            }
        }
    return t;
}

void jacobi_eigen(int n, std::vector<double> a, std::vector<double> &e, std::vector<double> &v)
{
    v.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) v[i + (size_t)n * i] = 1.0;
    auto A = [&](int i, int j) -> double & { return a[i + (size_t)n * j]; };
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int j = 0; j < n; ++j) {
            diag += A(j, j) * A(j, j);
            for (int i = 0; i < j; ++i) off += A(i, j) * A(i, j);
        }
        if (off <= 1e-32 * diag) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A(p, q);
                if (std::fabs(apq) < 1e-300) continue;
                const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {  // columns p, q
                    const double akp = A(k, p), akq = A(k, q);
                    A(k, p) = c * akp - s * akq;
                    A(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {  // rows p, q
                    const double apk = A(p, k), aqk = A(q, k);
                    A(p, k) = c * apk - s * aqk;
                    A(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = v[k + (size_t)n * p], vkq = v[k + (size_t)n * q];
                    v[k + (size_t)n * p] = c * vkp - s * vkq;
                    v[k + (size_t)n * q] = s * vkp + c * vkq;
                }
            }
    }
    e.resize(n);
    for (int i = 0; i < n; ++i) e[i] = A(i, i);
}

// Y = (W (x) W (x) W) X along the third, second, then first axis
// (TOOTHEIGMULT tooth.f90:178-204).
static void eigmult3(int n, const std::vector<double> &x, std::vector<double> &y,
                     const std::vector<double> &w)
{
    const size_t n3 = (size_t)n * n * n;
    std::vector<double> x1(n3), x2(n3);
    y.assign(n3, 0.0);
    auto I3 = [n](int i, int j, int k) { return (size_t)i + (size_t)n * ((size_t)j + (size_t)n * k); };
#pragma omp parallel for collapse(2)
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < n; ++k) {
                double s = 0.0;
                for (int l = 0; l < n; ++l) s += w[k + (size_t)n * l] * x[I3(i, j, l)];
                x1[I3(i, j, k)] = s;
            }
#pragma omp parallel for collapse(2)
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                double s = 0.0;
                for (int l = 0; l < n; ++l) s += w[j + (size_t)n * l] * x1[I3(i, l, k)];
                x2[I3(i, j, k)] = s;
            }
#pragma omp parallel for collapse(2)
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double s = 0.0;
                for (int l = 0; l < n; ++l) s += w[i + (size_t)n * l] * x2[I3(l, j, k)];
                y[I3(i, j, k)] = s;
            }
}

std::vector<double> getinverse(int nout, int nbig, int nsmall, double delta)
{
    const double pi = 4.0 * std::atan(1.0);
    const int nb = 2 * nbig + 1, ns = 2 * nsmall + 1;
    // R = delta^3/|r| on the big grid (RVECTOR tooth.f90:134-156)
    std::vector<double> r((size_t)nb * nb * nb);
    auto RB = [&](int i, int j, int k) -> double & {
        return r[(size_t)(i + nbig) + (size_t)nb * ((size_t)(j + nbig) + (size_t)nb * (k + nbig))];
    };
#pragma omp parallel for
    for (int k = -nbig; k <= nbig; ++k)
        for (int j = -nbig; j <= nbig; ++j)
            for (int i = -nbig; i <= nbig; ++i) {
                const double x = i * delta, y = j * delta, z = k * delta;
                const double rad = std::sqrt(x * x + y * y + z * z);
                RB(i, j, k) = (rad == 0.0) ? 0.0 : delta * delta * delta / rad;
            }
    // TR = -T_big R on the small grid (RVECTOR tooth.f90:160-170)
    std::vector<double> tcol(2 * nb + 1);  // T(a,b) by a-b in [-(nb-1), nb-1] ... covers |i-p| <= nbig+nsmall
    const int off = nb;
    for (int d = -nb; d <= nb; ++d)
        tcol[d + off] = (d == 0) ? pi * pi / (6.0 * delta * delta)
                                 : ((d % 2 == 0) ? 1.0 : -1.0) / (delta * delta * (double)(d * d));
    std::vector<double> tr((size_t)ns * ns * ns);
#pragma omp parallel for collapse(2)
    for (int k = -nsmall; k <= nsmall; ++k)
        for (int j = -nsmall; j <= nsmall; ++j)
            for (int i = -nsmall; i <= nsmall; ++i) {
                double acc = 0.0;
                for (int p = -nbig; p <= nbig; ++p)
                    acc = acc - (tcol[i - p + off] * RB(p, j, k) + tcol[j - p + off] * RB(i, p, k) +
                                 tcol[k - p + off] * RB(i, j, p));
                tr[(size_t)(i + nsmall) + (size_t)ns * ((size_t)(j + nsmall) + (size_t)ns * (k + nsmall))] = acc;
            }
    tr[(size_t)nsmall + (size_t)ns * ((size_t)nsmall + (size_t)ns * nsmall)] += 2 * pi;
    // T_small eigen-decomposition (the reference calls DSYEV('V','U'))
    std::vector<double> ts((size_t)ns * ns);
    for (int j = 0; j < ns; ++j)
        for (int i = 0; i < ns; ++i) ts[i + (size_t)ns * j] = tcol[i - j + off];
    std::vector<double> e, w;
    jacobi_eigen(ns, ts, e, w);
    std::vector<double> wt((size_t)ns * ns);
    for (int j = 0; j < ns; ++j)
        for (int i = 0; i < ns; ++i) wt[i + (size_t)ns * j] = w[j + (size_t)ns * i];
    std::vector<double> qq, q;
    eigmult3(ns, tr, qq, wt);
    for (int k = 0; k < ns; ++k)
        for (int j = 0; j < ns; ++j)
            for (int i = 0; i < ns; ++i) qq[(size_t)i + (size_t)ns * ((size_t)j + (size_t)ns * k)] /= (e[i] + e[j] + e[k]);
    eigmult3(ns, qq, q, w);
    for (int k = -nsmall; k <= nsmall; ++k)
        for (int j = -nsmall; j <= nsmall; ++j)
            for (int i = -nsmall; i <= nsmall; ++i)
                RB(i, j, k) += q[(size_t)(i + nsmall) + (size_t)ns * ((size_t)(j + nsmall) + (size_t)ns * (k + nsmall))];
    const int no = 2 * nout + 1;
    std::vector<double> out((size_t)no * no * no);
    for (int k = -nout; k <= nout; ++k)
        for (int j = -nout; j <= nout; ++j)
            for (int i = -nout; i <= nout; ++i)
                out[(size_t)(i + nout) + (size_t)no * ((size_t)(j + nout) + (size_t)no * (k + nout))] = RB(i, j, k);
    return out;
}

// ---------------------------------------------------------------- dense

int herm_sqrt_pair(int k, const std::vector<cplx> &g, std::vector<cplx> &ginv,
                   std::vector<cplx> &gsq)
{
    const Lapack &L = lapack();
    if (!L.ok) return set_error(DE_E_LAPACK, "host LAPACK not found (set DE_LAPACK_LIB)");
    std::vector<cplx> a = g, u((size_t)k * k), vt((size_t)k * k);
    std::vector<double> sv(k);
    const int lwork = 10 * k * k + 100;
    std::vector<cplx> zwork(20 * k * k + 100);
    std::vector<double> rwork(20 * k * k + 100);
    std::vector<int> iwork(100 * k);
    int info = 0;
    L.zgesdd("A", &k, &k, a.data(), &k, sv.data(), u.data(), &k, vt.data(), &k, zwork.data(),
             &lwork, rwork.data(), iwork.data(), &info, 1);
    if (info != 0) return set_error(DE_E_SVD, "zgesdd info=%d", info);
    std::vector<double> s1(k), s2(k);
    for (int i = 0; i < k; ++i) {
        double v = sv[i];
        if (v != 0.0) v = 1.0 / v;  // tol = 0 in the reference call
        s1[i] = std::sqrt(v);
        s2[i] = std::sqrt(sv[i]);
    }
    ginv.assign((size_t)k * k, 0.0);
    gsq.assign((size_t)k * k, 0.0);
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < k; ++i) {
            cplx a1 = 0.0, a2 = 0.0;
            for (int l = 0; l < k; ++l) {
                const cplx t = std::conj(vt[l + (size_t)k * i]) * std::conj(u[j + (size_t)k * l]);
                a1 += t * s1[l];
                a2 += t * s2[l];
            }
            ginv[i + (size_t)k * j] = a1;
            gsq[i + (size_t)k * j] = a2;
        }
    return DE_OK;
}

int solve_gevp(int kdim, int nev, std::vector<cplx> kp, std::vector<cplx> mp,
               std::vector<cplx> &vr_out, std::vector<cplx> *eigs)
{
    const Lapack &L = lapack();
    if (!L.ok) return set_error(DE_E_LAPACK, "host LAPACK not found (set DE_LAPACK_LIB)");
    std::vector<cplx> alpha(kdim), beta(kdim), vr((size_t)kdim * kdim), vl(1);
    const int lwork = 10 * std::max(1, 2 * kdim);
    std::vector<cplx> work(lwork);
    std::vector<double> rwork(8 * kdim);
    int info = 0, one = 1;
    L.zggev("N", "V", &kdim, kp.data(), &kdim, mp.data(), &kdim, alpha.data(), beta.data(),
            vl.data(), &one, vr.data(), &kdim, work.data(), &lwork, rwork.data(), &info, 1, 1);
    if (info != 0) return set_error(DE_E_GEVP, "SOLVE OF THE PROJECTED EIGENVALUE PROBLEM FAILED (zggev info=%d)", info);
    // EIGSORT gplmr.F90:640-660: nev smallest |alpha/beta|, first minimum on ties
    std::vector<double> y(kdim);
    for (int i = 0; i < kdim; ++i) y[i] = std::abs(alpha[i] / beta[i]);
    const double mx = *std::max_element(y.begin(), y.end());
    vr_out.assign((size_t)kdim * nev, 0.0);
    if (eigs) eigs->assign(nev, 0.0);
    for (int kq = 0; kq < nev; ++kq) {
        int im = 0;
        for (int i = 1; i < kdim; ++i)
            if (y[i] < y[im]) im = i;
        for (int r = 0; r < kdim; ++r) vr_out[r + (size_t)kdim * kq] = vr[r + (size_t)kdim * im];
        if (eigs) (*eigs)[kq] = alpha[im] / beta[im];
        y[im] = mx + 1;
    }
    return DE_OK;
}

}  // namespace de
