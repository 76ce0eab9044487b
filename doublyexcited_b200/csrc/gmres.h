// gmres.h -- control flow of the PETSc-path inner solve: GMRES in the
// configuration PETSCSOLVE (petscsolve.F90:142-279) gives KSPGMRES,
// PETSc's defaults otherwise.  That is restart 30, classical Gram-Schmidt
// without refinement, no preconditioner, zero initial guess, and the stop
// test |g_{k+1}| <= max(rtol ||b||, 1e-50) on the Arnoldi residual
// estimate; max_it counts operator applications inside cycles (a restart's
// residual r = b - A x is not counted), as KSPGMRESCycle does.
//
// Header-only and free of CUDA: the vector operations come from an Ops
// object.  The solver uses device Ops (gplmr.cpp); a host Ops instance
// checks this control flow on the CPU.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace de {

// Givens least-squares state of one GMRES cycle: the rotated Hessenberg
// columns R, the rotated right-hand side g, and the rotations.
struct GmresLS {
    using cplx = std::complex<double>;
    int mk, k = 0;
    std::vector<cplx> hh, g, cs, sn, c;

    explicit GmresLS(int restart)
        : mk(restart), hh((size_t)(restart + 1) * restart), g(restart + 1), cs(restart), sn(restart), c(restart + 1)
    {
    }

    void start(double beta)
    {
        std::fill(g.begin(), g.end(), cplx(0.0));
        g[0] = beta;
        k = 0;
    }

    // Column k of the Arnoldi relation: coef[0..k] = <v_i, w> and tt = |w -
    // sum v_i coef_i|.  Returns 0, 1 for a happy breakdown (the column is
    // kept), or 2 when the rotation is undefined (KSP_DIVERGED_NULL: the
    // column is dropped).  res receives |g_{k+1}|.
    int add(const cplx *coef, double tt, double &res)
    {
        for (int i = 0; i <= k; ++i) c[i] = coef[i];
        c[k + 1] = tt;
        for (int i = 0; i < k; ++i) {  // earlier rotations
            const cplx a0 = c[i], a1 = c[i + 1];
            c[i] = std::conj(cs[i]) * a0 + sn[i] * a1;
            c[i + 1] = -std::conj(sn[i]) * a0 + cs[i] * a1;
        }
        const double hapbnd = std::min(g[k] != 0.0 ? std::abs(tt / g[k]) : 1e-30, 1e-30);
        const bool hap = tt < hapbnd;
        const double den = std::sqrt(std::norm(c[k]) + std::norm(c[k + 1]));
        if (den == 0.0) {
            res = std::abs(g[k]);
            return 2;
        }
        cs[k] = c[k] / den;
        sn[k] = c[k + 1] / den;
        c[k] = den;
        c[k + 1] = 0.0;
        g[k + 1] = -std::conj(sn[k]) * g[k];
        g[k] = std::conj(cs[k]) * g[k];
        for (int i = 0; i <= k + 1; ++i) hh[i + (size_t)(mk + 1) * k] = c[i];
        res = std::abs(g[k + 1]);
        ++k;
        return hap ? 1 : 0;
    }

    // y = R^-1 g over the k columns kept (back substitution)
    std::vector<cplx> solve() const
    {
        std::vector<cplx> y(k);
        for (int i = k - 1; i >= 0; --i) {
            cplx t = g[i];
            for (int j = i + 1; j < k; ++j) t -= hh[i + (size_t)(mk + 1) * j] * y[j];
            y[i] = t / hh[i + (size_t)(mk + 1) * i];
        }
        return y;
    }
};

// Ops: int sqnorm_b(double &n2); int sqnorm_r(double &n2);
//      int copy_b_to_r(); int r_to_v0();            (v0 = r / |r|, |r| just measured)
//      int arnoldi(int k, std::complex<double> *coef, double &tt);
//                       (w = A v_k into v_{k+1}; coef = V^H w; w -= V coef; tt = |w|)
//      int normalize_v(int k);                      (v_k /= |v_k|, |v_k| just measured)
//      int set_x(const std::vector<std::complex<double>> &y, int k, bool accumulate);
//                       (x = V y, or x += V y)
//      int zero_x(); int zero_result();
//      int residual();                              (r = b - A x)
//      int x_to_result();
// Each returns 0 on success or a status that is passed through.
template <class Ops>
int gmres_run(Ops &o, int max_it, double rtol, int restart, int *its_out)
{
    using cplx = std::complex<double>;
    const int mk = std::min(max_it, restart);
    double bn2 = 0.0;
    int s;
    if ((s = o.sqnorm_b(bn2)) != 0) return s;
    const double bnorm = std::sqrt(bn2), ttol = std::max(rtol * bnorm, 1e-50);
    *its_out = 0;
    if (bnorm <= ttol) return o.zero_result();  // converged at iteration 0: x = 0
    if ((s = o.copy_b_to_r()) != 0) return s;
    GmresLS ls(mk);
    std::vector<cplx> coef(mk + 1);
    int its = 0;
    bool first = true, done = false;
    double beta2 = bn2;
    while (!done) {
        if (!first && (s = o.sqnorm_r(beta2)) != 0) return s;
        if ((s = o.r_to_v0()) != 0) return s;
        ls.start(std::sqrt(beta2));
        while (ls.k < mk && its < max_it) {
            double tt = 0.0, res = 0.0;
            if ((s = o.arnoldi(ls.k, coef.data(), tt)) != 0) return s;
            const int st = ls.add(coef.data(), tt, res);
            ++its;
            if (st == 2 || res <= ttol || st == 1 || its >= max_it) {
                done = true;
                break;
            }
            if ((s = o.normalize_v(ls.k)) != 0) return s;
        }
        if (ls.k > 0) {
            if ((s = o.set_x(ls.solve(), ls.k, !first)) != 0) return s;
        } else if (first && (s = o.zero_x()) != 0) {
            return s;
        }
        first = false;
        if (!done && (s = o.residual()) != 0) return s;
    }
    *its_out = its;
    return o.x_to_result();
}

}  // namespace de
