// Host instance of the GMRES control flow in doublyexcited_b200/csrc/gmres.h,
// for tests/test_gmres_host.py: dense complex A and b from a file, the same
// Ops contract as the solver's device instance, x and the iteration count out.
// Input file: int32 n, max_it, restart; float64 rtol; then A (n x n,
// column-major) and b, as complex128.  Output file: int32 status, its; then x.
#include <complex>
#include <cstdio>
#include <cstdint>
#include <vector>

#include "gmres.h"

using cplx = std::complex<double>;

struct HostOps {
    int n;
    const std::vector<cplx> &a;
    std::vector<cplx> b, r, x, result;
    std::vector<std::vector<cplx>> v;
    double last_n2 = 0.0;

    std::vector<cplx> apply(const std::vector<cplx> &u) const
    {
        std::vector<cplx> y(n, 0.0);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) y[i] += a[i + (size_t)n * j] * u[j];
        return y;
    }
    static double sq(const std::vector<cplx> &u)
    {
        double s = 0.0;
        for (const cplx &z : u) s += std::norm(z);
        return s;
    }
    int sqnorm_b(double &n2) { return n2 = last_n2 = sq(b), 0; }
    int sqnorm_r(double &n2) { return n2 = last_n2 = sq(r), 0; }
    int copy_b_to_r() { return r = b, 0; }
    int r_to_v0()
    {
        const double f = 1.0 / std::sqrt(last_n2);
        v[0] = r;
        for (cplx &z : v[0]) z *= f;
        return 0;
    }
    int arnoldi(int k, cplx *coef, double &tt)
    {
        std::vector<cplx> w = apply(v[k]);
        for (int i = 0; i <= k; ++i) {  // classical: every coefficient on the unmodified w
            cplx s = 0.0;
            for (int t = 0; t < n; ++t) s += std::conj(v[i][t]) * w[t];
            coef[i] = s;
        }
        for (int i = 0; i <= k; ++i)
            for (int t = 0; t < n; ++t) w[t] -= v[i][t] * coef[i];
        last_n2 = sq(w);
        tt = std::sqrt(last_n2);
        v[k + 1] = w;
        return 0;
    }
    int normalize_v(int k)
    {
        const double f = 1.0 / std::sqrt(last_n2);
        for (cplx &z : v[k]) z *= f;
        return 0;
    }
    int set_x(const std::vector<cplx> &y, int k, bool accumulate)
    {
        if (!accumulate) x.assign(n, 0.0);
        for (int i = 0; i < k; ++i)
            for (int t = 0; t < n; ++t) x[t] += v[i][t] * y[i];
        return 0;
    }
    int zero_x() { return x.assign(n, 0.0), 0; }
    int zero_result() { return result.assign(n, 0.0), 0; }
    int residual()
    {
        std::vector<cplx> ax = apply(x);
        for (int t = 0; t < n; ++t) r[t] = b[t] - ax[t];
        return 0;
    }
    int x_to_result() { return result = x, 0; }
};

int main(int argc, char **argv)
{
    if (argc != 3) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    int32_t hdr[3];
    double rtol;
    if (std::fread(hdr, sizeof hdr, 1, f) != 1 || std::fread(&rtol, sizeof rtol, 1, f) != 1) return 4;
    const int n = hdr[0], max_it = hdr[1], restart = hdr[2];
    std::vector<cplx> a((size_t)n * n), b(n);
    if (std::fread(a.data(), sizeof(cplx), a.size(), f) != a.size()) return 5;
    if (std::fread(b.data(), sizeof(cplx), b.size(), f) != b.size()) return 6;
    std::fclose(f);
    HostOps o{n, a, b, {}, {}, {}, std::vector<std::vector<cplx>>(std::min(max_it, restart) + 1)};
    int its = 0;
    const int32_t status = de::gmres_run(o, max_it, rtol, restart, &its);
    FILE *g = std::fopen(argv[2], "wb");
    if (!g) return 7;
    const int32_t out[2] = {status, its};
    std::fwrite(out, sizeof out, 1, g);
    std::fwrite(o.result.data(), sizeof(cplx), o.result.size(), g);
    std::fclose(g);
    return 0;
}
