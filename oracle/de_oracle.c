/*
 * de_oracle.c -- CPU oracle for the two-electron complex-scaled sinc-DVR
 * Hamiltonian matvec of doublyexcited (helium, 3-D Cartesian grid).
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates the reference Fortran loops
 * so that the CUDA product can be checked against them.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may
 * load the library built from it; the product never links or calls it.
 *
 * Layout conventions follow the reference exactly:
 *   one-electron index  p = i + NN*j + NN^2*k   (0-based; Fortran 1-based
 *                        linear index P-1, decoded in hammod.F90:559-569)
 *   two-electron vector X(p,q), column-major, p (electron 1) fastest
 *                        (hammod.F90:149, gplmr.F90:27)
 *   T is the COMPLEX NN x NN kinetic matrix already divided by SCALE^2
 *                        (initmod.F90:207-208), column-major T[l + NN*i].
 *   V is the COMPLEX diagonal potential already divided by SCALE
 *                        (initmod.F90:224).
 *
 * The loops deliberately keep the reference's complex*complex arithmetic
 * (KEMULTS with complex T), its explicit transposes (MPITRANSPOSE at NP=1 is
 * Y = TRANSPOSE(X), hammod.F90:898-899) and its OpenMP decomposition over
 * columns (hammod.F90:164-179), so timing this file is timing the
 * reference's algorithm on the host cores.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex zc;

/* KEMATRIX, hammod.F90:235-260 (real part; caller divides by SCALE^2). */
void or_kematrix(int nn, double delta, double *t)
{
    const double pi = 4.0 * atan(1.0);
    for (int j = 0; j < nn; ++j)
        for (int i = 0; i < nn; ++i) {
            if (i == j) {
                t[i + nn * j] = (pi / delta) * (pi / delta) / 6.0;
            } else {
                int d = i - j;
                double sgn = (d % 2 == 0) ? 1.0 : -1.0;
                t[i + nn * j] = sgn / (delta * delta * (double)(d * d));
            }
        }
}

/* RVECTOR, tooth.f90:106-172.
 *   R(i,j,k)  = delta^3/|r| on the big grid (-nbig..nbig)^3, 0 at the origin
 *   TR(i,j,k) = -sum_p [T(i,p) R(p,j,k) + T(j,p) R(i,p,k) + T(k,p) R(i,j,p)]
 *               on the small grid (-nsmall..nsmall)^3.                      */
void or_rvector(int nbig, int nsmall, double delta, double *r, double *tr)
{
    const double pi = 4.0 * atan(1.0);
    const int nb = 2 * nbig + 1, ns = 2 * nsmall + 1;
#define RB(i, j, k) r[((i) + nbig) + (size_t)nb * (((j) + nbig) + (size_t)nb * ((k) + nbig))]
#pragma omp parallel for schedule(static)
    for (int k = -nbig; k <= nbig; ++k)
        for (int j = -nbig; j <= nbig; ++j)
            for (int i = -nbig; i <= nbig; ++i) {
                double x = i * delta, y = j * delta, z = k * delta;
                double rad = sqrt(x * x + y * y + z * z);
                RB(i, j, k) = (rad == 0.0) ? 0.0 : delta * delta * delta / rad;
            }
#pragma omp parallel for schedule(static)
    for (int k = -nsmall; k <= nsmall; ++k)
        for (int j = -nsmall; j <= nsmall; ++j)
            for (int i = -nsmall; i <= nsmall; ++i) {
                double acc = 0.0;
                for (int p = -nbig; p <= nbig; ++p) {
                    double t1 = pi * pi / (6.0 * delta * delta), t2 = t1, t3 = t1;
                    if (i != p) t1 = (((i - p) % 2 == 0) ? 1.0 : -1.0) / (delta * delta * (double)((i - p) * (i - p)));
                    if (j != p) t2 = (((j - p) % 2 == 0) ? 1.0 : -1.0) / (delta * delta * (double)((j - p) * (j - p)));
                    if (k != p) t3 = (((k - p) % 2 == 0) ? 1.0 : -1.0) / (delta * delta * (double)((k - p) * (k - p)));
                    acc = acc - (t1 * RB(p, j, k) + t2 * RB(i, p, k) + t3 * RB(i, j, p));
                }
                tr[(i + nsmall) + (size_t)ns * ((j + nsmall) + (size_t)ns * (k + nsmall))] = acc;
            }
#undef RB
}

/* TOOTHEIGMULT, tooth.f90:178-204: Y = (W (x) W (x) W) X, applied along the
 * third, then second, then first axis.  W is n x n column-major.          */
void or_tootheigmult(const double *x, double *y, const double *w, int n)
{
    size_t n3 = (size_t)n * n * n;
    double *x1 = (double *)malloc(n3 * sizeof(double));
    double *x2 = (double *)malloc(n3 * sizeof(double));
#define A3(a, i, j, k) a[(i) + (size_t)n * ((j) + (size_t)n * (k))]
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < n; ++k) {
                double s = 0.0;
                for (int l = 0; l < n; ++l) s += w[k + n * l] * A3(x, i, j, l);
                A3(x1, i, j, k) = s;
            }
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                double s = 0.0;
                for (int l = 0; l < n; ++l) s += w[j + n * l] * A3(x1, i, l, k);
                A3(x2, i, j, k) = s;
            }
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double s = 0.0;
                for (int l = 0; l < n; ++l) s += w[i + n * l] * A3(x2, l, j, k);
                A3(y, i, j, k) = s;
            }
#undef A3
    free(x1);
    free(x2);
}

/* POTENTIAL1, hammod.F90:432-498, one nucleus of charge z at the origin.
 * tinv is (-nb..nb)^3 column-major with nb = 2N+1.  Output is REAL; the
 * caller divides by SCALE.                                                  */
void or_potential1(int n, double delta, double charge, const double *tinv, double *v)
{
    const int nn = 2 * n + 1, nb = nn, nbd = 2 * nb + 1;
    const double a = -charge / (delta * delta * delta);
    for (int k = 0; k < nn; ++k)
        for (int j = 0; j < nn; ++j)
            for (int i = 0; i < nn; ++i) {
                int ii = i - n, jj = j - n, kk = k - n;
                double s = tinv[(ii + nb) + (size_t)nbd * ((jj + nb) + (size_t)nbd * (kk + nb))];
                v[i + nn * (j + nn * k)] = 0.0 + a * s;
            }
}

/* POTENTIAL2, hammod.F90:502-582: V(P,Q) = A*TINV(r_Q) + A*TINV(r_P)
 * + TINV(r_Q - r_P)/delta^3 with A = -Z/delta^3; the reference names the
 * coordinates of the column index Q (I1,J1,K1) and of the row P (I2,J2,K2).
 * Output is REAL (M*M); the caller divides by SCALE.                       */
void or_potential2(int n, double delta, double charge, const double *tinv, double *v)
{
    const int nn = 2 * n + 1, nb = nn, nbd = 2 * nb + 1;
    const int64_t m = (int64_t)nn * nn * nn;
    const double d3 = delta * delta * delta;
    const double a = -charge / d3;
#define TI(i, j, k) tinv[((i) + nb) + (size_t)nbd * (((j) + nb) + (size_t)nbd * ((k) + nb))]
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < m; ++q) {
        int k1 = (int)(q / (nn * nn)), j1 = (int)((q / nn) % nn), i1 = (int)(q % nn);
        i1 -= n; j1 -= n; k1 -= n;
        for (int64_t p = 0; p < m; ++p) {
            int k2 = (int)(p / (nn * nn)), j2 = (int)((p / nn) % nn), i2 = (int)(p % nn);
            i2 -= n; j2 -= n; k2 -= n;
            v[p + m * q] = 0.0 + a * TI(i1, j1, k1) + a * TI(i2, j2, k2) + TI(i1 - i2, j1 - j2, k1 - k2) / d3;
        }
    }
#undef TI
}

/* KEMULTS, hammod.F90:264-286, complex T, one NN^3 column. */
static void kemults(int nn, const zc *t, const zc *x, zc *y)
{
#define X3(i, j, k) x[(i) + nn * ((j) + nn * (k))]
    for (int k = 0; k < nn; ++k)
        for (int j = 0; j < nn; ++j)
            for (int i = 0; i < nn; ++i) {
                zc s1 = 0, s2 = 0, s3 = 0;
                for (int l = 0; l < nn; ++l) s1 += t[l + nn * i] * X3(l, j, k);
                for (int l = 0; l < nn; ++l) s2 += t[l + nn * j] * X3(i, l, k);
                for (int l = 0; l < nn; ++l) s3 += t[l + nn * k] * X3(i, j, l);
                y[i + nn * (j + nn * k)] = s1 + s2 + s3;
            }
#undef X3
}

/* Out-of-place transpose of an m x m column-major complex matrix, blocked. */
static void transpose(int64_t m, const zc *x, zc *y)
{
    const int64_t b = 32;
#pragma omp parallel for schedule(static)
    for (int64_t qb = 0; qb < m; qb += b)
        for (int64_t pb = 0; pb < m; pb += b)
            for (int64_t q = qb; q < qb + b && q < m; ++q)
                for (int64_t p = pb; p < pb + b && p < m; ++p) y[q + m * p] = x[p + m * q];
}

/* HAMMULT for NELEC=2 with NP=1 (hammod.F90:19-67 -> KEMULT2 :138-187):
 *   Y = T*X columnwise; W = X^T; Z = T*W columnwise; W = Z^T; Y = Y + W;
 *   Y = Y + V*X.
 * w and z are caller-provided work arrays of m*m elements (the reference's
 * SAVE'd W and Z, hammod.F90:153-159).                                     */
void or_hammult2(int nn, const zc *t, const zc *v, const zc *x, zc *y, zc *w, zc *z)
{
    const int64_t m = (int64_t)nn * nn * nn, mm = m * m;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < m; ++q) kemults(nn, t, x + m * q, y + m * q);
    transpose(m, x, w);
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < m; ++q) kemults(nn, t, w + m * q, z + m * q);
    transpose(m, z, w);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < mm; ++e) y[e] = y[e] + w[e] + v[e] * x[e];
}

/* HAMMULT for NELEC=1 with NP=1 (KEMULT1, hammod.F90:71-134, full index
 * ranges) followed by Y = Y + V*X.                                           */
void or_hammult1(int nn, const zc *t, const zc *v, const zc *x, zc *y)
{
    const int64_t m = (int64_t)nn * nn * nn;
    kemults(nn, t, x, y);
    for (int64_t e = 0; e < m; ++e) y[e] = y[e] + v[e] * x[e];
}
