// de_kernels.h -- launch interface of the sm_100a kernels (host side).
//
// Device vectors are double2 arrays (re, im) in the reference layout
// X(p,q), p = i + NN*j + NN^2*k fastest (hammod.F90:149).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace de {

// Process-wide count of kernels launched by this library.
void count_launch(int n = 1);
int64_t launch_count();
// Whether the even/odd matvec kernels are launched as programmatic dependent
// launches (they wait on the grid dependency after their table preload);
// on unless the environment sets DE_PDL=0.  Read once per process.
bool programmatic_launch();

constexpr int kMaxNN = 27;      // N <= 13 (the reference ran N = 5..15)
constexpr int kEvCoef = 12 * 12;  // even/odd coefficient tables, N <= 11
constexpr int kMaxCols = 128;   // columns per block-op operand list

// Operator data for one problem (HAMILTONIAN, structs.F90:87-102).
struct HamDev {
    int nn;                 // NN = 2N+1
    int nelec;              // 1 or 2
    int64_t m;              // NN^3
    double t[kMaxNN];       // T_real(0,d) = KEMATRIX first column, d = 0..NN-1
    double s2re, s2im;      // 1/SCALE^2 (initmod.F90:208)
    double vsre, vsim;      // 1/SCALE (initmod.F90:224)
    double sre, sim;        // SCALE = exp(i theta) (initmod.F90:48)
    const double *t1a;      // [M]  A*TINV(r_p), A = -Z/delta^3 (hammod.F90:576-577)
    const double *v12;      // [(2NN-1)^3] TINV(r_q - r_p)/delta^3 (hammod.F90:578)
    // FP32 copies for the mixed form (null when the problem is FP64 only)
    float tf[kMaxNN];
    const float *t1af;
    const float *v12f;
    // Matvec kernels per [storage: 0 complex128, 1 complex64][pass: 0 A, 1 B]:
    // fam 0 even/odd-split (hammult_ev.cu; streaming / cube where those are
    // not built), 1 FP64 tensor cores (hammult_tc.cu), 2 streaming / cube
    // (hammult.cu), 3 tcgen05 TF32 (hammult_tc32.cu, complex64 on NN 9..15;
    // even/odd elsewhere); ctas = resident CTAs per SM of the persistent
    // kernels, 0 = as many as fit.  Filled from the tuning table at creation
    // (tuning.cpp) or by de_set_matvec_kernel / de_set_matvec_launch.
    signed char fam[2][2];
    signed char ctas[2][2];
    // Even/odd-split coefficients of T for the grid (hammult_ev.cu), index
    // a * (N+1) + b: ev_ce(a,0) = t(a), ev_ce(a,b) = (t(|a-b|) + t(a+b))/2,
    // ev_co(a,b) = (t(|a-b|) - t(a+b))/2 (a, b >= 1); FP32 copies beside.
    double ev_ce[kEvCoef], ev_co[kEvCoef];
    float ev_cef[kEvCoef], ev_cof[kEvCoef];
};

// Fills ev_ce / ev_co (and the FP32 copies) from h.t for grid h.nn.
void fill_ev_coefficients(HamDev &h);

// The kinetic-eigenbasis preconditioner MSOLVECPLX22 (kinpc.cu): pass 0
// writes Y = P on the row cubes, pass 1 adds P on the column cubes; w_dev =
// W (NN x NN column-major eigenvectors of the real kinetic matrix), dinv_dev
// = 1 / ((lam_i + lam_j + lam_k) / SCALE^2 - shift) on the cube (M, i
// fastest).  NN odd, 3..19; y must not alias x.
bool kinetic_pc_supported(int nn);
cudaError_t kinetic_pc_launch(int nn, const double2 *x, double2 *y, int nvec, int64_t vstride, const double *w_dev,
                              const double2 *dinv_dev, int pass, cudaStream_t st);

// Tuning table (tuning.cpp): the entry of (storage 0 complex128 / 1
// complex64, NN, pass) in the table at path; false when the file or the
// entry is missing.  apply_tuning fills h.fam / h.ctas for h.nn from the
// default table (built-in choices where it has no entry).
bool tuning_lookup(const char *path, int storage, int nn, int pass, int &fam, int &ctas);
void apply_tuning(HamDev &h);

// Y(:,:,v) = H X(:,:,v) for v < nvec; vectors are vstride elements apart.
// Two passes: electron-2 axes + potential (strided cubes, writes Y), then
// electron-1 axes (contiguous cubes, Y += ...).  Deterministic (no atomics).
// shift: y = (H + shift) x, fused into the potential term of pass A.
cudaError_t hammult_launch(const HamDev &h, const double2 *x, double2 *y, int nvec,
                           int64_t vstride, cudaStream_t st, double2 shift = double2{0.0, 0.0});

// One pass of the above: pass 0 = electron-2 + potential (writes Y), pass 1 =
// electron-1 (Y += ...).
cudaError_t hammult_pass_launch(const HamDev &h, const double2 *x, double2 *y, int nvec,
                                int64_t vstride, int pass, cudaStream_t st, double2 shift = double2{0.0, 0.0});
// The same on complex64 vectors in FP32 arithmetic (needs h.tf / t1af / v12f).
cudaError_t hammult_pass_launch(const HamDev &h, const float2 *x, float2 *y, int nvec, int64_t vstride, int pass,
                                cudaStream_t st, double2 shift = double2{0.0, 0.0});

// Even/odd-split form of one pass (hammult_ev.cu) for the grids
// hammult_ev_supported accepts (complex128: NN = 9..13; complex64: NN =
// 9..17); shs is the diagonal shift times SCALE^2.
bool hammult_ev_supported(int nn, bool fp64);

// The complex64 passes with the kinetic contractions on the tensor cores
// (tcgen05 kind::tf32, head/tail split; hammult_tc32.cu) for the grids
// hammult_tc32_supported accepts (NN = 9..15); shs as above.  The kernels
// record a timed-out mbarrier wait in a device flag that
// hammult_tc32_error reads and clears (1 = a wait gave up, -1 = the read
// failed).
bool hammult_tc32_supported(int nn);
cudaError_t hammult_tc32_pass_launch(const HamDev &h, const float2 *x, float2 *y, int nvec, int64_t vstride,
                                     int pass, cudaStream_t st, double2 shs, int ctas = 0);
int hammult_tc32_error(cudaStream_t st);
cudaError_t hammult_ev_pass_launch(const HamDev &h, const double2 *x, double2 *y, int nvec, int64_t vstride,
                                   int pass, cudaStream_t st, double2 shs, int ctas = 0);
cudaError_t hammult_ev_pass_launch(const HamDev &h, const float2 *x, float2 *y, int nvec, int64_t vstride, int pass,
                                   cudaStream_t st, double2 shs, int ctas = 0);

// Tensor-core (DMMA) form of one pass, for the grids hammult_tc_supported
// accepts; the same arguments and results as hammult_pass_launch.
bool hammult_tc_supported(int nn);
cudaError_t hammult_tc_pass_launch(const HamDev &h, const double2 *x, double2 *y, int nvec, int64_t vstride, int pass,
                                   cudaStream_t st, double2 shift);
cudaError_t hammult_tc_pass_launch(const HamDev &h, const float2 *x, float2 *y, int nvec, int64_t vstride, int pass,
                                   cudaStream_t st, double2 shift);

// One-electron H (NELEC=1): KEMULT1 + V (hammod.F90:71-134).
cudaError_t hammult1_launch(const HamDev &h, const double *vfull, const double2 *x, double2 *y,
                            int nvec, int64_t vstride, cudaStream_t st);

// Column list: column c is a[c] - sigma * b[c] (b[c] may be null).  S is
// the storage type (double2, or float2 for the mixed form's inner solve);
// sums accumulate in FP64 either way.
template <class S>
struct ColListT {
    const S *a[kMaxCols];
    const S *b[kMaxCols];
    double2 sigma;
    int n;
};
using ColList = ColListT<double2>;
using ColListF = ColListT<float2>;

// G(i,j) = sum_r op(L_i[r]) R_j[r] over len rows; op = conj (herm=1) or
// identity (herm=0).  out is device memory, column-major with leading
// dimension ldo; nl <= 64, nr <= 128.  work must hold gram_work_elems().
int64_t gram_work_elems(int nl, int nr, int64_t len);
cudaError_t gram_launch(const ColList &L, const ColList &R, int64_t len, int herm, double2 *out,
                        int ldo, double2 *work, cudaStream_t st);
cudaError_t gram_launch(const ColListF &L, const ColListF &R, int64_t len, int herm, double2 *out, int ldo,
                        double2 *work, cudaStream_t st);

// Hermitian Gram G = Z^H Z of n <= 7 complex64 vectors (FP64 sums), all n x n
// entries written to DEVICE out (column-major, ldo); work as for gram.
cudaError_t gram_herm_launch(const ColListF &Z, int64_t len, double2 *out, int ldo, double2 *work, cudaStream_t st);

// Y_j = beta_j * Y_j + alpha * sum_i X_i C(i,j) for j < nout (nout <= 16,
// nin <= kMaxCols); C is DEVICE memory (complex, column-major, ldc).  Each
// row is read before it is written, so Y may alias X columns.
template <class SI, class SO>
struct UpdListT {
    const SI *x[kMaxCols];
    SO *y[16];
    double2 beta[16];
    double2 alpha;  // Y_j = beta_j Y_j + alpha * sum_i X_i C(i,j)
    int nin, nout;
};
using UpdList = UpdListT<double2, double2>;
cudaError_t update_launch(const UpdList &U, const double2 *c_dev, int ldc, int64_t len,
                          cudaStream_t st);
cudaError_t update_launch(const UpdListT<float2, float2> &U, const double2 *c_dev, int ldc, int64_t len,
                          cudaStream_t st);
cudaError_t update_launch(const UpdListT<float2, double2> &U, const double2 *c_dev, int ldc, int64_t len,
                          cudaStream_t st);

// out_j = a_j + s * c_j * b_j, c_j from DEVICE memory (j < n, n <= 64).
// c_dev may be null (c_j = 1).  out may alias a.
cudaError_t axpc_launch(double2 *const *out, const double2 *const *a, const double2 *const *b,
                        int n, double2 s, const double2 *c_dev, int64_t len, cudaStream_t st);
// out = (complex64) (a + s c b) for one column, c = c_dev[0] (device) or 1.
cudaError_t axpc_f32_launch(float2 *out, const double2 *a, const double2 *b, double2 s, const double2 *c_dev,
                            int64_t len, cudaStream_t st);

// d_j = sum_r conj(A_j[r]) B_j[r] (herm) for j < n (n <= 64) into DEVICE out.
int64_t dotdiag_work_elems(int n, int64_t len);
cudaError_t dotdiag_launch(const double2 *const *a, const double2 *const *b, int n, int64_t len,
                           int herm, double2 *out, double2 *work, cudaStream_t st);

// Gram-Schmidt step of the inner solve: q -= sum_i qp_i d_i, v -= sum_i
// vp_i d_i (d: m values in DEVICE memory), then q, v *= 1/sqrt(|<q,q>|); the
// factor is also left in cout[0].  work as for gram (ticket at work[0]).
cudaError_t gs_update_launch(const double2 *const *qp, const double2 *const *vp, int m, double2 *q, double2 *v,
                             const double2 *d, int64_t len, double2 *work, double2 *cout, cudaStream_t st);
cudaError_t gs_update_launch(const float2 *const *qp, const float2 *const *vp, int m, float2 *q, float2 *v,
                             const double2 *d, int64_t len, double2 *work, double2 *cout, cudaStream_t st);

// First pass of the fused two-pass Gram-Schmidt (m <= 16): q -= qp d,
// v -= vp d with pass-1 coefficients d, and the pass-2 coefficients
// <qp_i, q> reduced into dout[0..m) and |q|^2 into dout[64].  The second pass
// is gs_pass2_launch with d2 = dout.
cudaError_t gs_pass1_launch(const double2 *const *qp, const double2 *const *vp, int m, double2 *q, double2 *v,
                            const double2 *d, int64_t len, double2 *work, double2 *dout, cudaStream_t st);
cudaError_t gs_pass1_launch(const float2 *const *qp, const float2 *const *vp, int m, float2 *q, float2 *v,
                            const double2 *d, int64_t len, double2 *work, double2 *dout, cudaStream_t st);

// Second pass: q <- (q - qp d2)/|w|, v <- (v - vp d2)/|w| with
// |w|^2 = d2[64] - |d2[0..m)|^2; the factor also goes to cout[0].
cudaError_t gs_pass2_launch(const double2 *const *qp, const double2 *const *vp, int m, double2 *q, double2 *v,
                            const double2 *d2, int64_t len, double2 *cout, cudaStream_t st);
cudaError_t gs_pass2_launch(const float2 *const *qp, const float2 *const *vp, int m, float2 *q, float2 *v,
                            const double2 *d2, int64_t len, double2 *cout, cudaStream_t st);

// Electron-exchange symmetry of one M x M vector: out[0] = <X, X^T>
// (Hermitian; work as for gram, >= (M/32)^2 + 1 elements), and the in-place
// projection X <- (X + s X^T)/2.
cudaError_t exch_dot_launch(const double2 *x, int64_t m, double2 *out, double2 *work, cudaStream_t st);
// Y = sum_{i < nz} Z_i coef_i (complex64 columns, nz <= 8, coefficients on
// the device) written projected, Y <- (Y + s Y^T)/2, in one pass.
cudaError_t update_exch_launch(const float2 *const *z, int nz, const double2 *coef, double2 *y, int64_t m, double s,
                               cudaStream_t st);
cudaError_t exch_project_launch(double2 *x, int64_t m, double s, cudaStream_t st);

// Reflection sectors of one nn^6 vector (nn odd): out[r] = <x, R_r x> for
// the 8 products R_r of the axis reflections c -> nn-1-c (bit a of r:
// axis a, both electrons; work as for gram, >= 8 * 592 + 1 elements, work[0]
// untouched), and the in-place
// projection onto the sectors c with bit c of keep set, sector c being
// the eigenspace where R_r has eigenvalue (-1)^popcount(c & r).
cudaError_t refl_corr_launch(const double2 *x, int nn, double2 *out, double2 *work, cudaStream_t st);
cudaError_t refl_project_launch(double2 *x, int nn, unsigned keep, cudaStream_t st);

// Narrowing copies to FP32 (complex and real).
cudaError_t to_f32_launch(const double2 *x, float2 *y, int64_t n, cudaStream_t st);
cudaError_t to_f32_launch(const double *x, float *y, int64_t n, cudaStream_t st);

// Orthogonalise-and-normalise coefficients of one column against n
// orthonormal columns, from g = [Q^H b; b^H b] (n + 1 entries): coef =
// [-(Q^H b)/|w|; 1/|w|] with |w|^2 = b^H b - |Q^H b|^2; a |w|^2 not above
// 1e-28 b^H b raises flag bit 1 (cholQR breakdown).
cudaError_t orth_norm_coef_launch(const double2 *g, int n, double2 *coef, int *flag, cudaStream_t st);

// k x k (k <= 16) dense helpers that keep the solver on the device.
// flag bits: 1 Cholesky breakdown, 2 all-zero block, 4 orthonormality
// self-check failed, 8 singular 1 x 1 Gram.
cudaError_t small_cholinv_launch(const double2 *g, int k, double2 *rinv, int *flag, cudaStream_t st);
// The mixed inner solve's normal equations for one column (Gram g of the
// nz <= 9 power-basis vectors): the nz - 1 coefficients into DEVICE a.
cudaError_t small_sstep_solve_launch(const double2 *g, int nz, double2 *a, int *flag, cudaStream_t st);
cudaError_t small_hsqrt1_launch(const double2 *g, double2 *ginvh, double2 *gsq, int *flag, cudaStream_t st);
// |T - I| <= tol elementwise (the reference's self-check uses 1e-10).
cudaError_t small_ortho_check_launch(const double2 *t, int k, int *flag, cudaStream_t st, double tol = 1e-10);
cudaError_t small_gemm_launch(const double2 *a, const double2 *b, double2 *c, int m, int k, int n, cudaStream_t st);

// out = a + s b over n contiguous complex elements (may alias a or b
// element for element).
cudaError_t axpy_launch(double2 *out, const double2 *a, const double2 *b, double2 s, int64_t n, cudaStream_t st);
cudaError_t axpy_launch(float2 *out, const float2 *a, const float2 *b, double2 s, int64_t n, cudaStream_t st);

// x_j *= c_j (c from DEVICE, complex), in place.
cudaError_t scale_cols_launch(double2 *const *x, int n, const double2 *c_dev, int64_t len,
                              cudaStream_t st);

// c_j = 1/sqrt(|d_j|) on device (myhgramschmidt_many normalisation).
cudaError_t inv_sqrt_abs_launch(const double2 *d, double2 *c, int n, cudaStream_t st);

// Potential-table construction on device from the TINV table.
cudaError_t build_tables_launch(int nn, int n, double charge, double delta, const double *tinv,
                                int nbd, double *t1a, double *v12, cudaStream_t st);

}  // namespace de
