/*
 * doublyexcited.h -- C ABI of the B200 implementation of doublyexcited's
 * hot path: the complex-scaled two-electron sinc-DVR helium Hamiltonian
 * applied to blocks of vectors inside the GPLMR harmonic-Ritz block
 * eigensolver.
 *
 * Conventions
 *   - Every function returns an int status: DE_OK (0) or a DE_E_* code.
 *     Nothing aborts or exits; de_last_error() gives a message for the
 *     calling host thread.
 *   - Complex numbers are de_complex {re, im}: the memory layout of Fortran
 *     COMPLEX*16 and of C99 double _Complex, so reference-side buffers pass
 *     through unchanged.
 *   - Two-electron vectors are X(1:M, 1:M) column-major with electron 1
 *     (p) fastest, p = i + NN*j + NN^2*k, exactly as the reference stores
 *     them (hammod.F90:149, gplmr.F90:27).  Blocks are X(M, MB, NEV).
 *   - One de_problem handle owns all state (operator tables, device
 *     workspace, CUDA stream).  Calls on one handle are serialised by the
 *     caller; different handles may be used from different host threads.
 *     The reference's HAMMULT keeps SAVE'd state and is not reentrant
 *     (hammod.F90:31,153-159); this API is.
 *   - Functions without a suffix take HOST pointers and include the
 *     host<->device copies; the _d variants take DEVICE pointers and run on
 *     the handle's stream.
 *
 * Paths cited below are relative to complexscale-djhnow/code/ of the
 * reference.
 */
#ifndef DOUBLYEXCITED_B200_H
#define DOUBLYEXCITED_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DE_API __attribute__((visibility("default")))

typedef struct {
    double re, im;
} de_complex;

enum {
    DE_OK = 0,
    DE_E_INVALID = 1,      /* bad argument */
    DE_E_SIZE = 2,         /* size mismatch (reference: "SIZE ERRORRRR 66", doublyexcited.F90:33-36) */
    DE_E_CUDA = 3,         /* CUDA runtime error */
    DE_E_NOMEM = 4,        /* device or host allocation failed */
    DE_E_UNSUPPORTED = 5,  /* option the build does not provide (e.g. grids above N=11) */
    DE_E_CHOLESKY = 6,     /* zpotrf breakdown in cholQR (lamod.f90:169-175) */
    DE_E_GEVP = 7,         /* zggev failure (gplmr.F90:431-432) */
    DE_E_SVD = 8,          /* zgesdd failure (hr_eigen.f90:246-248) */
    DE_E_ORTHO = 9,        /* inner-solve orthonormality self-check (harmonic_ritz_small.F90:221-242) */
    DE_E_NOT_CONVERGED = 10,
    DE_E_IO = 11,          /* file error */
    DE_E_PARSE = 12,       /* Input.Inp / argument parse error */
    DE_E_LAPACK = 13,      /* host LAPACK library not found */
    DE_E_NAN = 14,         /* non-finite residual */
    DE_E_BUSY = 15         /* admission refused (serving) */
};

enum { DE_PREC_FP64 = 0, DE_PREC_MIXED = 1 };

/* Grid / physics parameters.  Mirrors PARAMETERS (structs.F90:28-57) and the
 * &grid/&molecule/&main namelist fields that feed INIT_STRUCTS
 * (input.F90:365-417). */
typedef struct {
    int n;            /* N: NN = 2N+1 points per axis (input.F90 &grid N) */
    double delta;     /* grid spacing (DELTA) */
    double radius;    /* box radius (RADIUS); delta = radius/N when autodelta */
    int autodelta;    /* AUTODELTA */
    double theta;     /* complex-scaling angle (THETA); SCALE = exp(i theta) */
    double charge;    /* nuclear charge (CHARGE), nucleus at the origin */
    int nelec;        /* 1 or 2 electrons */
    int nsmall;       /* NSMALL of the TINV solve (default 22) */
    int tfactor;      /* TFACTOR of the TINV solve (default 4) */
    int precision;    /* DE_PREC_FP64 or DE_PREC_MIXED */
    int device;       /* CUDA device ordinal */
} de_params;

/* Inner-solve options.  Mirrors GMRES_SOLVER (structs.F90:137-162). */
typedef struct {
    int max_inner_iter;          /* GM_MAX_INNER_ITER: Krylov order of PRECBLOCK_BASIC, or the
                                    GMRES iteration limit of the PETSc path */
    int usepetscflag;            /* 0 -> the PETSc path: per column, GMRES on H in KSPGMRES's
                                    configuration (PRECBLOCK_PETSC gplmr.F90:507-563,
                                    PETSCSOLVE petscsolve.F90:142-279), FP64; else BASIC.
                                    The reference's flag is inverted (gplmr.F90:496-500); same here. */
    double tol;                  /* GM_TOL: the GMRES rtol (PETSc path only) */
    int compat_first_column_only;/* 1: reproduce allhmultsub's first-column-only matvec
                                    (gplmr.F90:704-716); other columns of the product are zero */
} de_gmres;

/* Solver statistics (the reference prints these, gplmr.F90:343-366). */
typedef struct {
    int iterations;
    int converged;
    int64_t matvecs;          /* vector-matvecs executed */
    int64_t matvecs_reference;/* HAMMULT calls the reference makes for the same solve (its ICALLED) */
    double max_residual;
    double t_total_s;         /* wall time of the solve */
    double t_matvec_s;        /* MATBLOCK time (TSPMV) */
    double t_prec_s;          /* PRECBLOCK time (TPREC) */
    double t_dense_s;         /* host dense LAPACK time */
} de_stats;

typedef struct de_problem de_problem;

/* ---- errors ---------------------------------------------------------- */
DE_API const char *de_strerror(int status);
DE_API const char *de_last_error(void);
DE_API const char *de_version(void);
/* Number of CUDA kernels this library has launched in the process. */
DE_API int64_t de_kernel_launches(void);

/* ---- parameters and set-up ------------------------------------------- */

/* Reference defaults (input.F90:1-124: N=2, DELTA=0.5, RADIUS=7, AUTODELTA,
 * THETA=0, CHARGE=2, NSMALL=22, TFACTOR=4) with nelec=2. */
DE_API void de_params_default(de_params *p);

/* Build the operator: T = KEMATRIX/SCALE^2, TINV by GETINVERSE, potential
 * tables (INIT_HAMILTONIAN initmod.F90:174-228, GETINVERSE tooth.f90:14-101,
 * POTENTIAL1/2 hammod.F90:432-582).  Allocates device tables only. */
DE_API int de_problem_create(const de_params *p, de_problem **out);
DE_API int de_problem_destroy(de_problem *h);
/* Release the device workspace a handle keeps between solves (GPLMR blocks,
 * staging) back to the stream-ordered pool; the operator tables stay.  The
 * reference keeps SAVE'd work arrays for the life of the process
 * (hammod.F90:153-159); this is the way to give them back. */
DE_API int de_problem_trim(de_problem *h);

/* NN, M = NN^3 and the vector length M^nelec of a handle. */
DE_API int de_problem_dims(const de_problem *h, int *nn, int64_t *m, int64_t *dim);

/* Run the handle's work on a caller's cudaStream_t from now on.  NULL is the
 * CUDA legacy default stream (as in the CUDA runtime); a new handle uses a
 * private non-blocking stream until this is called. */
DE_API int de_set_stream(de_problem *h, void *cuda_stream);

/* Device-time accounting of the matvec kernels: CUDA events recorded on the
 * handle's stream around the two passes of MATBLOCK calls (pass A:
 * electron-2 contraction + potential; pass B: electron-1 contraction).
 * on = 0: off (the default); 1: every call; n > 1: every n-th call of each
 * storage (complex128, complex64), which keeps the events' own cost (a few
 * microseconds a call) out of the timed work; the read-outs then cover the
 * sampled calls.  The reference times phases with MPI_WTIME
 * (gplmr.F90:42-57). */
DE_API int de_set_profiling(de_problem *h, int on);
/* Which matvec kernels a handle uses: DE_MATVEC_FMA (the default) the
 * fastest CUDA-core kernels per grid: even/odd-split contractions for the
 * mixed form's complex64 matvec at NN = 9..17 and the plain form's at NN =
 * 9..13, streaming kernels at NN = 15..19 otherwise, shared-memory cube
 * kernels elsewhere; DE_MATVEC_TENSOR the axis contractions on the FP64
 * tensor cores (DMMA) for NN = 9..19; DE_MATVEC_STREAM the streaming / cube
 * kernels everywhere (for comparison); DE_MATVEC_TF32 the mixed form's
 * complex64 matvec with its kinetic contractions on the 5th-generation
 * tensor cores (tcgen05, TF32 products of head/tail-split operands, FP32
 * accuracy) for NN = 9..15, the FMA kernels elsewhere and for complex128.
 * All give the reference's H x to rounding. */
enum { DE_MATVEC_FMA = 0, DE_MATVEC_TENSOR = 1, DE_MATVEC_STREAM = 2, DE_MATVEC_TF32 = 3 };
DE_API int de_set_matvec_kernel(de_problem *h, int kind);
/* The kernels of one matvec pass.  storage 0 = complex128 matvecs, 1 =
 * complex64 (the mixed form's inner solve); pass 0 = electron-2 axes and
 * potential, 1 = electron-1 axes; family a DE_MATVEC_* kind (where a
 * family is not built for the grid, the even/odd kernels run, or the
 * streaming / cube kernels where those are not built either);
 * ctas_per_sm caps the resident CTAs per SM of the persistent kernels
 * (0 = as many as fit).  A handle starts from the tuning table written by
 * `python -m doublyexcited_b200.tune`: the file DE_MATVEC_TUNING names (set
 * but empty: none), else matvec_tuning.txt beside the library; entries it
 * lacks keep the FMA kernels with all resident CTAs.  No reference
 * counterpart (the reference has one kernel). */
DE_API int de_set_matvec_launch(de_problem *h, int storage, int pass, int family, int ctas_per_sm);
DE_API int de_get_matvec_launch(de_problem *h, int storage, int pass, int *family, int *ctas_per_sm);
/* The kinetic-eigenbasis preconditioner MSOLVECPLX22 (littlesolver.F90:
 * 372-436) on nvec device vectors: with W the eigenvectors and lam the
 * eigenvalues of the real kinetic matrix (KINETIC_EIGS :709-740) and P = W
 * diag(1 / ((lam_i + lam_j + lam_k) / SCALE^2 - shift)) W^T on one
 * electron's cube, y = P on every column cube + P on every row cube.  Two
 * electrons, NN 3..19; y must not alias x. */
DE_API int de_kinetic_precond_d(de_problem *h, const de_complex *x_d, de_complex *y_d, int nvec, de_complex shift);
/* The preconditioner of the GMRES inner solve (de_gmres.usepetscflag = 0):
 * 0 none (the reference's hard-wired GM_PCOPT, input.F90:67), 2 the
 * kinetic eigenbasis above applied on the left, as the reference's
 * PETSc shell PC option 2 would (petscsolve.F90:109-114,179). */
DE_API int de_set_gmres_pc(de_problem *h, int pcopt);
/* A tuning table's entry for (storage, NN, pass), read on the host only;
 * DE_E_INVALID when the file or the entry is missing. */
DE_API int de_tuning_lookup(const char *path, int storage, int nn, int pass, int *family, int *ctas_per_sm);
/* Device milliseconds of pass A and pass B, MATBLOCK calls and vectors
 * multiplied since the last read (waits for the recorded events); resets. */
DE_API int de_profile_read(de_problem *h, double *pass_a_ms, double *pass_b_ms, int64_t *calls,
                           int64_t *vectors);
/* The same for the FP32 matvecs of the mixed form's inner solve (no
 * counterpart in the reference, which has one precision). */
DE_API int de_profile_read32(de_problem *h, double *pass_a_ms, double *pass_b_ms, int64_t *calls,
                             int64_t *vectors);

/* ---- operator: HAMMULT / MATBLOCK / MYMATMUL ------------------------- */

/* Y = H X for one vector of length mm (== M^nelec).  Replaces
 * HAMMULT(HAM,PARAMS,MPIDATA,X,Y,MM) hammod.F90:19-67 at NP=1. */
DE_API int de_hammult(de_problem *h, const de_complex *x, de_complex *y, int64_t mm);
DE_API int de_hammult_d(de_problem *h, const de_complex *x_d, de_complex *y_d, int64_t mm);

/* AX(:,:,j) = H X(:,:,j), j = 1..nev, in one launch.  Replaces MATBLOCK
 * gplmr.F90:443-462 and the MYMATMUL callback doublyexcited.F90:24-44
 * (m*mb must equal the vector length: DE_E_SIZE otherwise). */
DE_API int de_matblock(de_problem *h, const de_complex *x, de_complex *ax, int64_t m, int64_t mb,
                       int nev);
DE_API int de_matblock_d(de_problem *h, const de_complex *x_d, de_complex *ax_d, int64_t m,
                         int64_t mb, int nev);
/* MATBLOCK in the mixed form's precision: complex64 device vectors
 * ({float re, im} interleaved, same layout), FP32 arithmetic.  No
 * counterpart in the reference (one precision there); it is the inner-solve
 * matvec of DE_PREC_MIXED, exported for accuracy and throughput checks. */
DE_API int de_matblock32_d(de_problem *h, const void *x_d, void *ax_d, int64_t m, int64_t mb, int nev);

/* OUT(i,j) = <BRA_i, KET_j> over vectors of length size.  hermitian=1:
 * conj(BRA).KET (MYDOTSUB doublyexcited.F90:47-59, MPIHERMDOT
 * hammod.F90:383-403); hermitian=0: BRA.KET, the c-product (MPIDOT
 * hammod.F90:361-380).  out is nbra x nket column-major. */
DE_API int de_dots(de_problem *h, const de_complex *bras, const de_complex *kets, int64_t size,
                   int nbra, int nket, de_complex *out, int hermitian);
DE_API int de_dots_d(de_problem *h, const de_complex *bras_d, const de_complex *kets_d,
                     int64_t size, int nbra, int nket, de_complex *out_host, int hermitian);

/* Allocation-free device dot products.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc: code embedded in a host
 * application that owns all device memory through its own pool or a fixed
 * reservation (a serving process that reserved its HBM up front), where an
 * allocation by this library would fail or exceed the reservation.  Same
 * results as de_dots_d (hermitian=1: conj(BRA).KET; 0: the c-product),
 * written to DEVICE memory out_d (nbra x nket column-major) asynchronously on
 * cuda_stream (NULL: legacy default stream).  Needs no handle and calls no
 * allocating routine: the reduction scratch is a static device array of
 * 151,568 bytes that every GPU loading the library holds until exit.
 * Shapes: nket == 1 with nbra <= 32, or nbra, nket <= 8 with one of them <= 4
 * (at most 32 outputs); larger shapes return DE_E_INVALID.  The first call on
 * each device (and the first after a device reset) looks up the array's
 * device address; make that call before any stream capture.  All calls share
 * the array and each clears its reduction ticket first: calls that overlap
 * on the GPU (other streams, other host threads) race and must be serialised
 * by the caller. */
DE_API int de_dots_noalloc_d(const de_complex *bras_d, const de_complex *kets_d, int64_t size, int nbra,
                             int nket, de_complex *out_d, int hermitian, void *cuda_stream);

/* EXPECTS(j) = <psi_j|H|psi_j>/<psi_j|psi_j> (Hermitian; c-product when
 * cshiftopt).  GET_EXPECTS hammod.F90:1261-1301. */
DE_API int de_get_expects(de_problem *h, const de_complex *psi, int nvec, int cshiftopt,
                          de_complex *expects);

/* ---- initial guess: HELIUM_ORBITAL products + DIAGSUBSPACE ---------- */

/* The reference's start block for GPLMR (doublyexcited.F90:135-190).
 * The numorbs He+ levels of lowest real part come from the one-electron
 * operator of the handle's grid.  The reference converges them with block
 * Lanczos; here a dense ZGEEV is used, so numorbs <= M.  They are
 * Gram-Schmidt orthonormalised as in HELIUM_ORBITALGATHER
 * hammod.F90:1084-1113: c-products, or Hermitian products with hermopt.
 * The symmetrised products HELIUM_ORBITAL hammod.F90:1041-1080 follow
 * (i <= j for singlet, i < j otherwise).  H is diagonalised in their span,
 * as in DIAGSUBSPACE hammod.F90:1125-1256: A(I,J) = psi_I . H psi_J, ZGEEV,
 * then eigenvalues ordered by distance to etarget as in mysort
 * hammod.F90:1658-1690.  Outputs: the first numout eigenvalues in e0, and
 * the two-electron vectors in x (D x numout, column-major, unit Hermitian
 * norm).  At most 128 products and 16 outputs; numout above the number of
 * products returns DE_E_INVALID (the reference STOPs with "Reset NUMOUT").
 * _d: x is device memory.  Needs a nelec == 2 handle and host LAPACK. */
DE_API int de_subspace_guess_d(de_problem *h, int numorbs, int singlet, int hermopt, de_complex etarget,
                               int numout, de_complex *x_d, de_complex *e0);
DE_API int de_subspace_guess(de_problem *h, int numorbs, int singlet, int hermopt, de_complex etarget,
                             int numout, de_complex *x, de_complex *e0);

/* The He+ orbitals of the initial guess from a dense one-electron operator
 * h1 (M x M, column-major, M = (2n+1)^3, n <= 11).  Host only: no GPU
 * needed.  This replaces DIAGONALIZE (doublyexcited.F90:135-137) and
 * HELIUM_ORBITALGATHER (hammod.F90:1084-1113).  The numorbs levels of
 * lowest real part go to energies, and their right eigenvectors,
 * Gram-Schmidt orthonormalised in that order, go to orbitals (M x numorbs,
 * column-major).  The Gram-Schmidt uses c-products, or Hermitian products
 * with hermopt.  The eigenproblem is split into the 8 reflection-parity
 * sectors of the cube, one ZGEEV each.  de_subspace_guess uses this
 * routine. */
DE_API int de_heplus_orbitals(int n, const de_complex *h1, int numorbs, int hermopt, de_complex *energies,
                              de_complex *orbitals);

/* ---- eigensolver: GPLMR_EIG ----------------------------------------- */

/* Block GPLMR with harmonic projection and the BASIC inner solve.
 * Replaces GPLMR_EIG(HAM,PARAMS,MPIDATA,GMSOLVER,X,E,M,MB,SIGMA,NEV,NS,
 * MAXIT,TOL,PRECONDITIONER,OUTMODULUS) gplmr.F90:9-374.  x is X(M,MB,NEV)
 * in/out (start vectors in, Ritz vectors out), e receives NEV eigenvalues.
 * outmodulus > 0 prints the reference's progress lines to stdout every
 * outmodulus iterations; 0 is silent.  stats may be NULL. */
DE_API int de_gplmr_eig(de_problem *h, de_complex *x, de_complex *e, int64_t m, int64_t mb,
                        de_complex sigma, int nev, int ns, int maxit, double tol,
                        const de_gmres *gm, int outmodulus, de_stats *stats);
DE_API int de_gplmr_eig_d(de_problem *h, de_complex *x_d, de_complex *e, int64_t m, int64_t mb,
                          de_complex sigma, int nev, int ns, int maxit, double tol,
                          const de_gmres *gm, int outmodulus, de_stats *stats);

/* ---- configuration: Input.Inp namelists + command-line keys ---------- */

/* Everything get_input/get_args (input.F90:143-362) can set. */
typedef struct {
    de_params params;
    de_gmres gmres;
    int writevecs, readvecs;
    char invecfile[300], outvecfile[300];
    int numorbs, singlet, numskip;
    int outmodulus, takerealpart, hermopt, cshiftopt;
    int gplmr_nev, gplmr_ns, gplmr_maxit;
    double gplmr_tol;
    de_complex gplmr_shift;
    int kdim, lanblocksize, check;
    double lantol;
} de_input;

/* Defaults of input.F90:1-124 for every field. */
DE_API void de_input_default(de_input *in);

/* Read the &main &grid &molecule &lanczos &gmres &orbitals &gplmr
 * namelists from path (a missing file leaves the defaults, as the
 * reference does), then apply argv keys (N= Shift= Outfile= Infile=
 * NoPetsc Petsc Theta= R= Delta= Nev= Norbs= Gptol= Skip= Gmtol= Iter=
 * Read Takereal Notakereal Sing Trip).  argv may be NULL. */
DE_API int de_read_input(const char *path, int argc, const char *const *argv, de_input *in);

/* The Inp=<file> argument of get_inputfile (input.F90:257-276), or
 * "Input.Inp" when absent.  buf receives at most len bytes. */
DE_API int de_input_file_arg(int argc, const char *const *argv, char *buf, size_t len);

/* ---- eigenvector files (utils.F90:82-198) ---------------------------- */

/* Write NUM vectors of M x M complex to a Fortran unformatted sequential
 * file: header record (int32 M, int32 NUM, int64 16*M*M), then one record
 * per vector, 4-byte record markers with gfortran sub-records beyond 2 GiB. */
DE_API int de_write_vectors(const char *path, int64_t m, int num, const de_complex *psi);

/* Read num vectors into a grid of M = (2N+1)^3 points.  A file written for
 * another odd grid is zero-padded or cropped about the centre in all six
 * coordinates (SIXD_FIX utils.F90:186-198). */
DE_API int de_read_vectors(const char *path, int64_t m, int num, de_complex *psi);

/* Header of an eigenvector file: its M and number of vectors. */
DE_API int de_vectors_header(const char *path, int64_t *m, int *num);

/* ---- the whole program: PROGRAM ATOM ---------------------------------- */

typedef struct {
    int totget;              /* start vectors formed or read (TOTGET) */
    int nexpects;            /* TOTGET - NUMSKIP */
    de_complex e0[16];       /* subspace eigenvalues after NUMSKIP (zero when vectors were read) */
    de_complex expects[16];  /* expectation values of the start vectors (GET_EXPECTS) */
    de_complex shift;        /* the shift GPLMR ran with */
    de_stats stats;
} de_run_info;

/* PROGRAM ATOM doublyexcited.F90:60-262 on a parsed input.  Steps:
 *  1. TOTGET = min(MAXGET, NEV+NUMSKIP+5) start vectors from the initial
 *     guess (de_subspace_guess, etarget = gplmr_shift), or NEV+NUMSKIP read
 *     from invecfile when readvecs.  NEV+NUMSKIP above MAXGET returns
 *     DE_E_INVALID (the reference STOPs: "GPLMR_NEV TOO BIG FOR NUMORBS").
 *  2. NUMSKIP leading vectors are dropped.
 *  3. GET_EXPECTS runs on the rest.  The shift is the mean of the first NEV
 *     expectation values, real part only with takerealpart.
 *  4. GPLMR_EIG runs with the input's NS, MAXIT, TOL and gmres options.
 *  5. The NEV eigenvectors are written to outvecfile when writevecs.
 * e receives NEV eigenvalues; x (may be NULL) the D x NEV eigenvectors;
 * info (may be NULL) the intermediate values.  verbose prints the
 * reference's report lines (SUBSPACE EIGENVALS, CHOSEN SHIFT, the GPLMR
 * iterations every outmodulus, FINAL EIGVALS).  At most 16 start vectors.
 * Argument errors return before any GPU work. */
DE_API int de_run(const de_input *in, int verbose, de_complex *e, de_complex *x, de_run_info *info);

/* ---- batched and served solves ----------------------------------------
 * No counterpart in the reference, which runs one GPLMR_EIG per MPI job
 * (doublyexcited.F90:238-241); these entry points run many independent
 * GPLMR_EIG solves of uneven size on one GPU at once.
 *
 * A server owns `workers` host threads, each with its own CUDA stream and
 * handles, so the kernels of different solves overlap on the device.
 * Requests are admitted in arrival order (first come, first served; the
 * head of the queue waits rather than being overtaken) when a worker is
 * free and the request's device footprint fits in what is left of
 * `max_bytes`; a request whose footprint alone exceeds max_bytes is
 * refused at submission with DE_E_BUSY.  A request's Krylov blocks stay on
 * the device for the whole solve; its host buffers x and e must stay valid
 * until its result has been collected. */
typedef struct {
    int device;        /* CUDA device ordinal */
    int workers;       /* concurrent solves (streams), >= 1 */
    int64_t max_bytes; /* device bytes for admitted solves; 0 = 90% of the free memory at creation */
} de_server_opts;

typedef struct {
    de_params params;   /* operator and precision of this solve (params.device is ignored) */
    de_complex sigma;   /* GPLMR shift */
    int nev, ns, maxit;
    double tol;
    de_gmres gm;
    de_complex *x;      /* host, M^2 x NEV column-major: start vectors in, Ritz vectors out */
    de_complex *e;      /* host, NEV eigenvalues out */
} de_request;

typedef struct {
    uint64_t id;
    int status;                     /* DE_OK or the solve's error */
    de_stats stats;
    double t_submit_s, t_start_s, t_end_s;  /* server clock, seconds since creation */
    int64_t footprint_bytes;        /* device bytes reserved for the solve */
    int worker;
} de_result;

/* Device bytes a request reserves: the GPLMR blocks (X AX W AW P AP, S AS,
 * the inner solve's Krylov blocks, complex64 in the mixed form), staging
 * and the operator tables. */
DE_API int de_request_footprint(const de_request *r, int64_t *bytes);
DE_API int de_server_create(const de_server_opts *o, void **server);
/* Queue a request; its id is returned in *id. */
DE_API int de_server_submit(void *server, const de_request *r, uint64_t *id);
/* Wait for request id (timeout_s < 0: no limit); DE_E_BUSY on timeout. */
DE_API int de_server_wait(void *server, uint64_t id, double timeout_s, de_result *out);
/* Wait for any finished request not yet collected. */
DE_API int de_server_wait_any(void *server, double timeout_s, de_result *out);
/* Seconds on the server clock. */
DE_API double de_server_now(void *server);
/* Requests queued, running, and device bytes reserved right now. */
DE_API int de_server_load(void *server, int *queued, int *running, int64_t *bytes_reserved);
/* Finishes the running solves, drops the queued ones, frees everything. */
DE_API int de_server_destroy(void *server);

#ifdef __cplusplus
}
#endif

#endif /* DOUBLYEXCITED_B200_H */
