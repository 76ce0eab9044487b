// run.cpp -- PROGRAM ATOM (doublyexcited.F90:60-262) as one call.  From a
// parsed input it forms the GPLMR start block: the initial guess
// (de_subspace_guess) or vectors read from a file.  It drops NUMSKIP
// leading vectors and takes the shift from their expectation values.  Then
// it runs GPLMR_EIG and writes the eigenvectors back.  Every step is a C-ABI
// call of this library; this file only sequences them as the reference
// program does.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "de_internal.h"

using namespace de;

namespace {

struct Owned {
    de_problem *h = nullptr;
    ~Owned()
    {
        if (h) de_problem_destroy(h);
    }
};

void print_values(const cplx *v, int from, int to, const cplx *other)
{
    for (int i = from; i < to; ++i) {
        if (other)
            printf("%20.14f%20.14f      %20.14f\n", v[i].real(), v[i].imag(), std::abs(v[i] - other[i]));
        else
            printf("%20.14f%20.14f\n", v[i].real(), v[i].imag());
    }
}

}  // namespace

extern "C" DE_API int de_run(const de_input *in, int verbose, de_complex *e, de_complex *x, de_run_info *info)
{
    if (!in || !e) return set_error(DE_E_INVALID, "null argument");
    const int nev = in->gplmr_nev, skip = in->numskip, norbs = in->numorbs;
    if (nev < 1 || skip < 0) return set_error(DE_E_INVALID, "GPLMR_NEV %d / NUMSKIP %d out of range", nev, skip);
    if (in->params.nelec != 2) return set_error(DE_E_INVALID, "PROGRAM ATOM solves the two-electron problem");
    // TOTGET doublyexcited.F90:139-151
    int totget = nev + skip;
    if (!in->readvecs) {
        if (norbs < 1) return set_error(DE_E_INVALID, "NUMORBS %d < 1", norbs);
        const int maxget = in->singlet ? norbs * (norbs + 1) / 2 : norbs * (norbs - 1) / 2;
        if (nev + skip > maxget)
            return set_error(DE_E_INVALID, "FOR INITIAL GUESS, GPLRM_NEV TOO BIG FOR NUMORBS. %d %d %d", nev, skip,
                             norbs);
        totget = std::min(maxget, nev + skip + 5);
    }
    if (totget > 16) return set_error(DE_E_INVALID, "TOTGET %d exceeds the 16 start vectors supported", totget);
    if (in->readvecs) {  // the file is checked before any GPU work
        int64_t fm = 0;
        int fnum = 0;
        DE_TRY(de_vectors_header(in->invecfile, &fm, &fnum));
        if (fnum < totget)
            return set_error(DE_E_IO, "%s holds %d vectors, %d requested", in->invecfile, fnum, totget);
    }

    Owned P;
    DE_TRY(de_problem_create(&in->params, &P.h));
    int nn = 0;
    int64_t m = 0, d = 0;
    DE_TRY(de_problem_dims(P.h, &nn, &m, &d));
    std::vector<cplx> psi((size_t)d * totget), e0(totget, 0.0), expects(totget, 0.0);
    de_complex *psi_c = reinterpret_cast<de_complex *>(psi.data());
    if (in->readvecs) {
        DE_TRY(de_read_vectors(in->invecfile, m, totget, psi_c));
    } else {
        if (verbose) printf("COMPUTING INITIAL GUESSES...\n");
        DE_TRY(de_subspace_guess(P.h, norbs, in->singlet, in->hermopt, in->gplmr_shift, totget, psi_c,
                                 reinterpret_cast<de_complex *>(e0.data())));
    }
    // NUMSKIP doublyexcited.F90:186-189
    if (skip > 0) {
        std::copy(psi.begin() + (size_t)d * skip, psi.end(), psi.begin());
        std::copy(e0.begin() + skip, e0.end(), e0.begin());
    }
    const int nuse = totget - skip;
    DE_TRY(de_get_expects(P.h, psi_c, nuse, in->cshiftopt, reinterpret_cast<de_complex *>(expects.data())));
    if (verbose) {
        if (!in->readvecs) {
            printf("SUBSPACE EIGENVALS:\n");
            print_values(e0.data(), 0, nev, expects.data());
            printf(" --xx-- \n");
            print_values(e0.data(), nev, nuse, expects.data());
        }
        printf("SUBSPACE EXPECTATION VALS:\n");
        print_values(expects.data(), 0, nev, nullptr);
        printf(" --xx-- \n");
        print_values(expects.data(), nev, nuse, nullptr);
    }
    // the shift: mean of the first NEV expectation values doublyexcited.F90:205-217
    cplx shift = 0.0;
    for (int j = 0; j < nev; ++j) shift += expects[j];
    shift /= (double)nev;
    if (in->takerealpart) shift = cplx(shift.real(), 0.0);
    if (verbose) printf("CHOSEN SHIFT: %20.10f%20.10f\n", shift.real(), shift.imag());
    fflush(stdout);

    de_stats st{};
    DE_TRY(de_gplmr_eig(P.h, psi_c, e, m, m, de_complex{shift.real(), shift.imag()}, nev, in->gplmr_ns,
                        in->gplmr_maxit, in->gplmr_tol, &in->gmres, verbose ? in->outmodulus : 0, &st));
    if (verbose) {
        printf(" FINAL EIGVALS:\n");
        for (int j = 0; j < nev; ++j) printf("%20.12f%20.12f\n", e[j].re, e[j].im);
        fflush(stdout);
    }
    if (in->writevecs) DE_TRY(de_write_vectors(in->outvecfile, m, nev, psi_c));
    if (x) std::memcpy(x, psi.data(), (size_t)d * nev * sizeof(cplx));
    if (info) {
        std::memset(info, 0, sizeof *info);
        info->totget = totget;
        info->nexpects = nuse;
        for (int j = 0; j < nuse; ++j) {
            info->e0[j] = de_complex{e0[j].real(), e0[j].imag()};
            info->expects[j] = de_complex{expects[j].real(), expects[j].imag()};
        }
        info->shift = de_complex{shift.real(), shift.imag()};
        info->stats = st;
    }
    return DE_OK;
}
