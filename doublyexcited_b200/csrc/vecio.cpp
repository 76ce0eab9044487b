// vecio.cpp -- eigenvector files in the reference's Fortran unformatted
// sequential format.
//
// Reference: READWRITE_EIGENVECTORS utils.F90:82-184 and SIXD_FIX :186-198.
// Layout written by gfortran: every record is framed by 4-byte length
// markers; a record longer than 2147483639 bytes is split into sub-records
// whose leading marker is negative when another sub-record follows and
// whose trailing marker is negative when a sub-record precedes it.
//   record 1: int32 M, int32 NUM, int64 SIZEOF(ALLPSI) = 16*M*M
//   records 2..NUM+1: M*M complex*16, electron 1 fastest.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "de_internal.h"

using namespace de;

namespace {

constexpr int64_t kMaxSub = 2147483639LL;

struct File {
    FILE *f = nullptr;
    ~File()
    {
        if (f) fclose(f);
    }
};

int write_record(FILE *f, const void *data, int64_t bytes)
{
    const char *p = (const char *)data;
    int64_t left = bytes;
    bool first = true;
    do {
        const int64_t n = std::min(left, kMaxSub);
        const bool more = left > n;
        int32_t lead = (int32_t)(more ? -n : n), trail = (int32_t)(first ? n : -n);
        if (fwrite(&lead, 4, 1, f) != 1) return DE_E_IO;
        if (n && fwrite(p, 1, (size_t)n, f) != (size_t)n) return DE_E_IO;
        if (fwrite(&trail, 4, 1, f) != 1) return DE_E_IO;
        p += n;
        left -= n;
        first = false;
    } while (left > 0);
    return DE_OK;
}

// Reads one logical record into out (resized); returns DE_OK or DE_E_IO.
int read_record(FILE *f, std::vector<char> &out, int64_t limit)
{
    out.clear();
    while (true) {
        int32_t lead = 0, trail = 0;
        if (fread(&lead, 4, 1, f) != 1) return DE_E_IO;
        const int64_t n = lead < 0 ? -(int64_t)lead : lead;
        if ((int64_t)out.size() + n > limit) return DE_E_IO;
        const size_t o = out.size();
        out.resize(o + (size_t)n);
        if (n && fread(out.data() + o, 1, (size_t)n, f) != (size_t)n) return DE_E_IO;
        if (fread(&trail, 4, 1, f) != 1) return DE_E_IO;
        if ((trail < 0 ? -(int64_t)trail : trail) != n) return DE_E_IO;
        if (lead >= 0) return DE_OK;
    }
}

int odd_cube_root(int64_t m)
{
    const int r = (int)std::floor(std::cbrt((double)m) + 0.5);
    if ((int64_t)r * r * r != m || r % 2 != 1) return -1;
    return r;
}

}  // namespace

extern "C" {

DE_API int de_write_vectors(const char *path, int64_t m, int num, const de_complex *psi)
{
    if (!path || !psi || m < 1 || num < 0) return set_error(DE_E_INVALID, "bad argument");
    File F;
    F.f = fopen(path, "wb");
    if (!F.f) return set_error(DE_E_IO, "cannot open %s for writing", path);
    struct {
        int32_t m, num;
        int64_t sz;
    } __attribute__((packed)) hdr{(int32_t)m, (int32_t)num, (int64_t)16 * m * m};
    if (write_record(F.f, &hdr, sizeof hdr) != DE_OK) return set_error(DE_E_IO, "write failed: %s", path);
    for (int v = 0; v < num; ++v)
        if (write_record(F.f, psi + (int64_t)v * m * m, 16 * m * m) != DE_OK)
            return set_error(DE_E_IO, "write failed: %s", path);
    return DE_OK;
}

DE_API int de_vectors_header(const char *path, int64_t *m, int *num)
{
    if (!path) return set_error(DE_E_INVALID, "null path");
    File F;
    F.f = fopen(path, "rb");
    if (!F.f) return set_error(DE_E_IO, "cannot open %s", path);
    std::vector<char> rec;
    if (read_record(F.f, rec, 64) != DE_OK || rec.size() != 16) return set_error(DE_E_IO, "bad header record in %s", path);
    int32_t mi, ni;
    std::memcpy(&mi, rec.data(), 4);
    std::memcpy(&ni, rec.data() + 4, 4);
    if (m) *m = mi;
    if (num) *num = ni;
    return DE_OK;
}

DE_API int de_read_vectors(const char *path, int64_t m, int num, de_complex *psi)
{
    if (!path || !psi || m < 1 || num < 0) return set_error(DE_E_INVALID, "bad argument");
    File F;
    F.f = fopen(path, "rb");
    if (!F.f) return set_error(DE_E_IO, "cannot open %s", path);
    std::vector<char> rec;
    if (read_record(F.f, rec, 64) != DE_OK || rec.size() != 16) return set_error(DE_E_IO, "bad header record in %s", path);
    int32_t m_in, num_in;
    int64_t insz;
    std::memcpy(&m_in, rec.data(), 4);
    std::memcpy(&num_in, rec.data() + 4, 4);
    std::memcpy(&insz, rec.data() + 8, 8);
    const int nn_here = odd_cube_root(m), nn_there = odd_cube_root(m_in);
    const bool fix = (m_in != m);
    if (fix && (nn_here < 0 || nn_there < 0))
        return set_error(DE_E_IO, "I DON'T UNDERSTAND %lld %d", (long long)m, (int)m_in);
    if (insz != (int64_t)16 * m_in * m_in)
        return set_error(DE_E_IO, "BOOGA STOP 8842 CODE BANANA. %lld %lld", (long long)insz, (long long)16 * m_in * m_in);
    if (num > num_in) return set_error(DE_E_IO, "%s holds %d vectors, %d requested", path, num_in, num);
    const int n_here = (nn_here - 1) / 2, n_there = (nn_there - 1) / 2;
    const int nmin = std::min(n_here, n_there);
    for (int v = 0; v < num; ++v) {
        if (read_record(F.f, rec, (int64_t)16 * m_in * m_in) != DE_OK || (int64_t)rec.size() != (int64_t)16 * m_in * m_in)
            return set_error(DE_E_IO, "short vector record %d in %s", v + 1, path);
        de_complex *out = psi + (int64_t)v * m * m;
        if (!fix) {
            std::memcpy(out, rec.data(), rec.size());
            continue;
        }
        // SIXD_FIX: zero-pad / crop the 6-D array about its centre
        std::memset(out, 0, (size_t)m * m * sizeof(de_complex));
        const de_complex *in = (const de_complex *)rec.data();
        const int64_t nt = nn_there, nh = nn_here;
        for (int k2 = -nmin; k2 <= nmin; ++k2)
            for (int j2 = -nmin; j2 <= nmin; ++j2)
                for (int i2 = -nmin; i2 <= nmin; ++i2)
                    for (int k1 = -nmin; k1 <= nmin; ++k1)
                        for (int j1 = -nmin; j1 <= nmin; ++j1)
                            for (int i1 = -nmin; i1 <= nmin; ++i1) {
                                const int64_t pt = (i1 + n_there) + nt * ((j1 + n_there) + nt * (k1 + n_there));
                                const int64_t qt = (i2 + n_there) + nt * ((j2 + n_there) + nt * (k2 + n_there));
                                const int64_t ph = (i1 + n_here) + nh * ((j1 + n_here) + nh * (k1 + n_here));
                                const int64_t qh = (i2 + n_here) + nh * ((j2 + n_here) + nh * (k2 + n_here));
                                out[ph + m * qh] = in[pt + (int64_t)m_in * qt];
                            }
    }
    return DE_OK;
}

}  // extern "C"
