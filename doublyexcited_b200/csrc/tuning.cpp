// tuning.cpp -- the matvec tuning table: which kernel family and how many
// resident CTAs per SM each pass of each grid runs with.
//
// The table is text, one entry per line (blank lines and '#' comments are
// skipped):
//
//     <storage> <NN> <pass> <family> <ctas_per_sm> [ms_per_vector ...]
//
// storage "c128" or "c64", pass "A" or "B", family "ev", "dmma", "stream" or
// "tf32" (see HamDev::fam), ctas_per_sm 0 for as many as fit; anything after
// the fifth field (the measured time) is ignored.  `python -m
// doublyexcited_b200.tune` writes it from timings on the GPU.  A problem
// handle reads it at creation: the file DE_MATVEC_TUNING names (set but
// empty: no table), else matvec_tuning.txt beside the library.  Grids,
// passes or files without an entry keep the built-in choice (even/odd
// kernels where built, all resident CTAs).
#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "de_kernels.h"

namespace de {
namespace {

using Key = std::tuple<int, int, int>;  // storage, NN, pass
struct Choice {
    int fam, ctas;
};
using Table = std::map<Key, Choice>;

int family_code(const char *s)
{
    if (!std::strcmp(s, "ev")) return 0;
    if (!std::strcmp(s, "dmma")) return 1;
    if (!std::strcmp(s, "stream")) return 2;
    if (!std::strcmp(s, "tf32")) return 3;
    return -1;
}

// Parses path; false when the file cannot be read.  Malformed lines are
// skipped.
bool parse(const std::string &path, Table &t)
{
    FILE *f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    char line[512];
    while (std::fgets(line, sizeof line, f)) {
        char *hash = std::strchr(line, '#');
        if (hash) *hash = 0;
        char sto[16], pass[16], fam[16];
        int nn = 0, ctas = 0;
        if (std::sscanf(line, "%15s %d %15s %15s %d", sto, &nn, pass, fam, &ctas) != 5) continue;
        const int s = !std::strcmp(sto, "c128") ? 0 : !std::strcmp(sto, "c64") ? 1 : -1;
        const int p = !std::strcmp(pass, "A") ? 0 : !std::strcmp(pass, "B") ? 1 : -1;
        const int fc = family_code(fam);
        if (s < 0 || p < 0 || fc < 0 || nn < 3 || nn > kMaxNN || ctas < 0 || ctas > 32) continue;
        t[Key{s, nn, p}] = Choice{fc, ctas};
    }
    std::fclose(f);
    return true;
}

std::mutex g_mu;
std::map<std::string, Table> g_cache;

const Table *cached(const std::string &path)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_cache.find(path);
    if (it == g_cache.end()) {
        Table t;
        if (!parse(path, t)) return nullptr;
        it = g_cache.emplace(path, std::move(t)).first;
    }
    return &it->second;
}

std::string default_path()
{
    const char *env = std::getenv("DE_MATVEC_TUNING");
    if (env) return env;  // "" = no table
    Dl_info info{};
    if (!dladdr(reinterpret_cast<void *>(&default_path), &info) || !info.dli_fname) return "";
    std::string lib = info.dli_fname;
    const size_t slash = lib.rfind('/');
    return (slash == std::string::npos ? std::string(".") : lib.substr(0, slash)) + "/matvec_tuning.txt";
}

}  // namespace

bool tuning_lookup(const char *path, int storage, int nn, int pass, int &fam, int &ctas)
{
    const Table *t = path ? cached(path) : nullptr;
    if (!t) return false;
    auto it = t->find(Key{storage, nn, pass});
    if (it == t->end()) return false;
    fam = it->second.fam;
    ctas = it->second.ctas;
    return true;
}

void apply_tuning(HamDev &h)
{
    const std::string path = default_path();
    for (int s = 0; s < 2; ++s)
        for (int p = 0; p < 2; ++p) {
            int fam = 0, ctas = 0;
            if (!path.empty()) tuning_lookup(path.c_str(), s, h.nn, p, fam, ctas);
            h.fam[s][p] = (signed char)fam;
            h.ctas[s][p] = (signed char)ctas;
        }
}

}  // namespace de
