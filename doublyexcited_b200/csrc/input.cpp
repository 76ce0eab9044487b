// input.cpp -- Input.Inp namelist reader and command-line keys.
//
// Reference: module INPUT defaults input.F90:1-124, get_input :143-254
// (seven namelists, each read from the start of the file; a missing group
// keeps its defaults), get_inputfile :257-276 and get_args :278-362.
// Fortran namelist rules honoured here: case-insensitive names, '!'
// comments, values separated by blanks/commas/newlines, the LAST assignment
// of a name wins (Input.Inp files rely on it), d/D exponents, .TRUE./T
// logicals, quoted strings and (re,im) complex constants.  An unknown name
// inside a group is an error (DE_E_PARSE); the reference's read would stop
// at that point with a non-zero IOSTAT.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "de_internal.h"

using namespace de;

namespace {

std::string upper(std::string s)
{
    for (auto &c : s) c = (char)std::toupper((unsigned char)c);
    return s;
}

std::string trim(const std::string &s)
{
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

bool parse_real(std::string v, double &out)
{
    v = trim(v);
    for (auto &c : v)
        if (c == 'd' || c == 'D') c = 'e';
    if (v.empty()) return false;
    char *end = nullptr;
    out = std::strtod(v.c_str(), &end);
    return end && *end == '\0';
}

bool parse_int(const std::string &v, int &out)
{
    std::string t = trim(v);
    if (t.empty()) return false;
    char *end = nullptr;
    long x = std::strtol(t.c_str(), &end, 10);
    if (!end || *end != '\0') return false;
    out = (int)x;
    return true;
}

bool parse_logical(const std::string &v, int &out)
{
    std::string t = upper(trim(v));
    size_t i = 0;
    if (i < t.size() && t[i] == '.') ++i;
    if (i >= t.size()) return false;
    if (t[i] == 'T') out = 1;
    else if (t[i] == 'F') out = 0;
    else return false;
    return true;
}

bool parse_complex(const std::string &v, de_complex &out)
{
    std::string t = trim(v);
    if (!t.empty() && t.front() == '(') {
        if (t.back() != ')') return false;
        std::string in = t.substr(1, t.size() - 2);
        size_t c = in.find(',');
        if (c == std::string::npos) return false;
        double re, im;
        if (!parse_real(in.substr(0, c), re) || !parse_real(in.substr(c + 1), im)) return false;
        out = de_complex{re, im};
        return true;
    }
    double re;
    if (!parse_real(t, re)) return false;
    out = de_complex{re, 0.0};
    return true;
}

bool parse_string(const std::string &v, char *dst, size_t cap)
{
    std::string t = trim(v);
    if (t.size() >= 2 && (t.front() == '\'' || t.front() == '"') && t.back() == t.front())
        t = t.substr(1, t.size() - 2);
    if (t.size() + 1 > cap) return false;
    std::memcpy(dst, t.c_str(), t.size() + 1);
    return true;
}

// Split "a=1, b = (1,2) c='x y'" into name/value pairs.
bool split_assignments(const std::string &body, std::vector<std::pair<std::string, std::string>> &out,
                       std::string &err)
{
    size_t i = 0, n = body.size();
    auto skip = [&]() {
        while (i < n && (std::isspace((unsigned char)body[i]) || body[i] == ',')) ++i;
    };
    while (true) {
        skip();
        if (i >= n) return true;
        size_t s = i;
        while (i < n && (std::isalnum((unsigned char)body[i]) || body[i] == '_' || body[i] == '%')) ++i;
        std::string name = body.substr(s, i - s);
        if (name.empty()) {
            err = "unexpected character '" + std::string(1, body[i]) + "'";
            return false;
        }
        while (i < n && std::isspace((unsigned char)body[i])) ++i;
        if (i >= n || body[i] != '=') {
            err = "expected '=' after " + name;
            return false;
        }
        ++i;
        while (i < n && std::isspace((unsigned char)body[i])) ++i;
        size_t v0 = i;
        if (i < n && (body[i] == '\'' || body[i] == '"')) {
            char q = body[i++];
            while (i < n && body[i] != q) ++i;
            if (i < n) ++i;
        } else if (i < n && body[i] == '(') {
            while (i < n && body[i] != ')') ++i;
            if (i < n) ++i;
        } else {
            while (i < n && !std::isspace((unsigned char)body[i]) && body[i] != ',') ++i;
        }
        out.emplace_back(upper(name), body.substr(v0, i - v0));
    }
}

// Text of group &name ... / (first occurrence), comments removed.
bool find_group(const std::string &text, const std::string &group, std::string &body)
{
    const std::string U = upper(text);
    const std::string key = "&" + upper(group);
    size_t p = 0;
    while ((p = U.find(key, p)) != std::string::npos) {
        size_t e = p + key.size();
        if (e < U.size() && (std::isalnum((unsigned char)U[e]) || U[e] == '_')) {
            p = e;
            continue;
        }
        // body ends at the first '/' outside quotes, or at &END
        size_t i = e;
        char q = 0;
        for (; i < text.size(); ++i) {
            char c = text[i];
            if (q) {
                if (c == q) q = 0;
            } else if (c == '\'' || c == '"') {
                q = c;
            } else if (c == '/') {
                break;
            } else if (c == '&' && U.compare(i, 4, "&END") == 0) {
                break;
            }
        }
        body = text.substr(e, i - e);
        return true;
    }
    return false;
}

std::string strip_comments(const std::string &text)
{
    std::string out;
    out.reserve(text.size());
    char q = 0;
    for (size_t i = 0; i < text.size(); ++i) {
        char c = text[i];
        if (q) {
            if (c == q) q = 0;
            out += c;
        } else if (c == '\'' || c == '"') {
            q = c;
            out += c;
        } else if (c == '!') {
            while (i < text.size() && text[i] != '\n') ++i;
            out += '\n';
        } else {
            out += c;
        }
    }
    return out;
}

struct Field {
    const char *name;
    enum Kind { kInt, kReal, kLog, kStr, kCplx, kIgnoreInt, kIgnoreReal, kIgnoreLog, kIgnoreStr } kind;
    void *ptr;
    size_t cap;
};

int apply(const char *group, const std::string &body, const std::vector<Field> &fields)
{
    std::vector<std::pair<std::string, std::string>> kv;
    std::string err;
    if (!split_assignments(body, kv, err)) return set_error(DE_E_PARSE, "namelist %s: %s", group, err.c_str());
    for (auto &a : kv) {
        const Field *f = nullptr;
        for (auto &c : fields)
            if (upper(c.name) == a.first) f = &c;
        if (!f) return set_error(DE_E_PARSE, "namelist %s: unknown name %s", group, a.first.c_str());
        bool ok = true;
        int iv;
        double dv;
        char sbuf[300];
        switch (f->kind) {
        case Field::kInt: ok = parse_int(a.second, *(int *)f->ptr); break;
        case Field::kReal: ok = parse_real(a.second, *(double *)f->ptr); break;
        case Field::kLog: ok = parse_logical(a.second, *(int *)f->ptr); break;
        case Field::kStr: ok = parse_string(a.second, (char *)f->ptr, f->cap); break;
        case Field::kCplx: ok = parse_complex(a.second, *(de_complex *)f->ptr); break;
        case Field::kIgnoreInt: ok = parse_int(a.second, iv); break;
        case Field::kIgnoreReal: ok = parse_real(a.second, dv); break;
        case Field::kIgnoreLog: ok = parse_logical(a.second, iv); break;
        case Field::kIgnoreStr: ok = parse_string(a.second, sbuf, sizeof sbuf); break;
        }
        if (!ok) return set_error(DE_E_PARSE, "namelist %s: bad value for %s: '%s'", group, a.first.c_str(), a.second.c_str());
    }
    return DE_OK;
}

bool starts(const std::string &s, const char *p) { return s.compare(0, std::strlen(p), p) == 0; }

std::string list_token(const std::string &s)
{
    std::string t = trim(s);
    if (!t.empty() && (t.front() == '\'' || t.front() == '"')) {
        size_t e = t.find(t.front(), 1);
        return t.substr(1, e == std::string::npos ? std::string::npos : e - 1);
    }
    size_t e = t.find_first_of(" ,/");
    return t.substr(0, e);
}

}  // namespace

extern "C" {

DE_API void de_input_default(de_input *in)
{
    if (!in) return;
    std::memset(in, 0, sizeof *in);
    de_params_default(&in->params);
    in->gmres.max_inner_iter = 5;
    in->gmres.usepetscflag = 1;
    in->gmres.tol = 1e-3;
    in->gmres.compat_first_column_only = 0;
    in->writevecs = 0;
    in->readvecs = 0;
    std::strcpy(in->invecfile, "eigvecs");
    std::strcpy(in->outvecfile, "eigvecs");
    in->numorbs = 14;
    in->singlet = 0;
    in->numskip = 0;
    in->outmodulus = 5;
    in->takerealpart = 1;
    in->hermopt = 0;
    in->cshiftopt = 0;
    in->gplmr_nev = 1;
    in->gplmr_ns = 5;
    in->gplmr_maxit = 100;
    in->gplmr_tol = 1e-12;
    in->gplmr_shift = de_complex{-999.0, 0.0};
    in->kdim = 2001;
    in->lanblocksize = 3;
    in->check = 10;
    in->lantol = 1e-6;
}

DE_API int de_input_file_arg(int argc, const char *const *argv, char *buf, size_t len)
{
    if (!buf || len == 0) return set_error(DE_E_INVALID, "null buffer");
    std::string f = "Input.Inp";
    for (int i = 0; argv && i < argc; ++i) {
        std::string a = trim(argv[i] ? argv[i] : "");
        if (starts(a, "Inp=")) f = a.substr(4);
    }
    if (f.size() + 1 > len) return set_error(DE_E_INVALID, "buffer too small");
    std::memcpy(buf, f.c_str(), f.size() + 1);
    return DE_OK;
}

DE_API int de_read_input(const char *path, int argc, const char *const *argv, de_input *in)
{
    if (!in) return set_error(DE_E_INVALID, "null input struct");
    de_params &p = in->params;
    int charge_i = (int)p.charge;
    int nuc_on_grid = 1, nuclei = 1, numpoints = 10;
    if (path && path[0]) {
        std::ifstream f(path);
        if (f) {  // a missing file keeps every default (get_input :203-208)
            std::stringstream ss;
            ss << f.rdbuf();
            const std::string text = strip_comments(ss.str());
            std::string body;
            int theta_set = 0;
            (void)theta_set;
            if (find_group(text, "main", body)) {
                std::vector<Field> fs = {
                    {"STRETCH", Field::kIgnoreLog, nullptr, 0},
                    {"MODBASIS", Field::kIgnoreLog, nullptr, 0},
                    {"VQUAD", Field::kIgnoreLog, nullptr, 0},
                    {"WRITEVALS", Field::kIgnoreLog, nullptr, 0},
                    {"WRITEVECS", Field::kLog, &in->writevecs, 0},
                    {"READVECS", Field::kLog, &in->readvecs, 0},
                    {"INVECFILE", Field::kStr, in->invecfile, sizeof in->invecfile},
                    {"OUTVECFILE", Field::kStr, in->outvecfile, sizeof in->outvecfile},
                    {"CORRFILE", Field::kIgnoreStr, nullptr, 0},
                    {"ENERGY_CURVE_FILE", Field::kIgnoreStr, nullptr, 0},
                    {"THETA", Field::kReal, &p.theta, 0}};
                DE_TRY(apply("main", body, fs));
            }
            if (find_group(text, "grid", body)) {
                std::vector<Field> fs = {{"N", Field::kInt, &p.n, 0},
                                         {"DELTA", Field::kReal, &p.delta, 0},
                                         {"NSMALL", Field::kInt, &p.nsmall, 0},
                                         {"TFACTOR", Field::kInt, &p.tfactor, 0},
                                         {"NCOR", Field::kIgnoreInt, nullptr, 0},
                                         {"RADIUS", Field::kReal, &p.radius, 0},
                                         {"AUTODELTA", Field::kLog, &p.autodelta, 0}};
                DE_TRY(apply("grid", body, fs));
            }
            if (find_group(text, "molecule", body)) {
                std::vector<Field> fs = {{"NUCLEI", Field::kInt, &nuclei, 0},
                                         {"CHARGE", Field::kInt, &charge_i, 0},
                                         {"NUMPOINTS", Field::kInt, &numpoints, 0},
                                         {"NUC_ON_GRID", Field::kLog, &nuc_on_grid, 0}};
                DE_TRY(apply("molecule", body, fs));
            }
            if (find_group(text, "lanczos", body)) {
                std::vector<Field> fs = {{"KDIM", Field::kInt, &in->kdim, 0},
                                         {"LANBLOCKSIZE", Field::kInt, &in->lanblocksize, 0},
                                         {"CHECK", Field::kInt, &in->check, 0},
                                         {"LANTOL", Field::kReal, &in->lantol, 0}};
                DE_TRY(apply("lanczos", body, fs));
            }
            if (find_group(text, "gmres", body)) {
                int maxrst = 0, pout = 0;
                std::vector<Field> fs = {{"GM_USEPETSCFLAG", Field::kInt, &in->gmres.usepetscflag, 0},
                                         {"GM_MAX_INNER_ITER", Field::kInt, &in->gmres.max_inner_iter, 0},
                                         {"GM_MAXRST", Field::kInt, &maxrst, 0},
                                         {"GM_PRINT_OUTPUT", Field::kLog, &pout, 0},
                                         {"GM_TOL", Field::kReal, &in->gmres.tol, 0}};
                DE_TRY(apply("gmres", body, fs));
            }
            if (find_group(text, "orbitals", body)) {
                std::vector<Field> fs = {{"NUMORBS", Field::kInt, &in->numorbs, 0},
                                         {"SINGLET", Field::kLog, &in->singlet, 0},
                                         {"NUMSKIP", Field::kInt, &in->numskip, 0}};
                DE_TRY(apply("orbitals", body, fs));
            }
            if (find_group(text, "gplmr", body)) {
                std::vector<Field> fs = {{"OUTMODULUS", Field::kInt, &in->outmodulus, 0},
                                         {"TAKEREALPART", Field::kLog, &in->takerealpart, 0},
                                         {"HERMOPT", Field::kLog, &in->hermopt, 0},
                                         {"CSHIFTOPT", Field::kLog, &in->cshiftopt, 0},
                                         {"GPLMR_NEV", Field::kInt, &in->gplmr_nev, 0},
                                         {"GPLMR_NS", Field::kInt, &in->gplmr_ns, 0},
                                         {"GPLMR_MAXIT", Field::kInt, &in->gplmr_maxit, 0},
                                         {"GPLMR_TOL", Field::kReal, &in->gplmr_tol, 0},
                                         {"GPLMR_SHIFT", Field::kCplx, &in->gplmr_shift, 0}};
                DE_TRY(apply("gplmr", body, fs));
            }
        }
    }
    p.charge = charge_i;
    if (nuclei != 1 || !nuc_on_grid)
        return set_error(DE_E_UNSUPPORTED, "only one nucleus on the grid (NUCLEI=1, NUC_ON_GRID) is built");
    // command-line keys (get_args input.F90:278-362), in order
    for (int i = 0; argv && i < argc; ++i) {
        const std::string a = trim(argv[i] ? argv[i] : "");
        auto num = [&](size_t off, auto &dst) -> int {
            const std::string v = list_token(a.substr(off));
            bool ok;
            if constexpr (std::is_same<std::decay_t<decltype(dst)>, int>::value) ok = parse_int(v, dst);
            else ok = parse_real(v, dst);
            return ok ? DE_OK : set_error(DE_E_PARSE, "bad argument '%s'", a.c_str());
        };
        if (starts(a, "N=")) DE_TRY(num(2, p.n));
        if (starts(a, "Shift=")) {
            if (!parse_complex(a.substr(6), in->gplmr_shift)) return set_error(DE_E_PARSE, "bad argument '%s'", a.c_str());
        }
        if (starts(a, "Outfile=")) parse_string(list_token(a.substr(8)), in->outvecfile, sizeof in->outvecfile);
        if (starts(a, "Infile=")) parse_string(list_token(a.substr(7)), in->invecfile, sizeof in->invecfile);
        if (starts(a, "NoPetsc")) in->gmres.usepetscflag = 0;
        if (starts(a, "Petsc")) in->gmres.usepetscflag = 1;
        if (starts(a, "Theta=")) DE_TRY(num(6, p.theta));
        if (starts(a, "R=")) {
            p.autodelta = 1;
            DE_TRY(num(2, p.radius));
        }
        if (starts(a, "Delta=")) {
            p.autodelta = 0;
            DE_TRY(num(6, p.delta));
        }
        if (starts(a, "Nev=")) DE_TRY(num(4, in->gplmr_nev));
        if (starts(a, "Norbs=")) DE_TRY(num(6, in->numorbs));
        if (starts(a, "Gptol=")) DE_TRY(num(6, in->gplmr_tol));
        if (starts(a, "Skip=")) DE_TRY(num(5, in->numskip));
        if (starts(a, "Gmtol=")) DE_TRY(num(6, in->gmres.tol));
        if (starts(a, "Iter=")) DE_TRY(num(5, in->gmres.max_inner_iter));
        if (starts(a, "Read")) {
            in->numskip = 0;
            in->readvecs = 1;
        }
        if (starts(a, "Takereal")) in->takerealpart = 1;
        if (starts(a, "Notakereal")) in->takerealpart = 0;
        if (starts(a, "Sing")) in->singlet = 1;
        if (starts(a, "Trip")) in->singlet = 0;
    }
    return DE_OK;
}

}  // extern "C"
