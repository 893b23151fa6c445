// Batched XYZ ingestion: many .xyz files parsed on host threads straight into
// one packed ragged buffer (charges (A,), coords (A, 3), offsets (M + 1,)),
// the layout every descriptor launch reads. The caller passes page-locked
// buffers, so one asynchronous host-to-device copy per array follows.
//
// Parsing rules of Molecule.read_xyz (fml/fml.py:109-132):
//   * the file is split into lines on \n, \r\n or \r (Python text mode);
//   * line 1 holds the declared atom count (int(lines[0]));
//   * line 2 is a comment;
//   * from line 3 on, each line is split on whitespace; the first line with
//     fewer than 4 tokens ends the atom list; otherwise token 1 is the element
//     symbol (looked up in the caller's charge table, NUCLEAR_CHARGE of
//     fml/data.py) and tokens 2-4 are x, y, z (float()).
// Whitespace and number syntax follow Python's str.split(), int() and float()
// for ASCII text: tokens split on space, \t, \v, \f and \x1c-\x1f; int()
// strips space, \t, \v and \f around the count; numbers are an optional
// sign and decimal digits with single underscores between digits (PEP 515),
// for float() also a fraction, an exponent, or inf / infinity / nan in any
// case. Non-ASCII digits and whitespace, which Python also accepts, are
// rejected, and so are declared counts outside the int32 range.
// The atom list length, not the declared count, sizes the molecule, as in
// the reference (natoms is only stored).
#include <ctype.h>
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "fmlb.h"

namespace fmlb {
void set_error(const char *fmt, ...);
}

namespace {

bool read_file(const char *path, std::string &out) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    out.clear();
    char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) out.append(buf, n);
    const bool ok = !ferror(f);
    fclose(f);
    return ok;
}

// Splits text into lines like Python's universal newlines.
void split_lines(const std::string &s, std::vector<std::pair<size_t, size_t>> &lines) {
    lines.clear();
    size_t b = 0, i = 0;
    const size_t n = s.size();
    while (i < n) {
        if (s[i] == '\n' || s[i] == '\r') {
            lines.emplace_back(b, i);
            if (s[i] == '\r' && i + 1 < n && s[i + 1] == '\n') ++i;
            b = ++i;
        } else {
            ++i;
        }
    }
    if (b < n) lines.emplace_back(b, n);
}

// ASCII whitespace of Python's str.split() (newlines never occur inside a line)
bool is_ws(char c) {
    return c == ' ' || c == '\t' || c == '\v' || c == '\f' || (c >= '\x1c' && c <= '\x1f');
}

// Whitespace tokens of s[b, e), at most 4 (the rest are ignored).
int tokens(const std::string &s, size_t b, size_t e, std::string tok[4]) {
    int k = 0;
    size_t i = b;
    while (i < e) {
        while (i < e && is_ws(s[i])) ++i;
        if (i >= e) break;
        const size_t t0 = i;
        while (i < e && !is_ws(s[i])) ++i;
        if (k < 4) tok[k] = s.substr(t0, i - t0);
        ++k;
    }
    return k;
}

bool is_digit(char c) { return c >= '0' && c <= '9'; }

// Removes the digit-group underscores of a PEP 515 literal into `out`; false
// when an underscore does not sit between two digits.
bool strip_underscores(const std::string &t, std::string &out) {
    out.clear();
    for (size_t i = 0; i < t.size(); ++i) {
        if (t[i] != '_') {
            out.push_back(t[i]);
            continue;
        }
        if (i == 0 || i + 1 == t.size() || !is_digit(t[i - 1]) || !is_digit(t[i + 1]))
            return false;
    }
    return true;
}

bool equals_nocase(const char *a, size_t n, const char *word) {
    if (strlen(word) != n) return false;
    for (size_t i = 0; i < n; ++i)
        if (tolower((unsigned char)a[i]) != word[i]) return false;
    return true;
}

// float() of one token (no surrounding whitespace): [sign] then inf, infinity
// or nan in any case, or digits [. digits] / . digits with an optional
// exponent e[sign]digits. The value comes from strtod on the validated text
// (correctly rounded, like Python's own conversion).
bool parse_double(const std::string &tok, double &v) {
    std::string t;
    if (tok.empty() || !strip_underscores(tok, t)) return false;
    const char *p = t.c_str();
    size_t i = (t[0] == '+' || t[0] == '-') ? 1 : 0;
    const size_t rest = t.size() - i;
    if (equals_nocase(p + i, rest, "inf") || equals_nocase(p + i, rest, "infinity") ||
        equals_nocase(p + i, rest, "nan")) {
        v = strtod(p, nullptr);
        return true;
    }
    size_t digits = 0;
    while (i < t.size() && is_digit(t[i])) ++i, ++digits;
    if (i < t.size() && t[i] == '.') {
        ++i;
        while (i < t.size() && is_digit(t[i])) ++i, ++digits;
    }
    if (digits == 0) return false;
    if (i < t.size() && (t[i] == 'e' || t[i] == 'E')) {
        ++i;
        if (i < t.size() && (t[i] == '+' || t[i] == '-')) ++i;
        size_t exp_digits = 0;
        while (i < t.size() && is_digit(t[i])) ++i, ++exp_digits;
        if (exp_digits == 0) return false;
    }
    if (i != t.size()) return false;
    v = strtod(p, nullptr);
    return true;
}

// The whitespace int() strips around its argument: C isspace, narrower than
// str.split()'s (\x1c-\x1f are not stripped)
bool is_strip_ws(char c) { return c == ' ' || c == '\t' || c == '\v' || c == '\f'; }

// int() of s[b, e): surrounding whitespace, [sign] digits with PEP 515
// underscores; values outside the int32 range are rejected.
bool parse_int(const std::string &s, size_t b, size_t e, int &v) {
    while (b < e && is_strip_ws(s[b])) ++b;
    while (e > b && is_strip_ws(s[e - 1])) --e;
    if (b == e) return false;
    std::string t;
    if (!strip_underscores(s.substr(b, e - b), t)) return false;
    size_t i = (t[0] == '+' || t[0] == '-') ? 1 : 0;
    if (i == t.size()) return false;
    for (size_t k = i; k < t.size(); ++k)
        if (!is_digit(t[k])) return false;
    errno = 0;
    const long long x = strtoll(t.c_str(), nullptr, 10);
    if (errno || x < -2147483647LL || x > 2147483647LL) return false;
    v = (int)x;
    return true;
}

struct FileResult {
    int rc = 0;          // 0, or an FMLB_* code
    int line = 0;        // 1-based line of the failure
    std::string what;    // failing token
    int declared = 0;
    int parsed = 0;
};

// Parses one file. With `charges` null only counts the atom lines.
void parse_one(const char *path, const std::unordered_map<std::string, int> *table,
               const double *table_charges, double *charges, double *coords, int *symbol_index,
               int capacity, FileResult &r) {
    std::string text;
    if (!read_file(path, text)) {
        r.rc = FMLB_EINVAL;
        r.what = "cannot read file";
        return;
    }
    std::vector<std::pair<size_t, size_t>> lines;
    split_lines(text, lines);
    if (lines.empty() || !parse_int(text, lines[0].first, lines[0].second, r.declared)) {
        r.rc = FMLB_EINVAL;
        r.line = 1;
        r.what = lines.empty() ? "empty file" : text.substr(lines[0].first,
                                                          lines[0].second - lines[0].first);
        return;
    }
    std::string tok[4];
    int a = 0;
    for (size_t li = 2; li < lines.size(); ++li) {
        if (tokens(text, lines[li].first, lines[li].second, tok) < 4) break;
        if (charges) {
            if (a >= capacity) {
                r.rc = FMLB_EINVAL;
                r.line = (int)li + 1;
                r.what = "more atom lines than at the first pass";
                return;
            }
            auto it = table->find(tok[0]);
            if (it == table->end()) {
                r.rc = FMLB_EINVAL;
                r.line = (int)li + 1;
                r.what = "unknown element " + tok[0];
                return;
            }
            double xyz[3];
            for (int c = 0; c < 3; ++c) {
                if (!parse_double(tok[1 + c], xyz[c])) {
                    r.rc = FMLB_EINVAL;
                    r.line = (int)li + 1;
                    r.what = "not a number: " + tok[1 + c];
                    return;
                }
            }
            charges[a] = table_charges[it->second];
            coords[3 * (size_t)a + 0] = xyz[0];
            coords[3 * (size_t)a + 1] = xyz[1];
            coords[3 * (size_t)a + 2] = xyz[2];
            if (symbol_index) symbol_index[a] = it->second;
        }
        ++a;
    }
    r.parsed = a;
}

template <class F>
void parallel_for(int n, int nthreads, F fn) {
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    nthreads = std::min(nthreads, std::max(n, 1));
    std::atomic<int> next(0);
    auto work = [&] {
        for (int i = next++; i < n; i = next++) fn(i);
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; ++t) th.emplace_back(work);
    work();
    for (auto &t : th) t.join();
}

int report(const char *fn, const char *const *paths, const std::vector<FileResult> &res) {
    for (size_t i = 0; i < res.size(); ++i)
        if (res[i].rc) {
            fmlb::set_error("%s: %s line %d: %s", fn, paths[i], res[i].line, res[i].what.c_str());
            return res[i].rc;
        }
    return FMLB_OK;
}

}  // namespace

extern "C" int fmlb_xyz_scan(const char *const *paths, int nfiles, int *natoms_declared,
                             int *natoms_parsed, int nthreads) {
    if (nfiles < 0 || (nfiles > 0 && (!paths || !natoms_parsed))) {
        fmlb::set_error("fmlb_xyz_scan: bad arguments");
        return FMLB_EINVAL;
    }
    std::vector<FileResult> res(nfiles);
    parallel_for(nfiles, nthreads, [&](int i) {
        parse_one(paths[i], nullptr, nullptr, nullptr, nullptr, nullptr, 0, res[i]);
    });
    for (int i = 0; i < nfiles; ++i) {
        natoms_parsed[i] = res[i].parsed;
        if (natoms_declared) natoms_declared[i] = res[i].declared;
    }
    return report("fmlb_xyz_scan", paths, res);
}

extern "C" int fmlb_xyz_parse(const char *const *paths, int nfiles, const int *offsets,
                              const char *const *table_symbols, const double *table_charges,
                              int ntable, double *charges, double *coords, int *symbol_index,
                              int nthreads) {
    if (nfiles < 0 || ntable < 0 || (nfiles > 0 && (!paths || !offsets)) ||
        (ntable > 0 && (!table_symbols || !table_charges))) {
        fmlb::set_error("fmlb_xyz_parse: bad arguments");
        return FMLB_EINVAL;
    }
    // a batch without atoms (every file an empty molecule) needs no output
    // buffers; its files are still parsed, into a dummy of capacity zero
    double dummy[3] = {0.0, 0.0, 0.0};
    if (nfiles > 0 && offsets[nfiles] == 0) {
        if (!charges) charges = dummy;
        if (!coords) coords = dummy;
    }
    if (nfiles > 0 && (!charges || !coords)) {
        fmlb::set_error("fmlb_xyz_parse: bad arguments");
        return FMLB_EINVAL;
    }
    std::unordered_map<std::string, int> table;
    for (int t = 0; t < ntable; ++t) table.emplace(table_symbols[t], t);
    std::vector<FileResult> res(nfiles);
    parallel_for(nfiles, nthreads, [&](int i) {
        const int a0 = offsets[i], cap = offsets[i + 1] - offsets[i];
        if (a0 < 0 || cap < 0) {
            res[i].rc = FMLB_EINVAL;
            res[i].what = "bad offsets";
            return;
        }
        parse_one(paths[i], &table, table_charges, charges + a0, coords + 3 * (size_t)a0,
                  symbol_index ? symbol_index + a0 : nullptr, cap, res[i]);
        if (!res[i].rc && res[i].parsed != cap) {
            res[i].rc = FMLB_EINVAL;
            res[i].what = "atom count differs from the offsets";
        }
    });
    return report("fmlb_xyz_parse", paths, res);
}
