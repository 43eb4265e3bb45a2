// matrix_market.cu -- MatrixMarket coordinate files <-> host CSR `spmat`
// (host code; the reference test harness loads R, AC and P this way).
//
// Reading follows code/src/lib/parser.c:126-330 (MMRead -> MMtoCOO ->
// COOtoCSR, wrapped by MMtoCSR): the banner and size line as the NIST mmio
// routines read them, then "row col [value]" items read as a stream of
// whitespace-separated tokens (fscanf semantics: an item may span lines),
// 1-based indices made 0-based, pattern values 1.0, symmetric files expanded
// by mirroring every off-diagonal item right after it, and each row's
// entries kept in the file's order (the reference's default build checks no
// column order).  The file is parsed by host threads: a first pass counts
// tokens per chunk, a second parses each chunk knowing its first token's
// global index; rows are then filled by one stable pass.
//
// Where the reference has undefined behaviour this reader reports an error
// instead (NULL plus a message on stderr, the reference's error convention):
// fewer or more items than the size line declares, an index outside the
// declared shape, complex or array (dense) files, and unparsable tokens.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "sp3mm_b200.h"

namespace {

void mm_error(const char* path, const char* what) {
    fprintf(stderr, "sp3mm_b200: MatrixMarket %s: %s\n", path ? path : "(null)", what);
}

inline bool is_space(char c) {
    return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f';
}

// Host threads for n work items (one for small inputs).
int mm_threads(size_t n) {
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t per = size_t(1) << 20;
    size_t t = (n + per - 1) / per;
    if (t > 16) t = 16;
    if (hw && t > hw) t = hw;
    return t < 1 ? 1 : static_cast<int>(t);
}

template <typename F>
void mm_parallel(int t, F&& f) {
    if (t <= 1) {
        f(0);
        return;
    }
    std::vector<std::thread> th;
    for (int k = 0; k < t; ++k) th.emplace_back([&f, k] { f(k); });
    for (auto& x : th) x.join();
}

// An unsigned index token as %lu reads it: optional sign, decimal digits
// (a leading '-' negates modulo 2^64, as strtoul does).
bool parse_index(const char* b, const char* e, unsigned long long* out) {
    bool neg = false;
    if (b < e && (*b == '+' || *b == '-')) {
        neg = *b == '-';
        ++b;
    }
    if (b == e) return false;
    unsigned long long v = 0;
    for (; b < e; ++b) {
        if (*b < '0' || *b > '9') return false;
        v = v * 10 + static_cast<unsigned>(*b - '0');
    }
    *out = neg ? 0ULL - v : v;
    return true;
}

// A value token as %lf reads it (correctly rounded decimal, inf, nan; other
// forms strtod accepts, such as hexadecimal, go through strtod).
bool parse_value(const char* b, const char* e, double* out) {
    const char* s = b;
    if (s < e && *s == '+') ++s;
    auto r = std::from_chars(s, e, *out, std::chars_format::general);
    if (r.ec == std::errc() && r.ptr == e) return true;
    std::string tok(b, e);
    char* end = nullptr;
    errno = 0;
    const double v = std::strtod(tok.c_str(), &end);
    if (end != tok.c_str() + tok.size()) return false;
    *out = v;
    return true;
}

// Next line [p, eol) of [p, e); returns the start of the following line.
const char* next_line(const char* p, const char* e, const char** eol) {
    const char* q = static_cast<const char*>(memchr(p, '\n', static_cast<size_t>(e - p)));
    *eol = q ? q : e;
    return q ? q + 1 : e;
}

std::string lower(std::string s) {
    for (char& c : s) c = static_cast<char>(tolower(static_cast<unsigned char>(c)));
    return s;
}

struct Banner {
    bool pattern = false;
    bool symmetric = false;
};

// Banner line: "%%MatrixMarket object format field symmetry".
bool read_banner(const char* path, const char* b, const char* e, Banner* out) {
    char tok[5][64] = {};
    std::string line(b, e);
    if (sscanf(line.c_str(), "%63s %63s %63s %63s %63s", tok[0], tok[1], tok[2], tok[3],
               tok[4]) != 5) {
        mm_error(path, "banner line is incomplete");
        return false;
    }
    if (strcmp(tok[0], "%%MatrixMarket") != 0) {
        mm_error(path, "missing %%MatrixMarket banner");
        return false;
    }
    const std::string obj = lower(tok[1]), fmt = lower(tok[2]), field = lower(tok[3]),
                      sym = lower(tok[4]);
    if (obj != "matrix") {
        mm_error(path, "invalid matrix: not a matrix");
        return false;
    }
    if (fmt == "array") {
        mm_error(path, "invalid matrix: dense (array) files are not supported");
        return false;
    }
    if (fmt != "coordinate") {
        mm_error(path, "unsupported storage format");
        return false;
    }
    if (field == "complex") {
        mm_error(path, "complex matrices are not supported");
        return false;
    }
    if (field != "real" && field != "integer" && field != "pattern") {
        mm_error(path, "unsupported data type");
        return false;
    }
    if (sym != "general" && sym != "symmetric" && sym != "skew-symmetric" && sym != "hermitian") {
        mm_error(path, "unsupported symmetry");
        return false;
    }
    out->pattern = field == "pattern";
    // Only "symmetric" is expanded (skew-symmetric and hermitian files are
    // read as general, as the reference reads them).
    out->symmetric = sym == "symmetric";
    return true;
}

spmat* fail_free(spmat* m) {
    if (m) {
        free(m->IRP);
        free(m->JA);
        free(m->AS);
        free(m);
    }
    return nullptr;
}

}  // namespace

extern "C" {

SP3MM_API spmat* MMtoCSR(char* matPath) {
    const char* path = matPath;
    if (!path) {
        mm_error(path, "NULL path");
        return nullptr;
    }
    FILE* f = fopen(path, "rb");
    if (!f) {
        perror("fopen");
        mm_error(path, "cannot open");
        return nullptr;
    }
    std::vector<char> buf;
    {
        if (fseek(f, 0, SEEK_END) != 0) {
            fclose(f);
            mm_error(path, "cannot seek");
            return nullptr;
        }
        const long sz = ftell(f);
        if (sz < 0 || fseek(f, 0, SEEK_SET) != 0) {
            fclose(f);
            mm_error(path, "cannot size");
            return nullptr;
        }
        buf.resize(static_cast<size_t>(sz) + 1);
        const size_t got = sz > 0 ? fread(buf.data(), 1, static_cast<size_t>(sz), f) : 0;
        fclose(f);
        if (got != static_cast<size_t>(sz)) {
            mm_error(path, "short read");
            return nullptr;
        }
        buf[static_cast<size_t>(sz)] = '\n';
    }
    const char* p = buf.data();
    const char* const end = buf.data() + buf.size();
    const char* eol = nullptr;

    Banner bn;
    const char* nl = next_line(p, end, &eol);
    if (!read_banner(path, p, eol, &bn)) return nullptr;
    p = nl;
    // Comment lines, then the size line (blank lines before it are skipped,
    // as mm_read_mtx_crd_size does).
    long long M = -1, N = -1, NZ = -1;
    while (p < end) {
        nl = next_line(p, end, &eol);
        if (*p == '%') {
            p = nl;
            continue;
        }
        std::string line(p, eol);
        p = nl;
        long long a, b, c;
        char extra;
        const int got = sscanf(line.c_str(), "%lld %lld %lld %c", &a, &b, &c, &extra);
        if (got >= 3) {
            M = a;
            N = b;
            NZ = c;
            break;
        }
        bool blank = true;
        for (char ch : line) blank = blank && is_space(ch);
        if (!blank) {
            mm_error(path, "malformed size line");
            return nullptr;
        }
    }
    if (M < 0 || N < 0 || NZ < 0) {
        mm_error(path, "missing or negative sizes");
        return nullptr;
    }
    if (M > INT32_MAX || N > INT32_MAX || NZ > INT32_MAX) {
        mm_error(path, "sizes beyond the 32-bit range the format's size line is read with");
        return nullptr;
    }

    // Items: k tokens each.
    const int k = bn.pattern ? 2 : 3;
    const size_t body = static_cast<size_t>(end - p);
    const int T = mm_threads(body);
    std::vector<const char*> cb(T + 1);
    cb[0] = p;
    cb[T] = end;
    for (int t = 1; t < T; ++t) {
        const char* q = p + body * t / T;
        while (q < end && !is_space(*q)) ++q;   // chunk starts between tokens
        cb[t] = std::max(q, cb[t - 1]);
    }
    std::vector<long long> ntok(T + 1, 0);
    mm_parallel(T, [&](int t) {
        long long n = 0;
        for (const char* q = cb[t]; q < cb[t + 1];) {
            while (q < cb[t + 1] && is_space(*q)) ++q;
            if (q >= cb[t + 1]) break;
            ++n;
            while (q < cb[t + 1] && !is_space(*q)) ++q;
        }
        ntok[t + 1] = n;
    });
    for (int t = 0; t < T; ++t) ntok[t + 1] += ntok[t];
    if (ntok[T] != NZ * k) {
        mm_error(path, ntok[T] < NZ * k ? "fewer entries than the size line declares"
                                        : "more entries than the size line declares "
                                          "(or an incomplete entry)");
        return nullptr;
    }
    std::vector<unsigned long long> rows(static_cast<size_t>(NZ)), cols(static_cast<size_t>(NZ));
    std::vector<double> vals(bn.pattern ? 0 : static_cast<size_t>(NZ));
    std::atomic<int> bad(0);
    mm_parallel(T, [&](int t) {
        long long g = ntok[t];
        for (const char* q = cb[t]; q < cb[t + 1];) {
            while (q < cb[t + 1] && is_space(*q)) ++q;
            if (q >= cb[t + 1]) break;
            const char* s = q;
            while (q < cb[t + 1] && !is_space(*q)) ++q;
            const long long item = g / k;
            const int fld = static_cast<int>(g % k);
            ++g;
            bool ok;
            if (fld == 0) ok = parse_index(s, q, &rows[item]);
            else if (fld == 1) ok = parse_index(s, q, &cols[item]);
            else ok = parse_value(s, q, &vals[item]);
            if (!ok) bad.store(1);
        }
    });
    if (bad.load()) {
        mm_error(path, "unparsable entry");
        return nullptr;
    }
    // Range check, row lengths (with mirrored items).
    std::vector<unsigned long long> rl(static_cast<size_t>(M) + 1, 0);
    long long total = 0;
    for (long long i = 0; i < NZ; ++i) {
        const unsigned long long r = rows[i], c = cols[i];
        if (r < 1 || r > static_cast<unsigned long long>(M) || c < 1 ||
            c > static_cast<unsigned long long>(N)) {
            mm_error(path, "entry index outside the declared shape");
            return nullptr;
        }
        ++rl[r - 1];
        ++total;
        if (bn.symmetric && r != c) {
            if (r > static_cast<unsigned long long>(N) || c > static_cast<unsigned long long>(M)) {
                mm_error(path, "mirrored entry outside the declared shape");
                return nullptr;
            }
            ++rl[c - 1];
            ++total;
        }
    }
    spmat* m = static_cast<spmat*>(calloc(1, sizeof(spmat)));
    if (!m) {
        mm_error(path, "spmat calloc failed");
        return nullptr;
    }
    m->M = static_cast<idx_t>(M);
    m->N = static_cast<idx_t>(N);
    m->NZ = static_cast<idx_t>(total);
    m->IRP = static_cast<idx_t*>(calloc(static_cast<size_t>(M) + 1, sizeof(idx_t)));
    m->JA = static_cast<idx_t*>(malloc(sizeof(idx_t) * std::max<long long>(total, 1)));
    m->AS = static_cast<double*>(malloc(sizeof(double) * std::max<long long>(total, 1)));
    if (!m->IRP || !m->JA || !m->AS) {
        mm_error(path, "CSR arrays allocation failed");
        return fail_free(m);
    }
    for (long long r = 0; r < M; ++r) m->IRP[r + 1] = m->IRP[r] + rl[r];
    // Fill in file order (each mirrored item right after its item).
    std::vector<idx_t> next(m->IRP, m->IRP + M);
    for (long long i = 0; i < NZ; ++i) {
        const idx_t r = rows[i] - 1, c = cols[i] - 1;
        const double v = bn.pattern ? 1.0 : vals[i];
        idx_t pos = next[r]++;
        m->JA[pos] = c;
        m->AS[pos] = v;
        if (bn.symmetric && r != c) {
            pos = next[c]++;
            m->JA[pos] = r;
            m->AS[pos] = v;
        }
    }
    return m;
}

SP3MM_API int sp3mm_write_mm(const spmat* m, int off, const char* path) {
    if (!m || !path || (off != 0 && off != 1)) return SP3MM_EINVAL;
    if (m->NZ > 0 && (!m->JA || !m->AS || !m->IRP)) return SP3MM_EINVAL;
    const long long M = static_cast<long long>(m->M);
    const long long nz = static_cast<long long>(m->NZ);
    if (!m->IRP && M > 0) return SP3MM_EINVAL;
    if (M > 0 && (static_cast<long long>(m->IRP[0]) != off ||
                  static_cast<long long>(m->IRP[M]) - off != nz))
        return SP3MM_EINVAL;
    for (long long r = 0; r < M; ++r)
        if (m->IRP[r + 1] < m->IRP[r]) return SP3MM_EINVAL;
    FILE* f = fopen(path, "wb");
    if (!f) return SP3MM_EINVAL;
    fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%% written by sp3mm_b200\n");
    fprintf(f, "%lld %lld %lld\n", M, static_cast<long long>(m->N), nz);
    // Rows formatted in parallel blocks, written in order.
    const int T = mm_threads(static_cast<size_t>(nz));
    std::vector<std::string> out(T);
    std::vector<long long> rb(T + 1);
    for (int t = 0; t <= T; ++t) rb[t] = M * t / T;
    std::atomic<int> bad(0);
    mm_parallel(T, [&](int t) {
        std::string& s = out[t];
        char line[96];
        for (long long r = rb[t]; r < rb[t + 1]; ++r) {
            for (idx_t j = m->IRP[r] - off; j < m->IRP[r + 1] - off; ++j) {
                const long long c = static_cast<long long>(m->JA[j]) - off;
                if (c < 0 || c >= static_cast<long long>(m->N)) bad.store(1);
                const int n = snprintf(line, sizeof line, "%lld %lld %.17g\n", r + 1, c + 1,
                                       m->AS[j]);
                s.append(line, static_cast<size_t>(n));
            }
        }
    });
    int rc = bad.load() ? SP3MM_EINVAL : SP3MM_OK;
    for (int t = 0; t < T && rc == SP3MM_OK; ++t)
        if (fwrite(out[t].data(), 1, out[t].size(), f) != out[t].size()) rc = SP3MM_EINVAL;
    if (fclose(f) != 0) rc = SP3MM_EINVAL;
    if (rc != SP3MM_OK) remove(path);
    return rc;
}

SP3MM_API int sp3mm_spmat_sort_rows(spmat* m, int off) {
    if (!m || (off != 0 && off != 1)) return SP3MM_EINVAL;
    const long long M = static_cast<long long>(m->M);
    if (M > 0 && !m->IRP) return SP3MM_EINVAL;
    if (m->NZ > 0 && (!m->JA || !m->AS)) return SP3MM_EINVAL;
    const int T = mm_threads(static_cast<size_t>(m->NZ));
    std::atomic<int> bad(0);
    mm_parallel(T, [&](int t) {
        std::vector<std::pair<idx_t, double>> row;
        for (long long r = M * t / T; r < M * (t + 1) / T; ++r) {
            const long long b = static_cast<long long>(m->IRP[r]) - off;
            const long long e = static_cast<long long>(m->IRP[r + 1]) - off;
            if (b < 0 || e < b || e > static_cast<long long>(m->NZ)) {
                bad.store(1);
                continue;
            }
            row.assign(static_cast<size_t>(e - b), {});
            for (long long j = b; j < e; ++j) row[j - b] = {m->JA[j], m->AS[j]};
            std::stable_sort(row.begin(), row.end(),
                             [](const auto& x, const auto& y) { return x.first < y.first; });
            for (long long j = b; j < e; ++j) {
                m->JA[j] = row[j - b].first;
                m->AS[j] = row[j - b].second;
            }
        }
    });
    return bad.load() ? SP3MM_EINVAL : SP3MM_OK;
}

}  // extern "C"
