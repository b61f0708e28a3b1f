// host_io.cpp -- host-side matrix I/O and format conversion of libtca_spmm:
// the smtx reader/writer, dense <-> CSR <-> COO, and the C++ drop-ins with the
// reference's signatures (smtx_input_to_Dense, smtx_input_to_CSR,
// convert_dense_to_csr, convert_csr_to_dense, destroy_csr, print_csr,
// format_conversion). Reference citations are file:line in the reference.
#include <algorithm>
#include <cerrno>
#include <climits>
#include <unistd.h>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>
#include "tca_internal.cuh"
#include "tca_spmm_compat.h"

namespace tca {
namespace {

// A cursor over one line split on a delimiter, with std::stoi's acceptance
// rules: leading blanks, optional sign, at least one digit; trailing
// characters after the digits end the number (as stoi does).
struct Tok {
    const char *p, *end;
    char delim;
    // 1 = token parsed, 0 = no more tokens, -1 = malformed token
    int next_int(long long *out)
    {
        if (p >= end)
            return 0;
        const char *t = p;
        while (t < end && *t != delim) t++;
        const char *s = p;
        p = (t < end) ? t + 1 : t;
        while (s < t && (*s == ' ' || *s == '\t' || *s == '\r')) s++;
        if (s == t && p >= end)
            return 0; // trailing delimiter / blank tail
        bool neg = false;
        if (s < t && (*s == '+' || *s == '-')) { neg = *s == '-'; s++; }
        if (s >= t || *s < '0' || *s > '9')
            return -1;
        long long v = 0;
        while (s < t && *s >= '0' && *s <= '9') {
            v = v * 10 + (*s - '0');
            if (v > 2147483647LL) return -1;
            s++;
        }
        *out = neg ? -v : v;
        return 1;
    }
};

const char *line_end(const char *p, const char *end)
{
    const char *e = static_cast<const char *>(std::memchr(p, '\n', (size_t)(end - p)));
    return e ? e : end;
}

bool blank(const char *p, const char *e)
{
    for (; p < e; p++)
        if (*p != ' ' && *p != '\t' && *p != '\r') return false;
    return true;
}

uint16_t f32_to_f16_bits(float f) { return __half_as_ushort(__float2half_rn(f)); }

int parse_smtx(const char *text, size_t len, int *M, int *K, int *nnz, std::vector<int> &rp, std::vector<int> &ci,
               std::vector<uint16_t> &vals)
{
    const char *end = text + len, *line = text, *eol = line_end(line, end);
    Tok hdr{line, eol, ','};
    long long h[3];
    for (int i = 0; i < 3; i++)
        if (hdr.next_int(&h[i]) != 1 || h[i] < 0)
            return set_error(TCA_ERR_FORMAT, "smtx header must be 'rows, cols, nnz'");
    *M = (int)h[0]; *K = (int)h[1]; *nnz = (int)h[2];
    rp.clear(); ci.clear(); vals.clear();
    rp.reserve((size_t)*M + 1);
    ci.reserve((size_t)*nnz);
    line = eol < end ? eol + 1 : end;
    eol = line_end(line, end);
    Tok t{line, eol, ' '};
    long long x;
    int r;
    while ((r = t.next_int(&x)) == 1) {
        if ((long long)rp.size() > *M) return set_error(TCA_ERR_FORMAT, "row_ptr line has more than rows+1 entries");
        rp.push_back((int)x);
    }
    if (r < 0) return set_error(TCA_ERR_FORMAT, "bad token in the row_ptr line");
    if ((long long)rp.size() != (long long)*M + 1)
        return set_error(TCA_ERR_FORMAT, "row_ptr line has %zu entries, expected %d", rp.size(), *M + 1);
    line = eol < end ? eol + 1 : end;
    // col_idx tokens until nnz have been read
    while (line < end && (int)ci.size() < *nnz) {
        eol = line_end(line, end);
        Tok c{line, eol, ' '};
        while ((r = c.next_int(&x)) == 1) {
            if ((int)ci.size() >= *nnz) return set_error(TCA_ERR_FORMAT, "more column indices than nnz");
            ci.push_back((int)x);
        }
        if (r < 0) return set_error(TCA_ERR_FORMAT, "bad token in the col_idx lines");
        line = eol < end ? eol + 1 : end;
    }
    if ((int)ci.size() != *nnz)
        return set_error(TCA_ERR_FORMAT, "%zu column indices, header says nnz=%d", ci.size(), *nnz);
    // optional values line (extension)
    while (line < end && blank(line, line_end(line, end))) {
        eol = line_end(line, end);
        line = eol < end ? eol + 1 : end;
    }
    if (line < end) {
        eol = line_end(line, end);
        std::string s(line, eol);
        const char *q = s.c_str();
        vals.reserve((size_t)*nnz);
        while (true) {
            while (*q == ' ' || *q == '\t' || *q == '\r') q++;
            if (!*q) break;
            char *nx = nullptr;
            errno = 0;
            const float v = std::strtof(q, &nx);
            if (nx == q) return set_error(TCA_ERR_FORMAT, "bad token in the values line");
            if ((int)vals.size() >= *nnz) return set_error(TCA_ERR_FORMAT, "more values than nnz");
            vals.push_back(f32_to_f16_bits(v));
            q = nx;
        }
        if ((int)vals.size() != *nnz)
            return set_error(TCA_ERR_FORMAT, "values line has %zu values, nnz=%d", vals.size(), *nnz);
        line = eol < end ? eol + 1 : end;
        if (line < end && !blank(line, end))
            return set_error(TCA_ERR_FORMAT, "unexpected text after the values line");
    } else {
        vals.assign((size_t)*nnz, (uint16_t)0x3c00u); // 1.0, src/file_input.cu:189
    }
    if (rp[0] != 0 || rp[*M] != *nnz) return set_error(TCA_ERR_FORMAT, "row_ptr must start at 0 and end at nnz");
    for (int i = 0; i < *M; i++)
        if (rp[i + 1] < rp[i]) return set_error(TCA_ERR_FORMAT, "row_ptr decreases at row %d", i);
    for (int i = 0; i < *nnz; i++)
        if (ci[i] < 0 || ci[i] >= *K) return set_error(TCA_ERR_FORMAT, "column %d outside [0, %d)", ci[i], *K);
    return TCA_OK;
}

template <typename T>
T *dup_malloc(const std::vector<T> &v)
{
    T *p = (T *)std::malloc(sizeof(T) * (v.empty() ? 1 : v.size()));
    if (p && !v.empty()) std::memcpy(p, v.data(), sizeof(T) * v.size());
    return p;
}

int read_file(const char *path, std::string &s)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) return set_error(TCA_ERR_IO, "cannot open %s", path);
    std::ostringstream ss;
    ss << f.rdbuf();
    s = ss.str();
    return TCA_OK;
}

bool g_exit_on_error = true;

void compat_fail(int st)
{
    std::fprintf(stderr, "tca-spmm error: %s: %s\n", tca_status_string(st), tca_last_error_string());
    if (g_exit_on_error)
        std::exit(EXIT_FAILURE);
}

// MatrixMarket coordinate text as the reference's mtx_input_to_CSR /
// mtx_input_to_Dense read it (src/file_input.cu:8-134): '%' lines are
// comments, the first other line is "rows cols nnz", every further line is
// "r c [v]" (1-based unless zero_based). pattern_only ignores a value and uses
// 1.0; otherwise a missing value is `missing` (0.0 in the reference's CSR
// reader, 1.0 in its dense reader). Entries keep the file's order within a
// row (no sorting, duplicates kept). Where the reference has undefined
// behaviour -- blank lines, '%' lines after the header, indices out of range,
// a count different from the header -- this returns TCA_ERR_FORMAT (blank
// lines are skipped).
struct MtxEntry {
    int r, c;
    float v;
};

// Whitespace-separated tokens of one line, read as stream extraction would.
struct WsTok {
    const char *p, *end;
    void skip() { while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\v' || *p == '\f')) p++; }
    bool next_int(long long *out)
    {
        skip();
        if (p >= end) return false;
        char *stop = nullptr;
        errno = 0;
        const long long v = std::strtoll(p, &stop, 10);
        if (stop == p || errno == ERANGE) return false;
        p = stop;
        *out = v;
        return true;
    }
    // false (value untouched) when no number starts here, as `>> float` leaves it
    bool next_float(float *out)
    {
        skip();
        if (p >= end) return false;
        const char c0 = *p;
        if (!(c0 == '+' || c0 == '-' || c0 == '.' || (c0 >= '0' && c0 <= '9'))) return false;
        std::string tok(p, (size_t)(end - p));
        char *stop = nullptr;
        const float v = std::strtof(tok.c_str(), &stop);
        if (stop == tok.c_str()) return false;
        p += stop - tok.c_str();
        *out = v;
        return true;
    }
};

int parse_mtx(const char *text, size_t len, bool zero_based, bool pattern_only, float missing, int *M, int *K,
              int *nnz, std::vector<MtxEntry> &ent)
{
    const char *p = text, *end = text + len;
    bool have_header = false;
    long long rows = 0, cols = 0, meta = 0;
    ent.clear();
    int line_no = 0;
    while (p < end) {
        const char *q = p;
        while (q < end && *q != '\n') q++;
        WsTok t{p, q};
        p = q < end ? q + 1 : q;
        line_no++;
        t.skip();
        if (t.p >= t.end) continue;    // blank line
        if (*t.p == '%') continue;     // comment (the reference skips them before the header only)
        if (!have_header) {
            if (!t.next_int(&rows) || !t.next_int(&cols) || !t.next_int(&meta) || rows < 0 || cols < 0 || meta < 0 ||
                rows > INT32_MAX || cols > INT32_MAX || meta > INT32_MAX)
                return set_error(TCA_ERR_FORMAT, "MatrixMarket line %d: expected \"rows cols nnz\"", line_no);
            have_header = true;
            ent.reserve((size_t)meta);
            continue;
        }
        long long r, c;
        if (!t.next_int(&r) || !t.next_int(&c))
            return set_error(TCA_ERR_FORMAT, "MatrixMarket line %d: expected \"row col [value]\"", line_no);
        float v = pattern_only ? 1.0f : missing;
        if (!pattern_only) t.next_float(&v);
        if (!zero_based) { r--; c--; }
        if (r < 0 || r >= rows || c < 0 || c >= cols)
            return set_error(TCA_ERR_FORMAT, "MatrixMarket line %d: entry (%lld, %lld) outside %lld x %lld", line_no,
                             r, c, rows, cols);
        ent.push_back(MtxEntry{(int)r, (int)c, v});
    }
    if (!have_header) return set_error(TCA_ERR_FORMAT, "MatrixMarket text has no \"rows cols nnz\" line");
    if ((long long)ent.size() != meta)
        return set_error(TCA_ERR_FORMAT, "MatrixMarket header announces %lld entries, the text has %zu", meta,
                         ent.size());
    *M = (int)rows;
    *K = (int)cols;
    *nnz = (int)meta;
    return TCA_OK;
}

} // namespace

bool compat_exit_on_error() { return g_exit_on_error; }
void compat_report(int st) { compat_fail(st); }

} // namespace tca

using namespace tca;

extern "C" {

void tca_free(void *p) { std::free(p); }

void tca_compat_set_exit_on_error(int enabled) { g_exit_on_error = enabled != 0; }

int tca_smtx_parse(const char *text, size_t len, int *M, int *K, int *nnz, int **row_ptr, int **col_idx,
                   void **vals_f16)
{
    clear_error();
    if (!text || !M || !K || !nnz) return set_error(TCA_ERR_INVALID_ARG, "NULL argument");
    std::vector<int> rp, ci;
    std::vector<uint16_t> v;
    TCA_TRY(parse_smtx(text, len, M, K, nnz, rp, ci, v));
    if (row_ptr) *row_ptr = dup_malloc(rp);
    if (col_idx) *col_idx = dup_malloc(ci);
    if (vals_f16) *vals_f16 = dup_malloc(v);
    return TCA_OK;
}

int tca_smtx_read(const char *path, int *M, int *K, int *nnz, int **row_ptr, int **col_idx, void **vals_f16)
{
    clear_error();
    if (!path) return set_error(TCA_ERR_INVALID_ARG, "path is NULL");
    std::string s;
    TCA_TRY(read_file(path, s));
    return tca_smtx_parse(s.data(), s.size(), M, K, nnz, row_ptr, col_idx, vals_f16);
}

int tca_mtx_parse(const char *text, size_t len, int zero_based, int pattern_only, float missing_value, int *M,
                  int *K, int *nnz, int **row_ptr, int **col_idx, void **vals_f16)
{
    clear_error();
    if (!text || !M || !K || !nnz) return set_error(TCA_ERR_INVALID_ARG, "NULL argument");
    std::vector<MtxEntry> ent;
    TCA_TRY(parse_mtx(text, len, zero_based != 0, pattern_only != 0, missing_value, M, K, nnz, ent));
    // rows in order, each row's entries in file order (a stable counting sort)
    std::vector<int> rp((size_t)*M + 1, 0), ci(ent.size());
    std::vector<uint16_t> v(ent.size());
    for (const MtxEntry &e : ent) rp[(size_t)e.r + 1]++;
    for (int i = 0; i < *M; i++) rp[(size_t)i + 1] += rp[i];
    std::vector<int> fill(rp.begin(), rp.end() - 1);
    for (const MtxEntry &e : ent) {
        const int j = fill[e.r]++;
        ci[j] = e.c;
        v[j] = __half_as_ushort(__float2half_rn(e.v));
    }
    if (row_ptr) *row_ptr = dup_malloc(rp);
    if (col_idx) *col_idx = dup_malloc(ci);
    if (vals_f16) *vals_f16 = dup_malloc(v);
    return TCA_OK;
}

int tca_mtx_read(const char *path, int zero_based, int pattern_only, float missing_value, int *M, int *K, int *nnz,
                 int **row_ptr, int **col_idx, void **vals_f16)
{
    clear_error();
    if (!path) return set_error(TCA_ERR_INVALID_ARG, "path is NULL");
    std::string s;
    TCA_TRY(read_file(path, s));
    return tca_mtx_parse(s.data(), s.size(), zero_based, pattern_only, missing_value, M, K, nnz, row_ptr, col_idx,
                         vals_f16);
}

int tca_smtx_write(const char *path, int M, int K, int nnz, const int *row_ptr, const int *col_idx,
                   const void *vals_f16)
{
    clear_error();
    if (!path || M < 0 || K < 0 || nnz < 0 || (M > 0 && !row_ptr) || (nnz > 0 && !col_idx))
        return set_error(TCA_ERR_INVALID_ARG, "invalid arguments");
    FILE *f = std::fopen(path, "w");
    if (!f) return set_error(TCA_ERR_IO, "cannot write %s", path);
    std::fprintf(f, "%d, %d, %d\n", M, K, nnz);
    for (int i = 0; i <= M; i++) std::fprintf(f, "%d ", row_ptr ? row_ptr[i] : 0);
    std::fprintf(f, "\n");
    for (int i = 0; i < nnz; i++) std::fprintf(f, "%d ", col_idx[i]);
    std::fprintf(f, "\n");
    if (vals_f16) {
        const uint16_t *v = (const uint16_t *)vals_f16;
        for (int i = 0; i < nnz; i++) std::fprintf(f, "%.9g ", (double)__half2float(__ushort_as_half(v[i])));
        std::fprintf(f, "\n");
    }
    const bool ok = std::fclose(f) == 0;
    return ok ? TCA_OK : set_error(TCA_ERR_IO, "write to %s failed", path);
}

int tca_dense_to_csr(const void *mat_f16, int M, int K, int *nnz, int **row_ptr, int **col_idx, void **vals_f16)
{
    clear_error();
    if ((M > 0 && K > 0 && !mat_f16) || M < 0 || K < 0 || !nnz)
        return set_error(TCA_ERR_INVALID_ARG, "invalid arguments");
    const uint16_t *a = (const uint16_t *)mat_f16;
    std::vector<int> rp((size_t)M + 1, 0), ci;
    std::vector<uint16_t> v;
    for (int r = 0; r < M; r++) {
        for (int c = 0; c < K; c++) {
            const uint16_t x = a[(size_t)r * K + c];
            if (__half2float(__ushort_as_half(x)) != 0.0f) { // -0.0 == 0; NaN != 0 (kept)
                ci.push_back(c);
                v.push_back(x);
            }
        }
        rp[r + 1] = (int)ci.size();
    }
    *nnz = (int)ci.size();
    if (row_ptr) *row_ptr = dup_malloc(rp);
    if (col_idx) *col_idx = dup_malloc(ci);
    if (vals_f16) *vals_f16 = dup_malloc(v);
    return TCA_OK;
}

int tca_csr_to_dense(int M, int K, int nnz, const int *row_ptr, const int *col_idx, const void *vals_f16,
                     void *mat_f16)
{
    clear_error();
    if (M < 0 || K < 0 || nnz < 0 || (M > 0 && (!row_ptr || (K > 0 && !mat_f16))) || (nnz > 0 && (!col_idx || !vals_f16)))
        return set_error(TCA_ERR_INVALID_ARG, "invalid arguments");
    uint16_t *a = (uint16_t *)mat_f16;
    const uint16_t *v = (const uint16_t *)vals_f16;
    if (M > 0 && K > 0) std::memset(a, 0, sizeof(uint16_t) * (size_t)M * K);
    for (int r = 0; r < M; r++) {
        if (row_ptr[r] < 0 || row_ptr[r + 1] < row_ptr[r] || row_ptr[r + 1] > nnz)
            return set_error(TCA_ERR_FORMAT, "invalid row_ptr at row %d", r);
        for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++) {
            if (col_idx[j] < 0 || col_idx[j] >= K) return set_error(TCA_ERR_FORMAT, "column outside [0, K)");
            a[(size_t)r * K + col_idx[j]] = v[j];
        }
    }
    return TCA_OK;
}

int tca_csr_to_coo(int M, int nnz, const int *row_ptr, int *row_idx)
{
    clear_error();
    if (M < 0 || nnz < 0 || (M > 0 && !row_ptr) || (nnz > 0 && !row_idx))
        return set_error(TCA_ERR_INVALID_ARG, "invalid arguments");
    for (int r = 0; r < M; r++) {
        if (row_ptr[r] < 0 || row_ptr[r + 1] < row_ptr[r] || row_ptr[r + 1] > nnz)
            return set_error(TCA_ERR_FORMAT, "invalid row_ptr at row %d", r);
        for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++) row_idx[j] = r;
    }
    return TCA_OK;
}

int tca_coo_to_csr(int M, int K, int nnz, const int *row_idx, const int *col_idx, const void *vals_f16, int *row_ptr,
                   int *col_out, void *vals_out)
{
    clear_error();
    if (M < 0 || K < 0 || nnz < 0 || !row_ptr || (nnz > 0 && (!row_idx || !col_idx || !vals_f16 || !col_out || !vals_out)))
        return set_error(TCA_ERR_INVALID_ARG, "invalid arguments");
    for (int i = 0; i < nnz; i++)
        if (row_idx[i] < 0 || row_idx[i] >= M || col_idx[i] < 0 || col_idx[i] >= K)
            return set_error(TCA_ERR_FORMAT, "entry %d outside the %d x %d matrix", i, M, K);
    std::vector<int> order((size_t)nnz);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return row_idx[a] != row_idx[b] ? row_idx[a] < row_idx[b] : col_idx[a] < col_idx[b];
    });
    const uint16_t *v = (const uint16_t *)vals_f16;
    uint16_t *vo = (uint16_t *)vals_out;
    std::fill(row_ptr, row_ptr + M + 1, 0);
    for (int i = 0; i < nnz; i++) {
        const int j = order[i];
        col_out[i] = col_idx[j];
        vo[i] = v[j];
        row_ptr[row_idx[j] + 1]++;
    }
    for (int r = 0; r < M; r++) row_ptr[r + 1] += row_ptr[r];
    return TCA_OK;
}

} // extern "C"

// ------------------------------------------------------------------ C++ drop-ins

static CSR *make_csr(int M, int K, int nnz, int *rp, int *ci, half *v)
{
    CSR *c = (CSR *)std::malloc(sizeof(CSR));
    c->nRow = M; c->nCol = K; c->nnz = nnz;
    c->row_offset = rp; c->col_idx = ci; c->value = v;
    return c;
}

void smtx_input_to_Dense(std::ifstream &fin, half **mat, char *filename, int *nRow, int *nCol, int *nnz)
{
    (void)filename; // unused, as in the reference
    std::ostringstream ss;
    ss << fin.rdbuf();
    const std::string s = ss.str();
    int *rp = nullptr, *ci = nullptr;
    void *v = nullptr;
    const int st = tca_smtx_parse(s.data(), s.size(), nRow, nCol, nnz, &rp, &ci, &v);
    if (st != TCA_OK) { compat_report(st); *mat = nullptr; return; }
    *mat = (half *)std::malloc(sizeof(half) * (size_t)(*nRow) * (*nCol) + 1);
    tca_csr_to_dense(*nRow, *nCol, *nnz, rp, ci, v, *mat);
    std::free(rp); std::free(ci); std::free(v);
}

void smtx_input_to_CSR(std::ifstream &fin, CSR **csr_mat, Arguments *arg)
{
    (void)arg; // unused, as the reference's declaration (src/file_input.cuh:9)
    std::ostringstream ss;
    ss << fin.rdbuf();
    const std::string s = ss.str();
    int M, K, nnz, *rp = nullptr, *ci = nullptr;
    void *v = nullptr;
    const int st = tca_smtx_parse(s.data(), s.size(), &M, &K, &nnz, &rp, &ci, &v);
    if (st != TCA_OK) { compat_report(st); *csr_mat = nullptr; return; }
    *csr_mat = make_csr(M, K, nnz, rp, ci, (half *)v);
}

void convert_dense_to_csr(half *mat, CSR **descr, int nRow, int nCol)
{
    int nnz = 0, *rp = nullptr, *ci = nullptr;
    void *v = nullptr;
    const int st = tca_dense_to_csr(mat, nRow, nCol, &nnz, &rp, &ci, &v);
    if (st != TCA_OK) { compat_report(st); *descr = nullptr; return; }
    *descr = make_csr(nRow, nCol, nnz, rp, ci, (half *)v);
}

void convert_csr_to_dense(CSR *d, half **mat)
{
    *mat = (half *)std::malloc(sizeof(half) * (size_t)d->nRow * d->nCol + 1);
    const int st = tca_csr_to_dense(d->nRow, d->nCol, d->nnz, d->row_offset, d->col_idx, d->value, *mat);
    if (st != TCA_OK) compat_report(st);
}

void destroy_csr(CSR *d)
{
    if (!d) return;
    std::free(d->col_idx);
    std::free(d->row_offset);
    std::free(d->value);
    std::free(d);
}

void destroy_coo(COO *d)
{
    if (!d) return;
    std::free(d->row_idx);
    std::free(d->col_idx);
    std::free(d->value);
    std::free(d);
}

void print_csr(CSR *d) // src/miscalleneous.cu:90-112
{
    std::puts("row_index");
    for (int i = 0; i < d->nRow; i++) std::printf("%d ", d->row_offset[i]);
    std::puts("");
    std::puts("col_index");
    for (int i = 0; i < d->nnz; i++) std::printf("%d ", d->col_idx[i]);
    std::puts("");
    std::puts("value");
    for (int i = 0; i < d->nnz; i++) std::printf("%f ", __half2float(d->value[i]));
    std::puts("");
}

static int bad_pair(mat_format in, mat_format out, mat_format want_in, mat_format want_out)
{
    if (in != want_in || out != want_out)
        return set_error(TCA_ERR_INVALID_ARG, "format_conversion %d -> %d does not match the argument types", (int)in,
                         (int)out);
    return TCA_OK;
}

int format_conversion(mat_format in, mat_format out, const half *src, int nRow, int nCol, CSR **dst)
{
    TCA_TRY(bad_pair(in, out, dense, csr));
    int nnz, *rp, *ci;
    void *v;
    TCA_TRY(tca_dense_to_csr(src, nRow, nCol, &nnz, &rp, &ci, &v));
    *dst = make_csr(nRow, nCol, nnz, rp, ci, (half *)v);
    return TCA_OK;
}

int format_conversion(mat_format in, mat_format out, const CSR *src, half **dst)
{
    TCA_TRY(bad_pair(in, out, csr, dense));
    *dst = (half *)std::malloc(sizeof(half) * (size_t)src->nRow * src->nCol + 1);
    return tca_csr_to_dense(src->nRow, src->nCol, src->nnz, src->row_offset, src->col_idx, src->value, *dst);
}

int format_conversion(mat_format in, mat_format out, const CSR *src, COO **dst)
{
    TCA_TRY(bad_pair(in, out, csr, coo));
    COO *c = (COO *)std::malloc(sizeof(COO));
    c->nRow = src->nRow; c->nCol = src->nCol; c->nnz = src->nnz;
    c->row_idx = (int *)std::malloc(sizeof(int) * (size_t)(src->nnz + 1));
    c->col_idx = (int *)std::malloc(sizeof(int) * (size_t)(src->nnz + 1));
    c->value = (half *)std::malloc(sizeof(half) * (size_t)(src->nnz + 1));
    std::memcpy(c->col_idx, src->col_idx, sizeof(int) * (size_t)src->nnz);
    std::memcpy(c->value, src->value, sizeof(half) * (size_t)src->nnz);
    const int st = tca_csr_to_coo(src->nRow, src->nnz, src->row_offset, c->row_idx);
    if (st != TCA_OK) { destroy_coo(c); return st; }
    *dst = c;
    return TCA_OK;
}

int format_conversion(mat_format in, mat_format out, const COO *src, CSR **dst)
{
    TCA_TRY(bad_pair(in, out, coo, csr));
    int *rp = (int *)std::malloc(sizeof(int) * (size_t)(src->nRow + 1));
    int *ci = (int *)std::malloc(sizeof(int) * (size_t)(src->nnz + 1));
    half *v = (half *)std::malloc(sizeof(half) * (size_t)(src->nnz + 1));
    const int st = tca_coo_to_csr(src->nRow, src->nCol, src->nnz, src->row_idx, src->col_idx, src->value, rp, ci, v);
    if (st != TCA_OK) { std::free(rp); std::free(ci); std::free(v); return st; }
    *dst = make_csr(src->nRow, src->nCol, src->nnz, rp, ci, v);
    return TCA_OK;
}

int format_conversion(mat_format in, mat_format out, const half *src, int nRow, int nCol, COO **dst)
{
    TCA_TRY(bad_pair(in, out, dense, coo));
    CSR *c = nullptr;
    TCA_TRY(format_conversion(dense, csr, src, nRow, nCol, &c));
    const int st = format_conversion(csr, coo, c, dst);
    destroy_csr(c);
    return st;
}

int format_conversion(mat_format in, mat_format out, const COO *src, half **dst)
{
    TCA_TRY(bad_pair(in, out, coo, dense));
    CSR *c = nullptr;
    TCA_TRY(format_conversion(coo, csr, src, &c));
    const int st = format_conversion(csr, dense, c, dst);
    destroy_csr(c);
    return st;
}

// ------------------------------------------------------------------ MatrixMarket drop-ins

Arguments::Arguments()
    : M(1024), N(1024), K(1024), num_iter(10), pattern_only(false), input_is_zero_based(true),
      input_file_exists(false), target_sparsity(0.8f), tolerance(1e-3f), a_type(fp16), b_type(fp16), c_type(fp32),
      input_fname(nullptr), ell_block_size(32)
{
}

Arguments::Arguments(int argc, char *argv[]) : Arguments()
{
    ParseArgs(argc, argv);
}

namespace {

// std::stoi / std::stof acceptance (leading blanks, a number, anything after
// it ignored), without the exception: false when no number starts the text.
bool opt_int(const char *s, int *out)
{
    errno = 0;
    char *end = nullptr;
    const long v = std::strtol(s, &end, 10);
    if (end == s || errno == ERANGE || v < INT_MIN || v > INT_MAX)
        return false;
    *out = (int)v;
    return true;
}

bool opt_float(const char *s, float *out)
{
    errno = 0;
    char *end = nullptr;
    const float v = std::strtof(s, &end);
    if (end == s || errno == ERANGE)
        return false;
    *out = v;
    return true;
}

// The reference exits on these errors (src/arg_parse.h:113-116, :121-124);
// with exit-on-error off the error is recorded and parsing goes on.
void args_fail(const char *fmt, const char *what)
{
    tca::set_error(TCA_ERR_INVALID_ARG, fmt, what);
    compat_fail(TCA_ERR_INVALID_ARG);
}

} // namespace

// The options of src/arg_parse.h:54-133 ("m:n:k:i:t:s:f:d:p:b:e:").
void Arguments::ParseArgs(int argc, char *argv[])
{
    optind = 1; // every call parses its own argv from the start
    int c;
    while ((c = getopt(argc, argv, "m:n:k:i:t:s:f:d:p:b:e:")) != -1) {
        int iv = 0;
        float fv = 0.f;
        switch (c) {
        case 'm': case 'n': case 'k': case 'i': case 'e': case 'p': case 'b': case 'd':
            if (!opt_int(optarg, &iv)) {
                args_fail("option value '%s' is not an integer", optarg);
                break;
            }
            if (c == 'm') M = iv;
            else if (c == 'n') N = iv;
            else if (c == 'k') K = iv;
            else if (c == 'i') num_iter = iv;
            else if (c == 'e') ell_block_size = iv;
            else if (c == 'p') pattern_only = iv == 1;
            else if (c == 'b') input_is_zero_based = iv == 0;
            else if (iv == (int)fp16) { a_type = b_type = fp16; c_type = fp32; }
            else if (iv == (int)fp64) { a_type = b_type = c_type = fp64; }
            else args_fail("Not Implemented error for the specified dtype (-d %s)", optarg);
            break;
        case 't': case 's':
            if (!opt_float(optarg, &fv)) {
                args_fail("option value '%s' is not a number", optarg);
                break;
            }
            if (c == 't') tolerance = fv;
            else target_sparsity = fv;
            break;
        case 'f': {
            const size_t n = std::strlen(optarg);
            input_fname = (char *)std::malloc(n + 1);
            std::memcpy(input_fname, optarg, n + 1);
            break;
        }
        default: // getopt reported the unknown option; skipped as in the reference
            break;
        }
    }
    input_file_exists = false;
    if (input_fname != nullptr) {
        if (access(input_fname, F_OK) != 0)
            args_fail("Input file not exists error: %s", input_fname);
        else
            input_file_exists = true;
    }
}

// src/arg_parse.h:135-160 (the reference's layout of the same settings).
void Arguments::print()
{
    static const char *dt[] = {"FP16", "FP32", "FP64"};
    std::printf("===================== Arguments ==========================\n");
    std::printf("Tolerance : %f\n", tolerance);
    std::printf("A type : %s, B type : %s, C type : %s\n", dt[a_type], dt[b_type], dt[c_type]);
    std::printf("N iter : %d\n", num_iter);
    std::printf("Ell block size : %d \n", ell_block_size);
    if (input_fname == nullptr) {
        std::printf("No input file have been passed ... generate synthetic with random entries\n");
        std::printf("The matrix size .. M: %d , N: %d, K: %d\n", M, N, K);
        std::printf("Target Sparsity : %f\n", target_sparsity);
    } else {
        std::printf("Input file name : %s\n", input_fname);
    }
    if (pattern_only)
        std::printf("Matrix is specified as pattern only matrix\n");
    if (!input_is_zero_based)
        std::printf("Input matrix is specified as one based index matrix\n");
    std::printf("================== End of Arguments ======================\n");
}

static std::string slurp(std::ifstream &fin)
{
    std::ostringstream ss;
    ss << fin.rdbuf();
    return ss.str();
}

void mtx_input_to_CSR(std::ifstream &fin, CSR **csr_mat, Arguments *arg)
{
    const std::string s = slurp(fin);
    const Arguments def;
    const Arguments &a = arg ? *arg : def;
    int M, K, nnz, *rp = nullptr, *ci = nullptr;
    void *v = nullptr;
    const int st = tca_mtx_parse(s.data(), s.size(), a.input_is_zero_based, a.pattern_only, 0.0f, &M, &K, &nnz, &rp,
                                 &ci, &v);
    if (st != TCA_OK) { compat_report(st); *csr_mat = nullptr; return; }
    *csr_mat = make_csr(M, K, nnz, rp, ci, (half *)v);
}

void mtx_input_to_Dense(std::ifstream &fin, half **mat, Arguments *arg)
{
    const std::string s = slurp(fin);
    const Arguments def;
    const Arguments &a = arg ? *arg : def;
    int M, K, nnz, *rp = nullptr, *ci = nullptr;
    void *v = nullptr;
    // the reference's dense reader always reads a value and keeps 1.0 where there is none
    const int st = tca_mtx_parse(s.data(), s.size(), a.input_is_zero_based, 0, 1.0f, &M, &K, &nnz, &rp, &ci, &v);
    if (st != TCA_OK) { compat_report(st); *mat = nullptr; return; }
    *mat = (half *)std::malloc(sizeof(half) * (size_t)M * K + 1);
    tca_csr_to_dense(M, K, nnz, rp, ci, v, *mat);
    std::free(rp); std::free(ci); std::free(v);
}
