/*
 * tca_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A plain-C CPU restatement of the reference TCA-SpMM hot path, used by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the
 * checker. Nothing in the product library links or calls this file.
 *
 * Parity is pinned by tests/golden/: fixtures generated by running the
 * reference's own CPU functions (smtx_input_to_Dense, convert_dense_to_csr,
 * convert_csr_to_dense, naive_gemm), compiled from the reference sources into
 * oracle/_ref/ by oracle/Makefile, on the reference's data fixture and on
 * seeded inputs (tests/golden/make_golden.py).
 *
 * Reference file:line citations are relative to the reference project root.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* IEEE binary16 <-> binary32, round-to-nearest-even (IEEE 754-2008).  */
/* ------------------------------------------------------------------ */
float orc_h2f(uint16_t h)
{
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1fu;
    uint32_t man = h & 0x3ffu;
    uint32_t bits;
    if (exp == 0) {
        if (man == 0) {
            bits = sign;
        } else { /* subnormal: value = man * 2^-24 */
            float v = (float)man * 5.9604644775390625e-08f;
            memcpy(&bits, &v, 4);
            bits |= sign;
        }
    } else if (exp == 31) {
        bits = sign | 0x7f800000u | (man << 13);
    } else {
        bits = sign | ((exp + 112u) << 23) | (man << 13);
    }
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

uint16_t orc_f2h(float f)
{
    uint32_t x;
    memcpy(&x, &f, 4);
    uint16_t sign = (uint16_t)((x >> 16) & 0x8000u);
    uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) /* inf or nan */
        return (uint16_t)(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u : 0u));
    if (ax >= 0x477ff000u) /* rounds to >= 65520 -> inf */
        return (uint16_t)(sign | 0x7c00u);
    if (ax < 0x38800000u) { /* below the smallest normal half: subnormal or zero */
        /* value * 2^24 rounded to nearest even integer gives the mantissa */
        float a;
        memcpy(&a, &ax, 4);
        float scaled = a * 16777216.0f; /* exact (power of two) */
        float r = nearbyintf(scaled);   /* default rounding mode: nearest-even */
        return (uint16_t)(sign | (uint16_t)r);
    }
    uint32_t e = (ax >> 23) - 112u;  /* half exponent */
    uint32_t m = ax & 0x7fffffu;
    uint32_t hm = m >> 13;
    uint32_t rem = m & 0x1fffu;
    uint32_t h = (e << 10) | hm;
    if (rem > 0x1000u || (rem == 0x1000u && (hm & 1u)))
        h += 1u; /* carries into the exponent correctly */
    return (uint16_t)(sign | h);
}

/* ------------------------------------------------------------------ */
/* smtx parsing: restates smtx_input_to_Dense (src/file_input.cu:135-193)
 * Header line "rows, cols, nnz" split on ',' (:141-148); line 2 holds the
 * row_ptr tokens split on ' ' (:155-162); every further line holds col_idx
 * tokens split on ' ' (:171-180). Returns 0 on success, -1 on a malformed
 * file (the reference throws from stoi or overruns its arrays instead).
 * Call with row_ptr == NULL to learn the sizes only.                    */
/* ------------------------------------------------------------------ */
static int orc_next_int(const char **p, const char *end, char delim, long *out, int *got)
{
    /* one getline(..., delim) token: characters up to delim or end. */
    const char *s = *p;
    if (s >= end) { *got = 0; return 0; }
    const char *t = s;
    while (t < end && *t != delim) t++;
    *p = (t < end) ? t + 1 : t;
    /* stoi semantics: skip leading whitespace, optional sign, digits */
    const char *q = s;
    while (q < t && (*q == ' ' || *q == '\t' || *q == '\r')) q++;
    int neg = 0;
    if (q < t && (*q == '+' || *q == '-')) { neg = (*q == '-'); q++; }
    if (q >= t || *q < '0' || *q > '9') return -1; /* stoi would throw */
    long v = 0;
    while (q < t && *q >= '0' && *q <= '9') { v = v * 10 + (*q - '0'); if (v > 2147483647L) return -1; q++; }
    *out = neg ? -v : v;
    *got = 1;
    return 0;
}

int orc_smtx_parse(const char *text, long len, int *nRow, int *nCol, int *nnz,
                   int *row_ptr, int *col_idx)
{
    const char *end = text + len;
    const char *line = text;
    const char *eol = memchr(line, '\n', (size_t)(end - line));
    if (!eol) eol = end;
    long v[3];
    const char *p = line;
    for (int i = 0; i < 3; i++) {
        int got = 0;
        if (orc_next_int(&p, eol, ',', &v[i], &got) != 0 || !got) return -1;
    }
    if (v[0] < 0 || v[1] < 0 || v[2] < 0) return -1;
    *nRow = (int)v[0]; *nCol = (int)v[1]; *nnz = (int)v[2];
    if (!row_ptr) return 0;
    /* line 2: row_ptr */
    line = (eol < end) ? eol + 1 : end;
    eol = memchr(line, '\n', (size_t)(end - line));
    if (!eol) eol = end;
    p = line;
    long n_rp = 0;
    for (;;) {
        long x; int got = 0;
        if (p >= eol) break;
        if (orc_next_int(&p, eol, ' ', &x, &got) != 0) return -1;
        if (!got) break;
        if (n_rp > *nRow) return -1;
        row_ptr[n_rp++] = (int)x;
    }
    if (n_rp != (long)*nRow + 1) return -1;
    /* remaining lines: col_idx */
    long n_ci = 0;
    line = (eol < end) ? eol + 1 : end;
    while (line < end) {
        eol = memchr(line, '\n', (size_t)(end - line));
        if (!eol) eol = end;
        p = line;
        while (p < eol) {
            long x; int got = 0;
            if (orc_next_int(&p, eol, ' ', &x, &got) != 0) return -1;
            if (!got) break;
            if (n_ci >= *nnz) return -1;
            col_idx[n_ci++] = (int)x;
        }
        line = (eol < end) ? eol + 1 : end;
    }
    if (n_ci != *nnz) return -1;
    if (row_ptr[0] != 0 || row_ptr[*nRow] != *nnz) return -1;
    for (int r = 0; r < *nRow; r++)
        if (row_ptr[r + 1] < row_ptr[r]) return -1;
    for (long i = 0; i < n_ci; i++)
        if (col_idx[i] < 0 || col_idx[i] >= *nCol) return -1;
    return 0;
}

/* Pattern -> dense M x K half matrix with 1.0 at each (r, col) (src/file_input.cu:182-191). */
void orc_pattern_to_dense(int nRow, int nCol, const int *row_ptr, const int *col_idx, uint16_t *mat)
{
    memset(mat, 0, sizeof(uint16_t) * (size_t)nRow * (size_t)nCol);
    for (int r = 0; r < nRow; r++)
        for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++)
            mat[(size_t)r * nCol + col_idx[j]] = 0x3c00u; /* 1.0 */
}

/* ------------------------------------------------------------------ */
/* convert_dense_to_csr (src/miscalleneous.cu:29-65): an element is a   */
/* nonzero iff (float)x != 0.0f, so -0.0 is dropped and NaN is kept;    */
/* the row-major scan emits sorted columns. Returns nnz. With row_ptr   */
/* NULL only counts.                                                    */
/* ------------------------------------------------------------------ */
long orc_dense_to_csr(const uint16_t *mat, int nRow, int nCol, int *row_ptr, int *col_idx, uint16_t *val)
{
    long nnz = 0;
    if (!row_ptr) {
        for (size_t i = 0; i < (size_t)nRow * (size_t)nCol; i++)
            nnz += (orc_h2f(mat[i]) != 0.0f);
        return nnz;
    }
    row_ptr[0] = 0;
    for (int r = 0; r < nRow; r++) {
        for (int c = 0; c < nCol; c++) {
            uint16_t x = mat[(size_t)r * nCol + c];
            if (orc_h2f(x) != 0.0f) {
                col_idx[nnz] = c;
                val[nnz] = x;
                nnz++;
            }
        }
        row_ptr[r + 1] = (int)nnz;
    }
    return nnz;
}

/* convert_csr_to_dense (src/miscalleneous.cu:66-81): later duplicates overwrite. */
void orc_csr_to_dense(int nRow, int nCol, const int *row_ptr, const int *col_idx, const uint16_t *val, uint16_t *mat)
{
    memset(mat, 0, sizeof(uint16_t) * (size_t)nRow * (size_t)nCol);
    for (int r = 0; r < nRow; r++)
        for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++)
            mat[(size_t)r * nCol + col_idx[j]] = val[j];
}

/* ------------------------------------------------------------------ */
/* SpMM semantics of kernel_our_spmm_balanced (src/our_spmm.cu:290-346):
 * C[r, n] = sum_j val_j * B[col_j, n] over the nonzeros of row r, B and C
 * row-major with leading dimension N; rows with no nonzeros are never
 * written (the kernel skips warps whose row is -1, :303-305, and
 * workload_manager gives empty rows no warps, :366-369).
 * keep_empty != 0 reproduces that; 0 writes zeros there.               */
/* ------------------------------------------------------------------ */
void orc_spmm_f64(int M, int N, const int *row_ptr, const int *col_idx, const uint16_t *val,
                  const uint16_t *B, int ldb, double *C, int ldc, int keep_empty)
{
    double *acc = (double *)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
    for (int r = 0; r < M; r++) {
        if (row_ptr[r + 1] == row_ptr[r] && keep_empty) continue;
        for (int n = 0; n < N; n++) acc[n] = 0.0;
        for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++) {
            double a = (double)orc_h2f(val[j]);
            const uint16_t *b = B + (size_t)col_idx[j] * ldb;
            for (int n = 0; n < N; n++) acc[n] += a * (double)orc_h2f(b[n]);
        }
        for (int n = 0; n < N; n++) C[(size_t)r * ldc + n] = acc[n];
    }
    free(acc);
}

/* FP32 accumulation in CSR order. With sorted columns this is bit-identical
 * to naive_gemm (src/miscalleneous.cu:114-134) on the densified A: the
 * skipped terms are exact zeros, which leave an fp32 sum unchanged. This is
 * also the timed CPU baseline (OpenMP over rows, nthreads <= 0 = all). */
void orc_spmm_f32(int M, int N, const int *row_ptr, const int *col_idx, const uint16_t *val,
                  const uint16_t *B, int ldb, float *C, int ldc, int keep_empty, int nthreads)
{
#ifdef _OPENMP
    int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
    /* B converted to fp32 once (exact), so the inner loop is a plain fp32
     * multiply-add the compiler can vectorise without changing any rounding. */
    int K = 0;
    for (int j = 0; j < row_ptr[M]; j++)
        if (col_idx[j] + 1 > K) K = col_idx[j] + 1;
    float *Bf = (float *)malloc(sizeof(float) * (size_t)(K > 0 ? K : 1) * (size_t)(N > 0 ? N : 1));
#ifdef _OPENMP
#pragma omp parallel for num_threads(nt) schedule(static)
#endif
    for (int k = 0; k < K; k++)
        for (int n = 0; n < N; n++) Bf[(size_t)k * N + n] = orc_h2f(B[(size_t)k * ldb + n]);
#ifdef _OPENMP
#pragma omp parallel num_threads(nt)
#endif
    {
        float *acc = (float *)malloc(sizeof(float) * (size_t)(N > 0 ? N : 1));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
        for (int r = 0; r < M; r++) {
            if (row_ptr[r + 1] == row_ptr[r] && keep_empty) continue;
            for (int n = 0; n < N; n++) acc[n] = 0.0f;
            for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++) {
                const float a = orc_h2f(val[j]);
                const float *b = Bf + (size_t)col_idx[j] * N;
                for (int n = 0; n < N; n++) acc[n] += a * b[n];
            }
            for (int n = 0; n < N; n++) C[(size_t)r * ldc + n] = acc[n];
        }
        free(acc);
    }
    free(Bf);
}

/* naive_gemm restated (src/miscalleneous.cu:114-134): dense fp32 sum over k. */
void orc_gemm_f32(int M, int N, int K, const uint16_t *A, const uint16_t *B, float *C)
{
    for (int m = 0; m < M; m++)
        for (int n = 0; n < N; n++) {
            float s = 0.0f;
            for (int k = 0; k < K; k++)
                s += orc_h2f(A[(size_t)m * K + k]) * orc_h2f(B[(size_t)k * N + n]);
            C[(size_t)m * N + n] = s;
        }
}

/* compare_mat (src/general.cuh:71-123): element i fails only when both
 * |gold-x|/|gold| >= tol and |gold-x| >= tol. Returns the number of failing
 * elements (the reference stops printing after 10 and returns false). */
long orc_compare_mat(const float *gold, const float *x, long n, float tol)
{
    long bad = 0;
    for (long i = 0; i < n; i++) {
        float d = fabsf(gold[i] - x[i]);
        float rel = fabsf(d / gold[i]);
        if (rel >= tol && d >= tol) bad++;
    }
    return bad;
}

/* ------------------------------------------------------------------ */
/* workload_manager's per-row warp demand (src/our_spmm.cu:362-391).   */
/* Returned for documentation tests of the reference schedule.         */
/* ------------------------------------------------------------------ */
void orc_ref_warp_demand(int M, const int *row_ptr, int N, int warps_per_tb, int *demand)
{
    for (int i = 0; i < M; i++) {
        int nnz = row_ptr[i + 1] - row_ptr[i];
        int w;
        if (nnz == 0) w = 0;
        else if (nnz <= 8) w = 1;
        else if (nnz <= 16) w = 2;
        else if (nnz <= 32) w = 4;
        else if (nnz <= 64) w = 8;
        else {
            int a = (int)ceilf((float)nnz / 64.0f), b = N / 64;
            w = (a < b ? a : b) * warps_per_tb;
        }
        demand[i] = w;
    }
}

/* ------------------------------------------------------------------ */
/* Host restatement of the row-window, column-condensed tile format   */
/* that libtca_spmm builds on the GPU (tca_plan_create). Same inputs   */
/* give the same arrays, bit for bit:                                  */
/*  - rows ordered by nnz descending, ties by row index;               */
/*  - windows of 128 sorted rows; a window is tensor-core eligible when */
/*    every row has strictly increasing columns, K <= 131072 and the   */
/*    plan is not CUDA-core only; it is chosen when nnz_w > 0 and      */
/*    (path == 2 or nnz_w >= tc_min_density * 8192 * ceil(distinct/64));*/
/*  - per tensor-core window: distinct columns ascending, -1 padded to  */
/*    a multiple of 64; per 64-column chunk, entries ordered by (row,   */
/*    column), packed as local_row << 22 | local_col << 16 | fp16 bits. */
/* ------------------------------------------------------------------ */
typedef struct orc_plan {
    int M, K, nnz, n_windows, n_tc, n_cc, n_tc_chunks;
    long long tc_nnz;
    int *perm, *p_row_ptr, *p_col, *src;
    uint16_t *p_val;
    int *tc_windows, *cc_windows, *tile_first, *win_cols, *tile_ptr, *tile_src;
    uint32_t *tile_entries;
    int n_images;
    int *img_idx;
    uint16_t *images;
    int n_cc_items, n_all_items;
    int *cc_items, *all_items; /* pairs [first, end) of sorted rows */
    int n_pairs;
    int *tc_pairs; /* [2 * n_pairs] tensor-core window index pairs, second -1 when alone */
} orc_plan;

/* CUDA-core work items over the rows of the listed windows: maximal runs of
 * consecutive listed rows, cut greedily into items of at most 31 rows whose
 * nonzeros stay within 32 (a longer row is an item of its own). */
static int orc_build_items(const int *windows, int nw, const int *row_ptr, int M, int *items)
{
    int n = 0, w = 0;
    while (w < nw) {
        int a = windows[w] * 128, v = w + 1;
        while (v < nw && windows[v] == windows[v - 1] + 1) v++;
        int b = windows[v - 1] * 128 + 128;
        if (b > M) b = M;
        int i = a;
        while (i < b) {
            int r0 = i, nz = row_ptr[i + 1] - row_ptr[i];
            i++;
            while (i < b && i - r0 < 31 && nz + (row_ptr[i + 1] - row_ptr[i]) <= 32) {
                nz += row_ptr[i + 1] - row_ptr[i];
                i++;
            }
            if (items) { items[2 * n] = r0; items[2 * n + 1] = i; }
            n++;
        }
        w = v;
    }
    return n;
}

void orc_plan_free(orc_plan *p)
{
    free(p->perm); free(p->p_row_ptr); free(p->p_col); free(p->src); free(p->p_val);
    free(p->tc_windows); free(p->cc_windows); free(p->tile_first); free(p->win_cols);
    free(p->tile_ptr); free(p->tile_src); free(p->tile_entries); free(p->img_idx); free(p->images);
    free(p->cc_items); free(p->all_items); free(p->tc_pairs);
    memset(p, 0, sizeof(*p));
}

static const int *g_sort_nnz;
static int orc_cmp_rows(const void *a, const void *b)
{
    int ra = *(const int *)a, rb = *(const int *)b;
    int na = g_sort_nnz[ra], nb = g_sort_nnz[rb];
    if (na != nb) return na > nb ? -1 : 1;
    return ra < rb ? -1 : (ra > rb);
}

int orc_plan_build(const int *row_ptr, const int *col, const uint16_t *val, int M, int K, int nnz,
                   int sort_rows, float tc_min_density, int path, orc_plan *p)
{
    enum { WR = 128, CW = 64, MAX_TC_K = 1 << 17 };
    memset(p, 0, sizeof(*p));
    p->M = M; p->K = K; p->nnz = nnz;
    if (M <= 0) return 0;
    if (row_ptr[0] != 0 || row_ptr[M] != nnz) return -1;
    int *row_nnz = (int *)malloc(sizeof(int) * M), *row_sorted = (int *)malloc(sizeof(int) * M);
    for (int r = 0; r < M; r++) {
        int s = row_ptr[r], e = row_ptr[r + 1];
        if (s < 0 || e < s || e > nnz) { free(row_nnz); free(row_sorted); return -1; }
        row_nnz[r] = e - s;
        row_sorted[r] = 1;
        for (int j = s; j < e; j++) {
            if (col[j] < 0 || col[j] >= K) { free(row_nnz); free(row_sorted); return -1; }
            if (j > s && !(col[j - 1] < col[j])) row_sorted[r] = 0;
        }
    }
    p->perm = (int *)malloc(sizeof(int) * M);
    for (int i = 0; i < M; i++) p->perm[i] = i;
    if (sort_rows) { g_sort_nnz = row_nnz; qsort(p->perm, (size_t)M, sizeof(int), orc_cmp_rows); }
    p->p_row_ptr = (int *)malloc(sizeof(int) * (M + 1));
    p->p_col = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    p->p_val = (uint16_t *)malloc(sizeof(uint16_t) * (nnz > 0 ? nnz : 1));
    p->src = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    p->p_row_ptr[0] = 0;
    for (int i = 0; i < M; i++) {
        int r = p->perm[i], d = p->p_row_ptr[i];
        for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++) {
            p->p_col[d] = col[j]; p->p_val[d] = val[j]; p->src[d] = j; d++;
        }
        p->p_row_ptr[i + 1] = d;
    }
    int W = (M + WR - 1) / WR;
    p->n_windows = W;
    int tc_possible = (path != 1) && K <= MAX_TC_K && K > 0;
    int *rank = (int *)malloc(sizeof(int) * (K > 0 ? K : 1));
    int *is_tc = (int *)calloc((size_t)W, sizeof(int)), *nch = (int *)calloc((size_t)W, sizeof(int));
    int *wnnz = (int *)calloc((size_t)W, sizeof(int)), *direct = (int *)calloc((size_t)W, sizeof(int));
    int *wblk = (int *)calloc((size_t)W, sizeof(int));
    for (int w = 0; w < W; w++) {
        int r0 = w * WR, r1 = r0 + WR < M ? r0 + WR : M;
        int lo = p->p_row_ptr[r0], hi = p->p_row_ptr[r1];
        wnnz[w] = hi - lo;
        if (!tc_possible) continue;
        int elig = 1;
        for (int i = r0; i < r1; i++) elig &= row_sorted[p->perm[i]];
        for (int c = 0; c < K; c++) rank[c] = 0;
        for (int j = lo; j < hi; j++) rank[p->p_col[j]] = 1;
        int nu = 0, nblk = 0;
        for (int c = 0; c < K; c++) nu += rank[c];
        for (int b = 0; b * CW < K; b++) {
            int hit = 0;
            for (int c = b * CW; c < (b + 1) * CW && c < K; c++) hit |= rank[c];
            nblk += hit;
        }
        /* direct chunks (the touched 64-column blocks of K) when they need at
         * most twice the chunks of the condensed distinct columns */
        int nch_cond = (nu + CW - 1) / CW;
        direct[w] = nblk <= 2 * nch_cond;
        wblk[w] = nblk;
        nch[w] = direct[w] ? nblk : nch_cond;
        if (elig && wnnz[w] > 0) {
            if (path == 2) is_tc[w] = 1;
            else is_tc[w] = (double)wnnz[w] >= (double)tc_min_density * (double)(WR * CW) * (double)nch[w];
        }
    }
    for (int w = 0; w < W; w++) {
        if (is_tc[w]) { p->n_tc++; p->n_tc_chunks += nch[w]; p->tc_nnz += wnnz[w]; }
        else p->n_cc++;
    }
    p->tc_windows = (int *)malloc(sizeof(int) * (p->n_tc > 0 ? p->n_tc : 1));
    p->cc_windows = (int *)malloc(sizeof(int) * (p->n_cc > 0 ? p->n_cc : 1));
    p->tile_first = (int *)malloc(sizeof(int) * (p->n_tc + 1));
    p->win_cols = (int *)malloc(sizeof(int) * ((size_t)p->n_tc_chunks * CW + 1));
    p->tile_ptr = (int *)malloc(sizeof(int) * ((size_t)p->n_tc_chunks + 1));
    p->tile_entries = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(p->tc_nnz + 1));
    p->tile_src = (int *)malloc(sizeof(int) * (size_t)(p->tc_nnz + 1));
    p->tile_first[0] = 0;
    p->tile_ptr[0] = 0;
    int it = 0, ic = 0;
    long long base = 0;
    int *cur = (int *)malloc(sizeof(int) * WR);
    for (int w = 0; w < W; w++) {
        if (!is_tc[w]) { p->cc_windows[ic++] = w; continue; }
        p->tc_windows[it] = w;
        int c0 = p->tile_first[it];
        p->tile_first[it + 1] = c0 + nch[w];
        it++;
        int r0 = w * WR, r1 = r0 + WR < M ? r0 + WR : M;
        for (int c = 0; c < K; c++) rank[c] = 0;
        for (int j = p->p_row_ptr[r0]; j < p->p_row_ptr[r1]; j++) rank[p->p_col[j]] = 1;
        if (direct[w])
            for (int b = 0; b * CW < K; b++) {
                int hit = 0;
                for (int c = b * CW; c < (b + 1) * CW && c < K; c++) hit |= rank[c];
                for (int c = b * CW; c < (b + 1) * CW && c < K; c++) rank[c] = hit;
            }
        int nu = 0;
        for (int c = 0; c < K; c++) {
            if (rank[c]) { p->win_cols[(size_t)c0 * CW + nu] = c; rank[c] = nu++; }
            else rank[c] = -1;
        }
        for (int k = nu; k < nch[w] * CW; k++) p->win_cols[(size_t)c0 * CW + k] = -1;
        for (int i = r0; i < r1; i++) cur[i - r0] = p->p_row_ptr[i];
        for (int c = 0; c < nch[w]; c++) {
            p->tile_ptr[c0 + c] = (int)base;
            for (int i = r0; i < r1; i++) {
                int lr = i - r0, e = p->p_row_ptr[i + 1];
                while (cur[lr] < e && rank[p->p_col[cur[lr]]] < (c + 1) * CW) {
                    int j = cur[lr];
                    uint32_t lc = (uint32_t)(rank[p->p_col[j]] - c * CW);
                    p->tile_entries[base] = ((uint32_t)lr << 22) | (lc << 16) | p->p_val[j];
                    p->tile_src[base] = j;
                    base++;
                    cur[lr]++;
                }
            }
        }
        p->tile_ptr[c0 + nch[w]] = (int)base;
    }
    /* chunks with >= 512 entries (1/16 of the tile) also become a dense 128 x 64 FP16 tile in
     * the 128-byte swizzled K-major layout: element (r, c) at byte
     * r*128 + ((c/8) ^ (r%8))*16 + (c%8)*2 */
    p->img_idx = (int *)malloc(sizeof(int) * ((size_t)p->n_tc_chunks + 1));
    p->n_images = 0;
    for (int c = 0; c < p->n_tc_chunks; c++)
        p->img_idx[c] = (p->tile_ptr[c + 1] - p->tile_ptr[c] >= WR * CW / 16) ? p->n_images++ : -1;
    p->images = (uint16_t *)calloc((size_t)p->n_images * WR * CW + 1, sizeof(uint16_t));
    for (int c = 0; c < p->n_tc_chunks; c++) {
        if (p->img_idx[c] < 0) continue;
        uint16_t *img = p->images + (size_t)p->img_idx[c] * WR * CW;
        for (int e = p->tile_ptr[c]; e < p->tile_ptr[c + 1]; e++) {
            uint32_t v = p->tile_entries[e], r = v >> 22, lc = (v >> 16) & 63u;
            uint32_t byte = r * 128u + (((lc >> 3) ^ (r & 7u)) << 4) + ((lc & 7u) << 1);
            img[byte / 2] = (uint16_t)(v & 0xffffu);
        }
    }
    int *all = (int *)malloc(sizeof(int) * (size_t)W);
    for (int w = 0; w < W; w++) all[w] = w;
    p->n_cc_items = orc_build_items(p->cc_windows, p->n_cc, p->p_row_ptr, M, NULL);
    p->cc_items = (int *)malloc(sizeof(int) * (2 * (size_t)p->n_cc_items + 1));
    orc_build_items(p->cc_windows, p->n_cc, p->p_row_ptr, M, p->cc_items);
    p->n_all_items = orc_build_items(all, W, p->p_row_ptr, M, NULL);
    p->all_items = (int *)malloc(sizeof(int) * (2 * (size_t)p->n_all_items + 1));
    orc_build_items(all, W, p->p_row_ptr, M, p->all_items);
    free(all);
    /* window pairs for the pair kernel: consecutive tensor-core windows that
     * are direct and touch every 64-column block of K have the same chunk
     * columns; greedily paired in tensor-core order, any other window alone */
    p->tc_pairs = (int *)malloc(sizeof(int) * (2 * (size_t)p->n_tc + 1));
    p->n_pairs = 0;
    {
        const int nkb = (K + CW - 1) / CW;
        for (int t = 0; t < p->n_tc;) {
            int wa = p->tc_windows[t], wb = t + 1 < p->n_tc ? p->tc_windows[t + 1] : -1;
            int fa = direct[wa] && wblk[wa] == nkb, fb = wb >= 0 && direct[wb] && wblk[wb] == nkb;
            p->tc_pairs[2 * p->n_pairs] = t;
            p->tc_pairs[2 * p->n_pairs + 1] = (fa && fb) ? t + 1 : -1;
            p->n_pairs++;
            t += (fa && fb) ? 2 : 1;
        }
    }
    free(cur); free(rank); free(is_tc); free(nch); free(wnnz); free(direct); free(wblk); free(row_nnz); free(row_sorted);
    return 0;
}

/* ---------------------------------------------------------------------------
 * FP8-E4M3 quantization (the rebuild's reduced-precision mode; the reference
 * computes in FP16 only). E4M3: 1 sign, 4 exponent (bias 7), 3 mantissa bits,
 * no infinities, 0x7F / 0xFF are NaN, largest finite 448, smallest subnormal
 * 2^-9. Conversion: round to nearest, ties to even, saturating to +-448.
 * ------------------------------------------------------------------------- */
uint8_t orc_f32_to_e4m3(float x)
{
    if (isnan(x)) return 0x7F;
    const uint8_t sign = signbit(x) ? 0x80 : 0x00;
    const float a = fabsf(x);
    if (a >= 448.0f) return sign | 0x7E; /* saturate (448 = 1.75 * 2^8) */
    if (a < 0.015625f) {                  /* below 2^-6: subnormal, quantum 2^-9 */
        const float m = nearbyintf(a * 512.0f); /* exact scaling; ties to even */
        return sign | (uint8_t)m;          /* m == 8 is the smallest normal, 0x08 */
    }
    int e;
    frexpf(a, &e);                        /* a = f * 2^e, f in [0.5, 1) */
    int E = e - 1;                        /* a in [2^E, 2^(E+1)), E in [-6, 8] */
    float m = nearbyintf(ldexpf(a, 3 - E)); /* 8 .. 16 */
    if (m >= 16.0f) { m = 8.0f; E += 1; }
    if (E > 8) return sign | 0x7E;
    return sign | (uint8_t)(((E + 7) << 3) | ((int)m - 8));
}

float orc_e4m3_to_f32(uint8_t q)
{
    const float sign = (q & 0x80) ? -1.0f : 1.0f;
    const int ex = (q >> 3) & 0xF, man = q & 7;
    if ((q & 0x7F) == 0x7F) return NAN;
    if (ex == 0) return sign * ldexpf((float)man, -9);
    return sign * ldexpf(1.0f + man / 8.0f, ex - 7);
}

static float orc_scale_of(float amax) { return amax > 0.0f ? amax / 448.0f : 1.0f; }

/* Per row r of a CSR (FP16 values): scale[r] = max|v| / 448 (1 if 0), q[j] =
 * E4M3(v_j / scale[r]). */
void orc_quant_rows(int M, const int *row_ptr, const uint16_t *val, float *scale, uint8_t *q)
{
    for (int r = 0; r < M; r++) {
        float m = 0.0f;
        for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++) {
            const float a = fabsf(orc_h2f(val[j]));
            if (a > m) m = a;
        }
        const float s = orc_scale_of(m);
        scale[r] = s;
        for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++) q[j] = orc_f32_to_e4m3(orc_h2f(val[j]) / s);
    }
}

/* Per column n of B (K x N FP16, row stride ldb): scale[n] = max_k |B| / 448,
 * q[k * ldq + n] = E4M3(B[k, n] / scale[n]). */
void orc_quant_cols(int K, int N, const uint16_t *B, int ldb, uint8_t *q, int ldq, float *scale)
{
    for (int n = 0; n < N; n++) {
        float m = 0.0f;
        for (int k = 0; k < K; k++) {
            const float a = fabsf(orc_h2f(B[(size_t)k * ldb + n]));
            if (a > m) m = a;
        }
        scale[n] = orc_scale_of(m);
    }
    /* B is divided by its column scale as a product with the FP32 reciprocal
     * (one correctly rounded division per column, as the GPU kernels do) */
    for (int k = 0; k < K; k++)
        for (int n = 0; n < N; n++) {
            const float inv = 1.0f / scale[n];
            q[(size_t)k * ldq + n] = orc_f32_to_e4m3(orc_h2f(B[(size_t)k * ldb + n]) * inv);
        }
}

/* ---------------------------------------------------------------------------
 * MatrixMarket coordinate text (restates src/file_input.cu:63-134,
 * mtx_input_to_CSR, and :8-62, mtx_input_to_Dense, through `missing`): '%'
 * lines are comments; the first other line is "rows cols nnz"; each further
 * non-blank line is "r c [v]", 1-based unless zero_based. pattern_only: v =
 * 1.0; else a missing v is `missing`. Rows in order, file order within a row.
 * Returns nnz, or -1 when the text is malformed (no header, a bad entry line,
 * an index out of range, a count different from the header). Output arrays
 * are malloc'd (row_ptr M+1, col nnz, val nnz FP16 bits).
 * ------------------------------------------------------------------------- */
long orc_mtx_parse(const char *text, long len, int zero_based, int pattern_only, float missing, int *M, int *K,
                   int **row_ptr_out, int **col_out, uint16_t **val_out)
{
    const char *p = text, *end = text + len;
    long rows = -1, cols = -1, meta = -1, n = 0;
    int *er = NULL, *ec = NULL;
    float *ev = NULL;
    while (p < end) {
        const char *q = p;
        while (q < end && *q != '\n') q++;
        /* copy the line to a NUL-terminated buffer */
        char buf[512];
        long L = (long)(q - p);
        if (L > 511) L = 511;
        memcpy(buf, p, (size_t)L);
        buf[L] = 0;
        p = q < end ? q + 1 : q;
        char *s = buf;
        while (*s == ' ' || *s == '\t' || *s == '\r') s++;
        if (*s == 0 || *s == '%') continue;
        char *e1, *e2;
        if (rows < 0) {
            rows = strtol(s, &e1, 10);
            if (e1 == s) goto bad;
            cols = strtol(e1, &e2, 10);
            if (e2 == e1) goto bad;
            meta = strtol(e2, &s, 10);
            if (s == e2 || rows < 0 || cols < 0 || meta < 0) goto bad;
            er = (int *)malloc(sizeof(int) * (size_t)(meta + 1));
            ec = (int *)malloc(sizeof(int) * (size_t)(meta + 1));
            ev = (float *)malloc(sizeof(float) * (size_t)(meta + 1));
            continue;
        }
        long r = strtol(s, &e1, 10);
        if (e1 == s) goto bad;
        long c = strtol(e1, &e2, 10);
        if (e2 == e1) goto bad;
        float v = pattern_only ? 1.0f : missing;
        if (!pattern_only) {
            char *t = e2, *e3;
            while (*t == ' ' || *t == '\t') t++;
            if (*t == '+' || *t == '-' || *t == '.' || (*t >= '0' && *t <= '9')) {
                const float x = strtof(t, &e3);
                if (e3 != t) v = x;
            }
        }
        if (!zero_based) { r--; c--; }
        if (r < 0 || r >= rows || c < 0 || c >= cols || n >= meta) goto bad;
        er[n] = (int)r; ec[n] = (int)c; ev[n] = v; n++;
    }
    if (rows < 0 || n != meta) goto bad;
    {
        int *rp = (int *)calloc((size_t)rows + 1, sizeof(int));
        int *co = (int *)malloc(sizeof(int) * (size_t)(n + 1));
        uint16_t *va = (uint16_t *)malloc(sizeof(uint16_t) * (size_t)(n + 1));
        for (long i = 0; i < n; i++) rp[er[i] + 1]++;
        for (long i = 0; i < rows; i++) rp[i + 1] += rp[i];
        int *fill = (int *)malloc(sizeof(int) * (size_t)(rows + 1));
        memcpy(fill, rp, sizeof(int) * (size_t)(rows + 1));
        for (long i = 0; i < n; i++) {           /* stable: file order within a row */
            const int j = fill[er[i]]++;
            co[j] = ec[i];
            va[j] = orc_f2h(ev[i]);
        }
        free(fill); free(er); free(ec); free(ev);
        *M = (int)rows; *K = (int)cols;
        *row_ptr_out = rp; *col_out = co; *val_out = va;
        return n;
    }
bad:
    free(er); free(ec); free(ev);
    return -1;
}
