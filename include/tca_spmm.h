/*
 * tca_spmm.h -- C ABI of the B200 (sm_100a) TCA-SpMM library, libtca_spmm.so.
 *
 * Computes C = alpha * A * B + beta * C for a CSR sparse A (M x K, FP16 values,
 * int32 indices, 0-based) and a dense row-major B (K x N, FP16), accumulating
 * in FP32 and writing C (M x N, row-major) in FP16 or FP32.
 *
 * All array arguments named d_* are device pointers; h_* are host pointers.
 * Every entry point returns a tca_status_t; on failure
 * tca_last_error_string() describes the error (per host thread).
 * Streams are CUDA runtime streams (cudaStream_t); NULL is the legacy default
 * stream. Reference citations are file:line within the reference project.
 */
#ifndef TCA_SPMM_H
#define TCA_SPMM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define TCA_API __attribute__((visibility("default")))
#else
#define TCA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

struct CUstream_st;
typedef struct CUstream_st *tca_stream_t; /* identical to cudaStream_t */

typedef enum tca_status {
    TCA_OK = 0,
    TCA_ERR_INVALID_ARG = 1, /* bad size, pointer, alignment or option */
    TCA_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    TCA_ERR_ALLOC = 3,       /* device or host allocation failed */
    TCA_ERR_UNSUPPORTED = 4, /* valid request this build does not support */
    TCA_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
    TCA_ERR_FORMAT = 6,      /* malformed CSR or matrix file */
    TCA_ERR_IO = 7           /* file could not be read */
} tca_status_t;

typedef enum tca_dtype {
    TCA_DTYPE_F16 = 0,
    TCA_DTYPE_F32 = 1,
    TCA_DTYPE_E4M3 = 2
} tca_dtype_t;

/* Rows of A without nonzeros leave C untouched, as in the reference, whose
 * kernel never writes them (src/our_spmm.cu:303-305, :366-369). Without the
 * flag those rows become beta * C. */
#define TCA_FLAG_KEEP_EMPTY_ROWS 1u

/* Test hook for the device-side failure path, not for production use: in the
 * tensor-core kernel each CTA withholds the completion signal of its last
 * accumulator, so that the epilogue's bounded wait for it (about one second)
 * runs out. The launch then ends normally with those output rows unwritten,
 * and tca_plan_status reports TCA_ERR_TIMEOUT. */
#define TCA_FLAG_TEST_WITHHOLD_ACCUM (1u << 31)

/* ------------------------------------------------------------------ */
/* Library information and errors                                     */
/* ------------------------------------------------------------------ */
TCA_API const char *tca_version(void);
TCA_API const char *tca_last_error_string(void);
TCA_API const char *tca_status_string(int status);

/* ------------------------------------------------------------------ */
/* Plan-free forward on CUDA cores, straight from CSR.
 * Replaces the device part of our_spmm_balanced (src/our_spmm.cu:472-588,
 * kernel at :290-346) without the per-call host schedule
 * (workload_manager, :347-471). N % 8 == 0 with 16-byte aligned B and C rows
 * takes the vectorised path; any other N or alignment a scalar one.        */
/* ------------------------------------------------------------------ */
TCA_API int tca_spmm_csr(const int *d_row_ptr, const int *d_col_idx, const void *d_vals_f16,
                 int M, int K, int nnz,
                 const void *d_B_f16, int ldb, int N,
                 void *d_C, int ldc, int c_dtype,
                 float alpha, float beta, unsigned flags, tca_stream_t stream);

/* FP64 forward, plan-free, on CUDA cores: C = alpha * A * B + beta * C with
 * FP64 values, B and C and FP64 accumulation (TCA_FLAG_KEEP_EMPTY_ROWS as
 * for tca_spmm_csr). The reference names an FP64 data type
 * (src/arg_parse.h:102-105, src/general.cuh:58,65) but has no FP64 path. */
TCA_API int tca_spmm_csr_f64(const int *d_row_ptr, const int *d_col_idx, const double *d_vals, int M, int K, int nnz,
                             const double *d_B, int ldb, int N, double *d_C, int ldc, double alpha, double beta,
                             unsigned flags, tca_stream_t stream);

/* ------------------------------------------------------------------ */
/* Plans: the row-window, column-condensed tile format.
 * tca_plan_create builds it on the GPU from a device CSR (replacing the
 * reference's per-call host schedule workload_manager, src/our_spmm.cu:347-471):
 * rows are ordered by nonzero count, grouped into windows of 128 rows, each
 * window's distinct columns are condensed into 64-wide chunks, and each window
 * is assigned to the tensor-core path (tcgen05) or the CUDA-core path by its
 * condensed density. The plan keeps its own device copy of everything it
 * needs; the caller's CSR may be freed afterwards.                          */
/* ------------------------------------------------------------------ */
typedef struct tca_plan *tca_plan_t;

typedef struct tca_plan_opts {
    int sort_rows;        /* 1 (default): windows over rows sorted by nnz; 0: natural row order */
    float tc_min_density; /* windows with condensed density >= this use tensor cores (default 0.01) */
    int path;             /* 0 auto (default), 1 CUDA cores only, 2 tensor cores only */
    int pair_windows;     /* 0 (default): one tensor-core window per SM; 1: consecutive windows
                             with identical chunk columns run as pairs on two SMs (tcgen05
                             cta_group::2) for N-slices of 256 -- correct, but measured slower on
                             the sweep problems (FP16 kernel 63 vs 50 us, E4M3 59 vs 37 us) */
    int reserved[4];
} tca_plan_opts_t;

typedef struct tca_plan_info {
    int M, K, nnz;
    int n_windows;          /* windows of 128 rows */
    int n_tc_windows;       /* windows on the tensor-core path */
    int n_cc_windows;       /* windows on the CUDA-core path */
    int n_tc_chunks;        /* 64-column condensed chunks over all tensor-core windows */
    int n_images;           /* chunks also kept as dense pre-swizzled tiles */
    long long tc_nnz;       /* nonzeros carried by tensor-core tiles */
    long long format_bytes; /* device bytes the plan occupies */
} tca_plan_info_t;

/* Arrays of a plan, for tca_plan_export (element type in brackets). */
typedef enum tca_plan_array {
    TCA_ARR_ROW_PERM = 0,     /* [int, M]   sorted position -> caller's row */
    TCA_ARR_P_ROW_PTR = 1,    /* [int, M+1] CSR offsets in sorted row order */
    TCA_ARR_P_COL = 2,        /* [int, nnz] columns in sorted row order */
    TCA_ARR_P_VAL = 3,        /* [fp16, nnz] values in sorted row order */
    TCA_ARR_SRC = 4,          /* [int, nnz] caller's nonzero index of each entry */
    TCA_ARR_TC_WINDOWS = 5,   /* [int, n_tc_windows] */
    TCA_ARR_CC_WINDOWS = 6,   /* [int, n_cc_windows] */
    TCA_ARR_TILE_FIRST = 7,   /* [int, n_tc_windows+1] first chunk of each tensor-core window */
    TCA_ARR_WIN_COLS = 8,     /* [int, n_tc_chunks*64] condensed columns, -1 padded */
    TCA_ARR_TILE_PTR = 9,     /* [int, n_tc_chunks+1] entry offsets per chunk */
    TCA_ARR_TILE_ENTRIES = 10,/* [uint32, tc_nnz] local_row<<22 | local_col<<16 | fp16 bits */
    TCA_ARR_TILE_SRC = 11,    /* [int, tc_nnz] index of each entry into TCA_ARR_P_VAL */
    TCA_ARR_TILE_IMAGE_IDX = 12, /* [int, n_tc_chunks] dense image of each chunk, -1 = none */
    TCA_ARR_TILE_IMAGES = 13, /* [fp16, n_images*8192] dense 128x64 tiles, 128-byte swizzled K-major */
    TCA_ARR_CC_ITEMS = 14,    /* [int pairs] CUDA-core items [first, end) of sorted rows, CUDA-core windows */
    TCA_ARR_ALL_ITEMS = 15,   /* [int pairs] the same over all windows */
    TCA_ARR_ROW_SCALE = 16,   /* [float, M] E4M3 scale per sorted row (after tca_plan_quantize_fp8) */
    TCA_ARR_P_VAL_F8 = 17,    /* [u8, nnz] E4M3 values, sorted order */
    TCA_ARR_TILE_ENTRIES_F8 = 18, /* [u32] tile entries with the E4M3 value in the low byte */
    TCA_ARR_TILE_IMAGES_F8 = 19,  /* [u8, n_images*8192] dense 128x64 E4M3 tiles, 64-byte swizzled K-major */
    TCA_ARR_TC_PAIRS = 20     /* [int pairs] tensor-core window pairs (indices into TCA_ARR_TC_WINDOWS; second -1: alone) */
} tca_plan_array_t;

TCA_API void tca_plan_opts_default(tca_plan_opts_t *opts);
TCA_API int tca_plan_create(const int *d_row_ptr, const int *d_col_idx, const void *d_vals_f16,
                    int M, int K, int nnz, const tca_plan_opts_t *opts,
                    tca_stream_t stream, tca_plan_t *plan);
/* Re-gathers new values for the same sparsity pattern into the plan. */
TCA_API int tca_plan_update_values(tca_plan_t plan, const void *d_vals_f16, tca_stream_t stream);
TCA_API int tca_plan_info(tca_plan_t plan, tca_plan_info_t *info);
/* Copies one plan array (tca_plan_array_t) to host memory; *out_bytes gets its
 * size. With h_dst NULL only the size is returned. Used to check the GPU build
 * of the format bit for bit against a host build. */
TCA_API int tca_plan_export(tca_plan_t plan, int which, void *h_dst, size_t capacity_bytes, size_t *out_bytes);
/* Reads and clears the plan's device status word (synchronises):
 * TCA_ERR_TIMEOUT when a bounded device-side wait of a launch since the last
 * call gave up, else TCA_OK. The kernel that gave up ends normally (tensor
 * memory released, no copy left in flight), so the context stays usable. */
TCA_API int tca_plan_status(tca_plan_t plan);
TCA_API int tca_plan_destroy(tca_plan_t plan);

/* Forward with a plan: C = alpha * A * B + beta * C. Launches the
 * tensor-core kernel over the plan's tensor-core windows and the CUDA-core
 * kernel over the rest, in that order, on `stream`. N % 8 == 0, ldb % 8 == 0,
 * ldc * sizeof(C) % 16 == 0 and 16-byte aligned B and C are needed for the
 * tensor-core kernel; otherwise every window runs on CUDA cores.
 * Replaces the device work of our_spmm_balanced (src/our_spmm.cu:547-559). */
TCA_API int tca_spmm(tca_plan_t plan, const void *d_B_f16, int ldb, int N,
             void *d_C, int ldc, int c_dtype, float alpha, float beta,
             unsigned flags, tca_stream_t stream);
/* tca_spmm that also records four caller-created CUDA events (cudaEvent_t,
 * NULL entries skipped) on `stream`: events[0]/[1] around the tensor-core
 * kernel, events[2]/[3] around the CUDA-core kernel -- per-kernel device time
 * for profiling. Same work as tca_spmm. */
TCA_API int tca_spmm_events(tca_plan_t plan, const void *d_B_f16, int ldb, int N,
             void *d_C, int ldc, int c_dtype, float alpha, float beta,
             unsigned flags, tca_stream_t stream, void *const *events);
/* One forward of a batched launch. n_tile picks the tensor-core N-slice
 * width (64, 128 or 256; 0 = by N). */
typedef struct tca_batch_item {
    tca_plan_t plan;
    const void *d_B_f16;
    int ldb, N;
    void *d_C;
    int ldc;
    int n_tile;   /* tensor-core N-slice width: 64, 128, 256 (E4M3: 128, 256); 0 = by N */
    int cc_cols;  /* CUDA-core output columns per lane: 2, 4, 8; 16 = the FP16
                     mma.sync item kernel (E4M3 items: by N); 0 = by N */
} tca_batch_item_t;

/* Forwards of many plans (layers of different shapes and sparsity) in a
 * handful of launches: one tensor-core launch per N-slice width over every
 * item's tensor-core windows, then one CUDA-core launch per row width over
 * every item's remaining rows (at most 32 items per launch). Same results as
 * calling tca_spmm per item. events: as in tca_spmm_events (may be NULL).
 * No device memory is allocated: the work list travels as kernel parameters,
 * so the call can be captured in a CUDA graph. */
TCA_API int tca_spmm_batched(const tca_batch_item_t *items, int n_items, int c_dtype, float alpha,
                             float beta, unsigned flags, tca_stream_t stream, void *const *events);
/* ------------------------------------------------------------------ */
/* Adjoints of Y = A B (the reference has no backward pass; these follow
 * from its forward, src/our_spmm.cu:290-346, Y[r,:] = sum_j a_j B[c_j,:]).  */
/* ------------------------------------------------------------------ */
/* dA on A's pattern (SDDMM): out[j] = alpha * sum_n dY[r_j, n] * B[c_j, n]
 * for every nonzero j in the caller's CSR order; dY is M x N (ldy), B is
 * K x N (ldb), out is nnz values of out_dtype (F16 or F32). Where A is dense
 * enough (and M * K * 4 <= 256 MiB) it computes dY B^T with one cuBLAS GEMM
 * into stream-ordered scratch from the library's pool and samples it; else a
 * sparse kernel; FP32 accumulation either way. */
TCA_API int tca_sddmm(tca_plan_t plan, const void *d_dY_f16, int ldy, const void *d_B_f16, int ldb, int N,
                      void *d_out, int out_dtype, float alpha, tca_stream_t stream);
/* dB = alpha * A^T dY + beta * dB (dY M x N, dB K x N of dB_dtype). Runs the
 * forward kernels on a plan of A^T, which the first call builds on the GPU
 * (allocating; do that call, or tca_plan_build_transpose, outside stream
 * capture). tca_plan_update_values keeps A^T's values in step. */
TCA_API int tca_spmm_t(tca_plan_t plan, const void *d_dY_f16, int ldy, int N, void *d_dB, int lddb,
                       int dB_dtype, float alpha, float beta, tca_stream_t stream);
TCA_API int tca_plan_build_transpose(tca_plan_t plan, tca_stream_t stream);

/* How many tensor-core and CUDA-core kernel launches one tca_spmm with this
 * N makes (0 or 1 each). */
TCA_API int tca_plan_launch_counts(tca_plan_t plan, int N, int *n_tc_launches, int *n_cc_launches);

/* ---- FP8-E4M3 forward (no counterpart in the reference, which computes in
 * FP16 only; src/our_spmm.cu:109-145 uses FP16 mma.sync) ----
 * A is quantized per sorted row, B per column: s = max|x| / 448 (1 for an
 * all-zero row or column), q = E4M3(x / s) for A and q = E4M3(x * r) with
 * r = 1 / s rounded to FP32 for B, rounded to nearest even and saturated. The forward accumulates the exact products q_a * q_b in FP32 and
 * returns alpha * (sum * s_a[row] * s_b[col]) + beta * C. */

/* Builds (or, after new values, refreshes) the plan's E4M3 form of A.
 * tca_spmm_fp8 calls it on first use; tca_plan_update_values refreshes it. */
TCA_API int tca_plan_quantize_fp8(tca_plan_t plan, tca_stream_t stream);
/* B (K x N FP16, row stride ldb) -> Bq (K x N E4M3 bytes, row stride ldq,
 * ldq % 4 == 0) and scale[N] (FP32). */
TCA_API int tca_quantize_b_fp8(const void *d_B_f16, int ldb, int K, int N, void *d_Bq, int ldq, float *d_scale,
                               tca_stream_t stream);
/* E4M3 forward from FP16 B, which is quantized per call into a workspace
 * owned by the plan (allocated on first use, grown when N grows). Needs
 * N % 8 == 0 and a 16-byte aligned C with ldc * sizeof(C) % 16 == 0. Calls
 * on one plan must not overlap in time on different streams (they share the
 * workspace). */
TCA_API int tca_spmm_fp8(tca_plan_t plan, const void *d_B_f16, int ldb, int N, void *d_C, int ldc, int c_dtype,
                         float alpha, float beta, unsigned flags, tca_stream_t stream);
/* tca_spmm_fp8 over many forwards in as few launches as tca_spmm_batched; a
 * plan may appear once per batch. n_tile: 128 or 256 (0 = by N). */
TCA_API int tca_spmm_fp8_batched(const tca_batch_item_t *items, int n_items, int c_dtype, float alpha, float beta,
                                 unsigned flags, tca_stream_t stream, void *const *events);

/* tca_spmm_fp8 for callers that may not allocate device memory: those whose
 * memory is handed out by someone else (a framework's own caching allocator,
 * a fixed per-process budget) and those on a latency-critical path where a
 * cudaMalloc / cudaFree, which may synchronise the device, is not allowed.
 * This entry point has no counterpart in the reference.
 * Instead of the plan's workspace it quantizes B into one fixed array of
 * TCA_FP8_STATIC_SCRATCH_BYTES, part of the library on every GPU that loads
 * it (held until the process exits). Limit: K * round_up(N, 16) bytes, rounded
 * up to 256, plus 4 * round_up(N, 16) must fit; larger B is rejected with
 * TCA_ERR_INVALID_ARG (use tca_spmm_fp8). The plan's E4M3 form must exist
 * already (tca_plan_quantize_fp8, which allocates, called once at set-up).
 * The first call on each device looks up the array's device address; make
 * that first call before any stream capture. The address is kept for the
 * process: after a cudaDeviceReset of a device, do not call this on that
 * device again. Every call on a device shares the one array (the call clears
 * what it needs cleared): calls whose work overlaps on the GPU -- on
 * different streams, or from different threads -- race and give wrong
 * results. K == 0 writes C = beta * C through tca_spmm (no quantization, no
 * allocation). Otherwise as tca_spmm_fp8, with the same launches. */
#define TCA_FP8_STATIC_SCRATCH_BYTES (16u << 20)
TCA_API int tca_spmm_fp8_static(tca_plan_t plan, const void *d_B_f16, int ldb, int N, void *d_C, int ldc, int c_dtype,
                                float alpha, float beta, unsigned flags, tca_stream_t stream);

/* Device memory the library holds on the current device: its stream-ordered
 * pool (plans, their temporaries and workspaces, host-buffer calls), in
 * bytes reserved from the device, in use now, and the highest use since the
 * last reset (reset_high != 0 resets that mark to the current use first).
 * Any pointer may be NULL. Diagnostics; no counterpart in the reference,
 * which allocates with cudaMalloc per call (src/our_spmm.cu:497-506). */
TCA_API int tca_pool_stats(int reset_high, size_t *reserved_bytes, size_t *used_bytes, size_t *used_high_bytes);

/* ---- Batched forward as a CUDA graph, and its autotuner (no counterpart in
 * the reference: its launch geometry is fixed per call by workload_manager,
 * src/our_spmm.cu:347-471) ---- */
typedef enum { TCA_PRECISION_F16 = 0, TCA_PRECISION_E4M3 = 1 } tca_precision_t;
typedef struct tca_graph *tca_graph_t;

/* Captures tca_spmm_batched (precision F16) or tca_spmm_fp8_batched (E4M3)
 * over `items` into a CUDA graph. Runs the batch once eagerly first (one-time
 * set-up and validation; it writes the items' C), then captures a second run
 * on a private stream. The graph keeps the items' pointers: replaying it after
 * freeing any of them is undefined. */
TCA_API int tca_batch_graph_create(const tca_batch_item_t *items, int n_items, int c_dtype, float alpha, float beta,
                                   unsigned flags, int precision, tca_graph_t *graph);
/* tca_batch_graph_create that also captures four caller-created CUDA events
 * (cudaEvent_t, NULL entries skipped) into the graph, recorded around the
 * tensor-core and the CUDA-core launches of every replay: per-kernel device
 * time of the batch as it runs from the graph. */
TCA_API int tca_batch_graph_create_events(const tca_batch_item_t *items, int n_items, int c_dtype, float alpha,
                                          float beta, unsigned flags, int precision, void *const *events,
                                          tca_graph_t *graph);
/* One replay of the captured batch on `stream`. */
TCA_API int tca_batch_graph_launch(tca_graph_t graph, tca_stream_t stream);
TCA_API int tca_batch_graph_destroy(tca_graph_t graph);
/* Per item, times every (n_tile, cc_cols) candidate on the item alone (median
 * of `reps` runs, CUDA events on `stream`, synchronising); then, for batches
 * of more than one item, times those picks as a whole against every uniform
 * (n_tile, cc_cols) for all items, each as replays of a captured graph, and
 * stores the fastest into items[i].n_tile / items[i].cc_cols. Writes the
 * items' C. */
TCA_API int tca_batch_autotune(tca_batch_item_t *items, int n_items, int c_dtype, int precision, int reps,
                               tca_stream_t stream);

/* ------------------------------------------------------------------ */
/* Host-side matrix I/O and format conversion. Arrays returned through
 * pointer-to-pointer arguments are malloc'd; release them with tca_free.  */
/* ------------------------------------------------------------------ */
TCA_API void tca_free(void *p);

/* Parses .smtx text as smtx_input_to_Dense does (src/file_input.cu:135-193):
 * header "rows, cols, nnz" split on ',', the row_ptr line, then col_idx tokens
 * over any number of lines. Extension: one further line of nnz decimal values
 * (the reference's files carry none and it stores 1.0 at every nonzero; its
 * reader would misparse such a line). *vals_f16 receives those values, or 1.0
 * everywhere. Malformed text (bad tokens, wrong counts, decreasing row_ptr,
 * columns outside [0, cols)) gives TCA_ERR_FORMAT instead of the reference's
 * exception or overrun. */
TCA_API int tca_smtx_parse(const char *text, size_t len, int *M, int *K, int *nnz,
                           int **row_ptr, int **col_idx, void **vals_f16);
TCA_API int tca_smtx_read(const char *path, int *M, int *K, int *nnz,
                          int **row_ptr, int **col_idx, void **vals_f16);
/* MatrixMarket coordinate text, read as the reference's mtx_input_to_CSR
 * (src/file_input.cu:63-134): '%' lines are comments, the first other line
 * is "rows cols nnz", each further line "r c [v]" (1-based unless
 * zero_based). pattern_only: every value is 1.0 (a third token is ignored);
 * otherwise a missing value is missing_value (the reference's CSR reader:
 * 0.0; its dense reader, src/file_input.cu:8-62: 1.0). Rows come out in
 * order with each row's entries in file order (no sorting; duplicates kept);
 * values rounded to FP16. TCA_ERR_FORMAT for a count that differs from the
 * header, an index out of range or a line that is not "r c [v]" (blank
 * lines are skipped). Arrays are malloc'd; free with tca_free. */
TCA_API int tca_mtx_parse(const char *text, size_t len, int zero_based, int pattern_only, float missing_value,
                          int *M, int *K, int *nnz, int **row_ptr, int **col_idx, void **vals_f16);
TCA_API int tca_mtx_read(const char *path, int zero_based, int pattern_only, float missing_value, int *M, int *K,
                         int *nnz, int **row_ptr, int **col_idx, void **vals_f16);
/* Writes the smtx layout (values line only when vals_f16 is not NULL). */
TCA_API int tca_smtx_write(const char *path, int M, int K, int nnz, const int *row_ptr,
                           const int *col_idx, const void *vals_f16);

/* Dense row-major FP16 -> CSR, as convert_dense_to_csr (src/miscalleneous.cu:29-65):
 * an element is a nonzero iff its value compares != 0 (so -0.0 is dropped). */
TCA_API int tca_dense_to_csr(const void *mat_f16, int M, int K, int *nnz,
                             int **row_ptr, int **col_idx, void **vals_f16);
/* CSR -> dense into a caller buffer of M*K FP16 (convert_csr_to_dense,
 * src/miscalleneous.cu:66-81; a repeated column keeps the last value). */
TCA_API int tca_csr_to_dense(int M, int K, int nnz, const int *row_ptr, const int *col_idx,
                             const void *vals_f16, void *mat_f16);
/* CSR row offsets -> COO row indices (caller buffer of nnz ints). */
TCA_API int tca_csr_to_coo(int M, int nnz, const int *row_ptr, int *row_idx);
/* COO -> CSR into caller buffers (row_ptr M+1, col/vals nnz); entries are
 * ordered by (row, column), stably, duplicates kept. */
TCA_API int tca_coo_to_csr(int M, int K, int nnz, const int *row_idx, const int *col_idx,
                           const void *vals_f16, int *row_ptr, int *col_out, void *vals_out);

/* ------------------------------------------------------------------ */
/* Host-buffer forward with the reference's calling convention
 * (our_spmm_balanced, src/our_spmm.cu:472): copies A, B (and C when it is
 * read) to the device, builds a plan, runs the forward n_iter times, copies C
 * back. *elapsed_ms (may be NULL) receives the mean device time of one
 * forward, as the reference reports it (:552-574).                       */
/* ------------------------------------------------------------------ */
TCA_API int tca_spmm_host(const int *h_row_ptr, const int *h_col_idx, const void *h_vals_f16,
                  int M, int K, int nnz, const void *h_B_f16, int N,
                  void *h_C, int c_dtype, unsigned flags, int n_iter, double *elapsed_ms);

#ifdef __cplusplus
}
#endif
#endif /* TCA_SPMM_H */
