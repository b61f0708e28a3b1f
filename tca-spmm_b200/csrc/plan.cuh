// plan.cuh -- the row-window, column-condensed tile format (a tca_plan).
//
// Layout in HBM (all arrays device-resident, int32 unless stated):
//   perm[M]            sorted position -> caller's row (rows ordered by nnz,
//                      descending, ties by row index)
//   p_row_ptr[M+1], p_col[nnz], p_val[nnz] (FP16), src[nnz]
//                      the CSR re-ordered by perm; src maps each entry back to
//                      the caller's nonzero index (for value updates)
//   windows            w covers sorted positions [128 w, 128 w + 128)
//   tc_windows[n_tc], cc_windows[n_cc]
//                      windows on the tensor-core / CUDA-core path
//   tile_first[n_tc+1] first condensed chunk of each tensor-core window
//   win_cols[chunks*64] the window's distinct columns, ascending, 64 per chunk,
//                      -1 padding in the last chunk
//   tile_ptr[chunks+1], tile_entries[tc_nnz + 4] (uint32), tile_src[tc_nnz]
//                      per chunk, its nonzeros as (local_row << 22 |
//                      local_col << 16 | fp16 bits), ordered by (row, column);
//                      tile_src indexes p_val; 4 zero entries of padding let
//                      16-byte copies round the end of the last chunk up
//   img_idx[chunks], images[n_images * 8192] (FP16)
//                      chunks with >= 512 nonzeros (1/16 of the tile: at
//                      most 8x the bytes of their entries, and no scatter
//                      work on the kernel's critical path) are also kept
//                      as a dense 128 x 64 tile, already in the 128-byte
//                      swizzled K-major layout the tensor cores read from
//                      shared memory; img_idx is -1 for the other chunks
#pragma once
#include <functional>
#include <vector>
#include "tca_internal.cuh"

struct tca_plan {
    int M = 0, K = 0, nnz = 0;
    int n_windows = 0, n_tc = 0, n_cc = 0, n_tc_chunks = 0;
    long long tc_nnz = 0;
    tca_plan_opts_t opts{};
    int *perm = nullptr;
    int *p_row_ptr = nullptr;
    int *p_col = nullptr;
    __half *p_val = nullptr;
    int *src = nullptr;
    int *tc_windows = nullptr;
    int *cc_windows = nullptr;
    int *all_windows = nullptr;
    int *tile_first = nullptr;
    int4 *tc_win_info = nullptr; // per tensor-core window: {window, first chunk, chunk count, direct}
    // tensor-core windows in pairs (indices into tc_windows): consecutive
    // direct windows that touch every 64-column block of K have identical
    // chunk columns and pair up; any other window is alone (second -1)
    int2 *tc_pairs = nullptr;
    int n_pairs = 0, n_full_pairs = 0;
    int *win_cols = nullptr;
    int *tile_ptr = nullptr;
    uint32_t *tile_entries = nullptr;
    int *tile_src = nullptr;
    int *img_idx = nullptr;
    int *img_chunk = nullptr; // image -> chunk
    uint16_t *images = nullptr;
    int n_images = 0;
    // CUDA-core work items: runs of consecutive sorted rows [x, y) with at
    // most kItemRows rows and kItemNnz nonzeros (a longer row is an item of
    // its own), over the CUDA-core windows (cc_items) or over all windows
    // (all_items, used when the tensor-core kernel cannot run).
    int2 *cc_items = nullptr;
    int2 *all_items = nullptr;
    int n_cc_items = 0, n_all_items = 0;
    // host copy of tile_first: chunk offsets of the tensor-core windows
    // (n_tc + 1), for sizing launches on the host
    std::vector<int> h_tile_first;
    int *d_status = nullptr; // device error word written by bounded waits
    // The arrays above live in three device allocations, made when their
    // sizes become known: [0] the re-ordered CSR (perm .. src, d_status,
    // all_windows), [1] the window lists and tiles (tc_windows .. tile_src),
    // [2] the images and work items (img_idx, img_chunk, cc_items,
    // all_items, images).
    void *arena[3] = {nullptr, nullptr, nullptr};
    size_t bytes = 0;
    // A^T as a plan of its own (built on first use by tca_spmm_t or by
    // tca_plan_build_transpose), with t_src mapping each of its entries to the
    // caller's nonzero index and t_vals the values in that order.
    struct tca_plan *tplan = nullptr;
    int *t_src = nullptr;
    __half *t_vals = nullptr;
    // FP8-E4M3 representation of A (tca_plan_quantize_fp8): per sorted row an
    // FP32 scale (row absmax / 448), the quantized values in sorted order, the
    // tile entries with E4M3 bits in their low byte, and 8 KB dense images
    // (128 x 64 bytes, 64-byte swizzled K-major) for the imaged chunks.
    bool has_fp8 = false;
    float *row_scale = nullptr;
    uint8_t *p_val_f8 = nullptr;
    uint32_t *tile_entries_f8 = nullptr;
    uint8_t *images_f8 = nullptr;
    // workspace of tca_spmm_fp8: B quantized per column (K x N bytes) + N scales
    void *fp8_ws = nullptr;
    size_t fp8_ws_bytes = 0;
};

namespace tca {

// Chunks with at least this many nonzeros (1/16 of the tile) also get a
// pre-rendered dense image, which the tensor-core kernel loads with one bulk
// copy instead of scattering entries: the scatter sits on the chunk's
// critical path, while the image's extra HBM bytes (16 KB, up to 8x the
// entries of such a chunk) do not bound the kernel (measured on the
// 32-problem step at 80 %, threshold 2048 -> 512: FP16 tensor-core kernel
// 53.0 -> 50.4 us, E4M3 43.0 -> 36.9 us; 128 gave 50.1 us for twice the
// image memory of the sparsest chunks).
constexpr int kImageMinNnz = kWindowRows * kChunkCols / 16; // 512
constexpr int kEntryPad = 4;
constexpr int kItemRows = 31;
constexpr int kItemNnz = 32;

// Byte offset of element (r, c) of a 128 x 64 FP16 tile in the 128-byte
// swizzled K-major layout: 16-byte chunk index c/8 XOR-ed with r % 8.
__host__ __device__ inline uint32_t swz128_offset(uint32_t r, uint32_t c)
{
    return r * 128u + ((((c >> 3) ^ (r & 7u))) << 4) + ((c & 7u) << 1);
}

// Byte offset of element (r, c) of a 128 x 64 one-byte (E4M3) tile in the
// 64-byte swizzled K-major layout: 16-byte chunk index c/16 XOR-ed with
// (r / 2) % 4 (address bits 4-5 XOR bits 7-8).
__host__ __device__ inline uint32_t swz64_offset(uint32_t r, uint32_t c)
{
    return r * 64u + ((((c >> 4) ^ ((r >> 1) & 3u))) << 4) + (c & 15u);
}

constexpr float kE4M3Max = 448.f;

// Largest K for which windows may go to the tensor-core path: the builder
// keeps a K-bit column bitmap plus its prefix counts in shared memory.
constexpr int kMaxTcK = 1 << 17;

// Device status bits.
constexpr int kStatusTimeout = 1;
constexpr int kStatusLayout = 2; // shared memory base not 1024-byte aligned: the kernel did no work

// One forward of one plan, as the batched launchers see it.
struct SpmmJob {
    const tca_plan *p;
    const __half *B;
    void *C;
    int ldb, N, ldc;
    bool tc;    // the plan's tensor-core windows run on tensor cores
    int n_tile; // tensor-core N-slice width (64, 128, 256; 128 or 256 for E4M3)
    // E4M3 forward: B quantized per column (K x N bytes, row stride ldq) with
    // its column scales; A's E4M3 form lives in the plan.
    int cc_w = 0; // CUDA-core columns per lane (2, 4, 8), 16 = the mma.sync item kernel; 0 = by N
    bool f8 = false;
    const uint8_t *Bq = nullptr;
    int ldq = 0;
    const float *col_scale = nullptr;
};

// Kernel launches whose host-side preparation (argument blocks, TMA
// descriptors) is already done: running one only launches.
using LaunchList = std::vector<std::function<int(cudaStream_t)>>;

// Tensor-core (tcgen05) forward over the tensor-core windows of every job
// (jobs with tc set), in as few launches as the N-slice widths allow. With
// `defer` the prepared launches are appended to it instead of issued.
int launch_tc_jobs(const SpmmJob *jobs, int n_jobs, int c_dtype, float alpha, float beta, unsigned flags,
                   cudaStream_t s, LaunchList *defer = nullptr);

// Registers that one block of the tensor-core kernel holds on an SM (the
// largest over its FP16 or its E4M3 instantiations).
int tc_block_regs(bool f8, int *regs);

// CUDA-core forward over the remaining windows of every job (all windows of
// jobs without tc), in as few launches as the row widths allow. beside_regs >
// 0: the launches directly follow a tensor-core launch whose one block per SM
// holds that many registers (tc_block_regs); they are issued as programmatic
// dependents of it, which run beside it once its blocks are resident, with
// grids sized to fit beside it. 0: ordinary launches.
int launch_cc_jobs(const SpmmJob *jobs, int n_jobs, int c_dtype, float alpha, float beta, unsigned flags,
                   cudaStream_t s, LaunchList *defer = nullptr, int beside_regs = 0);

// Prepares both launch lists, then issues them with optional events (4
// caller-created cudaEvent_t or NULL) around the tensor-core and the
// CUDA-core launches, so that the events bracket device work only. Without
// events, the CUDA-core launches run concurrently with the tensor-core launch
// (programmatic dependents on the same stream; the two paths write disjoint
// rows of C). Allocates nothing.
int run_jobs_with_events(const SpmmJob *jobs, int n_jobs, int c_dtype, float alpha, float beta, unsigned flags,
                         cudaStream_t s, void *const *events);

// tca_plan_create with two extra controls for the host-buffer forward:
// vals_ready (an event after which the values may be read; NULL: at once)
// and sync_end (false: the build is only ordered on `stream`, not waited for).
int plan_create(const int *d_row_ptr, const int *d_col_idx, const void *d_vals_f16, int M, int K, int nnz,
                const tca_plan_opts_t *opts, cudaStream_t stream, cudaEvent_t vals_ready, bool sync_end,
                tca_plan_t *plan);

// The N-slice width a single forward of this plan uses.
int pick_tc_tile(const tca_plan *p, int N, bool batched, bool f8 = false);

// SDDMM over the plan's tensor-core windows on the tensor cores
// (sddmm_tc.cu); dY and B with 16-byte aligned rows. The nonzeros of the
// CUDA-core windows are left to the caller.
int sddmm_tc(const tca_plan *p, const __half *dY, int ldy, const __half *B, int ldb, int N, void *out, bool out_f16,
             float alpha, cudaStream_t s);

// E4M3 form of A (fp8.cu): refresh after new values (when it exists); release.
int plan_requantize_fp8(tca_plan *p, cudaStream_t s);
void plan_free_fp8(tca_plan *p);

// The plan of A^T (adjoint.cu): propagate new caller-order values; release.
int transpose_update_values(tca_plan *p, const __half *vals, cudaStream_t s);
void transpose_free(tca_plan *p);

// Whether B/C of a forward allow the vectorised and tensor-core kernels.
bool dense_operands_vec_ok(const void *B, int ldb, int N, const void *C, int ldc, int c_dtype);

} // namespace tca
