// plan.cu -- GPU builder of the row-window, column-condensed tile format,
// plan management and the planned forward (tca_spmm).
//
// This replaces the reference's per-call host schedule, workload_manager
// (src/our_spmm.cu:347-471), which bins each row's nnz into a warp count and
// first-fit packs rows into 8-warp thread blocks on the CPU at every call.
// Here the schedule is built once per sparsity pattern, on the GPU, and every
// step is deterministic (stable radix sort, prefix scans, no order-dependent
// atomics), so a host restatement reproduces it bit for bit:
//   1. check the CSR, count each row, flag rows with strictly increasing columns;
//   2. order rows by nnz (descending, ties by row index) and re-order the CSR;
//   3. per 128-row window: distinct columns and touched 64-column blocks of K
//      (a shared-memory bitmap), nnz, eligibility (all rows strictly
//      increasing);
//   4. on the host: a window's chunks are its touched 64-column blocks
//      ("direct": B rows contiguous) when there are at most twice as many of
//      them as chunks of its distinct columns, else its distinct columns 64
//      at a time ("condensed"); it goes to tensor cores when it is eligible
//      and nnz_w >= tc_min_density * 128 * 64 * chunks_w;
//   5. per tensor-core window: its chunk columns (one block per window), then
//      per chunk (one block each) the nonzeros of every row inside the chunk
//      -- counted, prefix-summed into tile_ptr, written as entries packed
//      (local_row << 22 | local_col << 16 | fp16 bits) ordered by (row, col);
//   6. dense 16 KB images of the chunks with >= 512 entries; CUDA-core
//      work items (host).
#include <cub/cub.cuh>
#include <vector>
#include <algorithm>
#include "tca_internal.cuh"
#include "plan.cuh"

namespace tca {
namespace {

constexpr int kErrRowPtr = 1, kErrColRange = 2;

// 1. Row checks: one warp per row.
__global__ void k_row_check(const int *__restrict__ row_ptr, const int *__restrict__ col, int M, int K, int nnz,
                            int *__restrict__ row_nnz, int *__restrict__ row_sorted, int *__restrict__ err)
{
    const int lane = threadIdx.x & 31;
    const long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= M)
        return;
    const int s = row_ptr[r], e = row_ptr[r + 1];
    if (s < 0 || e < s || e > nnz || (r == 0 && s != 0) || (r == M - 1 && e != nnz)) {
        if (lane == 0) {
            atomicOr(err, kErrRowPtr);
            row_nnz[r] = 0;
            row_sorted[r] = 0;
        }
        return;
    }
    bool ok = true, inc = true;
    for (int j = s + lane; j < e; j += 32) {
        const int c = col[j];
        ok &= (c >= 0 && c < K);
        if (j > s)
            inc &= (col[j - 1] < c);
    }
    ok = __all_sync(0xffffffffu, ok);
    inc = __all_sync(0xffffffffu, inc);
    if (lane == 0) {
        if (!ok)
            atomicOr(err, kErrColRange);
        row_nnz[r] = e - s;
        row_sorted[r] = inc ? 1 : 0;
    }
}

__global__ void k_iota(int *a, int n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        a[i] = (int)i;
}

__global__ void k_gather_int(const int *__restrict__ src, const int *__restrict__ idx, int *__restrict__ dst, int n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = src[idx[i]];
}

// 2b. Re-order the CSR: one warp per sorted row. Does nothing when the row
// checks found an error (the host reports it after its next wait).
__global__ void k_permute(const int *__restrict__ perm, const int *__restrict__ row_ptr,
                          const int *__restrict__ col, const __half *__restrict__ val,
                          const int *__restrict__ p_row_ptr, int M, const int *__restrict__ err,
                          int *__restrict__ p_col, __half *__restrict__ p_val, int *__restrict__ src)
{
    const int lane = threadIdx.x & 31;
    const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= M || *err)
        return;
    const int r = perm[i];
    const int s = row_ptr[r], e = row_ptr[r + 1], d = p_row_ptr[i];
    for (int j = lane; j < e - s; j += 32) {
        p_col[d + j] = col[s + j];
        p_val[d + j] = val[s + j];
        src[d + j] = s + j;
    }
}

// Sets the bit of every column of p_col[lo, hi) in the shared bitmap. Eight
// coalesced loads per thread are issued before their atomics, so that the
// loop is not one memory latency per column. A bit is only ever set, so a
// stale read costs at most one redundant atomic.
__device__ __forceinline__ void mark_columns(const int *__restrict__ p_col, int lo, int hi, uint32_t *bm)
{
    constexpr int U = 16; // loads in flight per thread: a window of 128 long rows is ~130K columns
    for (int j0 = lo + threadIdx.x; j0 < hi; j0 += blockDim.x * U) {
        int c[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int j = j0 + u * (int)blockDim.x;
            c[u] = j < hi ? __ldg(p_col + j) : -1;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            // dense windows set the same few words over and over: skip the
            // (serialising) shared atomic when the bit is already there
            if (c[u] >= 0) {
                const uint32_t bit = 1u << (c[u] & 31);
                if (!(*(volatile uint32_t *)&bm[c[u] >> 5] & bit))
                    atomicOr(&bm[c[u] >> 5], bit);
            }
        }
    }
}

// 3. Window statistics: one block per window, K-bit bitmap in shared memory.
// Does nothing when the row checks found an error (see k_permute).
__global__ void k_window_stats(const int *__restrict__ p_row_ptr, const int *__restrict__ p_col,
                               const int *__restrict__ p_sorted, int M, int K, const int *__restrict__ err,
                               int *__restrict__ win_nu, int *__restrict__ win_nnz, int *__restrict__ win_elig,
                               int *__restrict__ win_nblk, uint32_t *__restrict__ bitmaps)
{
    extern __shared__ uint32_t bm[];
    __shared__ int s_cnt, s_elig, s_nblk;
    const int w = blockIdx.x;
    if (*err)
        return; // uniform across the block
    const int nwords = (K + 31) >> 5;
    for (int i = threadIdx.x; i < nwords; i += blockDim.x) bm[i] = 0u;
    if (threadIdx.x == 0) { s_cnt = 0; s_elig = 1; s_nblk = 0; }
    __syncthreads();
    const int r0 = w * kWindowRows, r1 = min(M, r0 + kWindowRows);
    const int lo = p_row_ptr[r0], hi = p_row_ptr[r1];
    mark_columns(p_col, lo, hi, bm);
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x)
        if (!p_sorted[i]) atomicAnd(&s_elig, 0);
    __syncthreads();
    if (bitmaps) // kept for k_tile_cols, which would otherwise read the window's columns again
        for (int i = threadIdx.x; i < nwords; i += blockDim.x) bitmaps[(size_t)w * nwords + i] = bm[i];
    int cnt = 0;
    for (int i = threadIdx.x; i < nwords; i += blockDim.x) cnt += __popc(bm[i]);
    atomicAdd(&s_cnt, cnt); // integer sums: order-independent
    int nb = 0;
    for (int b = threadIdx.x; 2 * b < nwords; b += blockDim.x)
        nb += ((bm[2 * b] | (2 * b + 1 < nwords ? bm[2 * b + 1] : 0u)) != 0u);
    atomicAdd(&s_nblk, nb);
    __syncthreads();
    if (threadIdx.x == 0) {
        win_nu[w] = s_cnt;
        win_nnz[w] = hi - lo;
        win_elig[w] = s_elig;
        win_nblk[w] = s_nblk;
    }
}

// Block-wide exclusive scan of one int per thread (blockDim.x a multiple of
// 32, at most 1024); *total gets the sum. scratch holds >= 33 ints.
__device__ int block_exclusive_scan(int v, int *total, int *scratch)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) scratch[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int k = 0; k < nw; k++) { const int t = scratch[k]; scratch[k] = run; run += t; }
        scratch[32] = run;
    }
    __syncthreads();
    const int res = x - v + scratch[warp];
    *total = scratch[32];
    __syncthreads();
    return res;
}

// 5a. Window columns: one block of 1024 threads per tensor-core window builds
// the window's column bitmap (expanded to whole 64-column blocks for a direct
// window) and writes its columns, ascending, 64 per chunk, -1 padding.
__global__ void __launch_bounds__(1024)
k_tile_cols(const int4 *__restrict__ win_info, const int *__restrict__ p_row_ptr, const int *__restrict__ p_col,
            int M, int K, const uint32_t *__restrict__ bitmaps, int *__restrict__ win_cols)
{
    extern __shared__ uint32_t sm[];
    __shared__ int scratch[33];
    const int nwords = (K + 31) >> 5;
    uint32_t *bm = sm;
    int *pre = reinterpret_cast<int *>(sm + nwords);
    const int4 wi = win_info[blockIdx.x];
    const int w = wi.x, c0 = wi.y, nch = wi.z;
    const int r0 = w * kWindowRows, r1 = min(M, r0 + kWindowRows);
    const int lo = p_row_ptr[r0], hi = p_row_ptr[r1];

    if (bitmaps) { // the window's column bitmap, as k_window_stats built it
        for (int i = threadIdx.x; i < nwords; i += blockDim.x) bm[i] = bitmaps[(size_t)w * nwords + i];
    } else {
        for (int i = threadIdx.x; i < nwords; i += blockDim.x) bm[i] = 0u;
        __syncthreads();
        mark_columns(p_col, lo, hi, bm);
    }
    __syncthreads();
    if (wi.w) { // direct window: every column < K of each touched 64-column block
        for (int b = threadIdx.x; 2 * b < nwords; b += blockDim.x) {
            const bool hit = (bm[2 * b] | (2 * b + 1 < nwords ? bm[2 * b + 1] : 0u)) != 0u;
            for (int q = 0; q < 2 && 2 * b + q < nwords; q++) {
                const int base = (2 * b + q) * 32;
                const int valid = min(32, K - base);
                bm[2 * b + q] = hit ? (valid >= 32 ? 0xffffffffu : ((1u << valid) - 1u)) : 0u;
            }
        }
        __syncthreads();
    }
    // exclusive prefix of popcounts over words: each thread owns a contiguous segment
    const int seg = (nwords + blockDim.x - 1) / blockDim.x;
    const int wb = min(nwords, (int)threadIdx.x * seg), we = min(nwords, wb + seg);
    int local = 0;
    for (int i = wb; i < we; i++) local += __popc(bm[i]);
    int nu;
    int run = block_exclusive_scan(local, &nu, scratch);
    for (int i = wb; i < we; i++) { pre[i] = run; run += __popc(bm[i]); }
    __syncthreads();
    int *wc = win_cols + (size_t)c0 * kChunkCols;
    for (int i = threadIdx.x; i < nwords; i += blockDim.x) {
        uint32_t b = bm[i];
        int rk = pre[i];
        while (b) {
            const int bit = __ffs(b) - 1;
            wc[rk++] = i * 32 + bit;
            b &= b - 1;
        }
    }
    for (int k = nu + threadIdx.x; k < nch * kChunkCols; k += blockDim.x) wc[k] = -1;
}

// First position in the sorted columns p_col[a, b) whose column is >= v.
__device__ __forceinline__ int lower_bound_col(const int *__restrict__ p_col, int a, int b, int v)
{
    while (a < b) {
        const int mid = (a + b) >> 1;
        if (p_col[mid] < v) a = mid + 1; else b = mid;
    }
    return a;
}

// The nonzeros of local row lr of chunk c of window wi are p_col[*lo, *hi):
// the row's columns from the chunk's first column up to the next chunk's
// first column (a chunk holds at most 64 columns of a row).
__device__ __forceinline__ void chunk_row_range(const int4 &wi, int c, int lr, const int *__restrict__ p_row_ptr,
                                                const int *__restrict__ p_col, const int *__restrict__ wc, int M,
                                                int *lo, int *hi)
{
    const int i = wi.x * kWindowRows + lr;
    *lo = *hi = 0;
    if (i >= M)
        return;
    const int rs = p_row_ptr[i], re = p_row_ptr[i + 1];
    const int first = wc[c * kChunkCols];
    const int next = c + 1 < wi.z ? wc[(c + 1) * kChunkCols] : 0x7fffffff;
    *lo = lower_bound_col(p_col, rs, re, first);
    *hi = lower_bound_col(p_col, *lo, min(re, *lo + kChunkCols), next);
}

// 5b. Nonzeros per chunk: one block of 128 threads (= rows) per chunk; each
// row's range in the chunk is kept in row_range for 5c.
__global__ void __launch_bounds__(128)
k_tile_count(const int2 *__restrict__ chunk_win, const int4 *__restrict__ win_info,
             const int *__restrict__ p_row_ptr, const int *__restrict__ p_col, const int *__restrict__ win_cols,
             int M, int *__restrict__ chunk_nnz, int2 *__restrict__ row_range)
{
    __shared__ int scratch[33];
    const int2 cw = chunk_win[blockIdx.x];
    const int4 wi = win_info[cw.x];
    const int *wc = win_cols + (size_t)wi.y * kChunkCols;
    int lo, hi;
    chunk_row_range(wi, cw.y, threadIdx.x, p_row_ptr, p_col, wc, M, &lo, &hi);
    row_range[(size_t)blockIdx.x * kWindowRows + threadIdx.x] = make_int2(lo, hi);
    int total;
    block_exclusive_scan(hi - lo, &total, scratch);
    if (threadIdx.x == 0)
        chunk_nnz[blockIdx.x] = total;
}

// 5c. Entries of each chunk, ordered by (row, column): one block per chunk;
// tile_ptr (the exclusive sum of chunk_nnz) gives the chunk's first entry.
// Thread = row of the window; a row's columns and values in the chunk are
// read 8 at a time before any is used (the walk is otherwise one dependent
// load per entry).
__global__ void __launch_bounds__(128)
k_tile_write(const int2 *__restrict__ chunk_win, const int4 *__restrict__ win_info,
             const int *__restrict__ p_col, const __half *__restrict__ p_val, const int *__restrict__ win_cols,
             const int *__restrict__ tile_ptr, const int2 *__restrict__ row_range, uint32_t *__restrict__ entries,
             int *__restrict__ tile_src)
{
    constexpr int U = 8;
    __shared__ int scratch[33];
    __shared__ int s_cols[kChunkCols];
    const int2 cw = chunk_win[blockIdx.x];
    const int4 wi = win_info[cw.x];
    const int *wc = win_cols + (size_t)wi.y * kChunkCols;
    if (threadIdx.x < kChunkCols)
        s_cols[threadIdx.x] = wc[cw.y * kChunkCols + threadIdx.x];
    const int2 rr = row_range[(size_t)blockIdx.x * kWindowRows + threadIdx.x]; // from k_tile_count
    const int lo = rr.x, hi = rr.y;
    int total;
    const int off = block_exclusive_scan(hi - lo, &total, scratch); // its barriers also publish s_cols
    const long long base = (long long)tile_ptr[blockIdx.x] + off;
    const int first = s_cols[0];
    const uint32_t lr = threadIdx.x;
    for (int j0 = lo; j0 < hi; j0 += U) {
        int col[U];
        unsigned short val[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            col[u] = j0 + u < hi ? p_col[j0 + u] : 0;
            val[u] = j0 + u < hi ? __half_as_ushort(p_val[j0 + u]) : (unsigned short)0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (j0 + u >= hi)
                break;
            int rk;
            if (wi.w) {
                rk = col[u] - first; // direct chunk: 64 consecutive columns
            } else {                 // condensed chunk: position among its ascending columns (-1 padding last)
                int a = 0, b = kChunkCols;
                while (a < b) {
                    const int mid = (a + b) >> 1;
                    const int v = s_cols[mid];
                    if (v >= 0 && v < col[u]) a = mid + 1; else b = mid;
                }
                rk = a;
            }
            entries[base + (j0 + u - lo)] = (lr << 22) | ((uint32_t)rk << 16) | (uint32_t)val[u];
            tile_src[base + (j0 + u - lo)] = j0 + u;
        }
    }
}

__global__ void k_update_p_val(const int *__restrict__ src, const __half *__restrict__ vals, __half *__restrict__ p_val, int n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        p_val[i] = vals[src[i]];
}

__global__ void k_update_entries(const int *__restrict__ tile_src, const __half *__restrict__ p_val,
                                 uint32_t *__restrict__ entries, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        entries[i] = (entries[i] & 0xffff0000u) | (uint32_t)__half_as_ushort(p_val[tile_src[i]]);
}

// Dense tile images: one block per image chunk renders the 128 x 64 tile in
// shared memory -- zeroed, then every entry at its 128-byte-swizzled K-major
// position (positions are distinct within a chunk, so the result does not
// depend on thread order) -- and writes it out in 16-byte stores.
__global__ void __launch_bounds__(256)
k_render_images(const int *__restrict__ img_chunk, const int *__restrict__ tile_ptr,
                const uint32_t *__restrict__ entries, uint16_t *__restrict__ images)
{
    constexpr int kBytes = kWindowRows * kChunkCols * 2;
    __shared__ __align__(16) uint8_t tile[kBytes];
    const int m = blockIdx.x;
    const int c = img_chunk[m];
    for (int k = threadIdx.x; k < kBytes / 16; k += blockDim.x)
        reinterpret_cast<uint4 *>(tile)[k] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    const int e0 = tile_ptr[c], e1 = tile_ptr[c + 1];
    for (int e = e0 + (int)threadIdx.x; e < e1; e += 8 * (int)blockDim.x) { // 8 loads in flight per thread
        uint32_t v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int eu = e + u * (int)blockDim.x;
            v[u] = eu < e1 ? entries[eu] : 0xffffffffu;
        }
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (v[u] != 0xffffffffu)
                *reinterpret_cast<uint16_t *>(tile + swz128_offset(v[u] >> 22, (v[u] >> 16) & 63u)) =
                    (uint16_t)(v[u] & 0xffffu);
    }
    __syncthreads();
    uint4 *img = reinterpret_cast<uint4 *>(images + (size_t)m * kWindowRows * kChunkCols);
    for (int k = threadIdx.x; k < kBytes / 16; k += blockDim.x)
        img[k] = reinterpret_cast<const uint4 *>(tile)[k];
}

unsigned blocks_for(long long n, int per) { return (unsigned)((n + per - 1) / per); }

// The stream a plan is being built on: temporaries and plan arrays are
// stream-ordered allocations on it.
thread_local cudaStream_t tl_build_stream = nullptr;

struct BuildStream {
    cudaStream_t prev;
    explicit BuildStream(cudaStream_t s) : prev(tl_build_stream) { tl_build_stream = s; }
    ~BuildStream() { tl_build_stream = prev; }
};

struct DevBuf {
    void *p = nullptr;
    cudaStream_t s = tl_build_stream;
    ~DevBuf() { if (p) dev_free(p, s); }
};

template <typename T>
int dev_alloc(T **ptr, size_t count, size_t *bytes)
{
    const size_t b = sizeof(T) * (count > 0 ? count : 1);
    TCA_TRY(dev_malloc((void **)ptr, b, tl_build_stream));
    if (bytes) *bytes += b;
    return TCA_OK;
}

void free_plan(tca_plan *p)
{
    if (!p) return;
    cudaDeviceSynchronize(); // the plan's arrays may still be read by queued work on any stream
    transpose_free(p);
    plan_free_fp8(p);
    void *arrs[] = {p->perm, p->p_row_ptr, p->p_col, p->p_val, p->src, p->tc_windows, p->cc_windows,
                    p->all_windows, p->tile_first, p->win_cols, p->tile_ptr, p->tile_entries, p->tile_src,
                    p->img_idx, p->images, p->img_chunk, p->cc_items, p->all_items, p->tc_win_info,
                    p->tc_pairs, p->d_status};
    for (void *a : arrs)
        if (a) dev_free(a, nullptr);
    delete p;
}

// CUDA-core work items over the rows of `windows` (host, deterministic):
// maximal runs of consecutive listed rows are cut greedily into items of at
// most kItemRows rows whose nonzeros stay within kItemNnz (a row above that
// is an item of its own).
void build_items(const std::vector<int> &windows, const std::vector<int> &row_ptr, int M, std::vector<int2> &items)
{
    items.clear();
    size_t w = 0;
    while (w < windows.size()) {
        const int a = windows[w] * kWindowRows;
        size_t v = w + 1;
        while (v < windows.size() && windows[v] == windows[v - 1] + 1) v++;
        const int b = std::min(M, windows[v - 1] * kWindowRows + kWindowRows);
        int i = a;
        while (i < b) {
            const int r0 = i;
            int nz = row_ptr[i + 1] - row_ptr[i];
            i++;
            while (i < b && i - r0 < kItemRows && nz + (row_ptr[i + 1] - row_ptr[i]) <= kItemNnz) {
                nz += row_ptr[i + 1] - row_ptr[i];
                i++;
            }
            items.push_back(make_int2(r0, i));
        }
        w = v;
    }
}

// vals_ready: an event after which `val` may be read (the host-buffer path
// copies the values on a second stream); sync_end: wait for the whole build
// before returning (so that the plan is usable on any stream).
int build_plan(tca_plan *p, const int *row_ptr, const int *col, const __half *val, cudaStream_t s,
               cudaEvent_t vals_ready = nullptr, bool sync_end = true)
{
    BuildStream build_stream(s);
    const int M = p->M, K = p->K, nnz = p->nnz;
    size_t *bytes = &p->bytes;
    DevBuf t_row_nnz, t_row_sorted, t_err, t_iota, t_keys_out, t_p_sorted, t_scan_in, t_cub;
    int *row_nnz, *row_sorted, *err, *iota, *keys_out, *p_sorted, *scan_in;
    TCA_TRY(dev_alloc(&row_nnz, M, nullptr)); t_row_nnz.p = row_nnz;
    TCA_TRY(dev_alloc(&row_sorted, M, nullptr)); t_row_sorted.p = row_sorted;
    TCA_TRY(dev_alloc(&err, 1, nullptr)); t_err.p = err;
    TCA_TRY(dev_alloc(&iota, M, nullptr)); t_iota.p = iota;
    TCA_TRY(dev_alloc(&keys_out, M, nullptr)); t_keys_out.p = keys_out;
    TCA_TRY(dev_alloc(&p_sorted, M, nullptr)); t_p_sorted.p = p_sorted;
    TCA_TRY(dev_alloc(&scan_in, M + 1, nullptr)); t_scan_in.p = scan_in;

    TCA_TRY(dev_alloc(&p->perm, M, bytes));
    TCA_TRY(dev_alloc(&p->p_row_ptr, M + 1, bytes));
    TCA_TRY(dev_alloc(&p->p_col, nnz, bytes));
    TCA_TRY(dev_alloc(&p->p_val, nnz, bytes));
    TCA_TRY(dev_alloc(&p->src, nnz, bytes));
    TCA_TRY(dev_alloc(&p->d_status, 1, bytes));
    TCA_CUDA_TRY(cudaMemsetAsync(p->d_status, 0, sizeof(int), s));
    TCA_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));

    // 1. checks; the host reads their verdict with the window statistics
    // (step 3), the kernels that follow stand down on an error
    k_row_check<<<blocks_for((long long)M * 32, 256), 256, 0, s>>>(row_ptr, col, M, K, nnz, row_nnz, row_sorted, err);
    TCA_CUDA_TRY(cudaGetLastError());

    // 2. row order
    k_iota<<<blocks_for(M, 256), 256, 0, s>>>(iota, M);
    if (p->opts.sort_rows) {
        // row lengths are at most nnz: only their low bits take part
        int end_bit = 1;
        while (end_bit < 32 && ((long long)1 << end_bit) <= (long long)nnz) end_bit++;
        size_t tmp = 0;
        TCA_CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, row_nnz, keys_out, iota, p->perm, M, 0,
                                                               end_bit, s));
        void *tbuf;
        TCA_TRY(dev_alloc((char **)&tbuf, tmp, nullptr)); t_cub.p = tbuf;
        TCA_CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(tbuf, tmp, row_nnz, keys_out, iota, p->perm, M, 0,
                                                               end_bit, s));
    } else {
        TCA_CUDA_TRY(cudaMemcpyAsync(p->perm, iota, sizeof(int) * M, cudaMemcpyDeviceToDevice, s));
    }
    TCA_CUDA_TRY(cudaMemsetAsync(scan_in + M, 0, sizeof(int), s));
    k_gather_int<<<blocks_for(M, 256), 256, 0, s>>>(row_nnz, p->perm, scan_in, M);
    k_gather_int<<<blocks_for(M, 256), 256, 0, s>>>(row_sorted, p->perm, p_sorted, M);
    {
        size_t tmp = 0;
        TCA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp, scan_in, p->p_row_ptr, M + 1, s));
        DevBuf tb;
        char *tbuf;
        TCA_TRY(dev_alloc(&tbuf, tmp, nullptr)); tb.p = tbuf;
        TCA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tbuf, tmp, scan_in, p->p_row_ptr, M + 1, s));
    } // tb is released in stream order on s (DevBuf): no wait
    if (vals_ready)
        TCA_CUDA_TRY(cudaStreamWaitEvent(s, vals_ready, 0));
    k_permute<<<blocks_for((long long)M * 32, 256), 256, 0, s>>>(p->perm, row_ptr, col, val, p->p_row_ptr, M, err,
                                                                 p->p_col, p->p_val, p->src);
    TCA_CUDA_TRY(cudaGetLastError());

    // 3. windows. The host reads, in one copy after one wait, everything it
    // decides on: per window its distinct columns, nonzeros, sortedness and
    // touched 64-column blocks, the check verdict and the sorted row offsets
    // (for the work items, step 7), gathered in one device array.
    const int W = (M + kWindowRows - 1) / kWindowRows;
    p->n_windows = W;
    std::vector<int> h_all(W);
    for (int w = 0; w < W; w++) h_all[w] = w;
    TCA_TRY(dev_alloc(&p->all_windows, W, bytes));
    TCA_CUDA_TRY(cudaMemcpyAsync(p->all_windows, h_all.data(), sizeof(int) * W, cudaMemcpyHostToDevice, s));

    const size_t n_stage = 4 * (size_t)W + 1 + (size_t)M + 1;
    DevBuf t_stage;
    int *d_stage;
    TCA_TRY(dev_alloc(&d_stage, n_stage, nullptr)); t_stage.p = d_stage;
    int *d_nu = d_stage, *d_wn = d_stage + W, *d_el = d_stage + 2 * W, *d_nb = d_stage + 3 * W;
    const bool tc_possible = (p->opts.path != 1) && K <= kMaxTcK && K > 0 && W > 0;
    // the windows' column bitmaps, kept from the statistics for the tile
    // columns when they take at most 64 MB (else k_tile_cols rebuilds them)
    DevBuf t_bm;
    uint32_t *d_bm = nullptr;
    if (tc_possible && (size_t)W * ((K + 31) / 32) <= (size_t)(16u << 20)) {
        TCA_TRY(dev_alloc(&d_bm, (size_t)W * ((K + 31) / 32), nullptr));
        t_bm.p = d_bm;
    }
    if (tc_possible) {
        const size_t smem = sizeof(uint32_t) * ((K + 31) / 32);
        TCA_CUDA_TRY(cudaFuncSetAttribute(k_window_stats, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_window_stats<<<W, 1024, smem, s>>>(p->p_row_ptr, p->p_col, p_sorted, M, K, err, d_nu, d_wn, d_el, d_nb,
                                             d_bm);
        TCA_CUDA_TRY(cudaGetLastError());
    } else if (W > 0) {
        TCA_CUDA_TRY(cudaMemsetAsync(d_stage, 0, sizeof(int) * 4 * (size_t)W, s));
    }
    TCA_CUDA_TRY(cudaMemcpyAsync(d_stage + 4 * W, err, sizeof(int), cudaMemcpyDeviceToDevice, s));
    TCA_CUDA_TRY(cudaMemcpyAsync(d_stage + 4 * W + 1, p->p_row_ptr, sizeof(int) * ((size_t)M + 1),
                                 cudaMemcpyDeviceToDevice, s));
    std::vector<int> h_stage(n_stage);
    TCA_CUDA_TRY(cudaMemcpyAsync(h_stage.data(), d_stage, sizeof(int) * n_stage, cudaMemcpyDeviceToHost, s));
    TCA_CUDA_TRY(cudaStreamSynchronize(s));
    const int h_err = h_stage[4 * (size_t)W];
    if (h_err & kErrRowPtr)
        return set_error(TCA_ERR_FORMAT, "row_ptr is not a valid CSR offset array (must start at 0, be non-decreasing and end at nnz=%d)", nnz);
    if (h_err & kErrColRange)
        return set_error(TCA_ERR_FORMAT, "a column index lies outside [0, K=%d)", K);
    const int *h_nu = h_stage.data(), *h_nnz = h_nu + W, *h_elig = h_nu + 2 * W, *h_nblk = h_nu + 3 * W;
    const std::vector<int> h_rp(h_stage.begin() + 4 * (size_t)W + 1, h_stage.end());

    // 4. path decision (host, deterministic)
    // A window's chunks are "direct" (the 64-column blocks of K it touches,
    // whose B rows are contiguous and load as tiled TMA boxes) when that needs
    // at most twice the chunks of condensing its distinct columns (gathered
    // B rows); otherwise condensed.
    std::vector<int> tc_list, cc_list, h_first(1, 0), h_direct, h_full;
    const int n_kblocks = (K + kChunkCols - 1) / kChunkCols;
    long long ebase = 0; // nonzeros of the tensor-core windows so far
    for (int w = 0; w < W; w++) {
        const int nch_cond = (h_nu[w] + kChunkCols - 1) / kChunkCols;
        const bool direct = h_nblk[w] <= 2 * nch_cond;
        const int nch = direct ? h_nblk[w] : nch_cond;
        bool tc = false;
        if (tc_possible && h_elig[w] && h_nnz[w] > 0) {
            if (p->opts.path == 2)
                tc = true;
            else
                tc = (double)h_nnz[w] >= (double)p->opts.tc_min_density * (double)(kWindowRows * kChunkCols) * (double)nch;
        }
        if (tc) {
            tc_list.push_back(w);
            h_direct.push_back(direct ? 1 : 0);
            h_full.push_back(direct && h_nblk[w] == n_kblocks ? 1 : 0);
            h_first.push_back(h_first.back() + nch);
            ebase += h_nnz[w];
        } else {
            cc_list.push_back(w);
        }
    }
    p->n_tc = (int)tc_list.size();
    p->n_cc = (int)cc_list.size();
    p->n_tc_chunks = h_first.back();
    p->h_tile_first = h_first;
    p->tc_nnz = ebase;
    TCA_TRY(dev_alloc(&p->tc_windows, p->n_tc, bytes));
    TCA_TRY(dev_alloc(&p->cc_windows, p->n_cc, bytes));
    TCA_TRY(dev_alloc(&p->tile_first, p->n_tc + 1, bytes));
    if (p->n_tc)
        TCA_CUDA_TRY(cudaMemcpyAsync(p->tc_windows, tc_list.data(), sizeof(int) * p->n_tc, cudaMemcpyHostToDevice, s));
    if (p->n_cc)
        TCA_CUDA_TRY(cudaMemcpyAsync(p->cc_windows, cc_list.data(), sizeof(int) * p->n_cc, cudaMemcpyHostToDevice, s));
    TCA_CUDA_TRY(cudaMemcpyAsync(p->tile_first, h_first.data(), sizeof(int) * (p->n_tc + 1), cudaMemcpyHostToDevice, s));
    std::vector<int4> h_wi((size_t)p->n_tc);
    for (int t = 0; t < p->n_tc; t++)
        h_wi[t] = make_int4(tc_list[t], h_first[t], h_first[t + 1] - h_first[t], h_direct[t]);
    TCA_TRY(dev_alloc(&p->tc_win_info, (size_t)p->n_tc, bytes));
    if (p->n_tc)
        TCA_CUDA_TRY(cudaMemcpyAsync(p->tc_win_info, h_wi.data(), sizeof(int4) * p->n_tc, cudaMemcpyHostToDevice, s));
    // window pairs for the pair kernel: greedily, consecutive windows whose
    // chunks are all 64-column blocks of K (identical columns)
    std::vector<int2> h_pairs;
    p->n_full_pairs = 0;
    for (int t = 0; t < p->n_tc;) {
        if (h_full[t] && t + 1 < p->n_tc && h_full[t + 1]) {
            h_pairs.push_back(make_int2(t, t + 1));
            p->n_full_pairs++;
            t += 2;
        } else {
            h_pairs.push_back(make_int2(t, -1));
            t += 1;
        }
    }
    p->n_pairs = (int)h_pairs.size();
    TCA_TRY(dev_alloc(&p->tc_pairs, (size_t)p->n_pairs, bytes));
    if (p->n_pairs)
        TCA_CUDA_TRY(cudaMemcpyAsync(p->tc_pairs, h_pairs.data(), sizeof(int2) * p->n_pairs, cudaMemcpyHostToDevice, s));

    // 5. tiles
    TCA_TRY(dev_alloc(&p->win_cols, (size_t)p->n_tc_chunks * kChunkCols, bytes));
    TCA_TRY(dev_alloc(&p->tile_ptr, (size_t)p->n_tc_chunks + 1, bytes));
    TCA_TRY(dev_alloc(&p->tile_entries, (size_t)p->tc_nnz + kEntryPad, bytes));
    TCA_CUDA_TRY(cudaMemsetAsync(p->tile_entries + p->tc_nnz, 0, sizeof(uint32_t) * kEntryPad, s));
    TCA_TRY(dev_alloc(&p->tile_src, (size_t)p->tc_nnz, bytes));
    if (p->n_tc > 0) {
        // chunk -> (tensor-core window, chunk within the window)
        std::vector<int2> h_cw;
        h_cw.reserve((size_t)p->n_tc_chunks);
        for (int t = 0; t < p->n_tc; t++)
            for (int c = 0; c < h_wi[t].z; c++) h_cw.push_back(make_int2(t, c));
        DevBuf t_cw, t_cn, t_scan, t_rr;
        int2 *d_cw, *d_rr;
        int *d_cn;
        TCA_TRY(dev_alloc(&d_cw, (size_t)p->n_tc_chunks, nullptr)); t_cw.p = d_cw;
        TCA_TRY(dev_alloc(&d_cn, (size_t)p->n_tc_chunks + 1, nullptr)); t_cn.p = d_cn;
        TCA_TRY(dev_alloc(&d_rr, (size_t)p->n_tc_chunks * kWindowRows, nullptr)); t_rr.p = d_rr;
        TCA_CUDA_TRY(cudaMemcpyAsync(d_cw, h_cw.data(), sizeof(int2) * h_cw.size(), cudaMemcpyHostToDevice, s));
        TCA_CUDA_TRY(cudaMemsetAsync(d_cn + p->n_tc_chunks, 0, sizeof(int), s));
        const size_t smem = 2 * sizeof(uint32_t) * ((K + 31) / 32);
        TCA_CUDA_TRY(cudaFuncSetAttribute(k_tile_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_tile_cols<<<p->n_tc, 1024, smem, s>>>(p->tc_win_info, p->p_row_ptr, p->p_col, M, K, d_bm, p->win_cols);
        k_tile_count<<<p->n_tc_chunks, 128, 0, s>>>(d_cw, p->tc_win_info, p->p_row_ptr, p->p_col, p->win_cols, M,
                                                    d_cn, d_rr);
        size_t tmp = 0;
        TCA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_cn, p->tile_ptr, p->n_tc_chunks + 1, s));
        void *tb;
        TCA_TRY(dev_alloc((char **)&tb, tmp, nullptr)); t_scan.p = tb;
        TCA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tb, tmp, d_cn, p->tile_ptr, p->n_tc_chunks + 1, s));
        k_tile_write<<<p->n_tc_chunks, 128, 0, s>>>(d_cw, p->tc_win_info, p->p_col, p->p_val, p->win_cols,
                                                    p->tile_ptr, d_rr, p->tile_entries, p->tile_src);
        TCA_CUDA_TRY(cudaGetLastError());
    } else {
        TCA_CUDA_TRY(cudaMemsetAsync(p->tile_ptr, 0, sizeof(int), s));
    }

    // 6. dense tile images for chunks holding at least kImageMinNnz nonzeros
    std::vector<int> h_ptr((size_t)p->n_tc_chunks + 1, 0), h_img((size_t)p->n_tc_chunks, -1), h_img_chunk;
    if (p->n_tc_chunks > 0)
        TCA_CUDA_TRY(cudaMemcpyAsync(h_ptr.data(), p->tile_ptr, sizeof(int) * h_ptr.size(), cudaMemcpyDeviceToHost, s));
    TCA_CUDA_TRY(cudaStreamSynchronize(s));
    for (int c = 0; c < p->n_tc_chunks; c++)
        if (h_ptr[c + 1] - h_ptr[c] >= kImageMinNnz) {
            h_img[c] = (int)h_img_chunk.size();
            h_img_chunk.push_back(c);
        }
    p->n_images = (int)h_img_chunk.size();
    TCA_TRY(dev_alloc(&p->img_idx, (size_t)p->n_tc_chunks, bytes));
    TCA_TRY(dev_alloc(&p->img_chunk, (size_t)p->n_images, bytes));
    TCA_TRY(dev_alloc(&p->images, (size_t)p->n_images * kWindowRows * kChunkCols, bytes));
    if (p->n_tc_chunks > 0)
        TCA_CUDA_TRY(cudaMemcpyAsync(p->img_idx, h_img.data(), sizeof(int) * h_img.size(), cudaMemcpyHostToDevice, s));
    if (p->n_images > 0) {
        TCA_CUDA_TRY(cudaMemcpyAsync(p->img_chunk, h_img_chunk.data(), sizeof(int) * h_img_chunk.size(),
                                     cudaMemcpyHostToDevice, s));
        k_render_images<<<p->n_images, 256, 0, s>>>(p->img_chunk, p->tile_ptr, p->tile_entries, p->images);
        TCA_CUDA_TRY(cudaGetLastError());
    }

    // 7. CUDA-core work items. The host arrays copied to the device here (and
    // above) are pageable, so a copy returns once its data is staged; each
    // copy still has a source array of its own.
    std::vector<int2> cc_items, all_items;
    build_items(cc_list, h_rp, M, cc_items);
    p->n_cc_items = (int)cc_items.size();
    TCA_TRY(dev_alloc(&p->cc_items, cc_items.size(), bytes));
    if (!cc_items.empty())
        TCA_CUDA_TRY(cudaMemcpyAsync(p->cc_items, cc_items.data(), sizeof(int2) * cc_items.size(),
                                     cudaMemcpyHostToDevice, s));
    build_items(h_all, h_rp, M, all_items);
    p->n_all_items = (int)all_items.size();
    TCA_TRY(dev_alloc(&p->all_items, all_items.size(), bytes));
    if (!all_items.empty())
        TCA_CUDA_TRY(cudaMemcpyAsync(p->all_items, all_items.data(), sizeof(int2) * all_items.size(),
                                     cudaMemcpyHostToDevice, s));
    if (sync_end)
        TCA_CUDA_TRY(cudaStreamSynchronize(s)); // the plan is complete, for work on any stream
    return TCA_OK;
}

} // namespace
} // namespace tca

namespace tca {
int run_jobs_with_events(const SpmmJob *jobs, int n_jobs, int c_dtype, float alpha, float beta, unsigned flags,
                         cudaStream_t s, void *const *events)
{
    // Without events the CUDA-core launches follow the tensor-core launch as
    // programmatic dependents and run beside it; with events (which time each
    // path alone) the two run one after the other.
    LaunchList tc, cc;
    TCA_TRY(launch_tc_jobs(jobs, n_jobs, c_dtype, alpha, beta, flags, s, &tc));
    int beside = 0;
    for (int i = 0; !events && !tc.empty() && i < n_jobs; i++) {
        int r = 0;
        TCA_TRY(tc_block_regs(jobs[i].f8, &r));
        beside = std::max(beside, r);
    }
    TCA_TRY(launch_cc_jobs(jobs, n_jobs, c_dtype, alpha, beta, flags, s, &cc, beside));
    // Under stream capture a plain record only orders the graph; an external
    // record becomes a graph node that records the event at every replay.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (events)
        TCA_CUDA_TRY(cudaStreamIsCapturing(s, &cap));
    const unsigned rec_flags = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
    auto rec = [&](int i) -> int {
        if (events && events[i]) TCA_CUDA_TRY(cudaEventRecordWithFlags((cudaEvent_t)events[i], s, rec_flags));
        return TCA_OK;
    };
    TCA_TRY(rec(0));
    for (auto &f : tc) TCA_TRY(f(s));
    TCA_TRY(rec(1));
    TCA_TRY(rec(2));
    for (auto &f : cc) TCA_TRY(f(s));
    TCA_TRY(rec(3));
    return TCA_OK;
}
} // namespace tca

namespace tca {
int plan_create(const int *d_row_ptr, const int *d_col_idx, const void *d_vals_f16, int M, int K, int nnz,
                const tca_plan_opts_t *opts, cudaStream_t stream, cudaEvent_t vals_ready, bool sync_end,
                tca_plan_t *plan)
{
    clear_error();
    if (!plan)
        return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    *plan = nullptr;
    if (M < 0 || K < 0 || nnz < 0)
        return set_error(TCA_ERR_INVALID_ARG, "negative size (M=%d K=%d nnz=%d)", M, K, nnz);
    if ((M > 0 && !d_row_ptr) || (nnz > 0 && (!d_col_idx || !d_vals_f16)))
        return set_error(TCA_ERR_INVALID_ARG, "CSR array is NULL");
    tca_plan_opts_t o;
    tca_plan_opts_default(&o);
    if (opts) o = *opts;
    if (o.path < 0 || o.path > 2 || !(o.tc_min_density >= 0.f))
        return set_error(TCA_ERR_INVALID_ARG, "invalid plan options");
    tca_plan *p = new (std::nothrow) tca_plan();
    if (!p)
        return set_error(TCA_ERR_ALLOC, "host allocation failed");
    p->M = M; p->K = K; p->nnz = nnz; p->opts = o;
    int st = TCA_OK;
    if (M > 0)
        st = build_plan(p, d_row_ptr, d_col_idx, (const __half *)d_vals_f16, stream, vals_ready, sync_end);
    if (st != TCA_OK) {
        free_plan(p);
        return st;
    }
    *plan = p;
    return TCA_OK;
}
} // namespace tca

using namespace tca;

extern "C" {

void tca_plan_opts_default(tca_plan_opts_t *o)
{
    if (!o) return;
    *o = tca_plan_opts_t{};
    o->sort_rows = 1;
    o->tc_min_density = 0.02f;
    o->path = 0;
    o->pair_windows = 0;
}

int tca_plan_create(const int *d_row_ptr, const int *d_col_idx, const void *d_vals_f16, int M, int K, int nnz,
                    const tca_plan_opts_t *opts, tca_stream_t stream, tca_plan_t *plan)
{
    return plan_create(d_row_ptr, d_col_idx, d_vals_f16, M, K, nnz, opts, (cudaStream_t)stream, nullptr, true, plan);
}

int tca_plan_update_values(tca_plan_t p, const void *d_vals_f16, tca_stream_t stream)
{
    clear_error();
    if (!p) return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    if (p->nnz == 0) return TCA_OK;
    if (!d_vals_f16) return set_error(TCA_ERR_INVALID_ARG, "values are NULL");
    cudaStream_t s = (cudaStream_t)stream;
    k_update_p_val<<<blocks_for(p->nnz, 256), 256, 0, s>>>(p->src, (const __half *)d_vals_f16, p->p_val, p->nnz);
    if (p->tc_nnz > 0)
        k_update_entries<<<blocks_for(p->tc_nnz, 256), 256, 0, s>>>(p->tile_src, p->p_val, p->tile_entries, p->tc_nnz);
    if (p->n_images > 0)
        k_render_images<<<p->n_images, 256, 0, s>>>(p->img_chunk, p->tile_ptr, p->tile_entries, p->images);
    TCA_CUDA_TRY(cudaGetLastError());
    TCA_TRY(plan_requantize_fp8(p, s));
    return transpose_update_values(p, (const __half *)d_vals_f16, s);
}

int tca_plan_info(tca_plan_t p, tca_plan_info_t *info)
{
    clear_error();
    if (!p || !info) return set_error(TCA_ERR_INVALID_ARG, "NULL argument");
    *info = tca_plan_info_t{};
    info->M = p->M; info->K = p->K; info->nnz = p->nnz;
    info->n_windows = p->n_windows;
    info->n_tc_windows = p->n_tc;
    info->n_cc_windows = p->n_cc;
    info->n_tc_chunks = p->n_tc_chunks;
    info->tc_nnz = p->tc_nnz;
    info->format_bytes = (long long)p->bytes;
    info->n_images = p->n_images;
    return TCA_OK;
}

int tca_plan_export(tca_plan_t p, int which, void *h_dst, size_t capacity, size_t *out_bytes)
{
    clear_error();
    if (!p) return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    const void *src = nullptr;
    size_t n = 0;
    switch (which) {
    case TCA_ARR_ROW_PERM: src = p->perm; n = sizeof(int) * p->M; break;
    case TCA_ARR_P_ROW_PTR: src = p->p_row_ptr; n = p->M > 0 ? sizeof(int) * (p->M + 1) : 0; break;
    case TCA_ARR_P_COL: src = p->p_col; n = sizeof(int) * p->nnz; break;
    case TCA_ARR_P_VAL: src = p->p_val; n = 2 * (size_t)p->nnz; break;
    case TCA_ARR_SRC: src = p->src; n = sizeof(int) * p->nnz; break;
    case TCA_ARR_TC_WINDOWS: src = p->tc_windows; n = sizeof(int) * p->n_tc; break;
    case TCA_ARR_CC_WINDOWS: src = p->cc_windows; n = sizeof(int) * p->n_cc; break;
    case TCA_ARR_TILE_FIRST: src = p->tile_first; n = p->M > 0 ? sizeof(int) * (p->n_tc + 1) : 0; break;
    case TCA_ARR_WIN_COLS: src = p->win_cols; n = sizeof(int) * (size_t)p->n_tc_chunks * kChunkCols; break;
    case TCA_ARR_TILE_PTR: src = p->tile_ptr; n = p->M > 0 ? sizeof(int) * ((size_t)p->n_tc_chunks + 1) : 0; break;
    case TCA_ARR_TILE_ENTRIES: src = p->tile_entries; n = sizeof(uint32_t) * (size_t)p->tc_nnz; break;
    case TCA_ARR_TILE_SRC: src = p->tile_src; n = sizeof(int) * (size_t)p->tc_nnz; break;
    case TCA_ARR_TILE_IMAGE_IDX: src = p->img_idx; n = sizeof(int) * (size_t)p->n_tc_chunks; break;
    case TCA_ARR_TILE_IMAGES: src = p->images; n = sizeof(uint16_t) * (size_t)p->n_images * kWindowRows * kChunkCols; break;
    case TCA_ARR_CC_ITEMS: src = p->cc_items; n = sizeof(int2) * (size_t)p->n_cc_items; break;
    case TCA_ARR_ALL_ITEMS: src = p->all_items; n = sizeof(int2) * (size_t)p->n_all_items; break;
    case TCA_ARR_TC_PAIRS: src = p->tc_pairs; n = sizeof(int2) * (size_t)p->n_pairs; break;
    case TCA_ARR_ROW_SCALE: src = p->row_scale; n = p->has_fp8 ? sizeof(float) * (size_t)p->M : 0; break;
    case TCA_ARR_P_VAL_F8: src = p->p_val_f8; n = p->has_fp8 ? (size_t)p->nnz : 0; break;
    case TCA_ARR_TILE_ENTRIES_F8: src = p->tile_entries_f8; n = p->has_fp8 ? sizeof(uint32_t) * (size_t)p->tc_nnz : 0; break;
    case TCA_ARR_TILE_IMAGES_F8:
        src = p->images_f8;
        n = p->has_fp8 ? (size_t)p->n_images * kWindowRows * kChunkCols : 0;
        break;
    default: return set_error(TCA_ERR_INVALID_ARG, "unknown plan array %d", which);
    }
    if (out_bytes) *out_bytes = n;
    if (!h_dst || n == 0) return TCA_OK;
    if (capacity < n) return set_error(TCA_ERR_INVALID_ARG, "destination holds %zu bytes, %zu needed", capacity, n);
    TCA_CUDA_TRY(cudaMemcpy(h_dst, src, n, cudaMemcpyDeviceToHost));
    return TCA_OK;
}

int tca_plan_status(tca_plan_t p)
{
    clear_error();
    if (!p) return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    if (!p->d_status) return TCA_OK;
    int h = 0;
    TCA_CUDA_TRY(cudaMemcpy(&h, p->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (h != 0)
        TCA_CUDA_TRY(cudaMemset(p->d_status, 0, sizeof(int))); // read and clear
    if (h & kStatusTimeout)
        return set_error(TCA_ERR_TIMEOUT, "a bounded device-side wait gave up (status word 0x%x)", h);
    if (h & kStatusLayout)
        return set_error(TCA_ERR_UNSUPPORTED, "tensor-core kernel skipped: shared memory base not 1024-byte aligned");
    return TCA_OK;
}

int tca_plan_destroy(tca_plan_t p)
{
    clear_error();
    free_plan(p);
    return TCA_OK;
}

static int make_job(tca_plan_t p, const void *d_B_f16, int ldb, int N, void *d_C, int ldc, int c_dtype,
                    bool batched, SpmmJob *job)
{
    if (!p) return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    TCA_TRY(check_dense_args(d_B_f16, ldb, N, d_C, ldc, c_dtype, p->M, p->K));
    job->p = p;
    job->B = (const __half *)d_B_f16;
    job->C = d_C;
    job->ldb = ldb;
    job->N = N;
    job->ldc = ldc;
    job->tc = p->n_tc > 0 && dense_operands_vec_ok(d_B_f16, ldb, N, d_C, ldc, c_dtype);
    job->n_tile = pick_tc_tile(p, N, batched);
    return TCA_OK;
}

static int spmm_impl(tca_plan_t p, const void *d_B_f16, int ldb, int N, void *d_C, int ldc, int c_dtype,
                     float alpha, float beta, unsigned flags, cudaStream_t s, void *const *ev)
{
    clear_error();
    SpmmJob job;
    TCA_TRY(make_job(p, d_B_f16, ldb, N, d_C, ldc, c_dtype, false, &job));
    if (p->M == 0 || N == 0) return TCA_OK;
    return run_jobs_with_events(&job, 1, c_dtype, alpha, beta, flags, s, ev);
}

int tca_spmm(tca_plan_t p, const void *d_B_f16, int ldb, int N, void *d_C, int ldc, int c_dtype, float alpha,
             float beta, unsigned flags, tca_stream_t stream)
{
    return spmm_impl(p, d_B_f16, ldb, N, d_C, ldc, c_dtype, alpha, beta, flags, (cudaStream_t)stream, nullptr);
}

int tca_spmm_events(tca_plan_t p, const void *d_B_f16, int ldb, int N, void *d_C, int ldc, int c_dtype,
                    float alpha, float beta, unsigned flags, tca_stream_t stream, void *const *events)
{
    return spmm_impl(p, d_B_f16, ldb, N, d_C, ldc, c_dtype, alpha, beta, flags, (cudaStream_t)stream, events);
}

int tca_spmm_batched(const tca_batch_item_t *items, int n_items, int c_dtype, float alpha, float beta,
                     unsigned flags, tca_stream_t stream, void *const *events)
{
    clear_error();
    if (n_items < 0 || (n_items > 0 && !items))
        return set_error(TCA_ERR_INVALID_ARG, "invalid batch");
    std::vector<SpmmJob> jobs;
    jobs.reserve((size_t)n_items);
    for (int i = 0; i < n_items; i++) {
        SpmmJob j;
        const tca_batch_item_t &it = items[i];
        TCA_TRY(make_job(it.plan, it.d_B_f16, it.ldb, it.N, it.d_C, it.ldc, c_dtype, true, &j));
        if (it.n_tile == 64 || it.n_tile == 128 || it.n_tile == 256)
            j.n_tile = it.n_tile;
        j.cc_w = it.cc_cols;
        if (it.plan->M > 0 && it.N > 0)
            jobs.push_back(j);
    }
    return run_jobs_with_events(jobs.data(), (int)jobs.size(), c_dtype, alpha, beta, flags, (cudaStream_t)stream,
                                events);
}



int tca_plan_launch_counts(tca_plan_t p, int N, int *n_tc_launches, int *n_cc_launches)
{
    clear_error();
    if (!p) return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    const bool empty = p->M == 0 || N == 0;
    if (n_tc_launches) *n_tc_launches = (!empty && p->n_tc > 0) ? 1 : 0;
    if (n_cc_launches) *n_cc_launches = (!empty && (p->n_tc == 0 ? p->n_windows : p->n_cc) > 0) ? 1 : 0;
    return TCA_OK;
}

} // extern "C"
