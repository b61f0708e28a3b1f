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
#include <cstring>
#include <vector>
#include <algorithm>
#include "tca_internal.cuh"
#include "plan.cuh"

namespace tca {
namespace {

constexpr int kErrRowPtr = 1, kErrColRange = 2;

// 1. Row checks: one warp per row.
// Also fills all_windows (window w at index w) and clears the plan's status
// word.
__global__ void k_row_check(const int *__restrict__ row_ptr, const int *__restrict__ col, int M, int K, int nnz,
                            int *__restrict__ row_nnz, int *__restrict__ row_sorted, int *__restrict__ err,
                            int *__restrict__ all_windows, int W, int *__restrict__ status)
{
    const int lane = threadIdx.x & 31;
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g < W)
        all_windows[g] = (int)g;
    if (g == 0)
        *status = 0;
    const long long r = g >> 5;
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

// 2. Row order of a matrix with at most kOrderRows rows, in one block: a
// stable descending radix sort of the row lengths (ties keep row order; only
// the bits up to the longest row take part) carrying (row << 1 | sorted
// flag), the exclusive prefix sum of the sorted lengths (the sorted row
// offsets), and copies of the offsets and of the check verdict into the
// array the host reads after step 3. Global loads and stores are striped
// (coalesced), exchanged through shared memory with the sort's blocked order.
constexpr int kOrderThreads = 1024, kOrderItems = 8, kOrderRows = kOrderThreads * kOrderItems;

__global__ void __launch_bounds__(kOrderThreads)
k_order_small(const int *__restrict__ row_nnz, const int *__restrict__ row_sorted, int M, int sort,
              const int *__restrict__ err, int *__restrict__ perm, int *__restrict__ p_row_ptr,
              int *__restrict__ p_sorted, int *__restrict__ stage_err, int *__restrict__ stage_rp)
{
    using Sort = cub::BlockRadixSort<unsigned, kOrderThreads, kOrderItems, unsigned>;
    using Scan = cub::BlockScan<int, kOrderThreads>;
    using Xchg = cub::BlockExchange<unsigned, kOrderThreads, kOrderItems>;
    __shared__ union {
        typename Sort::TempStorage sort;
        typename Scan::TempStorage scan;
        typename Xchg::TempStorage xchg;
    } tmp;
    __shared__ unsigned longest;
    const int t = threadIdx.x;
    if (t == 0)
        longest = 0;
    unsigned key[kOrderItems], val[kOrderItems], mx = 0;
#pragma unroll
    for (int u = 0; u < kOrderItems; u++) { // striped: item u of thread t is row u * 1024 + t
        const int i = u * kOrderThreads + t;
        key[u] = i < M ? (unsigned)row_nnz[i] : 0u; // lengths are >= 0; padding sorts after the rows
        val[u] = i < M ? (unsigned)row_sorted[i] : 0u;
        mx = max(mx, key[u]);
    }
    __syncthreads(); // longest
    Xchg(tmp.xchg).StripedToBlocked(key, key);
    __syncthreads();
    Xchg(tmp.xchg).StripedToBlocked(val, val);
#pragma unroll
    for (int u = 0; u < kOrderItems; u++) // blocked: item u of thread t is row t * 8 + u
        val[u] = ((unsigned)(t * kOrderItems + u) << 1) | (val[u] & 1u);
    if (sort) {
        mx = __reduce_max_sync(0xffffffffu, mx);
        if ((t & 31) == 0)
            atomicMax(&longest, mx);
        __syncthreads();
        const int end_bit = longest ? 32 - __clz((int)longest) : 1;
        Sort(tmp.sort).SortDescending(key, val, 0, end_bit);
    }
    __syncthreads();
    int len[kOrderItems], off[kOrderItems], total;
#pragma unroll
    for (int u = 0; u < kOrderItems; u++)
        len[u] = (int)key[u];
    Scan(tmp.scan).ExclusiveSum(len, off, total);
    unsigned offs[kOrderItems];
#pragma unroll
    for (int u = 0; u < kOrderItems; u++)
        offs[u] = (unsigned)off[u];
    __syncthreads();
    Xchg(tmp.xchg).BlockedToStriped(offs, offs);
    __syncthreads();
    Xchg(tmp.xchg).BlockedToStriped(val, val);
#pragma unroll
    for (int u = 0; u < kOrderItems; u++) {
        const int i = u * kOrderThreads + t;
        if (i < M) {
            perm[i] = (int)(val[u] >> 1);
            p_sorted[i] = (int)(val[u] & 1u);
            p_row_ptr[i] = (int)offs[u];
            stage_rp[i] = (int)offs[u];
        }
    }
    if (t == 0) {
        p_row_ptr[M] = total;
        stage_rp[M] = total;
        *stage_err = *err;
    }
}

// Exclusive prefix sum of n values into out[0, n] (out[n] = the total), in
// one block: the tile offsets of up to kScanSmallMax chunks.
constexpr int kScanThreads = 1024, kScanItems = 8, kScanSmallMax = 8 * kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) k_scan_small(const int *__restrict__ in, int n, int *__restrict__ out)
{
    using Scan = cub::BlockScan<int, kScanThreads>;
    __shared__ typename Scan::TempStorage tmp;
    int carry = 0;
    for (int base = 0; base < n; base += kScanThreads * kScanItems) {
        int v[kScanItems], o[kScanItems], agg;
#pragma unroll
        for (int u = 0; u < kScanItems; u++) {
            const int i = base + (int)threadIdx.x * kScanItems + u;
            v[u] = i < n ? in[i] : 0;
        }
        Scan(tmp).ExclusiveSum(v, o, agg);
#pragma unroll
        for (int u = 0; u < kScanItems; u++) {
            const int i = base + (int)threadIdx.x * kScanItems + u;
            if (i < n)
                out[i] = carry + o[u];
        }
        carry += agg;
        __syncthreads(); // tmp is reused by the next tile
    }
    if (threadIdx.x == 0)
        out[n] = carry;
}

__global__ void k_iota(int *a, int n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        a[i] = (int)i;
}

// Clears and copies of the build's own arrays are kernels: a memset or a
// device-to-device copy may run on a copy engine, queued behind the
// host-to-device copies of the values and B on the host-buffer path's second
// stream, which steps 1-5 do not wait for.
__global__ void k_zero_words(uint32_t *__restrict__ p, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = 0u;
}

__global__ void k_copy_words(const int *__restrict__ src, int *__restrict__ dst, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

__global__ void k_gather_int(const int *__restrict__ src, const int *__restrict__ idx, int *__restrict__ dst, int n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = src[idx[i]];
}

// 2b. Re-order the CSR: one warp per sorted row. Does nothing when the row
// checks found an error (the host reports it after its next wait). With val
// NULL the values are left for k_update_p_val (gathered through src).
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
        if (val)
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

// 3. Window statistics with each window's nonzeros split over `split`
// blocks, so that a few windows still spread over the GPU: a block marks its
// share of the columns in a shared-memory bitmap and ORs the set words into
// the window's global bitmap (zeroed beforehand, kept for k_tile_cols); the
// window's last block to finish (a per-window counter, zeroed beforehand)
// counts the distinct columns and touched 64-column blocks from it and
// checks the rows' flags. Does nothing when the row checks found an error.
__global__ void __launch_bounds__(512)
k_window_stats_split(const int *__restrict__ p_row_ptr, const int *__restrict__ p_col,
                     const int *__restrict__ p_sorted, int M, int K, const int *__restrict__ err, int split,
                     int *__restrict__ win_nu, int *__restrict__ win_nnz, int *__restrict__ win_elig,
                     int *__restrict__ win_nblk, uint32_t *__restrict__ bitmaps, int *__restrict__ done)
{
    extern __shared__ uint32_t bm[];
    __shared__ int s_cnt, s_elig, s_nblk, s_last;
    const int w = blockIdx.x / split, part = blockIdx.x % split;
    if (*err)
        return; // uniform across the grid
    const int nwords = (K + 31) >> 5;
    for (int i = threadIdx.x; i < nwords; i += blockDim.x) bm[i] = 0u;
    if (threadIdx.x == 0) { s_cnt = 0; s_elig = 1; s_nblk = 0; }
    __syncthreads();
    const int r0 = w * kWindowRows, r1 = min(M, r0 + kWindowRows);
    const int lo = p_row_ptr[r0], hi = p_row_ptr[r1];
    const int a = lo + (int)((long long)(hi - lo) * part / split);
    const int b = lo + (int)((long long)(hi - lo) * (part + 1) / split);
    mark_columns(p_col, a, b, bm);
    __syncthreads();
    uint32_t *gbm = bitmaps + (size_t)w * nwords;
    for (int i = threadIdx.x; i < nwords; i += blockDim.x)
        if (bm[i]) atomicOr(&gbm[i], bm[i]);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        s_last = atomicAdd(&done[w], 1) == split - 1;
    __syncthreads();
    if (!s_last)
        return;
    __threadfence(); // the other blocks' words are visible to the last one
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x)
        if (!p_sorted[i]) atomicAnd(&s_elig, 0);
    int cnt = 0, nb = 0;
    for (int i = threadIdx.x; i < nwords; i += blockDim.x) cnt += __popc(__ldcg(gbm + i));
    for (int q = threadIdx.x; 2 * q < nwords; q += blockDim.x)
        nb += ((__ldcg(gbm + 2 * q) | (2 * q + 1 < nwords ? __ldcg(gbm + 2 * q + 1) : 0u)) != 0u);
    atomicAdd(&s_cnt, cnt); // integer sums: order-independent
    atomicAdd(&s_nblk, nb);
    __syncthreads();
    if (threadIdx.x == 0) {
        win_nu[w] = s_cnt;
        win_nnz[w] = hi - lo;
        win_elig[w] = s_elig;
        win_nblk[w] = s_nblk;
    }
}

// 3 (bitmaps too large to keep). One block per window, K-bit bitmap in
// shared memory. Does nothing when the row checks found an error.
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

// The nonzeros of local row lr of chunk c of a window are the row's columns
// from the chunk's first column up to the next chunk's first (a chunk holds
// at most 64 columns of a row). First index j in [rs, re) with p_col[j] >= x,
// for a row whose columns increase strictly, by a warp: rounds of 32 samples (the last column of each
// of 32 equal segments) narrow the range to one segment, whose at most 32
// columns one warp-wide load then counts. A row of up to 1024 columns takes
// two dependent loads per lane instead of ~10.
__device__ __forceinline__ int warp_lower_bound(const int *__restrict__ p_col, int rs, int re, int x, int lane)
{
    int a = rs, n = re - rs;
    while (n > 32) {
        const int seg = (n + 31) >> 5;
        const int j = a + min(n, (lane + 1) * seg) - 1; // last column of segment `lane` (or of the row)
        const int k = __popc(__ballot_sync(0xffffffffu, p_col[j] < x)); // segments wholly below x
        if (k * seg >= n)
            return re;
        a += k * seg;
        n = min(seg, n - k * seg);
    }
    return a + __popc(__ballot_sync(0xffffffffu, lane < n && p_col[a + lane] < x));
}

// Tile count and tile write: 4 blocks of 32 warps per chunk, a warp per row.
constexpr int kTileBlocksPerChunk = kWindowRows / 32;

// 5b. Nonzeros per chunk. A row's range in the chunk: its first column at or
// after the chunk's first (warp_lower_bound), its end among the next 64
// entries (64 columns, strictly increasing) by one warp-wide count. The range
// goes to row_range for 5c, its length (summed per block) to chunk_nnz,
// which is zeroed beforehand.
__global__ void __launch_bounds__(1024)
k_tile_count(const int2 *__restrict__ chunk_win, const int4 *__restrict__ win_info,
             const int *__restrict__ p_row_ptr, const int *__restrict__ p_col, const int *__restrict__ win_cols,
             int M, int *__restrict__ chunk_nnz, int2 *__restrict__ row_range)
{
    __shared__ int s_sum;
    const int chunk = blockIdx.x / kTileBlocksPerChunk;
    const int lane = threadIdx.x & 31, lr = (blockIdx.x % kTileBlocksPerChunk) * 32 + (threadIdx.x >> 5);
    if (threadIdx.x == 0)
        s_sum = 0;
    __syncthreads();
    const int2 cw = chunk_win[chunk];
    const int4 wi = win_info[cw.x];
    const int *wc = win_cols + (size_t)wi.y * kChunkCols;
    const int i = wi.x * kWindowRows + lr;
    int lo = 0, hi = 0;
    if (i < M) { // uniform across the warp
        const int rs = p_row_ptr[i], re = p_row_ptr[i + 1];
        const int first = wc[cw.y * kChunkCols];
        const int next = cw.y + 1 < wi.z ? wc[(cw.y + 1) * kChunkCols] : 0x7fffffff;
        lo = warp_lower_bound(p_col, rs, re, first, lane);
        const int e = min(re, lo + kChunkCols);
        const int j0 = lo + lane, j1 = lo + 32 + lane;
        const bool in0 = j0 < e && p_col[j0] < next, in1 = j1 < e && p_col[j1] < next;
        hi = lo + __popc(__ballot_sync(0xffffffffu, in0)) + __popc(__ballot_sync(0xffffffffu, in1));
    }
    if (lane == 0) {
        row_range[(size_t)chunk * kWindowRows + lr] = make_int2(lo, hi);
        if (hi > lo)
            atomicAdd(&s_sum, hi - lo);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_sum > 0)
        atomicAdd(&chunk_nnz[chunk], s_sum); // integer sums: order-independent
}

// 5c. Entries of each chunk, ordered by (row, column): a warp per row writes
// the row's (at most 64) entries with coalesced loads and stores. Each block
// scans the chunk's 128 row lengths for the rows' first entries; tile_ptr
// (the exclusive sum of chunk_nnz) gives the chunk's.
__global__ void __launch_bounds__(1024)
k_tile_write(const int2 *__restrict__ chunk_win, const int4 *__restrict__ win_info,
             const int *__restrict__ p_col, const __half *__restrict__ p_val, const int *__restrict__ win_cols,
             const int *__restrict__ tile_ptr, const int2 *__restrict__ row_range, uint32_t *__restrict__ entries,
             int *__restrict__ tile_src)
{
    __shared__ int scratch[33];
    __shared__ int s_off[kWindowRows];
    __shared__ int s_cols[kChunkCols];
    const int chunk = blockIdx.x / kTileBlocksPerChunk;
    const int lane = threadIdx.x & 31, lr = (blockIdx.x % kTileBlocksPerChunk) * 32 + (threadIdx.x >> 5);
    const int2 cw = chunk_win[chunk];
    const int4 wi = win_info[cw.x];
    if (threadIdx.x < kChunkCols)
        s_cols[threadIdx.x] = win_cols[((size_t)wi.y + cw.y) * kChunkCols + threadIdx.x];
    const int len = threadIdx.x < kWindowRows ? row_range[(size_t)chunk * kWindowRows + threadIdx.x].y -
                                                    row_range[(size_t)chunk * kWindowRows + threadIdx.x].x
                                              : 0;
    int total;
    const int off = block_exclusive_scan(len, &total, scratch); // its barriers also publish s_cols
    if (threadIdx.x < kWindowRows)
        s_off[threadIdx.x] = off;
    __syncthreads();
    const int2 r = row_range[(size_t)chunk * kWindowRows + lr];
    const long long base = (long long)tile_ptr[chunk] + s_off[lr];
    const int n = r.y - r.x, first = s_cols[0];
    int col[2];
    unsigned short val[2];
#pragma unroll
    for (int u = 0; u < 2; u++) { // both loads before any use
        const int k = lane + 32 * u;
        col[u] = k < n ? p_col[r.x + k] : 0;
        val[u] = k < n ? __half_as_ushort(p_val[r.x + k]) : (unsigned short)0;
    }
#pragma unroll
    for (int u = 0; u < 2; u++) {
        const int k = lane + 32 * u;
        if (k >= n)
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
        entries[base + k] = ((uint32_t)lr << 22) | ((uint32_t)rk << 16) | (uint32_t)val[u];
        tile_src[base + k] = r.x + k;
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

int zero_async(void *p, size_t bytes, cudaStream_t s) // bytes: a multiple of 4
{
    const size_t n = bytes / 4;
    if (n == 0)
        return TCA_OK;
    k_zero_words<<<std::min<unsigned>(blocks_for((long long)n, 256), 4 * kSMs), 256, 0, s>>>(
        static_cast<uint32_t *>(p), n);
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

int copy_async(const int *src, int *dst, size_t n, cudaStream_t s)
{
    if (n == 0)
        return TCA_OK;
    k_copy_words<<<std::min<unsigned>(blocks_for((long long)n, 256), 4 * kSMs), 256, 0, s>>>(src, dst, n);
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

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

// Offsets of arrays sharing one allocation, each at a 256-byte boundary (a
// pool allocation and its release cost ~2 us of host time each; a build
// makes a handful instead of dozens).
struct Carve {
    size_t size = 0;
    template <typename T>
    size_t take(size_t count)
    {
        const size_t off = size;
        size += (sizeof(T) * (count > 0 ? count : 1) + 255) & ~(size_t)255;
        return off;
    }
};

template <typename T>
T *at(void *base, size_t off)
{
    return reinterpret_cast<T *>(static_cast<char *>(base) + off);
}

void free_plan(tca_plan *p)
{
    if (!p) return;
    cudaDeviceSynchronize(); // the plan's arrays may still be read by queued work on any stream
    transpose_free(p);
    plan_free_fp8(p);
    for (void *a : p->arena)
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
//
// The plan's arrays come in three allocations (tca_plan::arena) and the
// temporaries of each step in one; host-made arrays go to the device in one
// copy per allocation. The host builds the CUDA-core work items while the
// device writes the tiles (step 5). With vals_ready the values are gathered
// only where they are first read (the tile entries), so that steps 1-5 run
// while they are still on their way.
int build_plan(tca_plan *p, const int *row_ptr, const int *col, const __half *val, cudaStream_t s,
               cudaEvent_t vals_ready = nullptr, bool sync_end = true)
{
    BuildStream build_stream(s);
    const int M = p->M, K = p->K, nnz = p->nnz;
    size_t *bytes = &p->bytes;
    const int W = (M + kWindowRows - 1) / kWindowRows;
    p->n_windows = W;
    const bool small = M <= kOrderRows;
    const bool tc_possible = (p->opts.path != 1) && K <= kMaxTcK && K > 0 && W > 0;
    // the windows' column bitmaps, kept from the statistics for the tile
    // columns when they take at most 64 MB (else k_tile_cols rebuilds them)
    const size_t bm_words = (size_t)W * ((K + 31) / 32);
    const bool keep_bm = tc_possible && bm_words <= (size_t)(16u << 20);

    {
        Carve c;
        const size_t o_perm = c.take<int>(M), o_rp = c.take<int>((size_t)M + 1), o_col = c.take<int>(nnz),
                     o_val = c.take<__half>(nnz), o_src = c.take<int>(nnz), o_status = c.take<int>(1),
                     o_all = c.take<int>(W);
        char *a;
        TCA_TRY(dev_alloc(&a, c.size, bytes));
        p->arena[0] = a;
        p->perm = at<int>(a, o_perm);
        p->p_row_ptr = at<int>(a, o_rp);
        p->p_col = at<int>(a, o_col);
        p->p_val = at<__half>(a, o_val);
        p->src = at<int>(a, o_src);
        p->d_status = at<int>(a, o_status);
        p->all_windows = at<int>(a, o_all);
    }

    // temporaries of steps 1-3; the stage array gathers what the host reads
    // after step 3: per window its distinct columns, nonzeros, sortedness and
    // touched 64-column blocks, then the check verdict and the sorted row
    // offsets (for the work items)
    const size_t n_stage = 4 * (size_t)W + 1 + (size_t)M + 1;
    int end_bit = 1; // row lengths are at most nnz: only their low bits take part
    while (end_bit < 32 && ((long long)1 << end_bit) <= (long long)nnz) end_bit++;
    size_t sort_tmp = 0, scan_tmp = 0;
    if (!small) {
        if (p->opts.sort_rows)
            TCA_CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(nullptr, sort_tmp, (const int *)nullptr,
                                                                   (int *)nullptr, (const int *)nullptr,
                                                                   (int *)nullptr, M, 0, end_bit, s));
        TCA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, (const int *)nullptr, (int *)nullptr, M + 1, s));
    }
    // err, the per-window block counters of step 3 and the kept bitmaps are
    // adjacent: one memset clears them
    Carve ct;
    const size_t o_nnz = ct.take<int>(M), o_sorted = ct.take<int>(M), o_psorted = ct.take<int>(M),
                 o_stage = ct.take<int>(n_stage), o_err = ct.take<int>(1 + (size_t)W),
                 o_bm = ct.take<uint32_t>(keep_bm ? bm_words : 0);
    const size_t zero_bytes = keep_bm ? o_bm - o_err + sizeof(uint32_t) * bm_words : sizeof(int) * (1 + (size_t)W);
    size_t o_iota = 0, o_keys = 0, o_scan_in = 0, o_sort_tmp = 0, o_scan_tmp = 0;
    if (!small) {
        o_iota = ct.take<int>(M);
        o_keys = ct.take<int>(M);
        o_scan_in = ct.take<int>((size_t)M + 1);
        o_sort_tmp = ct.take<char>(sort_tmp);
        o_scan_tmp = ct.take<char>(scan_tmp);
    }
    DevBuf t_steps13;
    char *tb;
    TCA_TRY(dev_alloc(&tb, ct.size, nullptr));
    t_steps13.p = tb;
    int *row_nnz = at<int>(tb, o_nnz), *row_sorted = at<int>(tb, o_sorted), *err = at<int>(tb, o_err);
    int *p_sorted = at<int>(tb, o_psorted), *d_stage = at<int>(tb, o_stage);
    uint32_t *d_bm = keep_bm ? at<uint32_t>(tb, o_bm) : nullptr;
    int *d_done = err + 1;
    TCA_TRY(zero_async(err, zero_bytes, s));

    // 1. checks; the host reads their verdict with the window statistics
    // (step 3), the kernels that follow stand down on an error
    k_row_check<<<blocks_for(std::max((long long)M * 32, (long long)W), 256), 256, 0, s>>>(
        row_ptr, col, M, K, nnz, row_nnz, row_sorted, err, p->all_windows, W, p->d_status);
    TCA_CUDA_TRY(cudaGetLastError());

    // 2. row order
    if (small) {
        k_order_small<<<1, kOrderThreads, 0, s>>>(row_nnz, row_sorted, M, p->opts.sort_rows ? 1 : 0, err, p->perm,
                                                  p->p_row_ptr, p_sorted, d_stage + 4 * W, d_stage + 4 * W + 1);
    } else {
        int *iota = at<int>(tb, o_iota), *keys_out = at<int>(tb, o_keys), *scan_in = at<int>(tb, o_scan_in);
        k_iota<<<blocks_for(M, 256), 256, 0, s>>>(iota, M);
        if (p->opts.sort_rows)
            TCA_CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(at<char>(tb, o_sort_tmp), sort_tmp, row_nnz,
                                                                   keys_out, iota, p->perm, M, 0, end_bit, s));
        else
            TCA_TRY(copy_async(iota, p->perm, M, s));
        TCA_TRY(zero_async(scan_in + M, sizeof(int), s));
        k_gather_int<<<blocks_for(M, 256), 256, 0, s>>>(row_nnz, p->perm, scan_in, M);
        k_gather_int<<<blocks_for(M, 256), 256, 0, s>>>(row_sorted, p->perm, p_sorted, M);
        TCA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(at<char>(tb, o_scan_tmp), scan_tmp, scan_in, p->p_row_ptr, M + 1, s));
        TCA_TRY(copy_async(err, d_stage + 4 * W, 1, s));
        TCA_TRY(copy_async(p->p_row_ptr, d_stage + 4 * W + 1, (size_t)M + 1, s));
    }
    TCA_CUDA_TRY(cudaGetLastError());
    bool vals_later = vals_ready != nullptr;
    k_permute<<<blocks_for((long long)M * 32, 256), 256, 0, s>>>(p->perm, row_ptr, col, vals_later ? nullptr : val,
                                                                 p->p_row_ptr, M, err, p->p_col, p->p_val, p->src);
    TCA_CUDA_TRY(cudaGetLastError());
    // after the host has seen a clean check (src is then complete)
    auto gather_vals = [&]() -> int {
        if (!vals_later)
            return TCA_OK;
        vals_later = false;
        TCA_CUDA_TRY(cudaStreamWaitEvent(s, vals_ready, 0));
        if (nnz > 0)
            k_update_p_val<<<blocks_for(nnz, 256), 256, 0, s>>>(p->src, val, p->p_val, nnz);
        TCA_CUDA_TRY(cudaGetLastError());
        return TCA_OK;
    };

    // 3. windows
    int *d_nu = d_stage, *d_wn = d_stage + W, *d_el = d_stage + 2 * W, *d_nb = d_stage + 3 * W;
    if (tc_possible && keep_bm) {
        // about two blocks per SM, each with at least ~4K nonzeros
        const long long per_window = (long long)nnz / W;
        const int split = std::max(1, std::min((2 * kSMs + W - 1) / W, (int)std::min(64LL, per_window / 4096)));
        const size_t smem = sizeof(uint32_t) * ((K + 31) / 32); // at most 16 KB (K <= kMaxTcK)
        k_window_stats_split<<<W * split, 512, smem, s>>>(p->p_row_ptr, p->p_col, p_sorted, M, K, err, split, d_nu,
                                                          d_wn, d_el, d_nb, d_bm, d_done);
        TCA_CUDA_TRY(cudaGetLastError());
    } else if (tc_possible) {
        const size_t smem = sizeof(uint32_t) * ((K + 31) / 32);
        k_window_stats<<<W, 1024, smem, s>>>(p->p_row_ptr, p->p_col, p_sorted, M, K, err, d_nu, d_wn, d_el, d_nb,
                                             nullptr);
        TCA_CUDA_TRY(cudaGetLastError());
    } else if (W > 0) {
        TCA_TRY(zero_async(d_stage, sizeof(int) * 4 * (size_t)W, s));
    }
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
    const int n_tc = p->n_tc, n_ch = p->n_tc_chunks;
    std::vector<int4> h_wi((size_t)n_tc);
    for (int t = 0; t < n_tc; t++)
        h_wi[t] = make_int4(tc_list[t], h_first[t], h_first[t + 1] - h_first[t], h_direct[t]);
    // window pairs for the pair kernel: greedily, consecutive windows whose
    // chunks are all 64-column blocks of K (identical columns)
    std::vector<int2> h_pairs;
    p->n_full_pairs = 0;
    for (int t = 0; t < n_tc;) {
        if (h_full[t] && t + 1 < n_tc && h_full[t + 1]) {
            h_pairs.push_back(make_int2(t, t + 1));
            p->n_full_pairs++;
            t += 2;
        } else {
            h_pairs.push_back(make_int2(t, -1));
            t += 1;
        }
    }
    p->n_pairs = (int)h_pairs.size();
    // chunk -> (tensor-core window, chunk within the window)
    std::vector<int2> h_cw;
    h_cw.reserve((size_t)n_ch);
    for (int t = 0; t < n_tc; t++)
        for (int c = 0; c < h_wi[t].z; c++) h_cw.push_back(make_int2(t, c));

    // the window lists (made here, copied in one piece) and the tiles
    int2 *d_cw;
    {
        Carve c;
        const size_t o_tcw = c.take<int>(n_tc), o_ccw = c.take<int>(p->n_cc), o_first = c.take<int>(n_tc + 1),
                     o_wi = c.take<int4>(n_tc), o_pairs = c.take<int2>(p->n_pairs), o_cw = c.take<int2>(n_ch);
        const size_t host_part = c.size;
        const size_t o_wc = c.take<int>((size_t)n_ch * kChunkCols), o_tp = c.take<int>((size_t)n_ch + 1),
                     o_te = c.take<uint32_t>((size_t)p->tc_nnz + kEntryPad), o_ts = c.take<int>((size_t)p->tc_nnz);
        char *a;
        TCA_TRY(dev_alloc(&a, c.size, bytes));
        p->arena[1] = a;
        p->tc_windows = at<int>(a, o_tcw);
        p->cc_windows = at<int>(a, o_ccw);
        p->tile_first = at<int>(a, o_first);
        p->tc_win_info = at<int4>(a, o_wi);
        p->tc_pairs = at<int2>(a, o_pairs);
        d_cw = at<int2>(a, o_cw);
        p->win_cols = at<int>(a, o_wc);
        p->tile_ptr = at<int>(a, o_tp);
        p->tile_entries = at<uint32_t>(a, o_te);
        p->tile_src = at<int>(a, o_ts);
        std::vector<char> h_part(host_part);
        auto put = [&](size_t off, const void *src, size_t n) { if (n) std::memcpy(h_part.data() + off, src, n); };
        put(o_tcw, tc_list.data(), sizeof(int) * n_tc);
        put(o_ccw, cc_list.data(), sizeof(int) * p->n_cc);
        put(o_first, h_first.data(), sizeof(int) * (n_tc + 1));
        put(o_wi, h_wi.data(), sizeof(int4) * n_tc);
        put(o_pairs, h_pairs.data(), sizeof(int2) * p->n_pairs);
        put(o_cw, h_cw.data(), sizeof(int2) * n_ch);
        // pageable: the copy returns once its source is staged
        TCA_CUDA_TRY(cudaMemcpyAsync(a, h_part.data(), host_part, cudaMemcpyHostToDevice, s));
    }
    TCA_TRY(zero_async(p->tile_entries + p->tc_nnz, sizeof(uint32_t) * kEntryPad, s));

    // 5. tiles
    DevBuf t_step5;
    std::vector<int> h_ptr((size_t)n_ch + 1, 0);
    if (n_tc > 0) {
        const bool small_scan = n_ch <= kScanSmallMax;
        size_t tmp = 0;
        if (!small_scan)
            TCA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp, (const int *)nullptr, (int *)nullptr, n_ch + 1, s));
        Carve c;
        const size_t o_cn = c.take<int>((size_t)n_ch + 1), o_rr = c.take<int2>((size_t)n_ch * kWindowRows),
                     o_tmp = c.take<char>(tmp);
        char *tb5;
        TCA_TRY(dev_alloc(&tb5, c.size, nullptr));
        t_step5.p = tb5;
        int *d_cn = at<int>(tb5, o_cn);
        int2 *d_rr = at<int2>(tb5, o_rr);
        const size_t smem = 2 * sizeof(uint32_t) * ((K + 31) / 32);
        TCA_CUDA_TRY(cudaFuncSetAttribute(k_tile_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_tile_cols<<<n_tc, 1024, smem, s>>>(p->tc_win_info, p->p_row_ptr, p->p_col, M, K, d_bm, p->win_cols);
        TCA_TRY(zero_async(d_cn, sizeof(int) * ((size_t)n_ch + 1), s));
        k_tile_count<<<(unsigned)n_ch * kTileBlocksPerChunk, 1024, 0, s>>>(d_cw, p->tc_win_info, p->p_row_ptr,
                                                                           p->p_col, p->win_cols, M, d_cn, d_rr);
        if (small_scan) {
            k_scan_small<<<1, kScanThreads, 0, s>>>(d_cn, n_ch, p->tile_ptr);
        } else {
            TCA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(at<char>(tb5, o_tmp), tmp, d_cn, p->tile_ptr, n_ch + 1, s));
        }
        TCA_TRY(gather_vals());
        k_tile_write<<<(unsigned)n_ch * kTileBlocksPerChunk, 1024, 0, s>>>(d_cw, p->tc_win_info, p->p_col, p->p_val,
                                                                           p->win_cols, p->tile_ptr, d_rr,
                                                                           p->tile_entries, p->tile_src);
        TCA_CUDA_TRY(cudaGetLastError());
    } else {
        TCA_TRY(zero_async(p->tile_ptr, sizeof(int), s));
    }

    // 7 (while the device writes the tiles). CUDA-core work items.
    std::vector<int> h_all(W);
    for (int w = 0; w < W; w++) h_all[w] = w;
    std::vector<int2> cc_items, all_items;
    build_items(cc_list, h_rp, M, cc_items);
    build_items(h_all, h_rp, M, all_items);
    p->n_cc_items = (int)cc_items.size();
    p->n_all_items = (int)all_items.size();

    // 6. dense tile images for chunks holding at least kImageMinNnz nonzeros
    if (n_ch > 0) {
        TCA_CUDA_TRY(cudaMemcpyAsync(h_ptr.data(), p->tile_ptr, sizeof(int) * h_ptr.size(), cudaMemcpyDeviceToHost, s));
        TCA_CUDA_TRY(cudaStreamSynchronize(s));
    }
    std::vector<int> h_img((size_t)n_ch, -1), h_img_chunk;
    for (int c = 0; c < n_ch; c++)
        if (h_ptr[c + 1] - h_ptr[c] >= kImageMinNnz) {
            h_img[c] = (int)h_img_chunk.size();
            h_img_chunk.push_back(c);
        }
    p->n_images = (int)h_img_chunk.size();
    {
        Carve c;
        const size_t o_idx = c.take<int>(n_ch), o_ich = c.take<int>(p->n_images),
                     o_cci = c.take<int2>(cc_items.size()), o_alli = c.take<int2>(all_items.size());
        const size_t host_part = c.size;
        const size_t o_img = c.take<uint16_t>((size_t)p->n_images * kWindowRows * kChunkCols);
        char *a;
        TCA_TRY(dev_alloc(&a, c.size, bytes));
        p->arena[2] = a;
        p->img_idx = at<int>(a, o_idx);
        p->img_chunk = at<int>(a, o_ich);
        p->cc_items = at<int2>(a, o_cci);
        p->all_items = at<int2>(a, o_alli);
        p->images = at<uint16_t>(a, o_img);
        std::vector<char> h_part(host_part);
        auto put = [&](size_t off, const void *src, size_t n) { if (n) std::memcpy(h_part.data() + off, src, n); };
        put(o_idx, h_img.data(), sizeof(int) * h_img.size());
        put(o_ich, h_img_chunk.data(), sizeof(int) * h_img_chunk.size());
        put(o_cci, cc_items.data(), sizeof(int2) * cc_items.size());
        put(o_alli, all_items.data(), sizeof(int2) * all_items.size());
        // pageable, as above: h_part may go out of scope when the call returns
        TCA_CUDA_TRY(cudaMemcpyAsync(a, h_part.data(), host_part, cudaMemcpyHostToDevice, s));
    }
    if (p->n_images > 0) {
        k_render_images<<<p->n_images, 256, 0, s>>>(p->img_chunk, p->tile_ptr, p->tile_entries, p->images);
        TCA_CUDA_TRY(cudaGetLastError());
    }
    TCA_TRY(gather_vals());
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
    o->tc_min_density = 0.01f;
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
