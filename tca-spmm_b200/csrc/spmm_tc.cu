// spmm_tc.cu -- tensor-core (tcgen05, sm_100a) forward over the dense-enough
// windows of one or many plans.
//
// The reference (src/our_spmm.cu:25-156) uses mma.sync m16n8k8 as a batched
// dot-product engine on one row's nonzeros, of which only the diagonal 8x8
// blocks are useful (:70-72, :123-124), and re-gathers a 64-column slice of B
// per nonzero. Here a 128-row window of sorted rows becomes a sequence of
// dense 128 x 64 A tiles over the window's condensed (distinct) columns; each
// tile multiplies the 64 matching rows of B on the 5th-generation tensor
// cores: D[128 x NT] (FP32, tensor memory) += A[128 x 64] * B[64 x NT].
//
// Work items are (job, window, NT-wide slice of N). The chunks of all items,
// in item order, are cut into one contiguous range per CTA of equal length
// (stream-K): a CTA's range covers the tail of one item, whole items and the
// head of another, so that every SM gets the same number of chunks whatever
// the item sizes. An item cut between CTAs is finished by the CTA that
// completes its part last: the other parts leave FP32 partial tiles in a
// workspace, the last one adds them in part order (a fixed order, so the
// result does not depend on which CTA finishes last) and stores C; no CTA
// waits for another. When the ranges would hold more items than a CTA's
// table, items go to CTAs in turn instead (item i to CTA i mod grid).
// Persistent CTAs (one per SM) stream the chunks of their segments through a
// ring of kStages (A tile, B tile, entry staging) stages, with decoupled
// roles:
//   * four loader warps, taking chunks in turn, move every byte through the
//     TMA engine: the 64 B rows of the chunk -- one tiled box per 64 columns
//     of N when its columns are 64 consecutive rows of B, else tile::gather4
//     of the condensed columns (4 rows x 128 bytes per instruction into a
//     128-byte swizzled N-major tile; padding columns and n >= N are out of
//     the tensor and arrive as zeros) -- and either the chunk's pre-rendered,
//     pre-swizzled dense A tile (chunks with >= 2048 nonzeros: one 16 KB
//     cp.async.bulk) or its packed entries (cp.async.bulk into the stage's
//     staging buffer);
//   * scatter warps (two groups taking chunks in turn), once a stage's
//     entries landed, zero its A tile and scatter them into the swizzled
//     K-major layout;
//   * one MMA lane issues 4 tcgen05.mma (K = 16 each) per chunk into the FP32
//     accumulator in tensor memory and releases the stage with tcgen05.commit;
//   * finally 4 warps read the accumulator (TMEM lane = row) and store
//     alpha * D + beta * C to C[perm[row]] (FP16 or FP32).
// Per-thread 16-byte cp.async was measured to issue only ~13 B/clock/SM for
// the B gather, which left the tensor cores idle; the TMA engine does not
// occupy the issuing threads.
// Every mbarrier wait is bounded (about one second of %globaltimer); on
// expiry the CTA records kStatusTimeout in the job's status word and runs to
// completion without hanging. No load uses cluster multicast.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <memory>
#include <mutex>
#include "tca_internal.cuh"
#include "plan.cuh"
#include "ptx.cuh"

namespace tca {
namespace {

constexpr int kScatterThreads = 128; // warps 0-3: sparse-entry scatter
constexpr int kLoaderWarp = 4;       // TMA issue, chunks g = 0 (mod kLoaders)
constexpr int kMmaWarp = 5;          // TMEM allocation, tcgen05.mma issue
constexpr int kEpiThreads = 128;     // warps 6-9: epilogue
constexpr int kLoaderWarp1 = 10;     // warps 10..: TMA issue, chunks g = 1, 2, .. (mod kLoaders)
constexpr int kLoaders = 4;          // loader warps, each issuing every kLoaders-th chunk
constexpr int kThreads = 320 + (kLoaders - 1) * 32;
constexpr int kMaxCtaItems = 32;      // work items (segments) per persistent CTA
constexpr int kEpiBar = 3;           // named barrier of the epilogue warps (1, 2: scatter groups)
constexpr int kStagingBytes = ((kImageMinNnz + 3) * 4 + 15) & ~15; // entries of a sparse chunk, 16-byte rounded
constexpr int kMaxJobs = 32;                                  // jobs per launch (kernel parameter space)

struct TcJob {
    CUtensorMap tmap_b;    // B as a 2-D tensor {N, K}, box {64, 1}, 128-byte swizzle (gather4 source)
    CUtensorMap tmap_tile; // the same tensor, box {64, 64}: 64 contiguous rows of B per instruction
    const int4 *win_info; // per tensor-core window: window, first chunk, chunk count
    const int *tile_ptr, *win_cols, *img_idx, *perm, *p_row_ptr;
    const uint32_t *entries;
    const uint8_t *images;   // dense tile images (16 KB FP16 or 8 KB E4M3 each)
    const float *row_scale;  // E4M3: per sorted row
    const float *col_scale;  // E4M3: per column of N
    const __half *B;
    void *C;
    int *status;
    int M, N, ldb, ldc, ntiles;
    int n_win; // tensor-core windows of the plan
    float alpha, beta;
    unsigned flags;
};

// Chunk ranges (stream-K): the items' chunks, job by job, window by window,
// N slice by N slice, are `units` chunk-units; CTA b covers units
// [b * units / grid, (b + 1) * units / grid), starting in item
// cta_start[b] = {job, window, N slice, chunk within the item}. A cut item's
// parts leave partial tiles in `partials` (two slots of 128 x NT floats per
// CTA: slot 2b for the CTA's first segment when that is cut, 2b + 1 for its
// last; tc_slot), which spmm_tc_fixup adds up after the launch.
struct TcBatch {
    int n_jobs;
    int item_start[kMaxJobs + 1];
    int split;        // 1: chunk ranges (above); 0: item i to CTA i mod grid
    long long units;
    float *partials;
    int *failed;      // split launches: set when a CTA gave up (zero before the launch); the sums are then skipped
    int4 cta_start[kSMs];
    TcJob job[kMaxJobs];
};

// The cut items of a split launch: {job << 16 | N slice, tensor-core window,
// first CTA, parts << 1 | head}, head: part 0 is its CTA's first segment.
struct TcCuts {
    int n;
    int4 cut[kSMs];
};

// The CTA whose range holds chunk-unit u (ranges of units / grid, floored).
__host__ __device__ inline int range_owner(long long u, long long units, int grid)
{
    return (int)(((u + 1) * grid - 1) / units);
}
__host__ __device__ inline long long range_lo(int b, long long units, int grid) { return (long long)b * units / grid; }

using namespace ptx;

// kind::f16 instruction descriptor: D FP32, A/B FP16, A K-major, B N-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_f16(int n)
{
    return (1u << 4) | (0u << 7) | (0u << 10) | (0u << 15) | (1u << 16) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
                 "l"(a), "l"(b), "r"(idesc), "r"(accum)
                 : "memory");
}
__device__ __forceinline__ void umma_f8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
                 "l"(a), "l"(b), "r"(idesc), "r"(accum)
                 : "memory");
}
__device__ __forceinline__ void store8_out(__half *p, const float *v, float alpha, float beta)
{
    uint4 u;
    __half2 *h = reinterpret_cast<__half2 *>(&u);
    if (beta != 0.f) {
        uint4 o = *reinterpret_cast<const uint4 *>(p);
        const __half2 *oh = reinterpret_cast<const __half2 *>(&o);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            float2 f = __half22float2(oh[i]);
            h[i] = __floats2half2_rn(fmaf(alpha, v[2 * i], beta * f.x), fmaf(alpha, v[2 * i + 1], beta * f.y));
        }
    } else {
#pragma unroll
        for (int i = 0; i < 4; i++) h[i] = __floats2half2_rn(alpha * v[2 * i], alpha * v[2 * i + 1]);
    }
    *reinterpret_cast<uint4 *>(p) = u;
}
__device__ __forceinline__ void store8_out(float *p, const float *v, float alpha, float beta)
{
    float o[8];
    if (beta != 0.f) {
        float4 a = reinterpret_cast<const float4 *>(p)[0], b = reinterpret_cast<const float4 *>(p)[1];
        const float old[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 8; i++) o[i] = fmaf(alpha, v[i], beta * old[i]);
    } else {
#pragma unroll
        for (int i = 0; i < 8; i++) o[i] = alpha * v[i];
    }
    reinterpret_cast<float4 *>(p)[0] = make_float4(o[0], o[1], o[2], o[3]);
    reinterpret_cast<float4 *>(p)[1] = make_float4(o[4], o[5], o[6], o[7]);
}

// Slot of part q of a cut item whose first part is on CTA b0 (head: that part
// is CTA b0's first segment): part q > 0 is the first segment of CTA b0 + q.
__host__ __device__ inline int tc_slot(int b0, int q, bool head)
{
    return q > 0 ? 2 * (b0 + q) : 2 * b0 + (head ? 0 : 1);
}

// E4M3 dequantisation of 16 accumulators of columns n..n+15: row scale x
// column scale (16-byte aligned scale vectors; columns >= N read as 0).
__device__ __forceinline__ void dequant16(float *v, float sa, const float *col_scale, int n, int N)
{
    const float4 *cs = reinterpret_cast<const float4 *>(col_scale + n);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float4 sv = (n + 4 * q < N) ? __ldg(cs + q) : make_float4(0.f, 0.f, 0.f, 0.f);
        v[4 * q] *= sa * sv.x;
        v[4 * q + 1] *= sa * sv.y;
        v[4 * q + 2] *= sa * sv.z;
        v[4 * q + 3] *= sa * sv.w;
    }
}

// Shared memory (1024-byte aligned base): kStages x (A tile | B tile),
// kStages entry staging buffers, per-stage chunk records, the CTA's item
// table, mbarriers, four broadcast flags and the TMEM slot.
// F8: E4M3 operands -- an 8 KB A tile (64-byte swizzled K-major) and 64 x NT
// byte B tiles, so the ring holds more stages.
template <int NT, bool F8> struct TcCfg {
    static constexpr int kElem = F8 ? 1 : 2;
    static constexpr int kATileBytes = kWindowRows * kChunkCols * kElem;
    static constexpr int kBoxCols = 128 / kElem; // N columns per 128-byte swizzle atom / TMA box
    static constexpr int kStages = F8 ? (NT == 256 ? 6 : 8) : (NT == 256 ? 4 : NT == 128 ? 5 : 6);
    static constexpr int kBTileBytes = kChunkCols * NT * kElem;
    static constexpr int kStage = kATileBytes + kBTileBytes;
    static constexpr int kStagingOff = kStages * kStage;
    static constexpr int kPendOff = kStagingOff + kStages * kStagingBytes; // int4 [kStages]: img, e0, e0a, e1
    static constexpr int kPend2Off = kPendOff + kStages * 16;              // int4 [kStages]: flags, buffer, item
    static constexpr int kItemOff = kPend2Off + kStages * 16;              // int4 [kMaxCtaItems]
    static constexpr int kPartOff = kItemOff + kMaxCtaItems * 16; // int4 [kMaxCtaItems]: cut-item parts
    static constexpr int kBarOff = kPartOff + kMaxCtaItems * 16;
    // full, empty, staged [kStages]; accum_full, accum_empty [2]; drain; 4 flags, TMEM slot, segment
    // count, epilogue flag
    static constexpr int kSmem = kBarOff + (3 * kStages + 5) * 8 + 32;
    static_assert(kSmem <= 227 * 1024, "shared memory budget");
    static_assert(kStage % 1024 == 0 && kATileBytes % 1024 == 0, "swizzled tiles need 1024-byte alignment");
    static_assert(kStagingOff % 16 == 0 && kStagingBytes % 16 == 0 && kPendOff % 16 == 0, "16-byte alignment");
    static_assert(kItemOff % 16 == 0 && kBarOff % 16 == 0, "16-byte aligned regions");
    static_assert(kLoaders <= kStages, "a loader may not lap a stage that an earlier loader still fills");
};

// Work item (job, tensor-core window, N slice) -> table entry {window,
// first chunk, chunk count, job << 16 | N-slice index}.
__device__ __forceinline__ int4 decode_item(const TcBatch &batch, int item)
{
    int j = 0;
    while (j + 1 < batch.n_jobs && batch.item_start[j + 1] <= item) j++;
    const TcJob &a = batch.job[j];
    const int local = item - batch.item_start[j];
    const int4 wi = a.win_info[local / a.ntiles];
    return make_int4(wi.x, wi.y, wi.z, (j << 16) | (local % a.ntiles));
}

// Persistent CTAs, one per SM: CTA b processes work items b, b + gridDim.x,
// ... (at most kMaxCtaItems), as one continuous stream of total_chunks chunks
// through the stage ring; every role runs over exactly those chunks. Roles
// (kThreads threads):
//   warps 4, 10, 11, 12 (loaders; loader l takes chunks g = l (mod kLoaders),
//     so that four chunks are being issued at once -- one warp issuing every
//     chunk in turn was measured to need ~0.9 us per chunk, three times the
//     tensor-core time of an N = 256 chunk): per chunk, acquire the stage
//     ("empty"), write the chunk's records (entries range and image for the
//     scatter warps; first / last chunk of its item and accumulator buffer for
//     the MMA lane), set the "full" transaction count and issue the dense A
//     image (cp.async.bulk) or the sparse entries (cp.async.bulk into staging,
//     completing on "staged"), then the B rows: tiled TMA boxes of 64
//     contiguous rows for direct chunks, tile::gather4 for condensed ones.
//     Chunk metadata (columns, image, entry range) is loaded into registers
//     one chunk of the same loader ahead.
//   warps 0-3 (scatter; two groups of two warps taking chunks in turn when
//     the ring has an even number of stages, else one group of four): per
//     chunk, wait "staged"; for a sparse chunk zero the A tile, scatter the
//     staged entries, fence.proxy.async; arrive "full". With two groups, a
//     group's previous use of a stage is its own (stage count even), so no
//     group waits on a phase more than one ahead of an mbarrier.
//   warp 5, lane 0 (MMA): per chunk wait "full"; on an item's first chunk
//     wait until its TMEM accumulator buffer (item parity) is drained
//     ("accum_empty"); 4 x tcgen05.mma (2 for E4M3); commit "empty"; on the
//     item's last chunk commit "accum_full".
//   warps 6-9 (epilogue): per item wait "accum_full", tcgen05.ld the rows
//     (warp w reads TMEM lanes 32 (w % 4) ..), alpha/beta, store to C[perm],
//     arrive "accum_empty" -- overlapping the next item's main loop.
template <int NT, typename OutT, bool F8>
__global__ void __launch_bounds__(kThreads, 1) spmm_tc_kernel(const __grid_constant__ TcBatch batch)
{
    using Cfg = TcCfg<NT, F8>;
    constexpr int S = Cfg::kStages;
    constexpr int kATileBytes = Cfg::kATileBytes;
    constexpr int kBoxes = NT / Cfg::kBoxCols; // 128-byte-wide boxes per B row slice
    constexpr int kGathers = 16 * kBoxes;      // gather4 instructions per condensed chunk
    extern __shared__ __align__(1024) uint8_t smem[];
    int4 *pend = reinterpret_cast<int4 *>(smem + Cfg::kPendOff);
    int4 *pend2 = reinterpret_cast<int4 *>(smem + Cfg::kPend2Off);
    int4 *items = reinterpret_cast<int4 *>(smem + Cfg::kItemOff);
    int4 *parts = reinterpret_cast<int4 *>(smem + Cfg::kPartOff); // per segment: first CTA, part, parts, head flag
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + Cfg::kBarOff);
    uint64_t *empty = full + S;
    uint64_t *staged = empty + S;
    uint64_t *acc_full = staged + S;  // [2]
    uint64_t *acc_empty = acc_full + 2; // [2]
    uint64_t *drain = acc_empty + 2;    // the MMA lane's last commit: every MMA it issued has completed
    volatile int *flag = reinterpret_cast<volatile int *>(drain + 1); // 2 slots per scatter group
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1) + 4;
    volatile int *seg_count = reinterpret_cast<volatile int *>(drain + 1) + 5;
    constexpr int kScatterGroups = S % 2 == 0 ? 2 : 1; // two groups need an even ring (see the scatter role)
    constexpr int kGroupThreads = kScatterThreads / kScatterGroups;

    // A CUDA-core launch that follows on the stream as a programmatic
    // dependent may start as soon as every block of this grid is resident: it
    // reads nothing this kernel writes (the two paths own disjoint rows of C).
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = batch.item_start[batch.n_jobs];
    const int rr_items = blockIdx.x < total ? min(kMaxCtaItems, (total - 1 - (int)blockIdx.x) / (int)gridDim.x + 1) : 0;
    if (smem_u32(smem) & 1023u) { // the swizzled tiles and TMA destinations need a 1024-byte aligned base
        if (threadIdx.x == 0)
            atomicOr(batch.job[0].status, kStatusLayout);
        return;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], kGroupThreads);
            mbar_init(&empty[s], 1);
            mbar_init(&staged[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kEpiThreads);
        }
        mbar_init(drain, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (batch.split) {
        // Warp 0 lists the segments of this CTA's chunk range: from its start
        // item on, one segment per item the range reaches, with the item's
        // cut (first CTA, part, number of parts) for the epilogue. The window
        // records of the next 32 windows are loaded at once, one per lane.
        if (warp == 0) {
            const long long units = batch.units;
            const int G = gridDim.x, b = blockIdx.x;
            long long u = range_lo(b, units, G);
            const long long hi = range_lo(b + 1, units, G);
            const int4 st = batch.cta_start[b];
            int j = st.x, w = st.y, t = st.z, i0 = st.w, n = 0;
            while (u < hi && n < kMaxCtaItems && j < batch.n_jobs) {
                const TcJob &a = batch.job[j];
                const int4 wl = (w + lane < a.n_win) ? __ldg(a.win_info + w + lane) : make_int4(0, 0, 0, 0);
                int l = 0;
                while (u < hi && n < kMaxCtaItems && l < 32 && w + l < a.n_win) {
                    const int wx = __shfl_sync(0xffffffffu, wl.x, l);
                    const int wy = __shfl_sync(0xffffffffu, wl.y, l);
                    const int z = __shfl_sync(0xffffffffu, wl.z, l);
                    const long long u0 = u - i0; // the item's first unit
                    const int cnt = (int)min((long long)(z - i0), hi - u);
                    const int b0 = range_owner(u0, units, G), b1 = range_owner(u0 + z - 1, units, G);
                    if (lane == 0) {
                        items[n] = make_int4(wx, wy + i0, cnt, (j << 16) | t);
                        parts[n] = make_int4(b0, b - b0, b1 - b0 + 1, range_lo(b0, units, G) == u0 ? 1 : 0);
                    }
                    n++;
                    u += cnt;
                    i0 = 0;
                    if (++t == a.ntiles) { t = 0; l++; }
                }
                w += l;
                if (w >= a.n_win) { j++; w = 0; }
            }
            if (lane == 0) {
                // The range's last segment, when cut, is the head of an item
                // another CTA finishes: it goes second (after the first,
                // itself cut or whole), so that both cut parts complete early
                // and the part that adds them up does so while this CTA's
                // whole items still run.
                if (n >= 3 && parts[n - 1].z > 1) {
                    const int4 li = items[n - 1], lp = parts[n - 1];
                    for (int k = n - 1; k > 1; k--) {
                        items[k] = items[k - 1];
                        parts[k] = parts[k - 1];
                    }
                    items[1] = li;
                    parts[1] = lp;
                }
                *seg_count = n;
                if (u < hi) // more segments than the table holds: the host sizes ranges so that this cannot be
                    atomicOr(batch.job[0].status, kStatusTable);
            }
        }
    } else if ((int)threadIdx.x < rr_items) {
        items[threadIdx.x] = decode_item(batch, blockIdx.x + threadIdx.x * gridDim.x);
        parts[threadIdx.x] = make_int4((int)blockIdx.x, 0, 1, 1);
    }
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * NT)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int n_items = batch.split ? *seg_count : rr_items;
    bool ok = true;
    int total_chunks = 0; // of this CTA's items: every role runs over exactly these
    for (int k = 0; k < n_items; k++) total_chunks += items[k].z;

    if (warp == kLoaderWarp || warp >= kLoaderWarp1) {
        // ---------------- loaders ----------------
        // Loader ld issues chunks g = ld, ld + kLoaders, ... of the CTA's chunk
        // stream; (k, i) is the item and chunk-within-item of its next chunk.
        const int ld = warp == kLoaderWarp ? 0 : warp - kLoaderWarp1 + 1;
        auto advance = [&](int &k, int &i) {
            while (k < n_items && i >= items[k].z) { i -= items[k].z; k++; }
        };
        // per-chunk metadata in registers: lanes 0-15 hold 4 columns each, every
        // lane the image index and entry range; fetched one chunk of this loader ahead
        struct Meta { int4 cols; int img, e0, e1; };
        auto fetch = [&](int k, int i, Meta &m) {
            m.cols = make_int4(-1, -1, -1, -1);
            m.img = -1;
            m.e0 = m.e1 = 0;
            if (k < n_items) {
                const int4 it = items[k];
                const TcJob &a = batch.job[it.w >> 16];
                const int c = it.y + i;
                if (lane < 16)
                    m.cols = __ldg(reinterpret_cast<const int4 *>(a.win_cols + (size_t)c * kChunkCols) + lane);
                m.img = __ldg(a.img_idx + c);
                m.e0 = __ldg(a.tile_ptr + c);
                m.e1 = __ldg(a.tile_ptr + c + 1);
            }
        };
        int k = 0, i = ld;
        advance(k, i);
        int g = ld;
        // One chunk: prefetch the metadata of this loader's next chunk into
        // `nxt`, acquire the stage, issue the chunk described by `cur`. The
        // loop below alternates the roles of two Meta variables (unrolled by
        // two), so that no register copy waits for a prefetch still in flight.
        auto step = [&](Meta &cur, Meta &nxt) -> bool {
            if (g >= total_chunks || !ok)
                return false;
            int k2 = k, i2 = i + kLoaders;
            advance(k2, i2);
            fetch(k2, i2, nxt);
            const int s = g % S;
            uint32_t got = 1;
            if (lane == 0 && g >= S)
                got = mbar_wait(&empty[s], ((g / S) - 1) & 1) ? 1u : 0u;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) { ok = false; return false; }
            const int4 it = items[k];
            const TcJob &a = batch.job[it.w >> 16];
            const int n0 = (it.w & 0xffff) * NT;
            const uint32_t a_s = smem_u32(smem + s * Cfg::kStage), b_s = a_s + kATileBytes;
            if (lane == 0) {
                const int img = cur.img, e0 = cur.e0, e1 = cur.e1, e0a = e0 & ~3;
                pend[s] = make_int4(img, e0, e0a, e1);
                pend2[s] = make_int4((i == 0 ? 1 : 0) | (i == it.z - 1 ? 2 : 0), k & 1, k, 0);
                mbar_expect_tx(&full[s], Cfg::kBTileBytes + (img >= 0 ? kATileBytes : 0));
                if (img >= 0) {
                    bulk_copy_g2s(a_s, a.images + (size_t)img * kATileBytes, kATileBytes, &full[s]);
                    mbar_arrive(&staged[s]);
                } else if (e1 > e0) {
                    const uint32_t bytes = (uint32_t)(((e1 - e0a) * 4 + 15) & ~15);
                    mbar_arrive_expect_tx(&staged[s], bytes);
                    bulk_copy_g2s(smem_u32(smem + Cfg::kStagingOff + s * kStagingBytes), a.entries + e0a, bytes,
                                  &staged[s]);
                } else {
                    mbar_arrive(&staged[s]);
                }
            }
            __syncwarp(); // the transaction count is set before any B load is issued
            const int col0 = __shfl_sync(0xffffffffu, cur.cols.x, 0);
            const int col63 = __shfl_sync(0xffffffffu, cur.cols.w, 15);
            if (col0 >= 0 && col63 == col0 + kChunkCols - 1) {
                // 64 contiguous B rows (direct chunks): one 8 KB tiled box per 128-byte column slab
                if (lane < kBoxes)
                    tma_tile2d(b_s + lane * (kChunkCols * 128), &a.tmap_tile, n0 + lane * Cfg::kBoxCols, col0,
                               &full[s]);
            } else {
                // condensed columns: gather q = lane, lane + 32, .. reads the 4 columns of lane q % 16
                const int src = lane & 15;
                const int y0 = __shfl_sync(0xffffffffu, cur.cols.x, src);
                const int y1 = __shfl_sync(0xffffffffu, cur.cols.y, src);
                const int y2 = __shfl_sync(0xffffffffu, cur.cols.z, src);
                const int y3 = __shfl_sync(0xffffffffu, cur.cols.w, src);
                for (int q = lane; q < kGathers; q += 32) {
                    const int box = q >> 4;
                    tma_gather4(b_s + box * (kChunkCols * 128) + src * 512, &a.tmap_b, n0 + box * Cfg::kBoxCols, y0,
                                y1, y2, y3, &full[s]);
                }
            }
            k = k2;
            i = i2;
            g += kLoaders;
            return true;
        };
        Meta ma, mb;
        fetch(k, i, ma);
        while (step(ma, mb) && step(mb, ma)) {
        }
    } else if (warp < 4) {
        // ---------------- scatter ----------------
        // kScatterGroups groups of warps take the chunks in turn (group q:
        // chunks g = q (mod kScatterGroups)), so that the scatter of one sparse
        // chunk overlaps the next one's.
        const int grp = kScatterGroups == 2 ? (warp >> 1) : 0;
        const int sid = (int)threadIdx.x - grp * kGroupThreads;
        int it = 0;
        for (int g = grp; g < total_chunks; g += kScatterGroups, it++) {
            const int s = g % S;
            volatile int *fl = flag + grp * 2 + (it & 1);
            if (sid == 0)
                *fl = mbar_wait(&staged[s], (g / S) & 1) ? 1 : 0;
            named_bar_sync(1 + grp, kGroupThreads); // also orders the staged data for every thread of the group
            if (*fl == 0) { ok = false; break; } // uniform across the group
            const int4 pd = pend[s];
            if (pd.x == -1) {
                uint8_t *At = smem + s * Cfg::kStage;
#pragma unroll
                for (int q = 0; q < kATileBytes / (16 * kGroupThreads); q++)
                    reinterpret_cast<uint4 *>(At)[sid + q * kGroupThreads] = make_uint4(0, 0, 0, 0);
                named_bar_sync(1 + grp, kGroupThreads);
                const uint32_t *st = reinterpret_cast<const uint32_t *>(smem + Cfg::kStagingOff + s * kStagingBytes);
                for (int e = pd.y + sid; e < pd.w; e += kGroupThreads) {
                    const uint32_t v = st[e - pd.z];
                    if constexpr (F8)
                        At[swz64_offset(v >> 22, (v >> 16) & 63u)] = (uint8_t)(v & 0xffu);
                    else
                        *reinterpret_cast<uint16_t *>(At + swz128_offset(v >> 22, (v >> 16) & 63u)) =
                            (uint16_t)(v & 0xffffu);
                }
                fence_proxy_async();
            }
            mbar_arrive(&full[s]);
        }
    } else if (warp == kMmaWarp) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_f16(NT); // E4M3 has format code 0 in kind::f8f6f4 as FP16 in kind::f16
            // test hook: the CTA's last accumulator is never announced, so the
            // epilogue's bounded wait for it runs out (TCA_FLAG_TEST_WITHHOLD_ACCUM)
            const bool withhold = (batch.job[0].flags & TCA_FLAG_TEST_WITHHOLD_ACCUM) != 0;
            for (int g = 0; g < total_chunks; g++) {
                const int s = g % S;
                if (!mbar_wait(&full[s], (g / S) & 1)) { ok = false; break; }
                const int4 f = pend2[s];
                const int b = f.y, k = f.z;
                if ((f.x & 1) && k >= 2 && !mbar_wait(&acc_empty[b], ((k >> 1) - 1) & 1)) { ok = false; break; }
                tc_fence_after();
                const uint32_t a_s = smem_u32(smem + s * Cfg::kStage), b_s = a_s + kATileBytes;
                const uint32_t d = tmem + (uint32_t)(b * NT);
                if constexpr (F8) {
                    // 2 x K = 32: A rows of 64 bytes (64-byte swizzle, 8-row groups 512 bytes apart),
                    // B k-rows of 128 bytes (128-byte swizzle, atoms along N 8 KB apart)
#pragma unroll
                    for (int kk = 0; kk < kChunkCols / 32; kk++) {
                        const uint64_t ad = smem_desc(a_s + kk * 32, 16, 512, 4);
                        const uint64_t bd = smem_desc(b_s + kk * 4096, kChunkCols * 128, 1024);
                        umma_f8(d, ad, bd, idesc, ((f.x & 1) && kk == 0) ? 0u : 1u);
                    }
                } else {
#pragma unroll
                    for (int kk = 0; kk < kChunkCols / 16; kk++) {
                        const uint64_t ad = smem_desc(a_s + kk * 32, 16, 1024);
                        const uint64_t bd = smem_desc(b_s + kk * 2048, kChunkCols * 128, 1024);
                        umma_f16(d, ad, bd, idesc, ((f.x & 1) && kk == 0) ? 0u : 1u);
                    }
                }
                umma_commit(&empty[s]);
                if ((f.x & 2) && !(withhold && k == n_items - 1))
                    umma_commit(&acc_full[b]);
            }
            // every MMA issued has completed before the tensor memory is
            // released, also when a role gave up early
            umma_commit(drain);
            if (!mbar_wait(drain, 0))
                ok = false;
        }
        __syncwarp();
    } else {
        // ---------------- epilogue ----------------
        // Per segment: wait for its accumulator; a whole item is stored to C
        // (alpha, beta, E4M3 scales); a cut item's part leaves its FP32
        // partial tile in its slot, for spmm_tc_fixup to add up after this
        // launch.
        const int quarter = warp & 3;
        const int row = quarter * 32 + lane; // TMEM lane = row of the window
        for (int k = 0; k < n_items; k++) {
            const int4 it = items[k];
            const int4 pt = parts[k];
            const TcJob &a = batch.job[it.w >> 16];
            const int n0 = (it.w & 0xffff) * NT;
            const int i = it.x * kWindowRows + row;
            int out_row = -1;
            if (i < a.M && !((a.flags & TCA_FLAG_KEEP_EMPTY_ROWS) && a.p_row_ptr[i + 1] == a.p_row_ptr[i]))
                out_row = a.perm[i];
            const int b = k & 1;
            uint32_t got = 0;
            if (lane == 0)
                got = mbar_wait(&acc_full[b], (k >> 1) & 1) ? 1u : 0u;
            got = __shfl_sync(0xffffffffu, got, 0);
            // the four warps agree, so that none is left at a later barrier
            if (!named_bar_and(kEpiBar, kEpiThreads, got != 0)) { ok = false; break; }
            tc_fence_after();
            const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * NT);
            if (pt.z > 1) {
                float *mine = batch.partials + ((size_t)tc_slot(pt.x, pt.y, pt.w != 0) * kWindowRows + row) * NT;
                for (int cb = 0; cb < NT / 16; cb++) {
                    if (n0 + cb * 16 >= a.N)
                        break; // uniform across the warp
                    uint32_t r[16];
                    tmem_ld16(taddr + cb * 16, r);
                    float4 *dst = reinterpret_cast<float4 *>(mine + cb * 16);
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        dst[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                             __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
                }
            } else {
                OutT *Crow = out_row >= 0 ? reinterpret_cast<OutT *>(a.C) + (size_t)out_row * a.ldc : nullptr;
                float sa = 1.f;
                if constexpr (F8)
                    sa = (i < a.M) ? a.row_scale[i] : 0.f;
                for (int cb = 0; cb < NT / 16; cb++) {
                    const int n = n0 + cb * 16;
                    if (n >= a.N)
                        break; // uniform across the warp
                    uint32_t r[16];
                    tmem_ld16(taddr + cb * 16, r);
                    float *v = reinterpret_cast<float *>(r);
                    if constexpr (F8)
                        dequant16(v, sa, a.col_scale, n, a.N);
                    if (Crow) {
                        store8_out(Crow + n, v, a.alpha, a.beta);
                        if (n + 8 < a.N)
                            store8_out(Crow + n + 8, v + 8, a.alpha, a.beta);
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&acc_empty[b]);
        }
    }

    tc_fence_before();
    if (__syncthreads_or(!ok)) {
        // A role gave up after a bounded wait: record it, then give bulk
        // copies that loaders issued and nobody consumed a bounded time
        // (1 ms; a copy lands within microseconds) to land before this
        // CTA's shared memory is released.
        if (threadIdx.x == 0) {
            if (n_items > 0)
                atomicOr(batch.job[items[0].w >> 16].status, kStatusTimeout);
            if (batch.split)
                atomicOr(batch.failed, 1); // its cut parts may be missing: no sums after this launch
            const uint64_t t0 = global_ns();
            while (global_ns() - t0 < 1000000ull) {
            }
        }
        __syncthreads();
    }
    if (warp == kMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * NT) : "memory");
    }
}

// After a split launch: block (c, r) adds up the parts of cut item c for
// rows 32 r .. 32 r + 31 of its window, in part order -- a fixed order, so the
// result does not depend on which CTA computed which part when -- and stores
// C as the tensor-core epilogue stores a whole item (E4M3 scales, alpha,
// beta, rows without nonzeros kept on request). A thread takes 8 columns of a
// row; the loads of up to four parts are issued before the first is added.
template <int NT, typename OutT, bool F8>
__global__ void __launch_bounds__(256)
spmm_tc_fixup(const __grid_constant__ TcBatch batch, const __grid_constant__ TcCuts cuts)
{
    if (*(volatile const int *)batch.failed)
        return; // a CTA of the launch gave up (its status word says so): C keeps what it had
    const int4 cu = cuts.cut[blockIdx.x];
    const TcJob &a = batch.job[cu.x >> 16];
    const int n0 = (cu.x & 0xffff) * NT;
    const int window = __ldg(&a.win_info[cu.y].x);
    const int b0 = cu.z, parts = cu.w >> 1;
    const bool head = (cu.w & 1) != 0;
    const int vpr = min(NT, a.N - n0) >> 3; // 8-column vectors a row (N % 8 == 0 on this path)
    for (int idx = threadIdx.x; idx < 32 * vpr; idx += blockDim.x) {
        const int rl = blockIdx.y * 32 + idx / vpr, c8 = (idx % vpr) * 8;
        const int i = window * kWindowRows + rl;
        if (i >= a.M)
            continue;
        const size_t off = (size_t)rl * NT + c8;
        float acc[8];
        for (int q0 = 0; q0 < parts; q0 += 4) {
            float4 x[4][2];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if (q0 + u < parts) {
                    const float4 *src = reinterpret_cast<const float4 *>(
                        batch.partials + (size_t)tc_slot(b0, q0 + u, head) * kWindowRows * NT + off);
                    x[u][0] = __ldcg(src);
                    x[u][1] = __ldcg(src + 1);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if (q0 + u < parts) {
                    const float e[8] = {x[u][0].x, x[u][0].y, x[u][0].z, x[u][0].w,
                                        x[u][1].x, x[u][1].y, x[u][1].z, x[u][1].w};
#pragma unroll
                    for (int k = 0; k < 8; k++) acc[k] = (q0 + u == 0) ? e[k] : acc[k] + e[k];
                }
            }
        }
        if ((a.flags & TCA_FLAG_KEEP_EMPTY_ROWS) && a.p_row_ptr[i + 1] == a.p_row_ptr[i])
            continue;
        const int n = n0 + c8;
        if constexpr (F8) {
            const float sa = a.row_scale[i];
            const float4 s0 = __ldg(reinterpret_cast<const float4 *>(a.col_scale + n));
            const float4 s1 = __ldg(reinterpret_cast<const float4 *>(a.col_scale + n) + 1);
            const float sb[8] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
#pragma unroll
            for (int k = 0; k < 8; k++) acc[k] *= sa * sb[k];
        }
        store8_out(reinterpret_cast<OutT *>(a.C) + (size_t)a.perm[i] * a.ldc + n, acc, a.alpha, a.beta);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

} // namespace

int encode_tensor_map_2d(CUtensorMap *map, CUtensorMapDataType dtype, const void *base, uint64_t d0, uint64_t d1,
                         uint64_t row_stride_bytes, uint32_t b0, uint32_t b1, CUtensorMapSwizzle swizzle)
{
    auto enc = tensor_map_encoder();
    if (!enc)
        return set_error(TCA_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[2] = {(cuuint64_t)d0, (cuuint64_t)(d1 > 0 ? d1 : 1)};
    const cuuint64_t strides[1] = {(cuuint64_t)row_stride_bytes};
    const cuuint32_t box[2] = {b0, b1};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(map, dtype, 2, const_cast<void *>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return set_error(TCA_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d): dims {%llu, %llu}, stride %llu, box {%u, %u}",
                         (int)r, (unsigned long long)d0, (unsigned long long)d1, (unsigned long long)row_stride_bytes,
                         b0, b1);
    return TCA_OK;
}

namespace {

// B (K x N, row-major, leading dimension ldb) as a TMA source: dims {N, K},
// row stride ldb * 2 bytes, box {64, rows}, 128-byte swizzle, zero fill.
int encode_b_map(const SpmmJob &sj, int K, int rows, CUtensorMap *map)
{
    return encode_tensor_map_2d(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, sj.B, (uint64_t)sj.N, (uint64_t)K,
                                (uint64_t)sj.ldb * 2, 64, (uint32_t)rows, CU_TENSOR_MAP_SWIZZLE_128B);
}

int make_job(const SpmmJob &sj, float alpha, float beta, unsigned flags, int NT, TcJob *out)
{
    const tca_plan *p = sj.p;
    TcJob &j = *out;
    if (sj.f8) {
        // E4M3 B (K x N bytes, row stride ldq): boxes of 128 columns
        TCA_TRY(encode_tensor_map_2d(&j.tmap_b, CU_TENSOR_MAP_DATA_TYPE_UINT8, sj.Bq, (uint64_t)sj.N, (uint64_t)p->K,
                                     (uint64_t)sj.ldq, 128, 1, CU_TENSOR_MAP_SWIZZLE_128B));
        TCA_TRY(encode_tensor_map_2d(&j.tmap_tile, CU_TENSOR_MAP_DATA_TYPE_UINT8, sj.Bq, (uint64_t)sj.N,
                                     (uint64_t)p->K, (uint64_t)sj.ldq, 128, kChunkCols, CU_TENSOR_MAP_SWIZZLE_128B));
        j.entries = p->tile_entries_f8;
        j.images = p->images_f8;
        j.row_scale = p->row_scale;
        j.col_scale = sj.col_scale;
    } else {
        TCA_TRY(encode_b_map(sj, p->K, 1, &j.tmap_b));
        TCA_TRY(encode_b_map(sj, p->K, kChunkCols, &j.tmap_tile));
        j.entries = p->tile_entries;
        j.images = reinterpret_cast<const uint8_t *>(p->images);
        j.row_scale = nullptr;
        j.col_scale = nullptr;
    }
    j.win_info = p->tc_win_info;
    j.tile_ptr = p->tile_ptr;
    j.win_cols = p->win_cols;
    j.img_idx = p->img_idx;
    j.perm = p->perm;
    j.p_row_ptr = p->p_row_ptr;
    j.B = sj.B;
    j.C = sj.C;
    j.status = p->d_status;
    j.M = p->M;
    j.N = sj.N;
    j.ldb = sj.ldb;
    j.ldc = sj.ldc;
    j.ntiles = (sj.N + NT - 1) / NT;
    j.n_win = p->n_tc;
    j.alpha = alpha;
    j.beta = beta;
    j.flags = flags;
    return TCA_OK;
}

// Chunk ranges (stream-K) for a batch whose jobs' plans are `plans`: the grid
// (at most one CTA per SM, at least kMinUnits chunks each, so that a cut item
// has few parts to add up) and each CTA's start item, from the plans' host
// copies of their windows' chunk offsets. False when some CTA's range would
// reach more items than its work table holds (then items go to CTAs in turn).
constexpr int kMinUnits = 8;

bool plan_ranges(TcBatch &b, const tca_plan *const *plans, int *grid_out, TcCuts *cuts)
{
    cuts->n = 0;
    long long units = 0;
    for (int j = 0; j < b.n_jobs; j++)
        units += (long long)plans[j]->n_tc_chunks * b.job[j].ntiles;
    if (units <= 0)
        return false;
    const int G = (int)std::min<long long>(kSMs, std::max<long long>(1, units / kMinUnits));
    int segs[kSMs] = {0};
    long long u0 = 0;
    for (int j = 0; j < b.n_jobs; j++) {
        const std::vector<int> &first = plans[j]->h_tile_first;
        for (int w = 0; w < b.job[j].n_win; w++) {
            const int z = first[w + 1] - first[w];
            for (int t = 0; t < b.job[j].ntiles; t++, u0 += z) {
                const int c0 = range_owner(u0, units, G), c1 = range_owner(u0 + z - 1, units, G);
                if (c1 > c0) {
                    if (cuts->n == kSMs)
                        return false; // cannot happen: a cut needs a range boundary inside the item
                    const int head = range_lo(c0, units, G) == u0 ? 1 : 0;
                    cuts->cut[cuts->n++] = make_int4((j << 16) | t, w, c0, ((c1 - c0 + 1) << 1) | head);
                }
                for (int c = c0; c <= c1; c++) {
                    if (++segs[c] > kMaxCtaItems)
                        return false;
                    const long long lo = range_lo(c, units, G);
                    if (lo >= u0)
                        b.cta_start[c] = make_int4(j, w, t, (int)(lo - u0));
                }
            }
        }
    }
    b.split = 1;
    b.units = units;
    *grid_out = G;
    return true;
}

template <int NT, typename OutT, bool F8>
int launch_group(const TcBatch &b, int grid, cudaStream_t s)
{
    const int smem = TcCfg<NT, F8>::kSmem;
    TCA_CUDA_TRY(cudaFuncSetAttribute(spmm_tc_kernel<NT, OutT, F8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    spmm_tc_kernel<NT, OutT, F8><<<grid, kThreads, smem, s>>>(b);
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

template <int NT, typename OutT, bool F8>
int launch_fixup(const TcBatch &b, const TcCuts &c, cudaStream_t s)
{
    spmm_tc_fixup<NT, OutT, F8><<<dim3((unsigned)c.n, kWindowRows / 32), 256, 0, s>>>(b, c);
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

template <typename OutT>
int launch_fixup_out(const TcBatch &b, const TcCuts &c, int NT, bool f8, cudaStream_t s)
{
    if (f8)
        return NT == 128 ? launch_fixup<128, OutT, true>(b, c, s) : launch_fixup<256, OutT, true>(b, c, s);
    switch (NT) {
    case 64: return launch_fixup<64, OutT, false>(b, c, s);
    case 128: return launch_fixup<128, OutT, false>(b, c, s);
    default: return launch_fixup<256, OutT, false>(b, c, s);
    }
}

template <typename OutT>
int launch_group_out(const TcBatch &b, int NT, bool f8, int grid, cudaStream_t s)
{
    if (f8)
        return NT == 128 ? launch_group<128, OutT, true>(b, grid, s) : launch_group<256, OutT, true>(b, grid, s);
    switch (NT) {
    case 64: return launch_group<64, OutT, false>(b, grid, s);
    case 128: return launch_group<128, OutT, false>(b, grid, s);
    default: return launch_group<256, OutT, false>(b, grid, s);
    }
}

int launch_group_typed(const TcBatch &b, int NT, bool f8, int c_dtype, int grid, cudaStream_t s)
{
    if (b.n_jobs == 0 || b.item_start[b.n_jobs] == 0)
        return TCA_OK;
    return c_dtype == TCA_DTYPE_F16 ? launch_group_out<__half>(b, NT, f8, grid, s)
                                    : launch_group_out<float>(b, NT, f8, grid, s);
}

} // namespace

int pick_tc_tile(const tca_plan *p, int N, bool batched, bool f8, bool split)
{
    const int lo = f8 ? 128 : 64; // E4M3 B tiles are whole 128-byte swizzle atoms
    int NT = N <= 64 ? 64 : N <= 128 ? 128 : 256;
    NT = std::max(NT, lo);
    if (batched)
        return NT;
    if (split) {
        // chunk ranges: halve the slice while the forward has fewer chunks
        // than kMinUnits per SM (a wider slice's chunk carries more work, but
        // fewer CTAs would share the forward)
        while (NT > lo && (long long)p->n_tc_chunks * ((N + NT - 1) / NT) < (long long)kMinUnits * kSMs)
            NT /= 2;
    } else {
        // items to CTAs in turn: halve the slice while that leaves fewer than
        // about three quarters of the SMs with an item (measured: A^T of
        // 512 x 2048, N = 4096, 4 windows: NT = 128, 128 items, 30.5 us;
        // NT = 64, 40.4 us)
        while (NT > lo && (long long)p->n_tc * ((N + NT - 1) / NT) < (3 * kSMs) / 4)
            NT /= 2;
    }
    return NT;
}

int tc_block_regs(bool f8, int *regs)
{
    static int worst[2] = {0, 0};
    if (worst[f8] == 0) {
        const void *f16_fns[] = {
            (const void *)spmm_tc_kernel<64, __half, false>, (const void *)spmm_tc_kernel<128, __half, false>,
            (const void *)spmm_tc_kernel<256, __half, false>, (const void *)spmm_tc_kernel<64, float, false>,
            (const void *)spmm_tc_kernel<128, float, false>, (const void *)spmm_tc_kernel<256, float, false>};
        const void *f8_fns[] = {
            (const void *)spmm_tc_kernel<128, __half, true>, (const void *)spmm_tc_kernel<256, __half, true>,
            (const void *)spmm_tc_kernel<128, float, true>, (const void *)spmm_tc_kernel<256, float, true>};
        int w = 0;
        for (const void *f : f16_fns) {
            if (f8) break;
            int r = 0;
            TCA_TRY(block_regs(f, kThreads, &r));
            w = std::max(w, r);
        }
        for (const void *f : f8_fns) {
            if (!f8) break;
            int r = 0;
            TCA_TRY(block_regs(f, kThreads, &r));
            w = std::max(w, r);
        }
        worst[f8] = w;
    }
    *regs = worst[f8];
    return TCA_OK;
}

int launch_tc_jobs(const SpmmJob *jobs, int n_jobs, int c_dtype, float alpha, float beta, unsigned flags,
                   cudaStream_t s, LaunchList *defer, TcWorkspace *ws, LaunchList *post)
{
    const int widths[3] = {64, 128, 256};
    auto emit = [&](TcBatch &b, const tca_plan *const *plans, int NT, bool f8) -> int {
        if (b.n_jobs == 0 || b.item_start[b.n_jobs] == 0)
            return TCA_OK;
        const int total = b.item_start[b.n_jobs];
        int grid = std::min(total, std::max(kSMs, (total + kMaxCtaItems - 1) / kMaxCtaItems));
        b.split = 0;
        b.units = 0;
        b.partials = nullptr;
        b.failed = nullptr;
        auto cuts = std::make_shared<TcCuts>();
        cuts->n = 0;
        size_t offset = 0; // this launch's partial tiles in the workspace (floats)
        if (ws && defer && post && plan_ranges(b, plans, &grid, cuts.get())) {
            offset = ws->partial_bytes / sizeof(float);
            // every launch of the call has a region of its own: the fixups run after all of them
            ws->partial_bytes += sizeof(float) * 2 * (size_t)grid * kWindowRows * NT;
        }
        if (!defer)
            return launch_group_typed(b, NT, f8, c_dtype, grid, s);
        auto held = std::make_shared<TcBatch>(b);
        defer->push_back([held, NT, f8, c_dtype, grid, ws, offset](cudaStream_t st) {
            if (held->split) {
                held->partials = ws->partials + offset;
                held->failed = ws->failed;
            }
            return launch_group_typed(*held, NT, f8, c_dtype, grid, st);
        });
        if (held->split && cuts->n > 0)
            post->push_back([held, cuts, NT, f8, c_dtype](cudaStream_t st) {
                return c_dtype == TCA_DTYPE_F16 ? launch_fixup_out<__half>(*held, *cuts, NT, f8, st)
                                                : launch_fixup_out<float>(*held, *cuts, NT, f8, st);
            });
        return TCA_OK;
    };
    for (bool f8 : {false, true}) {
        for (int NT : widths) {
            TcBatch b;
            const tca_plan *plans[kMaxJobs];
            b.n_jobs = 0;
            b.item_start[0] = 0;
            for (int i = 0; i < n_jobs; i++) {
                const SpmmJob &sj = jobs[i];
                if (!sj.tc || sj.f8 != f8 || sj.n_tile != NT || sj.p->n_tc == 0 || sj.N <= 0)
                    continue;
                TCA_TRY(make_job(sj, alpha, beta, flags, NT, &b.job[b.n_jobs]));
                plans[b.n_jobs] = sj.p;
                b.item_start[b.n_jobs + 1] = b.item_start[b.n_jobs] + sj.p->n_tc * b.job[b.n_jobs].ntiles;
                b.n_jobs++;
                if (b.n_jobs == kMaxJobs) {
                    TCA_TRY(emit(b, plans, NT, f8));
                    b.n_jobs = 0;
                }
            }
            TCA_TRY(emit(b, plans, NT, f8));
        }
    }
    return TCA_OK;
}

} // namespace tca
