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
// Work items are (job, window, NT-wide slice of N); persistent CTAs (one per
// SM) stream the chunks of their items through a ring of kStages (A tile,
// B tile, entry staging) stages, with decoupled roles:
//   * four loader warps, taking chunks in turn, move every byte through the
//     TMA engine: the 64 B rows of the chunk -- one tiled box per 64 columns
//     of N when its columns are 64 consecutive rows of B, else tile::gather4
//     of the condensed columns (4 rows x 128 bytes per instruction into a
//     128-byte swizzled N-major tile; padding columns and n >= N are out of
//     the tensor and arrive as zeros) -- and either the chunk's pre-rendered,
//     pre-swizzled dense A tile (chunks with >= 512 nonzeros: one 16 KB
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
constexpr int kMaxCtaItems = 32;      // work items per persistent CTA
constexpr int kEpiBar = 3;           // named barrier of the epilogue warps (1, 2: scatter groups)
constexpr int kEpiWarp0 = 6;         // first epilogue warp
constexpr int kStagingBytes = ((kImageMinNnz + 3) * 4 + 15) & ~15; // entries of a sparse chunk, 16-byte rounded
constexpr int kMaxJobs = 32;                                  // jobs per launch (kernel parameter space)

struct TcJob {
    CUtensorMap tmap_b;    // B as a 2-D tensor {N, K}, box {64, 1}, 128-byte swizzle (gather4 source)
    CUtensorMap tmap_tile; // the same tensor, box {64, 64}: 64 contiguous rows of B per instruction
    const int4 *win_info; // per tensor-core window: window, first chunk, chunk count
    const int2 *pairs;    // pair kernel: tensor-core window pairs (second -1: alone)
    const int *tile_ptr, *win_cols, *img_idx, *perm, *p_row_ptr;
    const uint32_t *entries;
    const uint8_t *images;   // dense tile images (16 KB FP16 or 8 KB E4M3 each)
    const float *row_scale;  // E4M3: per sorted row
    const float *col_scale;  // E4M3: per column of N
    const __half *B;
    void *C;
    int *status;
    int M, N, ldb, ldc, ntiles;
    float alpha, beta;
    unsigned flags;
};

// A launch's jobs. The kernel is also built for CAP = 1: a single forward's
// parameter block is then ~0.4 KB instead of ~12 KB (measured: the launch
// took 5-15 us of host time with the full block).
template <int CAP>
struct TcBatchT {
    int n_jobs;
    int item_start[CAP + 1];
    TcJob job[CAP];
};
using TcBatch = TcBatchT<kMaxJobs>;

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

// Shared memory (1024-byte aligned base): kStages x (A tile | B tile),
// kStages entry staging buffers, per-stage chunk records, the CTA's item
// table, mbarriers, four broadcast flags and the TMEM slot.
// F8: E4M3 operands -- an 8 KB A tile (64-byte swizzled K-major) and 64 x NT
// byte B tiles, so the ring holds more stages.
template <int NT, bool F8> struct TcCfg {
    static constexpr int kElem = F8 ? 1 : 2;
    static constexpr int kATileBytes = kWindowRows * kChunkCols * kElem;
    static constexpr int kBoxCols = 128 / kElem; // N columns per 128-byte swizzle atom / TMA box
    static constexpr int kStages = F8 ? (NT == 256 ? 8 : 12) : (NT == 256 ? 4 : NT == 128 ? 6 : 8);
    static constexpr int kBTileBytes = kChunkCols * NT * kElem;
    static constexpr int kStage = kATileBytes + kBTileBytes;
    static constexpr int kStagingOff = kStages * kStage;
    static constexpr int kPendOff = kStagingOff + kStages * kStagingBytes; // int4 [kStages]: img, e0, e0a, e1
    static constexpr int kPend2Off = kPendOff + kStages * 16;              // int4 [kStages]: flags, buffer, item
    static constexpr int kItemOff = kPend2Off + kStages * 16;              // int4 [kMaxCtaItems]
    static constexpr int kScaleOff = kItemOff + kMaxCtaItems * 16;         // E4M3: float [2][NT] column scales
    static constexpr int kBarOff = kScaleOff + (F8 ? 2 * NT * 4 : 0);
    // full, empty, staged [kStages]; accum_full, accum_empty [2]; drain; 4 flags, TMEM slot
    static constexpr int kSmem = kBarOff + (3 * kStages + 5) * 8 + 24;
    static_assert(kSmem <= 227 * 1024, "shared memory budget");
    static_assert(kStage % 1024 == 0 && kATileBytes % 1024 == 0, "swizzled tiles need 1024-byte alignment");
    static_assert(kStagingOff % 16 == 0 && kStagingBytes % 16 == 0 && kPendOff % 16 == 0, "16-byte alignment");
    static_assert(kItemOff % 16 == 0 && kBarOff % 16 == 0, "16-byte aligned regions");
    static_assert(kLoaders <= kStages, "a loader may not lap a stage that an earlier loader still fills");
};

// Work item (job, tensor-core window, N slice) -> table entry {window,
// first chunk, chunk count, job << 16 | N-slice index}.
template <typename Batch>
__device__ __forceinline__ int4 decode_item(const Batch &batch, int item)
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
template <int NT, typename OutT, bool F8, int CAP = kMaxJobs>
__global__ void __launch_bounds__(kThreads, 1) spmm_tc_kernel(const __grid_constant__ TcBatchT<CAP> batch)
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
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + Cfg::kBarOff);
    uint64_t *empty = full + S;
    uint64_t *staged = empty + S;
    uint64_t *acc_full = staged + S;  // [2]
    uint64_t *acc_empty = acc_full + 2; // [2]
    uint64_t *drain = acc_empty + 2;    // the MMA lane's last commit: every MMA it issued has completed
    volatile int *flag = reinterpret_cast<volatile int *>(drain + 1); // 2 slots per scatter group
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1) + 4;
    constexpr int kScatterGroups = S % 2 == 0 ? 2 : 1; // two groups need an even ring (see the scatter role)
    constexpr int kGroupThreads = kScatterThreads / kScatterGroups;

    // A CUDA-core launch that follows on the stream as a programmatic
    // dependent may start as soon as every block of this grid is resident: it
    // reads nothing this kernel writes (the two paths own disjoint rows of C).
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = batch.item_start[batch.n_jobs];
    const int n_items = blockIdx.x < total ? min(kMaxCtaItems, (total - 1 - (int)blockIdx.x) / (int)gridDim.x + 1) : 0;
    if (smem_u32(smem) & 1023u) { // the swizzled tiles and TMA destinations need a 1024-byte aligned base
        if (threadIdx.x == 0 && n_items > 0)
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
    if ((int)threadIdx.x < n_items)
        items[threadIdx.x] = decode_item(batch, blockIdx.x + threadIdx.x * gridDim.x);
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
                // windows of one problem start their chunk walks at different
                // chunks, so that they do not read the same rows of B at once
                const int c = it.y + (i + it.x % it.z) % it.z;
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
        const int quarter = warp & 3;
        for (int k = 0; k < n_items; k++) {
            const int4 it = items[k];
            const TcJob &a = batch.job[it.w >> 16];
            const int n0 = (it.w & 0xffff) * NT;
            const int i = it.x * kWindowRows + quarter * 32 + lane;
            int out_row = -1;
            if (i < a.M && !((a.flags & TCA_FLAG_KEEP_EMPTY_ROWS) && a.p_row_ptr[i + 1] == a.p_row_ptr[i]))
                out_row = a.perm[i];
            const int b = k & 1;
            if constexpr (F8) {
                // the item's column scales, once, into shared memory (buffer b
                // was last read for item k - 2, which every epilogue thread
                // finished before the barrier of item k - 1)
                float *sc = reinterpret_cast<float *>(smem + Cfg::kScaleOff) + b * NT;
                for (int c = quarter * 32 + lane; c < NT; c += kEpiThreads)
                    sc[c] = n0 + c < a.N ? __ldg(a.col_scale + n0 + c) : 0.f;
            }
            uint32_t got = 0;
            if (lane == 0)
                got = mbar_wait(&acc_full[b], (k >> 1) & 1) ? 1u : 0u;
            got = __shfl_sync(0xffffffffu, got, 0);
            // the four warps agree, so that none is left at a later barrier
            if (!named_bar_and(kEpiBar, kEpiThreads, got != 0)) { ok = false; break; }
            tc_fence_after();
            OutT *Crow = out_row >= 0 ? reinterpret_cast<OutT *>(a.C) + (size_t)out_row * a.ldc : nullptr;
            float sa = 1.f;
            if constexpr (F8)
                sa = (i < a.M) ? a.row_scale[i] : 0.f;
            for (int cb = 0; cb < NT / 16; cb++) {
                const int n = n0 + cb * 16;
                if (n >= a.N)
                    break; // uniform across the warp
                uint32_t r[16];
                tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * NT + cb * 16), r);
                if constexpr (F8) { // dequantise: row scale x column scale (staged above; the barrier orders it)
                    float *f = reinterpret_cast<float *>(r);
                    const float *sb = reinterpret_cast<const float *>(smem + Cfg::kScaleOff) + b * NT + cb * 16;
#pragma unroll
                    for (int q = 0; q < 16; q++) f[q] *= sa * sb[q];
                }
                if (Crow) {
                    store8_out(Crow + n, reinterpret_cast<const float *>(r), a.alpha, a.beta);
                    if (n + 8 < a.N)
                        store8_out(Crow + n + 8, reinterpret_cast<const float *>(r) + 8, a.alpha, a.beta);
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

// ---------------------------------------------------------------------------
// Window pairs on CTA pairs (tcgen05 cta_group::2).
//
// A chunk of the kernel above holds 48 KB (A tile 16 KB, B tile 64 x 256 x 2)
// and its ring fits 4 stages; the chunk time is the ring's round trip (loads
// land ~2 us after issue whatever their size, measured) over those 4 stages.
// Two windows whose chunks have the same columns (direct windows that touch
// every 64-column block of K) share every B tile, so a cluster of two CTAs on
// two SMs runs them as one M = 256 product: each CTA loads its own window's A
// tile and HALF of the B tile (128 of the 256 columns of N), the first CTA's
// single MMA lane multiplies both (tcgen05.mma.cta_group::2 reads the
// operands from both CTAs' shared memory) and each CTA's tensor memory holds
// its own window's 128 x 256 accumulator. A stage is then 32 KB (E4M3:
// 16 KB), so 6 (E4M3: 12) fit. A window without a partner runs with an empty
// one (zero A tile, no stores).
//   Opt-in (tca_plan_opts_t.pair_windows): correct, but measured slower on the
// 32-problem sweep step (FP16 63 us against 50 us for spmm_tc_kernel, E4M3 59
// against 37 us). Traces show each CTA's chunks completing one per ~0.9 us
// (FP16) / ~0.65 us (E4M3) whatever the stage count (4 to 12) and however the
// partner's completions are waited for -- half the per-SM throughput of the
// single-window kernel -- so the halved B bytes per SM buy nothing, and 192
// pair items on 74 CTA pairs balance worse than 352 items on 148 CTAs.
//   Per CTA the roles are those of spmm_tc_kernel. Synchronisation between
// the two: the second CTA's warp 5 forwards each stage's completion ("full",
// its loads landed and scattered) to the first CTA's "peer_full"; the MMA
// lane releases the stage in both CTAs and announces finished accumulators
// to both epilogues with multicast commits; each epilogue reports its drained
// accumulator to the first CTA's "acc_empty" (count 2). Every wait is bounded
// as above; waits on phases the partner completes poll with test_wait. At
// exit each CTA waits (bounded) until its partner has made its last access to
// this CTA's shared memory. No load uses multicast.
constexpr int kPairN = 256;

template <bool F8> struct Tc2Cfg {
    static constexpr int kElem = F8 ? 1 : 2;
    static constexpr int kATileBytes = kWindowRows * kChunkCols * kElem;
    static constexpr int kHalfCols = kPairN / 2;             // columns of N whose B rows this CTA loads
    static constexpr int kBoxCols = 128 / kElem;             // N columns per 128-byte swizzle atom / TMA box
    static constexpr int kBoxes = kHalfCols / kBoxCols;      // 2 (FP16) or 1 (E4M3)
    static constexpr int kBTileBytes = kChunkCols * kHalfCols * kElem;
    static constexpr int kStage = kATileBytes + kBTileBytes; // 32 KB / 16 KB
    static constexpr int kStages = F8 ? 12 : 6;
    static constexpr int kStagingOff = kStages * kStage;
    static constexpr int kPendOff = kStagingOff + kStages * kStagingBytes;
    static constexpr int kPend2Off = kPendOff + kStages * 16;
    static constexpr int kItemOff = kPend2Off + kStages * 16; // int4 [kMaxCtaItems][2]
    static constexpr int kScaleOff = kItemOff + kMaxCtaItems * 32;
    static constexpr int kBarOff = kScaleOff + (F8 ? 2 * kPairN * 4 : 0);
    // full, empty, staged, peer_full [kStages]; acc_full, acc_empty [2]; drain; bye; 4 flags, TMEM slot
    static constexpr int kSmem = kBarOff + (4 * kStages + 6) * 8 + 24;
    static_assert(kSmem <= 227 * 1024, "shared memory budget");
    static_assert(kStage % 1024 == 0 && kATileBytes % 1024 == 0, "swizzled tiles need 1024-byte alignment");
    static_assert(kPendOff % 16 == 0 && kItemOff % 16 == 0 && kBarOff % 16 == 0, "16-byte aligned regions");
    static_assert(kStages % 2 == 0 && kLoaders <= kStages, "two scatter groups; loaders may not lap a stage");
};

// kind::f16 / kind::f8f6f4 instruction descriptor for M = 256 across the pair
// (FP32 D, A K-major, B N-major, N = 256); E4M3 uses format code 0 as FP16.
__host__ __device__ constexpr uint32_t idesc_pair()
{
    return (1u << 4) | (1u << 16) | ((uint32_t)(kPairN >> 3) << 17) | ((uint32_t)(256 >> 4) << 24);
}

__device__ __forceinline__ void umma_pair_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                              uint32_t accum)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
                 "l"(a), "l"(b), "r"(idesc), "r"(accum)
                 : "memory");
}
__device__ __forceinline__ void umma_pair_f8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                             uint32_t accum)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::2.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
                 "l"(a), "l"(b), "r"(idesc), "r"(accum)
                 : "memory");
}
// Arrive on the mbarrier at `bar`'s offset in both CTAs of the pair once every
// tcgen05.mma this thread issued has completed.
__device__ __forceinline__ void umma_commit_pair(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;"
                 ::"r"(smem_u32(bar)), "h"((uint16_t)3)
                 : "memory");
}

// Pair work item (job, pair, 256-wide N slice) -> this CTA's two table
// entries: {A chunk base (-1: empty partner), B chunk base, chunk count,
// job << 16 | slice} and {window of its rows (-1: none), rotation base, 0, 0}.
// Both CTAs walk the chunks of the first window's list, so that both load
// the same B rows for the same chunk.
__device__ __forceinline__ void decode_pair_item(const TcBatch &batch, int item, uint32_t rank, int4 *e0, int4 *e1)
{
    int j = 0;
    while (j + 1 < batch.n_jobs && batch.item_start[j + 1] <= item) j++;
    const TcJob &a = batch.job[j];
    const int local = item - batch.item_start[j];
    const int2 pr = a.pairs[local / a.ntiles];
    const int4 w0 = a.win_info[pr.x];
    const int mine = rank == 0 ? pr.x : pr.y;
    const int4 wm = mine >= 0 ? a.win_info[mine] : make_int4(-1, -1, 0, 0);
    *e0 = make_int4(wm.y, w0.y, w0.z, (j << 16) | (local % a.ntiles));
    *e1 = make_int4(wm.x, w0.x, 0, 0);
}

template <typename OutT, bool F8>
__global__ void __launch_bounds__(kThreads, 1) spmm_tc_pair_kernel(const __grid_constant__ TcBatch batch)
{
    using Cfg = Tc2Cfg<F8>;
    constexpr int S = Cfg::kStages;
    constexpr int kATileBytes = Cfg::kATileBytes;
    constexpr int kGathers = 16 * Cfg::kBoxes; // gather4 instructions per condensed chunk
    extern __shared__ __align__(1024) uint8_t smem[];
    int4 *pend = reinterpret_cast<int4 *>(smem + Cfg::kPendOff);
    int4 *pend2 = reinterpret_cast<int4 *>(smem + Cfg::kPend2Off);
    int4 *items = reinterpret_cast<int4 *>(smem + Cfg::kItemOff); // [k][2]
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + Cfg::kBarOff);
    uint64_t *empty = full + S;
    uint64_t *staged = empty + S;
    uint64_t *peer_full = staged + S;    // first CTA: the partner's stage s is full
    uint64_t *acc_full = peer_full + S;  // [2]
    uint64_t *acc_empty = acc_full + 2;  // [2], first CTA: both epilogues drained it
    uint64_t *drain = acc_empty + 2;     // every MMA of the pair has completed
    uint64_t *bye = drain + 1;           // the partner is done with this CTA's shared memory
    volatile int *flag = reinterpret_cast<volatile int *>(bye + 1);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bye + 1) + 4;
    constexpr int kGroupThreads = kScatterThreads / 2;

    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

    const uint32_t rank = cluster_rank();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pair_id = (int)blockIdx.x >> 1, n_pairs_grid = (int)gridDim.x >> 1;
    const int total = batch.item_start[batch.n_jobs];
    const int n_items =
        pair_id < total ? min(kMaxCtaItems, (total - 1 - pair_id) / n_pairs_grid + 1) : 0;
    // both CTAs are resident before either touches the other's shared memory
    cluster_sync_all();
    if (smem_u32(smem) & 1023u) { // the same in both CTAs: both leave here, before any shared state
        if (threadIdx.x == 0 && n_items > 0)
            atomicOr(batch.job[0].status, kStatusLayout);
        return;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], kGroupThreads);
            mbar_init(&empty[s], 1);
            mbar_init(&staged[s], 1);
            mbar_init(&peer_full[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 2);
        }
        mbar_init(drain, 1);
        mbar_init(bye, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if ((int)threadIdx.x < n_items)
        decode_pair_item(batch, pair_id + (int)threadIdx.x * n_pairs_grid, rank, &items[2 * threadIdx.x],
                         &items[2 * threadIdx.x + 1]);
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * kPairN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    cluster_sync_all(); // barriers initialised and tensor memory allocated in both CTAs
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;
    int total_chunks = 0;
    for (int k = 0; k < n_items; k++) total_chunks += items[2 * k].z;

    if (warp == kLoaderWarp || warp >= kLoaderWarp1) {
        // ---------------- loaders (as in spmm_tc_kernel; B: this CTA's half of N) ----------------
        const int ld = warp == kLoaderWarp ? 0 : warp - kLoaderWarp1 + 1;
        auto advance = [&](int &k, int &i) {
            while (k < n_items && i >= items[2 * k].z) { i -= items[2 * k].z; k++; }
        };
        struct Meta { int4 cols; int img, e0, e1; };
        auto fetch = [&](int k, int i, Meta &m) {
            m.cols = make_int4(-1, -1, -1, -1);
            m.img = -1;
            m.e0 = m.e1 = 0;
            if (k < n_items) {
                const int4 it = items[2 * k], it2 = items[2 * k + 1];
                const TcJob &a = batch.job[it.w >> 16];
                const int r = (i + it2.y % it.z) % it.z; // the same chunk order in both CTAs
                if (lane < 16)
                    m.cols = __ldg(reinterpret_cast<const int4 *>(a.win_cols + (size_t)(it.y + r) * kChunkCols) + lane);
                if (it.x >= 0) { // else an empty partner: a zero A tile
                    m.img = __ldg(a.img_idx + it.x + r);
                    m.e0 = __ldg(a.tile_ptr + it.x + r);
                    m.e1 = __ldg(a.tile_ptr + it.x + r + 1);
                }
            }
        };
        int k = 0, i = ld;
        advance(k, i);
        int g = ld;
        auto step = [&](Meta &cur, Meta &nxt) -> bool {
            if (g >= total_chunks || !ok)
                return false;
            int k2 = k, i2 = i + kLoaders;
            advance(k2, i2);
            fetch(k2, i2, nxt);
            const int s = g % S;
            uint32_t got = 1;
            if (lane == 0 && g >= S)
                got = mbar_poll_cluster(&empty[s], ((g / S) - 1) & 1) ? 1u : 0u;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) { ok = false; return false; }
            const int4 it = items[2 * k];
            const TcJob &a = batch.job[it.w >> 16];
            const int n0 = (it.w & 0xffff) * kPairN + (int)rank * Cfg::kHalfCols;
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
            __syncwarp();
            const int col0 = __shfl_sync(0xffffffffu, cur.cols.x, 0);
            const int col63 = __shfl_sync(0xffffffffu, cur.cols.w, 15);
            if (col0 >= 0 && col63 == col0 + kChunkCols - 1) {
                if (lane < Cfg::kBoxes)
                    tma_tile2d(b_s + lane * (kChunkCols * 128), &a.tmap_tile, n0 + lane * Cfg::kBoxCols, col0,
                               &full[s]);
            } else {
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
        // ---------------- scatter (as in spmm_tc_kernel, two groups) ----------------
        const int grp = warp >> 1;
        const int sid = (int)threadIdx.x - grp * kGroupThreads;
        int it = 0;
        for (int g = grp; g < total_chunks; g += 2, it++) {
            const int s = g % S;
            volatile int *fl = flag + grp * 2 + (it & 1);
            if (sid == 0)
                *fl = mbar_wait(&staged[s], (g / S) & 1) ? 1 : 0;
            named_bar_sync(1 + grp, kGroupThreads);
            if (*fl == 0) { ok = false; break; }
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
        if (lane == 0) {
            if (rank == 0) {
                // ---------------- MMA issuer for the pair ----------------
                constexpr uint32_t idesc = idesc_pair();
                const bool withhold = (batch.job[0].flags & TCA_FLAG_TEST_WITHHOLD_ACCUM) != 0;
                for (int g = 0; g < total_chunks; g++) {
                    const int s = g % S;
                    if (!mbar_wait(&full[s], (g / S) & 1) || !mbar_poll_cluster(&peer_full[s], (g / S) & 1)) {
                        ok = false;
                        break;
                    }
                    const int4 f = pend2[s];
                    const int b = f.y, k = f.z;
                    if ((f.x & 1) && k >= 2 && !mbar_poll_cluster(&acc_empty[b], ((k >> 1) - 1) & 1)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t a_s = smem_u32(smem + s * Cfg::kStage), b_s = a_s + kATileBytes;
                    const uint32_t d = tmem + (uint32_t)(b * kPairN);
                    if constexpr (F8) {
#pragma unroll
                        for (int kk = 0; kk < kChunkCols / 32; kk++) {
                            const uint64_t ad = smem_desc(a_s + kk * 32, 16, 512, 4);
                            const uint64_t bd = smem_desc(b_s + kk * 4096, kChunkCols * 128, 1024);
                            umma_pair_f8(d, ad, bd, idesc, ((f.x & 1) && kk == 0) ? 0u : 1u);
                        }
                    } else {
#pragma unroll
                        for (int kk = 0; kk < kChunkCols / 16; kk++) {
                            const uint64_t ad = smem_desc(a_s + kk * 32, 16, 1024);
                            const uint64_t bd = smem_desc(b_s + kk * 2048, kChunkCols * 128, 1024);
                            umma_pair_f16(d, ad, bd, idesc, ((f.x & 1) && kk == 0) ? 0u : 1u);
                        }
                    }
                    umma_commit_pair(&empty[s]);
                    if ((f.x & 2) && !(withhold && k == n_items - 1))
                        umma_commit_pair(&acc_full[b]);
                }
                umma_commit_pair(drain);
            } else {
                // ---------------- relay: this CTA's stages to the first CTA ----------------
                for (int g = 0; g < total_chunks; g++) {
                    const int s = g % S;
                    if (!mbar_wait(&full[s], (g / S) & 1)) { ok = false; break; }
                    mbar_arrive_cluster(cluster_map(smem_u32(&peer_full[s]), 0u));
                }
            }
            // every MMA of the pair has completed (both CTAs' tensor memory and
            // shared memory are no longer read or written by it)
            if (!mbar_poll_cluster(drain, 0))
                ok = false;
        }
        __syncwarp();
    } else {
        // ---------------- epilogue: this CTA's window, all 256 columns ----------------
        const int quarter = warp & 3;
        for (int k = 0; k < n_items; k++) {
            const int4 it = items[2 * k], it2 = items[2 * k + 1];
            const TcJob &a = batch.job[it.w >> 16];
            const int n0 = (it.w & 0xffff) * kPairN;
            const int i = it2.x * kWindowRows + quarter * 32 + lane;
            int out_row = -1;
            if (it2.x >= 0 && i < a.M && !((a.flags & TCA_FLAG_KEEP_EMPTY_ROWS) && a.p_row_ptr[i + 1] == a.p_row_ptr[i]))
                out_row = a.perm[i];
            const int b = k & 1;
            if constexpr (F8) {
                float *sc = reinterpret_cast<float *>(smem + Cfg::kScaleOff) + b * kPairN;
                for (int c = quarter * 32 + lane; c < kPairN; c += kEpiThreads)
                    sc[c] = n0 + c < a.N ? __ldg(a.col_scale + n0 + c) : 0.f;
            }
            uint32_t got = 0;
            if (lane == 0)
                got = mbar_poll_cluster(&acc_full[b], (k >> 1) & 1) ? 1u : 0u;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!named_bar_and(kEpiBar, kEpiThreads, got != 0)) { ok = false; break; }
            tc_fence_after();
            OutT *Crow = out_row >= 0 ? reinterpret_cast<OutT *>(a.C) + (size_t)out_row * a.ldc : nullptr;
            float sa = 1.f;
            if constexpr (F8)
                sa = (it2.x >= 0 && i < a.M) ? a.row_scale[i] : 0.f;
            for (int cb = 0; it2.x >= 0 && cb < kPairN / 16; cb++) {
                const int n = n0 + cb * 16;
                if (n >= a.N)
                    break;
                uint32_t r[16];
                tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * kPairN + cb * 16), r);
                if constexpr (F8) {
                    float *f = reinterpret_cast<float *>(r);
                    const float *sb = reinterpret_cast<const float *>(smem + Cfg::kScaleOff) + b * kPairN + cb * 16;
#pragma unroll
                    for (int q = 0; q < 16; q++) f[q] *= sa * sb[q];
                }
                if (Crow) {
                    store8_out(Crow + n, reinterpret_cast<const float *>(r), a.alpha, a.beta);
                    if (n + 8 < a.N)
                        store8_out(Crow + n + 8, reinterpret_cast<const float *>(r) + 8, a.alpha, a.beta);
                }
            }
            tc_fence_before();
            named_bar_sync(kEpiBar, kEpiThreads); // the four warps are done with buffer b
            if (warp == kEpiWarp0 && lane == 0) {
                if (rank == 0)
                    mbar_arrive(&acc_empty[b]);
                else
                    mbar_arrive_cluster(cluster_map(smem_u32(&acc_empty[b]), 0u));
            }
        }
    }

    tc_fence_before();
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) {
            if (n_items > 0)
                atomicOr(batch.job[items[0].w >> 16].status, kStatusTimeout);
            const uint64_t t0 = global_ns();
            while (global_ns() - t0 < 1000000ull) {
            }
        }
        __syncthreads();
    }
    // The partner makes no further access to this CTA's shared memory once
    // it has arrived here (its roles are done, the MMAs it issued completed);
    // the wait is bounded like every other.
    if (threadIdx.x == 0) {
        mbar_arrive_cluster(cluster_map(smem_u32(bye), rank ^ 1u));
        if (!mbar_poll_cluster(bye, 0) && n_items > 0)
            atomicOr(batch.job[items[0].w >> 16].status, kStatusTimeout);
    }
    __syncthreads();
    if (warp == kMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kPairN) : "memory");
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
    j.pairs = p->tc_pairs;
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
    j.alpha = alpha;
    j.beta = beta;
    j.flags = flags;
    return TCA_OK;
}

template <int NT, typename OutT, bool F8, int CAP>
int launch_group_cap(const TcBatchT<CAP> &b, cudaStream_t s)
{
    const int smem = TcCfg<NT, F8>::kSmem;
    TCA_CUDA_TRY(cudaFuncSetAttribute(spmm_tc_kernel<NT, OutT, F8, CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem));
    // The whole 228 KB carveout: with the smallest one that holds this block
    // (196 KB for the E4M3 rings) no room is left for the 1 KB that each
    // CUDA-core block reserves, and the launch that should run beside this
    // one waits for it to end (measured: E4M3 step, CUDA-core blocks starting
    // as the first tensor-core blocks exit).
    TCA_CUDA_TRY(cudaFuncSetAttribute(spmm_tc_kernel<NT, OutT, F8, CAP>,
                                      cudaFuncAttributePreferredSharedMemoryCarveout,
                                      (int)cudaSharedmemCarveoutMaxShared));
    const int total = b.item_start[b.n_jobs];
    const int grid = std::min(total, std::max(kSMs, (total + kMaxCtaItems - 1) / kMaxCtaItems));
    spmm_tc_kernel<NT, OutT, F8, CAP><<<grid, kThreads, smem, s>>>(b);
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

template <int NT, typename OutT, bool F8>
int launch_group(const TcBatch &b, cudaStream_t s)
{
    if (b.n_jobs == 1) {
        TcBatchT<1> one;
        one.n_jobs = 1;
        one.item_start[0] = b.item_start[0];
        one.item_start[1] = b.item_start[1];
        one.job[0] = b.job[0];
        return launch_group_cap<NT, OutT, F8, 1>(one, s);
    }
    return launch_group_cap<NT, OutT, F8, kMaxJobs>(b, s);
}

template <typename OutT>
int launch_group_out(const TcBatch &b, int NT, bool f8, cudaStream_t s)
{
    if (f8)
        return NT == 128 ? launch_group<128, OutT, true>(b, s) : launch_group<256, OutT, true>(b, s);
    switch (NT) {
    case 64: return launch_group<64, OutT, false>(b, s);
    case 128: return launch_group<128, OutT, false>(b, s);
    default: return launch_group<256, OutT, false>(b, s);
    }
}

// Pair kernel: clusters of two CTAs (one per SM), persistent over the pair
// items, as many clusters as fit at once (or more when an item list would
// exceed kMaxCtaItems per cluster).
template <typename OutT, bool F8>
int launch_pair_group(const TcBatch &b, cudaStream_t s)
{
    const int smem = Tc2Cfg<F8>::kSmem;
    auto kernel = spmm_tc_pair_kernel<OutT, F8>;
    TCA_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    TCA_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      (int)cudaSharedmemCarveoutMaxShared));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    static int max_clusters = 0;
    if (max_clusters == 0) {
        cfg.gridDim = dim3(2 * (kSMs / 2));
        int n = 0;
        TCA_CUDA_TRY(cudaOccupancyMaxActiveClusters(&n, kernel, &cfg));
        if (n <= 0)
            return set_error(TCA_ERR_CUDA, "no CTA pair of the tensor-core pair kernel fits on this device");
        max_clusters = n;
    }
    const int total = b.item_start[b.n_jobs];
    const int clusters = std::min(total, std::max(max_clusters, (total + kMaxCtaItems - 1) / kMaxCtaItems));
    cfg.gridDim = dim3((unsigned)(2 * clusters));
    TCA_CUDA_TRY(cudaLaunchKernelEx(&cfg, kernel, b));
    return TCA_OK;
}

int launch_pair_typed(const TcBatch &b, bool f8, int c_dtype, cudaStream_t s)
{
    if (b.n_jobs == 0 || b.item_start[b.n_jobs] == 0)
        return TCA_OK;
    if (c_dtype == TCA_DTYPE_F16)
        return f8 ? launch_pair_group<__half, true>(b, s) : launch_pair_group<__half, false>(b, s);
    return f8 ? launch_pair_group<float, true>(b, s) : launch_pair_group<float, false>(b, s);
}

int launch_group_typed(const TcBatch &b, int NT, bool f8, int c_dtype, cudaStream_t s)
{
    if (b.n_jobs == 0 || b.item_start[b.n_jobs] == 0)
        return TCA_OK;
    return c_dtype == TCA_DTYPE_F16 ? launch_group_out<__half>(b, NT, f8, s) : launch_group_out<float>(b, NT, f8, s);
}

} // namespace

int pick_tc_tile(const tca_plan *p, int N, bool batched, bool f8)
{
    const int n_tc = p->n_tc;
    const int lo = f8 ? 128 : 64; // E4M3 B tiles are whole 128-byte swizzle atoms
    int NT = N <= 64 ? 64 : N <= 128 ? 128 : 256;
    NT = std::max(NT, lo);
    // a single forward halves the slice while that leaves fewer than about
    // three quarters of the SMs with an item (measured: A^T of 512 x 2048,
    // N = 4096, 4 windows: NT = 128, 128 items, 30.5 us; NT = 64, 40.4 us)
    if (!batched)
        while (NT > lo && (long long)n_tc * ((N + NT - 1) / NT) < (3 * kSMs) / 4)
            NT /= 2;
    return NT;
}

int tc_block_regs(bool f8, int *regs)
{
    static int worst[2] = {0, 0};
    if (worst[f8] == 0) {
        const void *f16_fns[] = {
            (const void *)spmm_tc_kernel<64, __half, false>, (const void *)spmm_tc_kernel<128, __half, false>,
            (const void *)spmm_tc_kernel<256, __half, false>, (const void *)spmm_tc_kernel<64, float, false>,
            (const void *)spmm_tc_kernel<128, float, false>, (const void *)spmm_tc_kernel<256, float, false>,
            (const void *)spmm_tc_pair_kernel<__half, false>, (const void *)spmm_tc_pair_kernel<float, false>,
            (const void *)spmm_tc_kernel<64, __half, false, 1>, (const void *)spmm_tc_kernel<128, __half, false, 1>,
            (const void *)spmm_tc_kernel<256, __half, false, 1>, (const void *)spmm_tc_kernel<64, float, false, 1>,
            (const void *)spmm_tc_kernel<128, float, false, 1>, (const void *)spmm_tc_kernel<256, float, false, 1>};
        const void *f8_fns[] = {
            (const void *)spmm_tc_kernel<128, __half, true>, (const void *)spmm_tc_kernel<256, __half, true>,
            (const void *)spmm_tc_kernel<128, float, true>, (const void *)spmm_tc_kernel<256, float, true>,
            (const void *)spmm_tc_pair_kernel<__half, true>, (const void *)spmm_tc_pair_kernel<float, true>,
            (const void *)spmm_tc_kernel<128, __half, true, 1>, (const void *)spmm_tc_kernel<256, __half, true, 1>,
            (const void *)spmm_tc_kernel<128, float, true, 1>, (const void *)spmm_tc_kernel<256, float, true, 1>};
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

// A window alone on a CTA pair keeps two SMs for one window's chunks, so the
// pair kernel takes a plan when at least two thirds of its tensor-core
// windows are paired.
bool pair_eligible(const tca_plan *p, int NT)
{
    return NT == kPairN && p->opts.pair_windows != 0 && p->tc_pairs != nullptr && 3 * p->n_full_pairs >= p->n_tc;
}

int launch_tc_jobs(const SpmmJob *jobs, int n_jobs, int c_dtype, float alpha, float beta, unsigned flags,
                   cudaStream_t s, LaunchList *defer)
{
    // widths of the single-window kernel, then (0) the pair kernel for N-slices of 256
    const int widths[4] = {64, 128, 256, 0};
    auto emit = [&](const TcBatch &b, int NT, bool f8) -> int {
        if (b.n_jobs == 0 || b.item_start[b.n_jobs] == 0)
            return TCA_OK;
        auto run = [NT, f8, c_dtype](const TcBatch &bb, cudaStream_t st) {
            return NT == 0 ? launch_pair_typed(bb, f8, c_dtype, st) : launch_group_typed(bb, NT, f8, c_dtype, st);
        };
        if (!defer)
            return run(b, s);
        auto held = std::make_shared<TcBatch>(b);
        defer->push_back([held, run](cudaStream_t st) { return run(*held, st); });
        return TCA_OK;
    };
    for (bool f8 : {false, true}) {
        for (int NT : widths) {
            TcBatch b;
            b.n_jobs = 0;
            b.item_start[0] = 0;
            for (int i = 0; i < n_jobs; i++) {
                const SpmmJob &sj = jobs[i];
                if (!sj.tc || sj.f8 != f8 || sj.p->n_tc == 0 || sj.N <= 0)
                    continue;
                const bool pair = pair_eligible(sj.p, sj.n_tile);
                if (NT == 0 ? !pair : (pair || sj.n_tile != NT))
                    continue;
                TCA_TRY(make_job(sj, alpha, beta, flags, NT == 0 ? kPairN : NT, &b.job[b.n_jobs]));
                const int units = NT == 0 ? sj.p->n_pairs : sj.p->n_tc;
                b.item_start[b.n_jobs + 1] = b.item_start[b.n_jobs] + units * b.job[b.n_jobs].ntiles;
                b.n_jobs++;
                if (b.n_jobs == kMaxJobs) {
                    TCA_TRY(emit(b, NT, f8));
                    b.n_jobs = 0;
                }
            }
            TCA_TRY(emit(b, NT, f8));
        }
    }
    return TCA_OK;
}

} // namespace tca
