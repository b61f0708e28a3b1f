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
// One CTA = one (job, window, NT-wide slice of N) work item, a ring of
// kStages (A tile, B tile, entry staging) stages and three decoupled roles:
//   * one loader warp moves every byte through the TMA engine: the 64 B rows
//     of the chunk's condensed columns by tile::gather4 (4 rows x 128 bytes
//     per instruction into a 128-byte swizzled N-major tile; padding columns
//     and n >= N are out of the tensor and arrive as zeros), and either the
//     chunk's pre-rendered, pre-swizzled dense A tile (chunks with >= 2048
//     nonzeros: one 16 KB cp.async.bulk) or its packed entries (cp.async.bulk
//     into the stage's staging buffer);
//   * scatter warps, once a stage's entries landed, zero its A tile and
//     scatter them into the 128-byte swizzled K-major layout;
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
#include <mutex>
#include "tca_internal.cuh"
#include "plan.cuh"

namespace tca {
namespace {

constexpr int kScatterThreads = 128; // warps 0-3: sparse-entry scatter
constexpr int kLoaderWarp = 4;       // TMA issue
constexpr int kMmaWarp = 5;          // TMEM allocation, tcgen05.mma issue
constexpr int kEpiThreads = 128;     // warps 6-9: epilogue
constexpr int kThreads = 320;
constexpr int kMetaRing = 8;          // chunk-metadata prefetch ring (prefetch distance kMetaRing - 1)
constexpr int kMetaSlotInts = 68;     // 64 columns, image index, first and end entry, pad
constexpr int kMaxCtaItems = 32;      // work items per persistent CTA
constexpr int kATileBytes = kWindowRows * kChunkCols * 2;     // 16 KB
constexpr int kStagingBytes = ((kImageMinNnz + 3) * 4 + 15) & ~15; // entries of a sparse chunk, 16-byte rounded
constexpr int kMaxJobs = 32;                                  // jobs per launch (kernel parameter space)

struct TcJob {
    CUtensorMap tmap_b;    // B as a 2-D tensor {N, K}, box {64, 1}, 128-byte swizzle (gather4 source)
    CUtensorMap tmap_tile; // the same tensor, box {64, 64}: 64 contiguous rows of B per instruction
    const int4 *win_info; // per tensor-core window: window, first chunk, chunk count
    const int *tile_ptr, *win_cols, *img_idx, *perm, *p_row_ptr;
    const uint32_t *entries;
    const uint16_t *images;
    const __half *B;
    void *C;
    int *status;
    int M, N, ldb, ldc, ntiles;
    float alpha, beta;
    unsigned flags;
};

struct TcBatch {
    int n_jobs;
    int item_start[kMaxJobs + 1];
    TcJob job[kMaxJobs];
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for the phase of `parity`: false after about one second.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(bar, parity))
            return true;
        if ((it & 255u) == 0u && global_ns() - t0 > 1000000000ull)
            return false;
    }
}

__device__ __forceinline__ void named_bar_sync(int id, int n)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// mbarrier arrive (count 1) that also adds `bytes` to the transaction count.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// TMA gather of 4 rows (y0..y3) x one 64-element box starting at column x of a
// 2-D tensor into shared memory, completing on `bar`. Rows or columns outside
// the tensor are zero-filled.
__device__ __forceinline__ void tma_gather4(uint32_t dst, const CUtensorMap *map, int x, int y0, int y1, int y2,
                                            int y3, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y0), "r"(y1), "r"(y2), "r"(y3)
                 : "memory");
}

// TMA load of a {64 columns x 64 rows} box of a 2-D tensor at (x, y) into
// shared memory, completing on `bar`; out-of-range elements are zero-filled.
__device__ __forceinline__ void tma_tile2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, 128-byte swizzle (layout type 2), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (2ull << 61);
}

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
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t *r)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                   "=r"(r[14]), "=r"(r[15])
                 : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
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
// kStages entry staging buffers, per-stage chunk records, the chunk-metadata
// ring, the CTA's item table, mbarriers and two broadcast flags + TMEM slot.
template <int NT> struct TcCfg {
    static constexpr int kStages = NT == 256 ? 4 : NT == 128 ? 5 : 6;
    static constexpr int kBTileBytes = kChunkCols * NT * 2;
    static constexpr int kStage = kATileBytes + kBTileBytes;
    static constexpr int kStagingOff = kStages * kStage;
    static constexpr int kPendOff = kStagingOff + kStages * kStagingBytes; // int4 [kStages]: img, e0, e0a, e1
    static constexpr int kPend2Off = kPendOff + kStages * 16;              // int4 [kStages]: flags, buffer, item
    static constexpr int kMetaOff = kPend2Off + kStages * 16;              // int [kMetaRing][kMetaSlotInts]
    static constexpr int kItemOff = kMetaOff + kMetaRing * kMetaSlotInts * 4; // int4 [kMaxCtaItems]
    static constexpr int kBarOff = kItemOff + kMaxCtaItems * 16;
    // full, empty, staged [kStages]; accum_full, accum_empty [2]
    static constexpr int kSmem = kBarOff + (3 * kStages + 4) * 8 + 16;
    static_assert(kSmem <= 227 * 1024, "shared memory budget");
    static_assert(kStage % 1024 == 0 && kATileBytes % 1024 == 0, "swizzled tiles need 1024-byte alignment");
    static_assert(kStagingOff % 16 == 0 && kStagingBytes % 16 == 0 && kPendOff % 16 == 0, "16-byte alignment");
    static_assert(kMetaOff % 16 == 0 && kItemOff % 16 == 0 && kBarOff % 16 == 0, "16-byte aligned regions");
};

__device__ __forceinline__ void cp_async4(uint32_t dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

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
// ... (at most kMaxCtaItems), as one continuous stream of chunks through the
// stage ring. Warp roles (320 threads):
//   warp 4 (loader): per chunk, acquire the stage ("empty"), write the
//     chunk's records (entries range and image for the scatter warps; first /
//     last chunk of its item and accumulator buffer for the MMA lane), set the
//     "full" transaction count and issue the dense A image (16 KB
//     cp.async.bulk) or the sparse entries (cp.async.bulk into staging,
//     completing on "staged"), then the B rows: tiled TMA boxes of 64
//     contiguous rows for direct chunks, tile::gather4 for condensed ones.
//     Chunk metadata is prefetched kMetaRing - 1 chunks ahead with cp.async.
//     After the last chunk it passes an end record through the ring.
//   warps 0-3 (scatter): per chunk, wait "staged"; for a sparse chunk zero the
//     A tile, scatter the staged entries, fence.proxy.async; arrive "full".
//   warp 5, lane 0 (MMA): per chunk wait "full"; on an item's first chunk
//     wait until its TMEM accumulator buffer (item parity) is drained
//     ("accum_empty"); 4 x tcgen05.mma; commit "empty"; on the item's last
//     chunk commit "accum_full".
//   warps 6-9 (epilogue): per item wait "accum_full", tcgen05.ld the rows
//     (warp w reads TMEM lanes 32 (w % 4) ..), alpha/beta, store to C[perm],
//     arrive "accum_empty" -- overlapping the next item's main loop.
template <int NT, typename OutT>
__global__ void __launch_bounds__(kThreads, 1) spmm_tc_kernel(const __grid_constant__ TcBatch batch)
{
    using Cfg = TcCfg<NT>;
    constexpr int S = Cfg::kStages;
    constexpr int kBoxes = NT / 64;       // 64-column boxes per B row slice
    constexpr int kGathers = 16 * kBoxes; // gather4 instructions per condensed chunk
    constexpr int P = kMetaRing - 1;      // metadata prefetch distance
    extern __shared__ __align__(1024) uint8_t smem[];
    int4 *pend = reinterpret_cast<int4 *>(smem + Cfg::kPendOff);
    int4 *pend2 = reinterpret_cast<int4 *>(smem + Cfg::kPend2Off);
    int *meta = reinterpret_cast<int *>(smem + Cfg::kMetaOff);
    int4 *items = reinterpret_cast<int4 *>(smem + Cfg::kItemOff);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + Cfg::kBarOff);
    uint64_t *empty = full + S;
    uint64_t *staged = empty + S;
    uint64_t *acc_full = staged + S;  // [2]
    uint64_t *acc_empty = acc_full + 2; // [2]
    volatile int *flag = reinterpret_cast<volatile int *>(acc_empty + 2); // 2 slots, alternating by chunk
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(acc_empty + 2) + 2;

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
            mbar_init(&full[s], kScatterThreads);
            mbar_init(&empty[s], 1);
            mbar_init(&staged[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kEpiThreads);
        }
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

    if (warp == kLoaderWarp) {
        // ---------------- loader ----------------
        // prefetch cursor: (item k, chunk i) of the next chunk whose metadata to fetch
        int pk = 0, pi = 0;
        auto prefetch = [&](int slot) {
            if (pk < n_items) {
                const int4 it = items[pk];
                const TcJob &a = batch.job[it.w >> 16];
                const int c = it.y + pi;
                const uint32_t dst = smem_u32(meta + slot * kMetaSlotInts);
                if (lane < 16)
                    cp_async16(dst + lane * 16, a.win_cols + (size_t)c * kChunkCols + lane * 4);
                else if (lane == 16)
                    cp_async4(dst + 64 * 4, a.img_idx + c);
                else if (lane == 17)
                    cp_async4(dst + 65 * 4, a.tile_ptr + c);
                else if (lane == 18)
                    cp_async4(dst + 66 * 4, a.tile_ptr + c + 1);
                if (++pi == it.z) { pi = 0; pk++; }
            }
            cp_async_commit();
        };
        for (int q = 0; q < P; q++) prefetch(q);
        int g = 0;
        for (int k = 0; k < n_items && ok; k++) {
            const int4 it = items[k];
            const TcJob &a = batch.job[it.w >> 16];
            const int n0 = (it.w & 0xffff) * NT;
            for (int i = 0; i < it.z; i++, g++) {
                const int s = g % S;
                uint32_t got = 1;
                if (lane == 0 && g >= S)
                    got = mbar_wait(&empty[s], ((g / S) - 1) & 1) ? 1u : 0u;
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) { ok = false; break; }
                cp_async_wait<P - 1>(); // this chunk's metadata has landed (this lane's share)
                __syncwarp();           // ... and every lane's
                const int *m = meta + (g % kMetaRing) * kMetaSlotInts;
                const int img = m[64];
                const uint32_t a_s = smem_u32(smem + s * Cfg::kStage), b_s = a_s + kATileBytes;
                if (lane == 0) {
                    const int e0 = m[65], e1 = m[66], e0a = e0 & ~3;
                    pend[s] = make_int4(img, e0, e0a, e1);
                    pend2[s] = make_int4((i == 0 ? 1 : 0) | (i == it.z - 1 ? 2 : 0), k & 1, k, 0);
                    mbar_expect_tx(&full[s], Cfg::kBTileBytes + (img >= 0 ? kATileBytes : 0));
                    if (img >= 0) {
                        bulk_copy_g2s(a_s, a.images + (size_t)img * (kATileBytes / 2), kATileBytes, &full[s]);
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
                if (m[0] >= 0 && m[kChunkCols - 1] == m[0] + kChunkCols - 1) {
                    // 64 contiguous B rows (direct chunks): one 8 KB tiled box per 64 columns
                    if (lane < kBoxes)
                        tma_tile2d(b_s + lane * (kChunkCols * 128), &a.tmap_tile, n0 + lane * 64, m[0], &full[s]);
                } else {
                    for (int q = lane; q < kGathers; q += 32) {
                        const int gg = q & 15, box = q >> 4;
                        tma_gather4(b_s + box * (kChunkCols * 128) + gg * 512, &a.tmap_b, n0 + box * 64, m[4 * gg],
                                    m[4 * gg + 1], m[4 * gg + 2], m[4 * gg + 3], &full[s]);
                    }
                }
                __syncwarp(); // every lane has read slot g before it is refilled
                prefetch((g + P) % kMetaRing);
            }
        }
        // end record: scatter warps and the MMA lane stop at it
        if (ok) {
            const int s = g % S;
            uint32_t got = 1;
            if (lane == 0 && g >= S)
                got = mbar_wait(&empty[s], ((g / S) - 1) & 1) ? 1u : 0u;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (got && lane == 0) {
                pend[s] = make_int4(-2, 0, 0, 0);
                mbar_arrive(&staged[s]);
            }
            if (!got) ok = false;
        }
        cp_async_wait<0>();
    } else if (warp < 4) {
        // ---------------- scatter ----------------
        const int sid = threadIdx.x;
        for (int g = 0;; g++) {
            const int s = g % S;
            if (sid == 0)
                flag[g & 1] = mbar_wait(&staged[s], (g / S) & 1) ? 1 : 0;
            named_bar_sync(1, kScatterThreads); // also orders the staged data for every scatter thread
            if (flag[g & 1] == 0) { ok = false; break; } // uniform across the scatter warps
            const int4 pd = pend[s];
            if (pd.x >= -1 && pd.x < 0) {
                uint8_t *At = smem + s * Cfg::kStage;
#pragma unroll
                for (int k = 0; k < kATileBytes / (16 * kScatterThreads); k++)
                    reinterpret_cast<uint4 *>(At)[sid + k * kScatterThreads] = make_uint4(0, 0, 0, 0);
                named_bar_sync(1, kScatterThreads);
                const uint32_t *st = reinterpret_cast<const uint32_t *>(smem + Cfg::kStagingOff + s * kStagingBytes);
                for (int e = pd.y + sid; e < pd.w; e += kScatterThreads) {
                    const uint32_t v = st[e - pd.z];
                    *reinterpret_cast<uint16_t *>(At + swz128_offset(v >> 22, (v >> 16) & 63u)) =
                        (uint16_t)(v & 0xffffu);
                }
                fence_proxy_async();
            }
            mbar_arrive(&full[s]);
            if (pd.x == -2)
                break; // end record
        }
    } else if (warp == kMmaWarp) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_f16(NT);
            for (int g = 0;; g++) {
                const int s = g % S;
                if (!mbar_wait(&full[s], (g / S) & 1)) { ok = false; break; }
                const int4 pd = pend[s];
                if (pd.x == -2)
                    break; // end record
                const int4 f = pend2[s];
                const int b = f.y, k = f.z;
                if ((f.x & 1) && k >= 2 && !mbar_wait(&acc_empty[b], ((k >> 1) - 1) & 1)) { ok = false; break; }
                tc_fence_after();
                const uint32_t a_s = smem_u32(smem + s * Cfg::kStage), b_s = a_s + kATileBytes;
                const uint32_t d = tmem + (uint32_t)(b * NT);
#pragma unroll
                for (int kk = 0; kk < kChunkCols / 16; kk++) {
                    const uint64_t ad = smem_desc(a_s + kk * 32, 16, 1024);
                    const uint64_t bd = smem_desc(b_s + kk * 2048, kChunkCols * 128, 1024);
                    umma_f16(d, ad, bd, idesc, ((f.x & 1) && kk == 0) ? 0u : 1u);
                }
                umma_commit(&empty[s]);
                if (f.x & 2)
                    umma_commit(&acc_full[b]);
            }
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
            uint32_t got = 0;
            if (lane == 0)
                got = mbar_wait(&acc_full[b], (k >> 1) & 1) ? 1u : 0u;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) { ok = false; break; }
            tc_fence_after();
            OutT *Crow = out_row >= 0 ? reinterpret_cast<OutT *>(a.C) + (size_t)out_row * a.ldc : nullptr;
            for (int cb = 0; cb < NT / 16; cb++) {
                const int n = n0 + cb * 16;
                if (n >= a.N)
                    break; // uniform across the warp
                uint32_t r[16];
                tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * NT + cb * 16), r);
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

    if (!ok && n_items > 0)
        atomicOr(batch.job[items[0].w >> 16].status, kStatusTimeout);
    tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * NT) : "memory");
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

// B (K x N, row-major, leading dimension ldb) as a TMA source: dims {N, K},
// row stride ldb * 2 bytes, box {64, rows}, 128-byte swizzle, zero fill.
int encode_b_map(const SpmmJob &sj, int K, int rows, CUtensorMap *map)
{
    auto enc = tensor_map_encoder();
    if (!enc)
        return set_error(TCA_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[2] = {(cuuint64_t)sj.N, (cuuint64_t)(K > 0 ? K : 1)};
    const cuuint64_t strides[1] = {(cuuint64_t)sj.ldb * 2};
    const cuuint32_t box[2] = {64, (cuuint32_t)rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<__half *>(sj.B), dims, strides, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return set_error(TCA_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) for B (N=%d, ldb=%d)", (int)r, sj.N, sj.ldb);
    return TCA_OK;
}

int make_job(const SpmmJob &sj, float alpha, float beta, unsigned flags, int NT, TcJob *out)
{
    const tca_plan *p = sj.p;
    TcJob &j = *out;
    TCA_TRY(encode_b_map(sj, p->K, 1, &j.tmap_b));
    TCA_TRY(encode_b_map(sj, p->K, kChunkCols, &j.tmap_tile));
    j.win_info = p->tc_win_info;
    j.tile_ptr = p->tile_ptr;
    j.win_cols = p->win_cols;
    j.img_idx = p->img_idx;
    j.perm = p->perm;
    j.p_row_ptr = p->p_row_ptr;
    j.entries = p->tile_entries;
    j.images = p->images;
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

template <int NT, typename OutT>
int launch_group(const TcBatch &b, cudaStream_t s)
{
    const int smem = TcCfg<NT>::kSmem;
    TCA_CUDA_TRY(cudaFuncSetAttribute(spmm_tc_kernel<NT, OutT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int total = b.item_start[b.n_jobs];
    const int grid = std::min(total, std::max(kSMs, (total + kMaxCtaItems - 1) / kMaxCtaItems));
    spmm_tc_kernel<NT, OutT><<<grid, kThreads, smem, s>>>(b);
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

int launch_group_typed(const TcBatch &b, int NT, int c_dtype, cudaStream_t s)
{
    if (b.n_jobs == 0 || b.item_start[b.n_jobs] == 0)
        return TCA_OK;
    if (c_dtype == TCA_DTYPE_F16) {
        switch (NT) {
        case 64: return launch_group<64, __half>(b, s);
        case 128: return launch_group<128, __half>(b, s);
        default: return launch_group<256, __half>(b, s);
        }
    }
    switch (NT) {
    case 64: return launch_group<64, float>(b, s);
    case 128: return launch_group<128, float>(b, s);
    default: return launch_group<256, float>(b, s);
    }
}

} // namespace

int pick_tc_tile(int n_tc, int N, bool batched)
{
    int NT = N <= 64 ? 64 : N <= 128 ? 128 : 256;
    if (!batched)
        while (NT > 64 && (long long)n_tc * ((N + NT - 1) / NT) < kSMs)
            NT /= 2;
    return NT;
}

int launch_tc_jobs(const SpmmJob *jobs, int n_jobs, int c_dtype, float alpha, float beta, unsigned flags,
                   cudaStream_t s)
{
    const int widths[3] = {64, 128, 256};
    for (int NT : widths) {
        TcBatch b;
        b.n_jobs = 0;
        b.item_start[0] = 0;
        for (int i = 0; i < n_jobs; i++) {
            const SpmmJob &sj = jobs[i];
            if (!sj.tc || sj.n_tile != NT || sj.p->n_tc == 0 || sj.N <= 0)
                continue;
            TCA_TRY(make_job(sj, alpha, beta, flags, NT, &b.job[b.n_jobs]));
            b.item_start[b.n_jobs + 1] = b.item_start[b.n_jobs] + sj.p->n_tc * b.job[b.n_jobs].ntiles;
            b.n_jobs++;
            if (b.n_jobs == kMaxJobs) {
                TCA_TRY(launch_group_typed(b, NT, c_dtype, s));
                b.n_jobs = 0;
            }
        }
        TCA_TRY(launch_group_typed(b, NT, c_dtype, s));
    }
    return TCA_OK;
}

} // namespace tca
