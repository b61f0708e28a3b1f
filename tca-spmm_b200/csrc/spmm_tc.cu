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
#include <mutex>
#include "tca_internal.cuh"
#include "plan.cuh"

namespace tca {
namespace {

constexpr int kScatterThreads = 128; // warps 0-3: scatter, then epilogue
constexpr int kLoaderWarp = 4;       // TMA issue
constexpr int kMmaWarp = 5;          // TMEM allocation, tcgen05.mma issue
constexpr int kThreads = 192;
constexpr int kATileBytes = kWindowRows * kChunkCols * 2;     // 16 KB
constexpr int kStagingBytes = ((kImageMinNnz + 3) * 4 + 15) & ~15; // entries of a sparse chunk, 16-byte rounded
constexpr int kMetaChunks = 8;                                // chunk metadata cached in shared memory
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
// kStages entry staging buffers, per-stage pending-chunk records, the loader's
// chunk metadata cache, mbarriers (full, empty, staged per stage; accumulator
// ready), two broadcast flags and the TMEM address slot.
template <int NT> struct TcCfg {
    static constexpr int kStages = NT == 256 ? 4 : NT == 128 ? 5 : 7;
    static constexpr int kBTileBytes = kChunkCols * NT * 2;
    static constexpr int kStage = kATileBytes + kBTileBytes;
    static constexpr int kStagingOff = kStages * kStage;
    static constexpr int kPendOff = kStagingOff + kStages * kStagingBytes;
    static constexpr int kMetaOff = kPendOff + kStages * 16;
    static constexpr int kMetaBytes = (kMetaChunks * kChunkCols + 2 * kMetaChunks + 1) * 4;
    static constexpr int kBarOff = (kMetaOff + kMetaBytes + 15) & ~15;
    static constexpr int kSmem = kBarOff + (3 * kStages + 1) * 8 + 16;
    static_assert(kSmem <= 227 * 1024, "shared memory budget");
    static_assert(kStage % 1024 == 0 && kATileBytes % 1024 == 0, "swizzled tiles need 1024-byte alignment");
    static_assert(kStagingOff % 16 == 0 && kStagingBytes % 16 == 0 && kPendOff % 16 == 0, "16-byte alignment");
    static_assert(kMetaOff % 16 == 0 && kBarOff % 16 == 0, "16-byte aligned regions");
};

// Warp roles (192 threads):
//   warp 4 (loader): per chunk, lane 0 acquires the stage ("empty"), records
//     the chunk in the stage's pending record, sets the "full" transaction
//     count, and issues the dense A image (16 KB cp.async.bulk) or the sparse
//     entries (cp.async.bulk into staging, completing on "staged"); then the
//     32 lanes issue the B gather: 16 row groups x NT/64 boxes of
//     tile::gather4 (4 rows x 128 bytes each, 128-byte swizzle), completing on
//     "full". Nothing in the loader waits for data, so it runs up to kStages
//     chunks ahead of the tensor core.
//   warps 0-3 (scatter): per chunk, wait "staged"; for a sparse chunk zero the
//     A tile, scatter the staged entries into the 128-byte swizzled K-major
//     layout and fence.proxy.async; arrive on "full".
//   warp 5, lane 0 (MMA): wait "full", 4 x tcgen05.mma, commit "empty"; after
//     the last chunk commit "accumulator ready".
//   warps 0-3 (epilogue): warp w reads TMEM lanes 32w .. 32w + 31 (rows).
template <int NT, typename OutT>
__global__ void __launch_bounds__(kThreads, 1) spmm_tc_kernel(const __grid_constant__ TcBatch batch)
{
    using Cfg = TcCfg<NT>;
    constexpr int S = Cfg::kStages;
    constexpr int kBoxes = NT / 64;      // 64-column boxes per B row slice
    constexpr int kGathers = 16 * kBoxes; // gather4 instructions per chunk
    extern __shared__ __align__(1024) uint8_t smem[];
    int4 *pend = reinterpret_cast<int4 *>(smem + Cfg::kPendOff);
    int *meta_cols = reinterpret_cast<int *>(smem + Cfg::kMetaOff); // kMetaChunks x 64 columns
    int *meta_img = meta_cols + kMetaChunks * kChunkCols;           // kMetaChunks image indices
    int *meta_eptr = meta_img + kMetaChunks;                        // kMetaChunks + 1 entry offsets
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + Cfg::kBarOff);
    uint64_t *empty = full + S;
    uint64_t *staged = empty + S;
    uint64_t *accum = staged + S;
    volatile int *flag = reinterpret_cast<volatile int *>(accum + 1); // 2 slots, alternating by chunk
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(accum + 1) + 2;

    // ---- work item -> (job, window, N slice)
    const int item = blockIdx.x;
    int j = 0;
    while (j + 1 < batch.n_jobs && batch.item_start[j + 1] <= item) j++;
    const TcJob &a = batch.job[j];
    const int local = item - batch.item_start[j];
    const int t = local / a.ntiles;
    const int n0 = (local % a.ntiles) * NT;
    const int4 wi = a.win_info[t];
    const int w = wi.x, c0 = wi.y, nch = wi.z;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (smem_u32(smem) & 1023u) { // the swizzled tiles and TMA destinations need a 1024-byte aligned base
        if (threadIdx.x == 0)
            atomicOr(a.status, kStatusLayout);
        return;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], kScatterThreads);
            mbar_init(&empty[s], 1);
            mbar_init(&staged[s], 1);
        }
        mbar_init(accum, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(NT)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    // The epilogue row of this thread (warps 0-3), fetched now so its latency
    // hides behind the main loop; -1 = no store.
    int out_row = -1;
    if (warp < 4) {
        const int i = w * kWindowRows + warp * 32 + lane;
        if (i < a.M && !((a.flags & TCA_FLAG_KEEP_EMPTY_ROWS) && a.p_row_ptr[i + 1] == a.p_row_ptr[i]))
            out_row = a.perm[i];
    }

    if (warp == kLoaderWarp) {
        // ---------------- loader ----------------
        for (int i = 0; i < nch; i++) {
            const int s = i % S, mi = i % kMetaChunks;
            if (mi == 0) { // metadata of the next up to kMetaChunks chunks
                const int cnt = min(kMetaChunks, nch - i);
                const int *src = a.win_cols + (size_t)(c0 + i) * kChunkCols;
                for (int k = lane; k < cnt * kChunkCols; k += 32) meta_cols[k] = __ldg(src + k);
                if (lane < cnt) meta_img[lane] = __ldg(a.img_idx + c0 + i + lane);
                if (lane <= cnt) meta_eptr[lane] = __ldg(a.tile_ptr + c0 + i + lane);
                __syncwarp();
            }
            uint32_t got = 1;
            if (lane == 0 && i >= S)
                got = mbar_wait(&empty[s], ((i / S) - 1) & 1) ? 1u : 0u;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) { ok = false; break; }
            const uint32_t a_s = smem_u32(smem + s * Cfg::kStage), b_s = a_s + kATileBytes;
            const int img = meta_img[mi];
            if (lane == 0) {
                const int e0 = meta_eptr[mi], e1 = meta_eptr[mi + 1], e0a = e0 & ~3;
                pend[s] = make_int4(img, e0, e0a, e1);
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
            __syncwarp(); // the transaction count is set before any gather is issued
            const int *cols = meta_cols + mi * kChunkCols;
            if (cols[0] >= 0 && cols[kChunkCols - 1] == cols[0] + kChunkCols - 1) {
                // 64 contiguous B rows (direct chunks): one 8 KB tiled box per 64 columns
                if (lane < kBoxes)
                    tma_tile2d(b_s + lane * (kChunkCols * 128), &a.tmap_tile, n0 + lane * 64, cols[0], &full[s]);
            } else {
                for (int q = lane; q < kGathers; q += 32) {
                    const int g = q & 15, box = q >> 4;
                    tma_gather4(b_s + box * (kChunkCols * 128) + g * 512, &a.tmap_b, n0 + box * 64, cols[4 * g],
                                cols[4 * g + 1], cols[4 * g + 2], cols[4 * g + 3], &full[s]);
                }
            }
            __syncwarp(); // the metadata cache is reloaded only after every lane used it
        }
    } else if (warp < 4) {
        // ---------------- scatter ----------------
        const int sid = threadIdx.x;
        for (int i = 0; i < nch; i++) {
            const int s = i % S;
            if (sid == 0)
                flag[i & 1] = mbar_wait(&staged[s], (i / S) & 1) ? 1 : 0;
            named_bar_sync(1, kScatterThreads); // also orders the staged data for every scatter thread
            if (flag[i & 1] == 0) { ok = false; break; } // uniform across the scatter warps
            const int4 pd = pend[s];
            if (pd.x < 0) {
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
        }
    } else if (warp == kMmaWarp && lane == 0) {
        // ---------------- MMA issuer ----------------
        constexpr uint32_t idesc = idesc_f16(NT);
        for (int i = 0; i < nch; i++) {
            const int s = i % S;
            if (!mbar_wait(&full[s], (i / S) & 1)) { ok = false; break; }
            tc_fence_after();
            const uint32_t a_s = smem_u32(smem + s * Cfg::kStage), b_s = a_s + kATileBytes;
#pragma unroll
            for (int k = 0; k < kChunkCols / 16; k++) {
                const uint64_t ad = smem_desc(a_s + k * 32, 16, 1024);
                const uint64_t bd = smem_desc(b_s + k * 2048, kChunkCols * 128, 1024);
                umma_f16(tmem, ad, bd, idesc, (i | k) != 0);
            }
            umma_commit(&empty[s]);
        }
        if (ok)
            umma_commit(accum);
    }

    if (warp < 4) {
        // ---------------- epilogue ----------------
        uint32_t got = 0;
        if (lane == 0)
            got = mbar_wait(accum, 0) ? 1u : 0u;
        got = __shfl_sync(0xffffffffu, got, 0);
        tc_fence_after();
        if (got) {
            const bool write = out_row >= 0;
            OutT *Crow = write ? reinterpret_cast<OutT *>(a.C) + (size_t)out_row * a.ldc : nullptr;
            for (int cb = 0; cb < NT / 16; cb++) {
                const int n = n0 + cb * 16;
                if (n >= a.N)
                    break; // uniform across the warp
                uint32_t r[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16), r);
                if (write) {
                    store8_out(Crow + n, reinterpret_cast<const float *>(r), a.alpha, a.beta);
                    if (n + 8 < a.N)
                        store8_out(Crow + n + 8, reinterpret_cast<const float *>(r) + 8, a.alpha, a.beta);
                }
            }
        } else {
            ok = false;
        }
    }

    if (!ok)
        atomicOr(a.status, kStatusTimeout);
    tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NT) : "memory");
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
    spmm_tc_kernel<NT, OutT><<<b.item_start[b.n_jobs], kThreads, smem, s>>>(b);
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
