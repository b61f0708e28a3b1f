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
// One CTA = one (job, window, NT-wide slice of N) work item; 5 warps:
//   warps 0-3 (producers), per chunk:
//     * dense chunks (>= 4096 nonzeros): one thread issues a 16 KB bulk copy
//       (cp.async.bulk, complete_tx on the stage's "full" mbarrier) of the
//       pre-rendered, pre-swizzled A tile straight into the stage;
//     * sparse chunks: zero the A tile; copy the packed entries into a
//       staging buffer with 16-byte cp.async; one chunk later, scatter them
//       into the 128-byte swizzled K-major tile;
//     * gather the 64 B rows (the chunk's condensed columns, preloaded in
//       shared memory) into a 128-byte swizzled N-major tile with 16-byte
//       cp.async, zero-filling padding columns and n >= N;
//     * fence.proxy.async, then arrive on "full".
//   warp 4, one lane: wait "full", issue 4 tcgen05.mma (K = 16 each),
//     tcgen05.commit the stage's "empty" barrier; after the last chunk commit
//     the "accumulator ready" barrier.
//   warps 0-3 (epilogue): tcgen05.ld the accumulator (TMEM lane = row),
//     alpha/beta, store to C[perm[row]] (FP16 or FP32).
// Every mbarrier wait is bounded (about one second of %globaltimer); on
// expiry the CTA records kStatusTimeout in the job's status word and runs to
// completion without hanging. No load uses cluster multicast.
#include "tca_internal.cuh"
#include "plan.cuh"

namespace tca {
namespace {

constexpr int kProducerThreads = 128;
constexpr int kThreads = kProducerThreads + 32;
constexpr int kATileBytes = kWindowRows * kChunkCols * 2; // 16 KB
constexpr int kStagingBytes = kImageMinNnz * 4 + 64;      // < 4096 entries, rounded out to 16 B
constexpr int kMetaChunks = 32;                           // chunk metadata cached in shared memory
constexpr int kMaxJobs = 32;                              // jobs per launch (kernel parameter space)

struct TcJob {
    const int *tc_windows, *tile_first, *tile_ptr, *win_cols, *img_idx, *perm, *p_row_ptr;
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

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
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

// Shared memory: kStages x (A tile | B tile), kStages entry staging buffers,
// chunk metadata, per-stage pending-chunk records, mbarriers.
template <int NT> struct TcCfg {
    static constexpr int kStages = NT == 256 ? 3 : 4;
    static constexpr int kBTileBytes = kChunkCols * NT * 2;
    static constexpr int kStage = kATileBytes + kBTileBytes;
    static constexpr int kStagingOff = kStages * kStage;
    static constexpr int kMetaOff = kStagingOff + kStages * kStagingBytes;
    static constexpr int kMetaBytes = (kMetaChunks * kChunkCols + 2 * kMetaChunks + 1) * 4;
    static constexpr int kPendOff = kMetaOff + kMetaBytes;
    static constexpr int kBarOff = (kPendOff + kStages * 16 + 15) & ~15;
    static constexpr int kBytes = kBarOff + (2 * kStages + 1) * 8 + 16;
    static constexpr int kSmem = kBytes + 1024; // alignment slack
    static_assert(kSmem <= 227 * 1024, "shared memory budget");
};

template <int NT, typename OutT>
__global__ void __launch_bounds__(kThreads, 1) spmm_tc_kernel(const __grid_constant__ TcBatch batch)
{
    using Cfg = TcCfg<NT>;
    constexpr int S = Cfg::kStages;
    constexpr int kPiecesPerRow = NT / 8; // 16-byte pieces of one B row slice
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    int *meta_cols = reinterpret_cast<int *>(smem + Cfg::kMetaOff);
    int *meta_eptr = meta_cols + kMetaChunks * kChunkCols; // kMetaChunks + 1
    int *meta_img = meta_eptr + kMetaChunks + 1;           // kMetaChunks
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + Cfg::kBarOff);
    uint64_t *empty = full + S;
    uint64_t *accum = empty + S;
    volatile int *flag = reinterpret_cast<volatile int *>(accum + 1);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(accum + 1) + 1;

    // ---- work item -> (job, window, N slice)
    const int item = blockIdx.x;
    int j = 0;
    while (j + 1 < batch.n_jobs && batch.item_start[j + 1] <= item) j++;
    const TcJob &a = batch.job[j];
    const int local = item - batch.item_start[j];
    const int t = local / a.ntiles;
    const int n0 = (local % a.ntiles) * NT;
    const int w = a.tc_windows[t];
    const int c0 = a.tile_first[t], nch = a.tile_first[t + 1] - c0;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], kProducerThreads);
            mbar_init(&empty[s], 1);
        }
        mbar_init(accum, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 4) {
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

    if (warp < 4) {
        // ---------------- producers ----------------
        // Chunk i is issued in iteration i and finished (copies waited for,
        // sparse entries scattered, "full" signalled) in iteration i + S - 1,
        // so up to S chunks of copies are in flight per CTA.
        const int tid = threadIdx.x;
        uint8_t *staging = smem + Cfg::kStagingOff;
        int4 *pend = reinterpret_cast<int4 *>(smem + Cfg::kPendOff); // per stage: img, e0, e0a, e1

        auto finish = [&](int idx, bool drain) {
            if (drain) cp_async_wait<0>(); else cp_async_wait<S - 1>();
            named_bar_sync(1, kProducerThreads); // every producer's copies of this chunk have landed
            const int s = idx % S;
            const int4 pd = pend[s];
            if (pd.x < 0) {
                uint8_t *At = smem + s * Cfg::kStage;
                const uint32_t *st = reinterpret_cast<const uint32_t *>(staging + s * kStagingBytes);
                for (int e = pd.y + tid; e < pd.w; e += kProducerThreads) {
                    const uint32_t v = st[e - pd.z];
                    *reinterpret_cast<uint16_t *>(At + swz128_offset(v >> 22, (v >> 16) & 63u)) =
                        (uint16_t)(v & 0xffffu);
                }
            }
            fence_proxy_async();
            mbar_arrive(&full[s]);
        };

        for (int i = 0; i < nch; i++) {
            const int s = i % S, mi = i % kMetaChunks;
            if (mi == 0) { // (re)load the metadata of up to kMetaChunks chunks
                named_bar_sync(1, kProducerThreads);
                const int cnt = min(kMetaChunks, nch - i);
                const int *src = a.win_cols + (size_t)(c0 + i) * kChunkCols;
                for (int k = tid; k < cnt * kChunkCols; k += kProducerThreads) meta_cols[k] = __ldg(src + k);
                for (int k = tid; k <= cnt; k += kProducerThreads) meta_eptr[k] = __ldg(a.tile_ptr + c0 + i + k);
                for (int k = tid; k < cnt; k += kProducerThreads) meta_img[k] = __ldg(a.img_idx + c0 + i + k);
                named_bar_sync(1, kProducerThreads);
            }
            if (tid == 0)
                *flag = (i < S) ? 1 : (mbar_wait(&empty[s], ((i / S) - 1) & 1) ? 1 : 0);
            named_bar_sync(1, kProducerThreads);
            if (*flag == 0) { ok = false; break; } // uniform across the producers
            uint8_t *At = smem + s * Cfg::kStage;
            const uint32_t a_s = smem_u32(At), b_s = a_s + kATileBytes;
            const int img = meta_img[mi];
            const int e0 = meta_eptr[mi], e1 = meta_eptr[mi + 1], e0a = e0 & ~3;
            if (tid == 0)
                pend[s] = make_int4(img, e0, e0a, e1); // read after the barrier in finish(i)
            if (img >= 0) {
                if (tid == 0) {
                    mbar_expect_tx(&full[s], kATileBytes);
                    bulk_copy_g2s(a_s, a.images + (size_t)img * (kATileBytes / 2), kATileBytes, &full[s]);
                }
            } else {
#pragma unroll
                for (int k = 0; k < kATileBytes / (16 * kProducerThreads); k++)
                    reinterpret_cast<uint4 *>(At)[tid + k * kProducerThreads] = make_uint4(0, 0, 0, 0);
                const uint32_t st_s = smem_u32(staging + s * kStagingBytes);
                const int pieces = (e1 - e0a + 3) >> 2;
                for (int k = tid; k < pieces; k += kProducerThreads)
                    cp_async16(st_s + k * 16, a.entries + e0a + 4 * k, 16u);
            }
            const int *cols = meta_cols + mi * kChunkCols;
#pragma unroll 4
            for (int piece = tid; piece < kChunkCols * kPiecesPerRow; piece += kProducerThreads) {
                const int k = piece / kPiecesPerRow, qq = piece % kPiecesPerRow;
                const int col = cols[k];
                const int n = n0 + qq * 8;
                const bool valid = (col >= 0) && (n < a.N);
                const __half *src = valid ? (a.B + (size_t)col * a.ldb + n) : a.B;
                const uint32_t dst = b_s + (qq >> 3) * (kChunkCols * 128) + k * 128 + ((((qq & 7) ^ (k & 7))) << 4);
                cp_async16(dst, src, valid ? 16u : 0u);
            }
            cp_async_commit();
            if (i >= S - 1)
                finish(i - (S - 1), false);
        }
        if (ok)
            for (int idx = max(0, nch - (S - 1)); idx < nch; idx++)
                finish(idx, true);
        cp_async_wait<0>(); // no copy outlives the CTA, also on the abort path
    } else if (lane == 0) {
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
            const int i = w * kWindowRows + warp * 32 + lane;
            const bool valid = i < a.M;
            bool write = valid;
            OutT *Crow = nullptr;
            if (valid) {
                if ((a.flags & TCA_FLAG_KEEP_EMPTY_ROWS) && a.p_row_ptr[i + 1] == a.p_row_ptr[i])
                    write = false;
                Crow = reinterpret_cast<OutT *>(a.C) + (size_t)a.perm[i] * a.ldc;
            }
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
    if (warp == 4) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NT) : "memory");
    }
}

TcJob make_job(const SpmmJob &sj, float alpha, float beta, unsigned flags, int NT)
{
    const tca_plan *p = sj.p;
    TcJob j;
    j.tc_windows = p->tc_windows;
    j.tile_first = p->tile_first;
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
    return j;
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
            const TcJob j = make_job(sj, alpha, beta, flags, NT);
            b.job[b.n_jobs] = j;
            b.item_start[b.n_jobs + 1] = b.item_start[b.n_jobs] + sj.p->n_tc * j.ntiles;
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
