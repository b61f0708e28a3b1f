// sddmm_tc.cu -- the SDDMM adjoint dA = alpha * (dY B^T) on A's pattern, on
// the tensor cores (tcgen05, sm_100a), over the plan's tensor-core windows.
//
// The reference has no backward pass; the adjoint follows from its forward
// (src/our_spmm.cu:290-346, Y[r, :] = sum_j a_j B[c_j, :]):
//   dL/da_j = sum_n dY[r_j, n] * B[c_j, n].
// For a tensor-core window (128 sorted rows) and one of its 64-column chunks,
// the tile D[128 x 64] = dY[window rows, :] B[chunk columns, :]^T holds the
// values of every nonzero of the chunk: a GEMM tile with K = N (the width of
// dY and B), A = dY rows (K-major) and B = B rows (K-major), accumulated in
// FP32 in tensor memory. Only chunks that hold nonzeros are computed, and the
// epilogue writes only the nonzeros (the chunk's tile entries), in the
// caller's nonzero order.
//
// Work unit: (window, group of up to 8 of its chunks -- 8 x 64 accumulator
// columns fill tensor memory --, part of the n range). Per 64-wide step of n
// the loader warp moves the window's dY rows (tile::gather4 of the rows
// perm[...], 16 KB) into a ring of dY stages and each chunk's B rows (one
// tiled box of 64 consecutive rows for direct chunks, tile::gather4 of the
// condensed columns otherwise; 8 KB) into a deeper ring of B stages; the MMA
// lane multiplies the dY stage with every chunk's B stage into the chunk's
// accumulator. No load uses cluster multicast; rows and columns outside the
// tensors (a window's rows beyond M, padding columns, n >= N) arrive as zeros.
//
// When the windows' groups are fewer than the SMs, the n range is cut into
// parts; each part leaves its values in a workspace slice (one float per
// tensor-core entry), and after the launch k_sddmm_sum adds the parts of
// every entry in part order -- a fixed order, so the result does not depend
// on which part finished when -- and writes dA. No CTA waits for another.
// Every mbarrier wait is bounded (about one second); on expiry the CTA records
// kStatusTimeout in the plan's status word (and in the launch's failure word,
// so that the sums are skipped) and ends.
#include <cuda.h>
#include <algorithm>
#include "tca_internal.cuh"
#include "plan.cuh"
#include "ptx.cuh"

namespace tca {
namespace {

using namespace ptx;

constexpr int kSdLoaderWarp = 0;
constexpr int kSdMmaWarp = 1;
constexpr int kSdEpiWarp0 = 2; // warps 2-5
constexpr int kSdThreads = 192;
constexpr int kSdEpiThreads = 128;
constexpr int kSdMaxChunks = 8;  // chunks per unit: 8 x 64 FP32 accumulator columns = all of tensor memory
constexpr int kSdYStages = 3;    // dY ring: 128 rows x 64 n, 16 KB each
constexpr int kSdBStages = 16;   // B ring: 64 rows x 64 n, 8 KB each
constexpr int kSdYBytes = kWindowRows * 64 * 2;
constexpr int kSdBBytes = kChunkCols * 64 * 2;
constexpr int kSdStageRow = 68;  // floats per row of the epilogue's staging tiles (64 + 4: fewer bank conflicts)
constexpr int kSdStageChunks = 4; // chunks staged at once in the epilogue
constexpr int kSdYOff = 0;
constexpr int kSdBOff = kSdYOff + kSdYStages * kSdYBytes;
constexpr int kSdBarOff = kSdBOff + kSdBStages * kSdBBytes;
// y_full, y_empty [kSdYStages]; b_full, b_empty [kSdBStages]; acc_full; drain; TMEM slot, flag
constexpr int kSdSmem = kSdBarOff + (2 * kSdYStages + 2 * kSdBStages + 2) * 8 + 16;
static_assert(kSdBarOff >= kSdStageChunks * kWindowRows * kSdStageRow * 4, "the rings hold the epilogue's staging tiles");
static_assert(kSdYBytes % 1024 == 0 && kSdBBytes % 1024 == 0, "swizzled tiles need 1024-byte alignment");
static_assert(kSdSmem <= 227 * 1024, "shared memory budget");

struct SdJob {
    CUtensorMap tmap_y;    // dY as {N, M}, box {64, 1}, 128-byte swizzle (gather4 of window rows)
    CUtensorMap tmap_b;    // B as {N, K}, box {64, 1} (gather4 of condensed columns)
    CUtensorMap tmap_tile; // B as {N, K}, box {64, 64} (64 consecutive rows: direct chunks)
    const int4 *win_info;  // per tensor-core window: window, first chunk, chunk count
    const int *win_cols, *tile_ptr, *perm, *src, *tile_src;
    const uint32_t *entries;
    void *out;             // nnz values in the caller's order (FP16 or FP32)
    float *partials;       // parts > 1: parts x tc_nnz floats
    int *failed;           // parts > 1: set when a CTA gave up (zero before the launch)
    int *status;
    int M, N, n_steps, parts, steps_per_part, out_f16;
    int n_win, groups_per_win; // tensor-core windows; chunk groups of the widest window
    long long tc_nnz;
    float alpha;
};

// kind::f16 instruction descriptor: D FP32, A/B FP16, both K-major, M = 128, N = 64.
constexpr uint32_t kSdIdesc = (1u << 4) | ((uint32_t)(64 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void sd_umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accum)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
                 "l"(a), "l"(b), "r"(kSdIdesc), "r"(accum)
                 : "memory");
}

// Unit u -> (tensor-core window t, chunk group gi: chunks [8 gi, 8 gi + 8)
// of the window, part q of the n range); units are ordered window, group,
// part. A window with fewer groups than the widest leaves its extra units
// empty: false.
struct SdUnit {
    int t, g0, nch, q, group;
};

__device__ __forceinline__ bool sd_decode(const SdJob &a, int u, SdUnit &x)
{
    x.q = u % a.parts;
    x.group = u / a.parts;
    x.t = x.group / a.groups_per_win;
    x.g0 = (x.group - x.t * a.groups_per_win) * kSdMaxChunks;
    if (x.t >= a.n_win)
        return false;
    const int z = __ldg(&a.win_info[x.t].z);
    x.nch = min(kSdMaxChunks, z - x.g0);
    return x.nch > 0;
}

__global__ void __launch_bounds__(kSdThreads, 1) k_sddmm_tc(const __grid_constant__ SdJob a)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t *y_full = reinterpret_cast<uint64_t *>(smem + kSdBarOff);
    uint64_t *y_empty = y_full + kSdYStages;
    uint64_t *b_full = y_empty + kSdYStages;
    uint64_t *b_empty = b_full + kSdBStages;
    uint64_t *acc_full = b_empty + kSdBStages;
    uint64_t *drain = acc_full + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    SdUnit x;
    if (!sd_decode(a, blockIdx.x, x))
        return; // uniform: no unit for this CTA
    if (smem_u32(smem) & 1023u) {
        if (threadIdx.x == 0)
            atomicOr(a.status, kStatusLayout);
        return;
    }
    const int4 wi = __ldg(a.win_info + x.t);
    const int c_first = wi.y + x.g0; // the group's first chunk (plan-wide index)
    const int ks0 = x.q * a.steps_per_part, ks1 = min(a.n_steps, ks0 + a.steps_per_part);
    int tcols = 32;
    while (tcols < x.nch * 64) tcols <<= 1;
    // the part's n steps, each window starting at a different one, so that
    // the windows do not read the same columns of B at once
    const int rot = x.t % max(1, ks1 - ks0);
    auto step_n = [&](int st) { return ks0 + (st + rot) % (ks1 - ks0); };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kSdYStages; s++) {
            mbar_init(&y_full[s], 1);
            mbar_init(&y_empty[s], 1);
        }
        for (int s = 0; s < kSdBStages; s++) {
            mbar_init(&b_full[s], 1);
            mbar_init(&b_empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(drain, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kSdMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(tcols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp == kSdLoaderWarp) {
        // ---------------- loader ----------------
        // the window's 128 rows of dY (caller rows; -1 beyond M: zero rows),
        // four per lane, and each chunk's 64 B rows (lanes 0-15: four each)
        int rows[4];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int i = wi.x * kWindowRows + 4 * lane + r;
            rows[r] = i < a.M ? __ldg(a.perm + i) : -1;
        }
        int4 cols[kSdMaxChunks];
        bool direct[kSdMaxChunks];
#pragma unroll
        for (int c = 0; c < kSdMaxChunks; c++) {
            cols[c] = make_int4(-1, -1, -1, -1);
            if (c < x.nch && lane < 16)
                cols[c] = __ldg(reinterpret_cast<const int4 *>(a.win_cols + (size_t)(c_first + c) * kChunkCols) + lane);
            const int col0 = __shfl_sync(0xffffffffu, cols[c].x, 0), col63 = __shfl_sync(0xffffffffu, cols[c].w, 15);
            direct[c] = col0 >= 0 && col63 == col0 + kChunkCols - 1;
        }
        int yt = 0, bt = 0;
        for (int st = 0; st < ks1 - ks0 && ok; st++, yt++) {
            const int n0 = step_n(st) * 64;
            const int sy = yt % kSdYStages;
            uint32_t got = 1;
            if (lane == 0 && yt >= kSdYStages)
                got = mbar_wait(&y_empty[sy], ((yt / kSdYStages) - 1) & 1) ? 1u : 0u;
            if (!__shfl_sync(0xffffffffu, got, 0)) { ok = false; break; }
            if (lane == 0)
                mbar_arrive_expect_tx(&y_full[sy], kSdYBytes);
            __syncwarp();
            tma_gather4(smem_u32(smem + kSdYOff + sy * kSdYBytes) + lane * 512, &a.tmap_y, n0, rows[0], rows[1],
                        rows[2], rows[3], &y_full[sy]);
#pragma unroll
            for (int c = 0; c < kSdMaxChunks; c++) {
                if (c >= x.nch || !ok)
                    break;
                const int sb = bt % kSdBStages;
                got = 1;
                if (lane == 0 && bt >= kSdBStages)
                    got = mbar_wait(&b_empty[sb], ((bt / kSdBStages) - 1) & 1) ? 1u : 0u;
                if (!__shfl_sync(0xffffffffu, got, 0)) { ok = false; break; }
                const uint32_t dst = smem_u32(smem + kSdBOff + sb * kSdBBytes);
                if (lane == 0)
                    mbar_arrive_expect_tx(&b_full[sb], kSdBBytes);
                __syncwarp();
                if (direct[c]) {
                    if (lane == 0)
                        tma_tile2d(dst, &a.tmap_tile, n0, cols[c].x, &b_full[sb]);
                } else if (lane < 16) {
                    tma_gather4(dst + lane * 512, &a.tmap_b, n0, cols[c].x, cols[c].y, cols[c].z, cols[c].w,
                                &b_full[sb]);
                }
                bt++;
            }
        }
    } else if (warp == kSdMmaWarp) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int yt = 0, bt = 0;
            for (int st = 0; st < ks1 - ks0 && ok; st++, yt++) {
                const int sy = yt % kSdYStages;
                if (!mbar_wait(&y_full[sy], (yt / kSdYStages) & 1)) { ok = false; break; }
                const uint32_t ys = smem_u32(smem + kSdYOff + sy * kSdYBytes);
                for (int c = 0; c < x.nch; c++, bt++) {
                    const int sb = bt % kSdBStages;
                    if (!mbar_wait(&b_full[sb], (bt / kSdBStages) & 1)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t bs = smem_u32(smem + kSdBOff + sb * kSdBBytes);
#pragma unroll
                    for (int kk = 0; kk < 4; kk++)
                        sd_umma(tmem + (uint32_t)(c * 64), smem_desc(ys + kk * 32, 16, 1024),
                                smem_desc(bs + kk * 32, 16, 1024), (st > 0 || kk > 0) ? 1u : 0u);
                    umma_commit(&b_empty[sb]);
                }
                umma_commit(&y_empty[sy]);
            }
            if (ok)
                umma_commit(acc_full);
            umma_commit(drain); // every MMA issued has completed before tensor memory is released
            if (!mbar_wait(drain, 0))
                ok = false;
        }
        __syncwarp();
    } else {
        // ---------------- epilogue ----------------
        const int quarter = warp & 3;
        const int row = quarter * 32 + lane; // TMEM lane = row of the window
        const int et = (int)threadIdx.x - kSdEpiWarp0 * 32;
        uint32_t got = 0;
        if (lane == 0)
            got = mbar_wait(acc_full, 0) ? 1u : 0u;
        got = __shfl_sync(0xffffffffu, got, 0);
        if (!named_bar_and(1, kSdEpiThreads, got != 0)) {
            ok = false;
        } else {
            tc_fence_after();
            // The MMAs are complete, so both rings are free: they hold the
            // staging tiles of up to kSdStageChunks chunks at a time (row-major,
            // kSdStageRow floats a row); then the entries of those chunks --
            // contiguous in the plan -- are read from them, four per thread in
            // flight.
            float *stage = reinterpret_cast<float *>(smem + kSdYOff);
            for (int g0 = 0; g0 < x.nch; g0 += kSdStageChunks) {
                const int ng = min(kSdStageChunks, x.nch - g0);
                for (int c = 0; c < ng; c++) {
#pragma unroll
                    for (int cb = 0; cb < 4; cb++) {
                        uint32_t r[16];
                        tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)((g0 + c) * 64 + cb * 16), r);
                        float4 *dst = reinterpret_cast<float4 *>(stage + (c * kWindowRows + row) * kSdStageRow + cb * 16);
#pragma unroll
                        for (int q = 0; q < 4; q++)
                            dst[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                                 __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
                    }
                }
                named_bar_sync(1, kSdEpiThreads);
                int bound[kSdStageChunks + 1];
#pragma unroll
                for (int c = 0; c <= kSdStageChunks; c++) bound[c] = __ldg(a.tile_ptr + c_first + g0 + min(c, ng));
                for (int e0 = bound[0] + et; e0 < bound[kSdStageChunks]; e0 += 4 * kSdEpiThreads) {
                    uint32_t v[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int e = e0 + u * kSdEpiThreads;
                        v[u] = e < bound[kSdStageChunks] ? __ldg(a.entries + e) : 0u;
                    }
                    int j[4];
                    if (a.parts == 1) {
#pragma unroll
                        for (int u = 0; u < 4; u++) {
                            const int e = e0 + u * kSdEpiThreads;
                            j[u] = e < bound[kSdStageChunks] ? __ldg(a.tile_src + e) : 0;
                        }
#pragma unroll
                        for (int u = 0; u < 4; u++) {
                            const int e = e0 + u * kSdEpiThreads;
                            j[u] = e < bound[kSdStageChunks] ? __ldg(a.src + j[u]) : 0;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int e = e0 + u * kSdEpiThreads;
                        if (e >= bound[kSdStageChunks])
                            break;
                        int c = 0;
#pragma unroll
                        for (int k = 1; k < kSdStageChunks; k++) c += e >= bound[k] ? 1 : 0;
                        const float d = stage[(c * kWindowRows + (v[u] >> 22)) * kSdStageRow + ((v[u] >> 16) & 63u)];
                        if (a.parts > 1)
                            a.partials[(size_t)x.q * a.tc_nnz + e] = d;
                        else if (a.out_f16)
                            reinterpret_cast<__half *>(a.out)[j[u]] = __float2half_rn(a.alpha * d);
                        else
                            reinterpret_cast<float *>(a.out)[j[u]] = a.alpha * d;
                    }
                }
                named_bar_sync(1, kSdEpiThreads); // the staging tiles are reused by the next group
            }
        }
    }

    tc_fence_before();
    if (__syncthreads_or(!ok)) {
        // a role gave up after a bounded wait: record it, then give bulk
        // copies in flight a bounded time (1 ms) to land before the CTA's
        // shared memory is released
        if (threadIdx.x == 0) {
            atomicOr(a.status, kStatusTimeout);
            if (a.failed)
                atomicOr(a.failed, 1);
            const uint64_t t0 = global_ns();
            while (global_ns() - t0 < 1000000ull) {
            }
        }
        __syncthreads();
    }
    if (warp == kSdMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols) : "memory");
    }
}

// After a launch with parts: dA of every tensor-core entry e = alpha x (part
// 0 + part 1 + ...) in part order, written in the caller's nonzero order;
// nothing when a CTA of the launch gave up.
template <typename OutT>
__global__ void __launch_bounds__(256)
k_sddmm_sum(const float *__restrict__ partials, long long tc_nnz, int parts, const int *__restrict__ tile_src,
            const int *__restrict__ src, const int *__restrict__ failed, OutT *__restrict__ out, float alpha)
{
    if (*(volatile const int *)failed)
        return;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tc_nnz;
         e += (long long)gridDim.x * blockDim.x) {
        float x[8];
        float d = 0.f;
        for (int q0 = 0; q0 < parts; q0 += 8) {
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (q0 + u < parts)
                    x[u] = __ldcg(partials + (size_t)(q0 + u) * tc_nnz + e);
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (q0 + u < parts)
                    d = (q0 + u == 0) ? x[u] : d + x[u];
        }
        const int j = __ldg(src + __ldg(tile_src + e));
        if constexpr (sizeof(OutT) == 2)
            out[j] = __float2half_rn(alpha * d);
        else
            out[j] = alpha * d;
    }
}

} // namespace

// The SDDMM over the plan's tensor-core windows on the tensor cores (see the
// top of this file). dY (M x N, row stride ldy) and B (K x N, row stride ldb)
// need 16-byte aligned rows. Values of the nonzeros outside tensor-core
// windows are not written (the caller's CUDA-core pass covers them).
int sddmm_tc(const tca_plan *p, const __half *dY, int ldy, const __half *B, int ldb, int N, void *out, bool out_f16,
             float alpha, cudaStream_t s)
{
    if (p->n_tc == 0 || N == 0)
        return TCA_OK;
    // units: (window, group of up to kSdMaxChunks chunks, part of the n range)
    int max_z = 0;
    for (int t = 0; t < p->n_tc; t++) max_z = std::max(max_z, p->h_tile_first[t + 1] - p->h_tile_first[t]);
    const int groups_per_win = (max_z + kSdMaxChunks - 1) / kSdMaxChunks;
    const int n_groups = p->n_tc * groups_per_win;
    const int n_steps = (N + 63) / 64;
    int parts = std::max(1, std::min(n_steps, kSMs / n_groups));
    const int steps_per_part = (n_steps + parts - 1) / parts;
    parts = (n_steps + steps_per_part - 1) / steps_per_part; // no empty part

    SdJob j{};
    TCA_TRY(encode_tensor_map_2d(&j.tmap_y, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, dY, (uint64_t)N, (uint64_t)p->M,
                                 (uint64_t)ldy * 2, 64, 1, CU_TENSOR_MAP_SWIZZLE_128B));
    TCA_TRY(encode_tensor_map_2d(&j.tmap_b, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, B, (uint64_t)N, (uint64_t)p->K,
                                 (uint64_t)ldb * 2, 64, 1, CU_TENSOR_MAP_SWIZZLE_128B));
    TCA_TRY(encode_tensor_map_2d(&j.tmap_tile, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, B, (uint64_t)N, (uint64_t)p->K,
                                 (uint64_t)ldb * 2, 64, kChunkCols, CU_TENSOR_MAP_SWIZZLE_128B));
    j.win_info = p->tc_win_info;
    j.win_cols = p->win_cols;
    j.tile_ptr = p->tile_ptr;
    j.perm = p->perm;
    j.src = p->src;
    j.tile_src = p->tile_src;
    j.entries = p->tile_entries;
    j.out = out;
    j.status = p->d_status;
    j.M = p->M;
    j.N = N;
    j.n_steps = n_steps;
    j.parts = parts;
    j.steps_per_part = steps_per_part;
    j.out_f16 = out_f16 ? 1 : 0;
    j.tc_nnz = p->tc_nnz;
    j.alpha = alpha;
    j.n_win = p->n_tc;
    j.groups_per_win = groups_per_win;

    // with parts: the failure word (cleared) and the partial values, for
    // this call only (stream-ordered; under capture the graph's own memory)
    void *ws = nullptr;
    if (parts > 1) {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        TCA_CUDA_TRY(cudaStreamIsCapturing(s, &cap));
        const size_t bytes = 256 + sizeof(float) * (size_t)parts * (size_t)p->tc_nnz;
        if (cap == cudaStreamCaptureStatusActive)
            TCA_CUDA_TRY(cudaMallocAsync(&ws, bytes, s));
        else
            TCA_TRY(dev_malloc(&ws, bytes, s));
        j.failed = static_cast<int *>(ws);
        j.partials = reinterpret_cast<float *>(static_cast<char *>(ws) + 256);
    }
    cudaError_t e = cudaSuccess;
    if (ws)
        e = cudaMemsetAsync(j.failed, 0, sizeof(int), s);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sddmm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kSdSmem);
    if (e == cudaSuccess) {
        k_sddmm_tc<<<n_groups * parts, kSdThreads, kSdSmem, s>>>(j);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && ws) {
        const unsigned grid = (unsigned)std::min<long long>((p->tc_nnz + 255) / 256, 8LL * kSMs);
        if (out_f16)
            k_sddmm_sum<__half><<<grid, 256, 0, s>>>(j.partials, p->tc_nnz, parts, p->tile_src, p->src, j.failed,
                                                      static_cast<__half *>(out), alpha);
        else
            k_sddmm_sum<float><<<grid, 256, 0, s>>>(j.partials, p->tc_nnz, parts, p->tile_src, p->src, j.failed,
                                                     static_cast<float *>(out), alpha);
        e = cudaGetLastError();
    }
    if (ws)
        cudaFreeAsync(ws, s);
    if (e != cudaSuccess)
        return set_error(TCA_ERR_CUDA, "tensor-core SDDMM launch failed: %s", cudaGetErrorString(e));
    return TCA_OK;
}

} // namespace tca
