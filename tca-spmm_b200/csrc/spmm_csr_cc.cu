// spmm_csr_cc.cu -- CSR x dense SpMM on CUDA cores.
//
// C[r, :] = alpha * sum_j val_j * B[col_j, :] + beta * C[r, :], FP32 accumulation.
// This restates the computation of kernel_our_spmm_balanced
// (src/our_spmm.cu:290-346) without its host-built warp schedule and without
// using mma.sync as a dot-product engine: a group of LPR lanes owns one row,
// each lane owns 8 consecutive output columns (one 16-byte vector of B), and
// the group walks the row's nonzeros, broadcasting (col, val) pairs by shuffle
// so that every B access is a fully used, coalesced 16-byte load with 8 loads
// in flight per lane.
//
// Kernels:
//   * plan-free (tca_spmm_csr): group g computes caller row g straight from
//     the CSR, 8 B loads in flight per lane;
//   * planned (tca_spmm / tca_spmm_batched): warps stream through work items
//     of consecutive sorted rows of one or many plans (spmm_cc_stream_kernel,
//     below; spmm_cc_items_kernel for operands that are not 16-byte aligned),
//     or compute them as small mma.sync products (spmm_cc_mma_kernel, an
//     autotuner candidate for FP16).
//
// Malformed CSR never faults: row ranges are clamped to [0, nnz] and
// nonzeros whose column is outside [0, K) contribute nothing.
#include <algorithm>
#include <memory>
#include <vector>
#include <cuda_fp8.h>
#include "tca_internal.cuh"
#include "plan.cuh"
#include "ptx.cuh"

namespace tca {
namespace {

__device__ __forceinline__ void fma8(float *acc, float a, const uint4 &b)
{
    const __half2 *h = reinterpret_cast<const __half2 *>(&b);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        float2 f = __half22float2(h[i]);
        acc[2 * i] = fmaf(a, f.x, acc[2 * i]);
        acc[2 * i + 1] = fmaf(a, f.y, acc[2 * i + 1]);
    }
}

__device__ __forceinline__ void load8(const __half *p, float *v)
{
    uint4 u = *reinterpret_cast<const uint4 *>(p);
    const __half2 *h = reinterpret_cast<const __half2 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        float2 f = __half22float2(h[i]);
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}
__device__ __forceinline__ void load8(const float *p, float *v)
{
    float4 a = reinterpret_cast<const float4 *>(p)[0];
    float4 b = reinterpret_cast<const float4 *>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void store8(__half *p, const float *v)
{
    uint4 u;
    __half2 *h = reinterpret_cast<__half2 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; i++) h[i] = __floats2half2_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<uint4 *>(p) = u;
}
__device__ __forceinline__ void store8(float *p, const float *v)
{
    reinterpret_cast<float4 *>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<float4 *>(p)[1] = make_float4(v[4], v[5], v[6], v[7]);
}

template <typename T> __device__ __forceinline__ float to_f(T x);
template <> __device__ __forceinline__ float to_f<__half>(__half x) { return __half2float(x); }
template <> __device__ __forceinline__ float to_f<float>(float x) { return x; }
template <typename T> __device__ __forceinline__ T from_f(float x);
template <> __device__ __forceinline__ __half from_f<__half>(float x) { return __float2half_rn(x); }
template <> __device__ __forceinline__ float from_f<float>(float x) { return x; }

// One row with LPR lanes, vectorised: N % 8 == 0, ldb % 8 == 0, 16-byte
// aligned B and C rows. Every lane of the group must call it.
template <typename OutT, int LPR>
__device__ __forceinline__ void row_vec(int start, int end, int K, const int *__restrict__ col_idx,
                                        const __half *__restrict__ vals, const __half *__restrict__ B, int ldb,
                                        int N, OutT *__restrict__ Crow, float alpha, float beta, int sub,
                                        unsigned gmask)
{
    constexpr int U = 8; // nonzeros in flight per lane
    for (int nb = 0; nb < N; nb += LPR * 8) {
        const int n0 = nb + sub * 8;
        const bool active = n0 < N;
        const __half *Bn = B + (active ? n0 : 0);
        float acc[8];
#pragma unroll
        for (int i = 0; i < 8; i++) acc[i] = 0.f;

        for (int base = start; base < end; base += LPR) {
            const int j = base + sub;
            int c = -1;
            float a = 0.f;
            if (j < end) {
                c = __ldg(col_idx + j);
                a = __half2float(vals[j]);
                if (c < 0 || c >= K) { c = -1; a = 0.f; }
            }
            const int cnt = min(LPR, end - base);
            int t = 0;
            for (; t + U <= cnt; t += U) {
                uint4 bv[U];
                float av[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int cu = __shfl_sync(gmask, c, t + u, LPR);
                    av[u] = __shfl_sync(gmask, a, t + u, LPR);
                    bv[u] = make_uint4(0, 0, 0, 0);
                    if (active && cu >= 0)
                        bv[u] = __ldg(reinterpret_cast<const uint4 *>(Bn + (size_t)cu * ldb));
                }
#pragma unroll
                for (int u = 0; u < U; u++) fma8(acc, av[u], bv[u]);
            }
            for (; t < cnt; t++) {
                const int cu = __shfl_sync(gmask, c, t, LPR);
                const float au = __shfl_sync(gmask, a, t, LPR);
                if (active && cu >= 0)
                    fma8(acc, au, __ldg(reinterpret_cast<const uint4 *>(Bn + (size_t)cu * ldb)));
            }
        }
        if (active) {
            OutT *cp = Crow + n0;
            float out[8];
            if (beta != 0.f) {
                float old[8];
                load8(cp, old);
#pragma unroll
                for (int i = 0; i < 8; i++) out[i] = fmaf(alpha, acc[i], beta * old[i]);
            } else {
#pragma unroll
                for (int i = 0; i < 8; i++) out[i] = alpha * acc[i];
            }
            store8(cp, out);
        }
    }
}

// One row with a full warp, scalar: any N, leading dimension and alignment.
template <typename OutT>
__device__ __forceinline__ void row_scalar(int start, int end, int K, const int *__restrict__ col_idx,
                                           const __half *__restrict__ vals, const __half *__restrict__ B,
                                           int ldb, int N, OutT *__restrict__ Crow, float alpha, float beta,
                                           int lane)
{
    for (int nb = 0; nb < N; nb += 32) {
        const int n = nb + lane;
        float acc = 0.f;
        for (int base = start; base < end; base += 32) {
            const int j = base + lane;
            int c = -1;
            float a = 0.f;
            if (j < end) {
                c = col_idx[j];
                a = __half2float(vals[j]);
                if (c < 0 || c >= K) { c = -1; a = 0.f; }
            }
            const int cnt = min(32, end - base);
            for (int t = 0; t < cnt; t++) {
                const int cu = __shfl_sync(0xffffffffu, c, t);
                const float au = __shfl_sync(0xffffffffu, a, t);
                if (n < N && cu >= 0)
                    acc = fmaf(au, __half2float(B[(size_t)cu * ldb + n]), acc);
            }
        }
        if (n < N) {
            float o = alpha * acc;
            if (beta != 0.f) o = fmaf(beta, to_f<OutT>(Crow[n]), o);
            Crow[n] = from_f<OutT>(o);
        }
    }
}

__device__ __forceinline__ void clamp_range(int &start, int &end, int nnz)
{
    start = max(0, min(start, nnz));
    end = max(start, min(end, nnz));
}

// Plan-free: group g of LPR lanes computes caller row g.
template <typename OutT, int LPR>
__global__ void __launch_bounds__(256)
spmm_csr_vec_kernel(const int *__restrict__ row_ptr, const int *__restrict__ col_idx,
                    const __half *__restrict__ vals, int M, int K, int nnz,
                    const __half *__restrict__ B, int ldb, int N,
                    OutT *__restrict__ C, int ldc, float alpha, float beta, unsigned flags)
{
    const int lane = threadIdx.x & 31;
    const int sub = lane & (LPR - 1);
    const long long group = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / LPR;
    const unsigned gmask = (LPR == 32) ? 0xffffffffu : (((1u << LPR) - 1u) << (lane & ~(LPR - 1)));
    if (group >= M)
        return; // the whole group leaves together
    const int r = (int)group;
    int start = row_ptr[r], end = row_ptr[r + 1];
    clamp_range(start, end, nnz);
    if (start == end && (flags & TCA_FLAG_KEEP_EMPTY_ROWS))
        return;
    row_vec<OutT, LPR>(start, end, K, col_idx, vals, B, ldb, N, C + (size_t)r * ldc, alpha, beta, sub, gmask);
}

template <typename OutT>
__global__ void __launch_bounds__(256)
spmm_csr_scalar_kernel(const int *__restrict__ row_ptr, const int *__restrict__ col_idx,
                       const __half *__restrict__ vals, int M, int K, int nnz,
                       const __half *__restrict__ B, int ldb, int N,
                       OutT *__restrict__ C, int ldc, float alpha, float beta, unsigned flags)
{
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= M)
        return;
    const int r = (int)warp;
    int start = row_ptr[r], end = row_ptr[r + 1];
    clamp_range(start, end, nnz);
    if (start == end && (flags & TCA_FLAG_KEEP_EMPTY_ROWS))
        return;
    row_scalar<OutT>(start, end, K, col_idx, vals, B, ldb, N, C + (size_t)r * ldc, alpha, beta, lane);
}

// Rows of plans, batched and streamed. Every job (one forward of one plan)
// contributes its work items: runs of consecutive sorted rows with about
// kItemNnz nonzeros in total. A group of L lanes takes one item and streams
// through its nonzeros -- which are contiguous in the plan's re-ordered CSR --
// with U = 8 independent 16-byte B loads in flight per lane, flushing a row's
// accumulators to C[perm[row]] whenever the stream crosses a row end. Short
// rows thus cost no dependent load chain per row, and a launch keeps
// thousands of items in flight.
constexpr int kMaxCcJobs = 32;

struct CcJob {
    const int2 *items;
    const int *perm, *p_row_ptr, *p_col;
    const __half *p_val;
    const __half *B;
    void *C;
    // E4M3 forward: values, B (row stride ldq bytes) and their scales
    const uint8_t *p_val8, *Bq;
    const float *row_scale, *col_scale;
    int ldq;
    int n_items;
    int M, K, N, ldb, ldc;
    float alpha, beta;
    unsigned flags;
};

// A launch's jobs; the stream kernel is also built for CAP = 1, whose
// parameter block launches faster for a single forward.
template <int CAP>
struct CcBatchT {
    int n_jobs;
    int block_start[CAP + 1]; // first block of each job (spmm_cc_items_kernel)
    int item_start[CAP + 1];  // first item of each job in the flattened list (spmm_cc_stream_kernel)
    CcJob job[CAP];
};
using CcBatch = CcBatchT<kMaxCcJobs>;

template <typename OutT, int L, bool VEC>
__global__ void __launch_bounds__(256) spmm_cc_items_kernel(const __grid_constant__ CcBatch b)
{
    constexpr int G = 256 / L;      // groups per block
    constexpr int W = VEC ? 8 : 1;  // output columns per lane per pass
    constexpr int U = 8;            // B loads in flight per lane
    __shared__ int s_rs[G][kItemRows + 1];
    __shared__ int s_out[G][kItemRows];
    const int lane = threadIdx.x & 31;
    const int sub = lane & (L - 1);
    const int g = (int)threadIdx.x / L;
    const unsigned gmask = (L == 32) ? 0xffffffffu : (((1u << L) - 1u) << (lane & ~(L - 1)));
    int j = 0;
    while (j + 1 < b.n_jobs && b.block_start[j + 1] <= (int)blockIdx.x) j++;
    const CcJob &a = b.job[j];
    const int item = ((int)blockIdx.x - b.block_start[j]) * G + g;
    if (item >= a.n_items)
        return; // whole group
    const int2 it = a.items[item];
    const int r0 = it.x, nrows = it.y - it.x;
    for (int k = sub; k <= nrows; k += L) {
        s_rs[g][k] = a.p_row_ptr[r0 + k];
        if (k < nrows)
            s_out[g][k] = a.perm[r0 + k];
    }
    __syncwarp(gmask);
    const int j0 = s_rs[g][0], j1 = s_rs[g][nrows];
    const bool keep = (a.flags & TCA_FLAG_KEEP_EMPTY_ROWS) != 0;

    for (int nb = 0; nb < a.N; nb += L * W) {
        const int n0 = nb + sub * W;
        const bool active = n0 < a.N;
        float acc[W];
#pragma unroll
        for (int i = 0; i < W; i++) acc[i] = 0.f;
        int cr = 0;
        int ce = s_rs[g][1];
        auto flush = [&]() {
            const bool empty_row = s_rs[g][cr] == ce;
            if (active && !(keep && empty_row)) {
                OutT *cp = reinterpret_cast<OutT *>(a.C) + (size_t)s_out[g][cr] * a.ldc + n0;
                float out[W];
                if (a.beta != 0.f) {
                    float old[W];
                    if constexpr (VEC) load8(cp, old); else old[0] = to_f<OutT>(*cp);
#pragma unroll
                    for (int i = 0; i < W; i++) out[i] = fmaf(a.alpha, acc[i], a.beta * old[i]);
                } else {
#pragma unroll
                    for (int i = 0; i < W; i++) out[i] = a.alpha * acc[i];
                }
                if constexpr (VEC) store8(cp, out); else *cp = from_f<OutT>(out[0]);
            }
#pragma unroll
            for (int i = 0; i < W; i++) acc[i] = 0.f;
            cr++;
            ce = (cr < nrows) ? s_rs[g][cr + 1] : 0x7fffffff;
        };
        const __half *Bn = a.B + (active ? n0 : 0);
        for (int base = j0; base < j1; base += L) {
            const int jj = base + sub;
            int c = -1;
            float v = 0.f;
            if (jj < j1) {
                c = __ldg(a.p_col + jj);
                v = __half2float(a.p_val[jj]);
            }
            const int cnt = min(L, j1 - base);
            for (int t = 0; t < cnt; t += U) {
                uint4 bv[U];
                float av[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int cu = __shfl_sync(gmask, c, (t + u) & (L - 1), L);
                    av[u] = __shfl_sync(gmask, v, (t + u) & (L - 1), L);
                    bv[u] = make_uint4(0, 0, 0, 0);
                    if (active && t + u < cnt) {
                        if constexpr (VEC)
                            bv[u] = __ldg(reinterpret_cast<const uint4 *>(Bn + (size_t)cu * a.ldb));
                        else
                            bv[u].x = __half_as_ushort(Bn[(size_t)cu * a.ldb]);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    if (t + u < cnt) { // uniform across the group
                        while (base + t + u >= ce) flush();
                        if constexpr (VEC) {
                            fma8(acc, av[u], bv[u]);
                        } else {
                            acc[0] = fmaf(av[u], __half2float(__ushort_as_half((unsigned short)bv[u].x)), acc[0]);
                        }
                    }
                }
            }
        }
        while (cr < nrows) flush();
    }
}

// ---------------------------------------------------------------------------
// Vectorised item stream: one warp per stream of items, persistent.
//
// Warp w takes items w, w + n_warps, ... of the flattened item list of all
// jobs. Each item's metadata is fetched by a three-deep software pipeline so
// that no dependent load chain is exposed between items: while item i is
// computed, the nonzeros (column, value) of item i+1, the row offsets and
// output rows of item i+2 and the descriptor of item i+3 are in flight.
// Lane k holds row offset k and output row k of its item and nonzero k of its
// first 32; every lane owns W consecutive output columns (W halves of B per
// load, 8 loads in flight per lane) and accumulates with mixed-precision FMA
// (FP16 x FP16 + FP32, one rounding -- the same value as converting both
// factors to FP32 and using fmaf).
// ---------------------------------------------------------------------------
template <int W> struct HalfVec;
template <> struct HalfVec<8> { using T = uint4; };
template <> struct HalfVec<4> { using T = uint2; };
template <> struct HalfVec<2> { using T = unsigned; };

using ptx::fma_f16_f32;

template <int W> __device__ __forceinline__ void load_out(const __half *p, float *v)
{
    using V = typename HalfVec<W>::T;
    const V u = *reinterpret_cast<const V *>(p);
    const __half *h = reinterpret_cast<const __half *>(&u);
#pragma unroll
    for (int i = 0; i < W; i++) v[i] = __half2float(h[i]);
}
template <int W> __device__ __forceinline__ void load_out(const float *p, float *v)
{
#pragma unroll
    for (int i = 0; i < W; i += 2) {
        const float2 f = reinterpret_cast<const float2 *>(p)[i / 2];
        v[i] = f.x;
        v[i + 1] = f.y;
    }
}
template <int W> __device__ __forceinline__ void store_out(__half *p, const float *v)
{
    using V = typename HalfVec<W>::T;
    V u;
    __half2 *h = reinterpret_cast<__half2 *>(&u);
#pragma unroll
    for (int i = 0; i < W / 2; i++) h[i] = __floats2half2_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<V *>(p) = u;
}
template <int W> __device__ __forceinline__ void store_out(float *p, const float *v)
{
    if constexpr (W >= 4) {
#pragma unroll
        for (int i = 0; i < W; i += 4)
            reinterpret_cast<float4 *>(p)[i / 4] = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
    } else {
        *reinterpret_cast<float2 *>(p) = make_float2(v[0], v[1]);
    }
}

struct ItemDesc {
    int job, r0, nrows; // nrows == 0: no item
};

template <typename Batch>
__device__ __forceinline__ ItemDesc load_desc(const Batch &b, int item)
{
    ItemDesc d{0, 0, 0};
    if (item < b.item_start[b.n_jobs]) {
        int j = 0, hi = b.n_jobs - 1; // the last job whose first item is <= item
        while (j < hi) {
            const int mid = (j + hi + 1) >> 1;
            if (b.item_start[mid] <= item)
                j = mid;
            else
                hi = mid - 1;
        }
        const int2 it = __ldg(b.job[j].items + (item - b.item_start[j]));
        d.job = j;
        d.r0 = it.x;
        d.nrows = it.y - it.x;
    }
    return d;
}

// B vectors of W elements: W halves, or W E4M3 bytes.
template <int W, bool F8> struct BVec { using T = typename HalfVec<W>::T; };
template <> struct BVec<8, true> { using T = uint2; };
template <> struct BVec<4, true> { using T = unsigned; };
template <> struct BVec<2, true> { using T = unsigned short; };

// One output row's W columns: t = acc (E4M3: x row scale sa x column scales
// sb), then alpha t + beta C.
template <typename OutT, int W, bool F8>
__device__ __forceinline__ void store_row(const CcJob &a, int orow, int n0, const float *acc, float sa,
                                          const float *sb)
{
    OutT *cp = reinterpret_cast<OutT *>(a.C) + (size_t)orow * a.ldc + n0;
    float t[W], o[W];
#pragma unroll
    for (int i = 0; i < W; i++) {
        if constexpr (F8)
            t[i] = acc[i] * (sa * sb[i]);
        else
            t[i] = acc[i];
    }
    if (a.beta != 0.f) {
        float old[W];
        load_out<W>(cp, old);
#pragma unroll
        for (int i = 0; i < W; i++) o[i] = fmaf(a.alpha, t[i], a.beta * old[i]);
    } else {
#pragma unroll
        for (int i = 0; i < W; i++) o[i] = a.alpha * t[i];
    }
    store_out<W>(cp, o);
}

// acc[i] = v * b[i] + acc[i] over one B vector (E4M3 pairs unpacked to FP16).
template <int W, bool F8, typename V>
__device__ __forceinline__ void fma_vec(float *acc, unsigned short v, const V &bv)
{
    if constexpr (F8) {
        const __nv_fp8x2_storage_t *q = reinterpret_cast<const __nv_fp8x2_storage_t *>(&bv);
#pragma unroll
        for (int i = 0; i < W / 2; i++) {
            const __half2_raw h = __nv_cvt_fp8x2_to_halfraw2(q[i], __NV_E4M3);
            acc[2 * i] = fma_f16_f32(v, h.x, acc[2 * i]);
            acc[2 * i + 1] = fma_f16_f32(v, h.y, acc[2 * i + 1]);
        }
    } else {
        const unsigned short *h = reinterpret_cast<const unsigned short *>(&bv);
#pragma unroll
        for (int i = 0; i < W; i++) acc[i] = fma_f16_f32(v, h[i], acc[i]);
    }
}

// F8: values and B are E4M3 (every E4M3 value is an FP16 value, so the
// products are formed exactly by the same mixed-precision FMA); the flush
// multiplies the FP32 sum by row scale x column scale, as the tensor-core
// epilogue does.
//
// Three blocks per SM (80 registers a thread). Beside the tensor-core
// kernel's block one of them is resident at a time (a warp's registers come
// from its SM sub-partition, and the tensor-core warps leave room for two
// more warps per sub-partition). U B loads are in flight per lane: 8, or 4
// at W = 8, which keeps the register budget without spills.
template <typename OutT, int W, bool F8, int CAP = kMaxCcJobs>
__global__ void __launch_bounds__(256, 3) spmm_cc_stream_kernel(const __grid_constant__ CcBatchT<CAP> b)
{
    using V = typename BVec<W, F8>::T;
    constexpr int U = W == 8 ? 4 : 8;
    // Launched as a programmatic dependent (beside the tensor-core kernel, or
    // behind another CUDA-core launch): let the next launch start as well.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int n_warps = (int)gridDim.x * 8;
    int item = (int)blockIdx.x * 8 + (int)(threadIdx.x >> 5);

    // row offsets (lane k <= nrows), output rows and E4M3 row scales (lane k < nrows) of an item
    auto load_rows = [&](const ItemDesc &d, int &rs, int &orow, float &sc) {
        rs = 0;
        orow = 0;
        sc = 0.f;
        if (lane <= d.nrows && d.nrows > 0) {
            const CcJob &a = b.job[d.job];
            rs = __ldg(a.p_row_ptr + d.r0 + lane);
            if (lane < d.nrows) {
                orow = __ldg(a.perm + d.r0 + lane);
                if constexpr (F8)
                    sc = __ldg(a.row_scale + d.r0 + lane);
            }
        }
    };
    auto value = [&](const CcJob &a, int j) -> unsigned short {
        if constexpr (F8)
            return __nv_cvt_fp8_to_halfraw((__nv_fp8_storage_t)a.p_val8[j], __NV_E4M3).x;
        else
            return __half_as_ushort(a.p_val[j]);
    };
    // the item's first 32 nonzeros, one per lane (values as FP16 bits)
    auto load_nz = [&](const ItemDesc &d, int rs, int &col, unsigned short &val) {
        const int j0 = __shfl_sync(full, rs, 0), j1 = __shfl_sync(full, rs, d.nrows & 31);
        col = 0;
        val = 0;
        if (d.nrows > 0 && j0 + lane < j1) {
            const CcJob &a = b.job[d.job];
            col = __ldg(a.p_col + j0 + lane);
            val = value(a, j0 + lane);
        }
    };

    ItemDesc d0 = load_desc(b, item), d1 = load_desc(b, item + n_warps), d2 = load_desc(b, item + 2 * n_warps);
    int rs0, out0, rs1, out1, col0;
    float sc0, sc1;
    unsigned short val0;
    load_rows(d0, rs0, out0, sc0);
    load_rows(d1, rs1, out1, sc1);
    load_nz(d0, rs0, col0, val0);

    while (d0.nrows > 0) {
        // ---- pipeline: nonzeros of i+1, rows of i+2, descriptor of i+3
        int col1;
        unsigned short val1;
        load_nz(d1, rs1, col1, val1);
        int rs2, out2;
        float sc2;
        load_rows(d2, rs2, out2, sc2);
        const ItemDesc d3 = load_desc(b, item + 3 * n_warps);

        // ---- item i
        const CcJob &a = b.job[d0.job];
        const int nrows = d0.nrows;
        const int j0 = __shfl_sync(full, rs0, 0), j1 = __shfl_sync(full, rs0, nrows);
        const bool keep = (a.flags & TCA_FLAG_KEEP_EMPTY_ROWS) != 0;
        // Items whose rows hold one nonzero each (the short-row tails of skewed
        // matrices): C[row] = alpha v B[col] (+ beta C[row]) row by row, with U
        // rows' B vectors in flight and no row-boundary tracking.
        const int rs_next = __shfl_down_sync(full, rs0, 1);
        const bool singles = __all_sync(full, lane >= nrows || rs_next - rs0 == 1);
        for (int nb = 0; singles && nb < a.N; nb += 32 * W) {
            const int n0 = nb + lane * W;
            const bool active = n0 < a.N;
            const uint8_t *Bn = F8 ? a.Bq + (active ? n0 : 0)
                                   : reinterpret_cast<const uint8_t *>(a.B + (active ? n0 : 0));
            const size_t brow = F8 ? (size_t)a.ldq : (size_t)a.ldb * 2; // bytes per B row
            float sb[F8 ? W : 1];
            if constexpr (F8) {
#pragma unroll
                for (int i = 0; i < W; i++) sb[i] = active ? __ldg(a.col_scale + n0 + i) : 0.f;
            }
            for (int t = 0; t < nrows; t += U) {
                V bv[U];
                unsigned short av[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int r = (t + u) & 31;
                    const int cu = __shfl_sync(full, col0, r);
                    av[u] = (unsigned short)__shfl_sync(full, (int)val0, r);
                    bv[u] = V{};
                    if (active && t + u < nrows)
                        bv[u] = __ldg(reinterpret_cast<const V *>(Bn + (size_t)cu * brow));
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int r = (t + u) & 31;
                    const int orow = __shfl_sync(full, out0, r);
                    float sa = 1.f;
                    if constexpr (F8)
                        sa = __shfl_sync(full, sc0, r);
                    if (active && t + u < nrows) {
                        float acc[W];
#pragma unroll
                        for (int i = 0; i < W; i++) acc[i] = 0.f;
                        fma_vec<W, F8>(acc, av[u], bv[u]);
                        store_row<OutT, W, F8>(a, orow, n0, acc, sa, sb);
                    }
                }
            }
        }
        for (int nb = 0; !singles && nb < a.N; nb += 32 * W) {
            const int n0 = nb + lane * W;
            const bool active = n0 < a.N;
            const uint8_t *Bn = F8 ? a.Bq + (active ? n0 : 0)
                                   : reinterpret_cast<const uint8_t *>(a.B + (active ? n0 : 0));
            const size_t brow = F8 ? (size_t)a.ldq : (size_t)a.ldb * 2; // bytes per B row
            float sb[F8 ? W : 1];
            if constexpr (F8) {
#pragma unroll
                for (int i = 0; i < W; i++) sb[i] = active ? __ldg(a.col_scale + n0 + i) : 0.f;
            }
            float acc[W];
#pragma unroll
            for (int i = 0; i < W; i++) acc[i] = 0.f;
            int cr = 0;
            int ce = __shfl_sync(full, rs0, 1);
            auto flush = [&]() {
                const int rstart = __shfl_sync(full, rs0, cr);
                const int orow = __shfl_sync(full, out0, cr);
                float sa = 1.f;
                if constexpr (F8)
                    sa = __shfl_sync(full, sc0, cr);
                if (active && !(keep && rstart == ce))
                    store_row<OutT, W, F8>(a, orow, n0, acc, sa, sb);
#pragma unroll
                for (int i = 0; i < W; i++) acc[i] = 0.f;
                cr++;
                const int nxt = __shfl_sync(full, rs0, min(cr + 1, 31));
                ce = cr < nrows ? nxt : 0x7fffffff;
            };
            for (int base = j0; base < j1; base += 32) {
                int c = col0;
                unsigned short v = val0;
                if (base != j0) { // a row longer than 32 nonzeros: the rest is loaded here
                    c = 0;
                    v = 0;
                    if (base + lane < j1) {
                        c = __ldg(a.p_col + base + lane);
                        v = value(a, base + lane);
                    }
                }
                const int m = min(32, j1 - base);
                for (int t = 0; t < m; t += U) {
                    V bv[U];
                    unsigned short av[U];
#pragma unroll
                    for (int u = 0; u < U; u++) {
                        const int cu = __shfl_sync(full, c, t + u);
                        av[u] = (unsigned short)__shfl_sync(full, (int)v, t + u);
                        bv[u] = V{};
                        if (active && t + u < m)
                            bv[u] = __ldg(reinterpret_cast<const V *>(Bn + (size_t)cu * brow));
                    }
#pragma unroll
                    for (int u = 0; u < U; u++) {
                        if (t + u < m) { // uniform across the warp
                            while (base + t + u >= ce) flush();
                            fma_vec<W, F8>(acc, av[u], bv[u]);
                        }
                    }
                }
            }
            while (cr < nrows) flush();
        }

        // ---- rotate the pipeline
        d0 = d1; rs0 = rs1; out0 = out1; sc0 = sc1; col0 = col1; val0 = val1;
        d1 = d2; rs1 = rs2; out1 = out2; sc1 = sc2;
        d2 = d3;
        item += n_warps;
    }
    // Complete no earlier than the launch this one depends on (a no-op for an
    // ordinary launch): work after this kernel on the stream then also finds
    // the tensor-core kernel done, whatever the stream's ordering rules for
    // programmatic dependents. That kernel never waits on this one and all of
    // its blocks were resident before this grid started, so the wait ends.
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename OutT, int LPR>
void launch_vec(const int *rp, const int *ci, const __half *v, int M, int K, int nnz, const __half *B, int ldb,
                int N, OutT *C, int ldc, float alpha, float beta, unsigned flags, cudaStream_t s)
{
    const long long threads = (long long)M * LPR;
    const unsigned grid = (unsigned)((threads + 255) / 256);
    spmm_csr_vec_kernel<OutT, LPR><<<grid, 256, 0, s>>>(rp, ci, v, M, K, nnz, B, ldb, N, C, ldc, alpha, beta, flags);
}

inline int pick_lpr(int N) { return N <= 32 ? 4 : N <= 64 ? 8 : N <= 128 ? 16 : 32; }

template <typename OutT>
void dispatch_vec(const int *rp, const int *ci, const __half *v, int M, int K, int nnz, const __half *B, int ldb,
                  int N, OutT *C, int ldc, float alpha, float beta, unsigned flags, cudaStream_t s)
{
    switch (pick_lpr(N)) {
    case 4: launch_vec<OutT, 4>(rp, ci, v, M, K, nnz, B, ldb, N, C, ldc, alpha, beta, flags, s); break;
    case 8: launch_vec<OutT, 8>(rp, ci, v, M, K, nnz, B, ldb, N, C, ldc, alpha, beta, flags, s); break;
    case 16: launch_vec<OutT, 16>(rp, ci, v, M, K, nnz, B, ldb, N, C, ldc, alpha, beta, flags, s); break;
    default: launch_vec<OutT, 32>(rp, ci, v, M, K, nnz, B, ldb, N, C, ldc, alpha, beta, flags, s); break;
    }
}

bool vec_ok(const void *B, int ldb, int N, const void *C, int ldc, int c_dtype)
{
    const size_t c_elem = (c_dtype == TCA_DTYPE_F16) ? 2 : 4;
    return (N % 8 == 0) && (ldb % 8 == 0) && aligned16(B) && aligned16(C) && ((ldc * c_elem) % 16 == 0);
}

} // namespace

int launch_spmm_csr_cc(const int *row_ptr, const int *col_idx, const __half *vals, int M, int K, int nnz,
                       const __half *B, int ldb, int N, void *C, int ldc, int c_dtype,
                       float alpha, float beta, unsigned flags, cudaStream_t stream)
{
    if (vec_ok(B, ldb, N, C, ldc, c_dtype)) {
        if (c_dtype == TCA_DTYPE_F16)
            dispatch_vec<__half>(row_ptr, col_idx, vals, M, K, nnz, B, ldb, N, (__half *)C, ldc, alpha, beta, flags, stream);
        else
            dispatch_vec<float>(row_ptr, col_idx, vals, M, K, nnz, B, ldb, N, (float *)C, ldc, alpha, beta, flags, stream);
    } else {
        const unsigned grid = (unsigned)(((long long)M * 32 + 255) / 256);
        if (c_dtype == TCA_DTYPE_F16)
            spmm_csr_scalar_kernel<__half><<<grid, 256, 0, stream>>>(row_ptr, col_idx, vals, M, K, nnz, B, ldb, N,
                                                                     (__half *)C, ldc, alpha, beta, flags);
        else
            spmm_csr_scalar_kernel<float><<<grid, 256, 0, stream>>>(row_ptr, col_idx, vals, M, K, nnz, B, ldb, N,
                                                                    (float *)C, ldc, alpha, beta, flags);
    }
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

bool dense_operands_vec_ok(const void *B, int ldb, int N, const void *C, int ldc, int c_dtype)
{
    return vec_ok(B, ldb, N, C, ldc, c_dtype);
}

namespace {

template <typename OutT, int LPR, bool VEC>
int launch_cc_group(const CcBatch &b, cudaStream_t s)
{
    if (b.n_jobs == 0 || b.block_start[b.n_jobs] == 0)
        return TCA_OK;
    spmm_cc_items_kernel<OutT, LPR, VEC><<<b.block_start[b.n_jobs], 256, 0, s>>>(b);
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

// ---------------------------------------------------------------------------
// Tensor-core item kernel (mma.sync, FP16): the CUDA-core windows' work items
// as tiny dense products. An item of R <= 31 rows and Z <= 32 nonzeros is
// C_item[R x N] = A_item[R x Z] * B_item[Z x N], where A_item holds each
// nonzero in its own column (row of the nonzero, position in the item) and
// B_item is the item's gathered B rows. Per 64-column slice of N, the warp
// stages B_item in shared memory (32 rows x 128 bytes, 16-byte chunks XOR-
// swizzled by row), reads it with ldmatrix.trans as m16n8k16 B fragments and
// issues 8 mma.sync per 16 rows and 16 nonzeros; A fragments come from the
// nonzeros in lane registers by shuffle. The accumulators go through shared
// memory so that every output row is stored as 128 contiguous bytes. A row
// longer than 32 nonzeros (an item of its own) is walked 32 nonzeros at a
// time into the same accumulators. Per output element this issues about a
// third of the instructions of the shuffle-and-FMA stream kernel; the
// products are exact in FP32 and sums accumulate in FP32.
// ---------------------------------------------------------------------------
constexpr int kMmaWarps = 8;
constexpr int kCcMma = 16; // cc_cols value that selects this kernel
constexpr int kMmaSliceCols = 64;
constexpr int kMmaAccStride = 72; // floats per staged accumulator row (2-way bank conflicts at most)
constexpr int kMmaWarpSmem = 16 * kMmaAccStride * 4; // >= 32 x 128 bytes of B staging

__device__ __forceinline__ void mma_16816(float *d, const uint32_t *a, uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldmatrix_x4_trans(uint32_t addr, uint32_t *r)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

template <typename OutT>
__global__ void __launch_bounds__(kMmaWarps * 32, 2) spmm_cc_mma_kernel(const __grid_constant__ CcBatch b)
{
    __shared__ __align__(16) uint8_t s_all[kMmaWarps * kMmaWarpSmem];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint8_t *ws = s_all + wid * kMmaWarpSmem;
    const uint32_t ws_addr = (uint32_t)__cvta_generic_to_shared(ws);
    float *acc_s = reinterpret_cast<float *>(ws);
    const int n_warps = (int)gridDim.x * kMmaWarps;
    int item = (int)blockIdx.x * kMmaWarps + wid;
    const int g = lane >> 2, c4 = lane & 3;

    auto load_rows = [&](const ItemDesc &d, int &rs, int &orow) {
        rs = 0;
        orow = 0;
        if (lane <= d.nrows && d.nrows > 0) {
            const CcJob &a = b.job[d.job];
            rs = __ldg(a.p_row_ptr + d.r0 + lane);
            if (lane < d.nrows)
                orow = __ldg(a.perm + d.r0 + lane);
        }
    };
    auto load_nz = [&](const ItemDesc &d, int rs, int &col, unsigned short &val) {
        const int j0 = __shfl_sync(full, rs, 0), j1 = __shfl_sync(full, rs, d.nrows & 31);
        col = 0;
        val = 0;
        if (d.nrows > 0 && j0 + lane < j1) {
            const CcJob &a = b.job[d.job];
            col = __ldg(a.p_col + j0 + lane);
            val = __half_as_ushort(a.p_val[j0 + lane]);
        }
    };

    ItemDesc d0 = load_desc(b, item), d1 = load_desc(b, item + n_warps), d2 = load_desc(b, item + 2 * n_warps);
    int rs0, out0, rs1, out1, col0;
    unsigned short val0;
    load_rows(d0, rs0, out0);
    load_rows(d1, rs1, out1);
    load_nz(d0, rs0, col0, val0);

    while (d0.nrows > 0) {
        int col1;
        unsigned short val1;
        load_nz(d1, rs1, col1, val1);
        int rs2, out2;
        load_rows(d2, rs2, out2);
        const ItemDesc d3 = load_desc(b, item + 3 * n_warps);

        const CcJob &a = b.job[d0.job];
        const int R = d0.nrows;
        const int j0 = __shfl_sync(full, rs0, 0), j1 = __shfl_sync(full, rs0, R);
        const int Z = j1 - j0;
        const int G = R > 16 ? 2 : 1; // 16-row groups
        const bool keep = (a.flags & TCA_FLAG_KEEP_EMPTY_ROWS) != 0;
        // local row of this lane's nonzero (rows of an item are consecutive)
        int rz = 0;
        for (int r = 1; r < R; r++) rz += (lane >= __shfl_sync(full, rs0, r) - j0) ? 1 : 0;

        for (int n0 = 0; n0 < a.N; n0 += kMmaSliceCols) {
            float acc[2][8][4];
#pragma unroll
            for (int gg = 0; gg < 2; gg++)
#pragma unroll
                for (int t = 0; t < 8; t++)
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[gg][t][q] = 0.f;
            for (int kb = 0; kb < Z; kb += 32) {
                int col = col0, zr = rz;
                unsigned short val = val0;
                if (kb > 0) { // a row longer than 32 nonzeros: its next 32
                    col = 0;
                    val = 0;
                    zr = 0;
                    if (kb + lane < Z) {
                        col = __ldg(a.p_col + j0 + kb + lane);
                        val = __half_as_ushort(a.p_val[j0 + kb + lane]);
                    }
                }
                const int zc = min(32, Z - kb);
                // stage B rows z = 4 i + lane / 8, 16-byte chunk lane % 8 of the slice
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int z = 4 * i + (lane >> 3), q = lane & 7;
                    const int cz = __shfl_sync(full, col, z);
                    uint4 v = make_uint4(0, 0, 0, 0);
                    if (z < zc && n0 + 8 * q < a.N)
                        v = __ldg(reinterpret_cast<const uint4 *>(a.B + (size_t)cz * a.ldb + n0 + 8 * q));
                    *reinterpret_cast<uint4 *>(ws + z * 128 + ((q ^ (z & 7)) << 4)) = v;
                }
                __syncwarp();
#pragma unroll
                for (int ks = 0; ks < 2; ks++) {
                    if (16 * ks >= zc)
                        break; // uniform
                    // A fragments: k = 16 ks + 2 c4 + {0, 1} (+ 8); rows 16 gg + g (+ 8)
                    uint32_t af[2][4];
                    int kk[4] = {16 * ks + 2 * c4, 16 * ks + 2 * c4 + 1, 16 * ks + 2 * c4 + 8, 16 * ks + 2 * c4 + 9};
                    int rk[4];
                    unsigned short vk[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        rk[u] = __shfl_sync(full, zr, kk[u]);
                        vk[u] = (unsigned short)__shfl_sync(full, (int)val, kk[u]);
                        if (kk[u] >= zc) rk[u] = -1;
                    }
#pragma unroll
                    for (int gg = 0; gg < 2; gg++) {
                        const int r_lo = 16 * gg + g, r_hi = r_lo + 8;
                        auto pk = [&](int u0, int u1, int row) -> uint32_t {
                            const uint32_t lo = rk[u0] == row ? vk[u0] : 0u;
                            const uint32_t hi = rk[u1] == row ? vk[u1] : 0u;
                            return lo | (hi << 16);
                        };
                        af[gg][0] = pk(0, 1, r_lo);
                        af[gg][1] = pk(0, 1, r_hi);
                        af[gg][2] = pk(2, 3, r_lo);
                        af[gg][3] = pk(2, 3, r_hi);
                    }
#pragma unroll
                    for (int p = 0; p < 4; p++) {
                        const int mi = lane >> 3;
                        const int krow = 16 * ks + (lane & 7) + (mi & 1) * 8;
                        const int nch = 2 * p + (mi >> 1);
                        uint32_t bf[4];
                        ldmatrix_x4_trans(ws_addr + krow * 128 + ((nch ^ (krow & 7)) << 4), bf);
                        mma_16816(acc[0][2 * p], af[0], bf[0], bf[1]);
                        mma_16816(acc[0][2 * p + 1], af[0], bf[2], bf[3]);
                        if (G == 2) {
                            mma_16816(acc[1][2 * p], af[1], bf[0], bf[1]);
                            mma_16816(acc[1][2 * p + 1], af[1], bf[2], bf[3]);
                        }
                    }
                }
            }
            // ---- epilogue of the slice, per 16-row group, through shared memory
#pragma unroll
            for (int gg = 0; gg < 2; gg++) {
                if (gg >= G)
                    break;
                __syncwarp();
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    *reinterpret_cast<float2 *>(acc_s + g * kMmaAccStride + 8 * t + 2 * c4) =
                        make_float2(acc[gg][t][0], acc[gg][t][1]);
                    *reinterpret_cast<float2 *>(acc_s + (g + 8) * kMmaAccStride + 8 * t + 2 * c4) =
                        make_float2(acc[gg][t][2], acc[gg][t][3]);
                }
                __syncwarp();
                const int rows = min(16, R - 16 * gg);
                for (int i = 0; 4 * i < rows; i++) {
                    const int rl = 4 * i + (lane >> 3); // row within the group
                    const int r = 16 * gg + rl;          // row within the item
                    const int orow = __shfl_sync(full, out0, r & 31);
                    const int rstart = __shfl_sync(full, rs0, r & 31), rend = __shfl_sync(full, rs0, (r + 1) & 31);
                    const int n = n0 + (lane & 7) * 8;
                    if (rl < rows && n < a.N && !(keep && rstart == rend)) {
                        const float4 v0 = *reinterpret_cast<const float4 *>(acc_s + rl * kMmaAccStride + (lane & 7) * 8);
                        const float4 v1 =
                            *reinterpret_cast<const float4 *>(acc_s + rl * kMmaAccStride + (lane & 7) * 8 + 4);
                        const float v[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
                        OutT *cp = reinterpret_cast<OutT *>(a.C) + (size_t)orow * a.ldc + n;
                        float o[8];
                        if (a.beta != 0.f) {
                            float old[8];
                            load_out<8>(cp, old);
#pragma unroll
                            for (int q = 0; q < 8; q++) o[q] = fmaf(a.alpha, v[q], a.beta * old[q]);
                        } else {
#pragma unroll
                            for (int q = 0; q < 8; q++) o[q] = a.alpha * v[q];
                        }
                        store_out<8>(cp, o);
                    }
                }
            }
        }

        d0 = d1; rs0 = rs1; out0 = out1; col0 = col1; val0 = val1;
        d1 = d2; rs1 = rs2; out1 = out2;
        d2 = d3;
        item += n_warps;
    }
}

// Persistent grid of the stream kernel: enough warps for every item, at most
// the resident blocks of all SMs.
// beside_regs > 0: the launch directly follows a tensor-core launch whose
// one block per SM holds that many registers. It is issued as a programmatic
// dependent of that launch (which triggers at entry), so its blocks start as
// soon as the tensor-core blocks are resident, and its grid is cut to the
// blocks that the SM's registers as a whole leave beside them (two per SM:
// the first starts at once, the second when the first ends -- measured
// faster than both a wider first block and claiming items from a counter
// with more blocks). The kernel reads nothing the tensor-core kernel writes,
// so it never waits on it.
template <typename OutT, int W, bool F8, int CAP>
int launch_stream_cap(const CcBatchT<CAP> &b, int beside_regs, cudaStream_t s)
{
    const int total = b.item_start[b.n_jobs];
    if (b.n_jobs == 0 || total == 0)
        return TCA_OK;
    static int per_sm = 0, regs = 0;
    if (per_sm == 0) {
        int n = 0;
        TCA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, spmm_cc_stream_kernel<OutT, W, F8, CAP>, 256, 0));
        TCA_TRY(block_regs((const void *)spmm_cc_stream_kernel<OutT, W, F8, CAP>, 256, &regs));
        per_sm = n > 0 ? n : 1;
    }
    const int fit = beside_regs > 0 ? std::max(1, std::min(per_sm, (kSmRegs - beside_regs) / regs)) : per_sm;
    const int grid = std::min((total + 7) / 8, kSMs * fit);
    if (beside_regs > 0) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)grid);
        cfg.blockDim = dim3(256);
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        TCA_CUDA_TRY(cudaLaunchKernelEx(&cfg, spmm_cc_stream_kernel<OutT, W, F8, CAP>, b));
        return TCA_OK;
    }
    spmm_cc_stream_kernel<OutT, W, F8, CAP><<<grid, 256, 0, s>>>(b);
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

template <typename OutT, int W, bool F8>
int launch_stream_group(const CcBatch &b, int beside_regs, cudaStream_t s)
{
    if (b.n_jobs == 1) {
        CcBatchT<1> one;
        one.n_jobs = 1;
        one.block_start[0] = b.block_start[0];
        one.block_start[1] = b.block_start[1];
        one.item_start[0] = b.item_start[0];
        one.item_start[1] = b.item_start[1];
        one.job[0] = b.job[0];
        return launch_stream_cap<OutT, W, F8, 1>(one, beside_regs, s);
    }
    return launch_stream_cap<OutT, W, F8, kMaxCcJobs>(b, beside_regs, s);
}

template <typename OutT>
int launch_mma_group(const CcBatch &b, cudaStream_t s)
{
    const int total = b.item_start[b.n_jobs];
    if (b.n_jobs == 0 || total == 0)
        return TCA_OK;
    static int per_sm = 0;
    if (per_sm == 0) {
        int n = 0;
        TCA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, spmm_cc_mma_kernel<OutT>, kMmaWarps * 32, 0));
        per_sm = n > 0 ? n : 1;
    }
    const int grid = std::min((total + kMmaWarps - 1) / kMmaWarps, kSMs * per_sm);
    spmm_cc_mma_kernel<OutT><<<grid, kMmaWarps * 32, 0, s>>>(b);
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

// Columns per lane of the stream kernel: 8 for N > 128, 4 for N > 64, else 2.
inline int pick_w(int N) { return N > 128 ? 8 : N > 64 ? 4 : 2; }

template <typename OutT, bool F8>
int launch_stream_w(const CcBatch &b, int w, int beside_regs, cudaStream_t s)
{
    switch (w) {
    case 2: return launch_stream_group<OutT, 2, F8>(b, beside_regs, s);
    case 4: return launch_stream_group<OutT, 4, F8>(b, beside_regs, s);
    default: return launch_stream_group<OutT, 8, F8>(b, beside_regs, s);
    }
}

template <typename OutT>
int launch_cc_typed(const CcBatch &b, int w, bool vec, bool f8, int beside_regs, cudaStream_t s)
{
    if (!vec) return launch_cc_group<OutT, 32, false>(b, s);
    if (w == kCcMma) return launch_mma_group<OutT>(b, s);
    return f8 ? launch_stream_w<OutT, true>(b, w, beside_regs, s) : launch_stream_w<OutT, false>(b, w, beside_regs, s);
}

} // namespace

int launch_cc_jobs(const SpmmJob *jobs, int n_jobs, int c_dtype, float alpha, float beta, unsigned flags,
                   cudaStream_t s, LaunchList *defer, int beside_regs)
{
    // groups: (columns per lane, vectorised, E4M3) -- stream kernel with 2/4/8 columns, scalar items
    // and the FP16 tensor-core item kernel (kCcMma)
    const int kinds[8][3] = {{2, 1, 0}, {4, 1, 0}, {8, 1, 0}, {kCcMma, 1, 0}, {32, 0, 0}, {2, 1, 1}, {4, 1, 1}, {8, 1, 1}};
    for (const auto &kd : kinds) {
        CcBatch b;
        b.n_jobs = 0;
        b.block_start[0] = 0;
        b.item_start[0] = 0;
        auto flush = [&]() -> int {
            if (b.n_jobs == 0)
                return TCA_OK;
            const int w = kd[0];
            const bool vec = kd[1] != 0, f8 = kd[2] != 0;
            auto run = [c_dtype, w, vec, f8, beside_regs](const CcBatch &bb, cudaStream_t st) {
                return (c_dtype == TCA_DTYPE_F16) ? launch_cc_typed<__half>(bb, w, vec, f8, beside_regs, st)
                                                  : launch_cc_typed<float>(bb, w, vec, f8, beside_regs, st);
            };
            int status = TCA_OK;
            if (defer) {
                auto held = std::make_shared<CcBatch>(b);
                defer->push_back([held, run](cudaStream_t st) { return run(*held, st); });
            } else {
                status = run(b, s);
            }
            b.n_jobs = 0;
            return status;
        };
        for (int i = 0; i < n_jobs; i++) {
            const SpmmJob &sj = jobs[i];
            const tca_plan *p = sj.p;
            const int n_items = sj.tc ? p->n_cc_items : p->n_all_items;
            if (n_items == 0 || sj.N <= 0)
                continue;
            // E4M3 jobs always qualify (B is the library's own aligned copy; C was checked)
            const bool vec = sj.f8 || vec_ok(sj.B, sj.ldb, sj.N, sj.C, sj.ldc, c_dtype);
            int lpr = 32;
            if (vec) {
                lpr = (sj.cc_w == 2 || sj.cc_w == 4 || sj.cc_w == 8) ? sj.cc_w : pick_w(sj.N);
                if (sj.cc_w == kCcMma && !sj.f8)
                    lpr = kCcMma;
            }
            if (lpr != kd[0] || (vec ? 1 : 0) != kd[1] || (sj.f8 ? 1 : 0) != kd[2])
                continue;
            CcJob &a = b.job[b.n_jobs];
            a.items = sj.tc ? p->cc_items : p->all_items;
            a.perm = p->perm;
            a.p_row_ptr = p->p_row_ptr;
            a.p_col = p->p_col;
            a.p_val = p->p_val;
            a.B = sj.B;
            a.C = sj.C;
            a.p_val8 = p->p_val_f8;
            a.Bq = sj.Bq;
            a.row_scale = p->row_scale;
            a.col_scale = sj.col_scale;
            a.ldq = sj.ldq;
            a.n_items = n_items;
            a.M = p->M;
            a.K = p->K;
            a.N = sj.N;
            a.ldb = sj.ldb;
            a.ldc = sj.ldc;
            a.alpha = alpha;
            a.beta = beta;
            a.flags = flags;
            const int per_block = vec ? 8 : 256 / lpr;
            b.block_start[b.n_jobs + 1] = b.block_start[b.n_jobs] + (a.n_items + per_block - 1) / per_block;
            b.item_start[b.n_jobs + 1] = b.item_start[b.n_jobs] + a.n_items;
            b.n_jobs++;
            if (b.n_jobs == kMaxCcJobs)
                TCA_TRY(flush());
        }
        TCA_TRY(flush());
    }
    return TCA_OK;
}

} // namespace tca
