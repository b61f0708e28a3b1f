// adjoint.cu -- the adjoints of Y = A B for a sparse A (pattern fixed by a
// plan): dA = (dY B^T) sampled on A's pattern (SDDMM) and dB = A^T dY
// (transpose SpMM). The reference has no backward pass; these follow from the
// forward's definition (src/our_spmm.cu:290-346: Y[r, :] = sum_j a_j B[c_j, :]):
//   dL/da_j   = sum_n dY[r_j, n] * B[c_j, n]
//   dL/dB[c,:] = sum_{j: c_j = c} a_j * dY[r_j, :]
//
// dB reuses the forward machinery on a plan of A^T, built on the GPU: the
// entries are sorted by the 64-bit key (column, original row) with a stable
// radix sort, so A^T's CSR -- and hence its plan -- is deterministic.
//
// dA on the tensor-core windows is a tcgen05 kernel of its own
// (sddmm_tc.cu): per window and chunk the tile dY[window rows] B[chunk
// columns]^T, of which the epilogue writes the nonzeros. The rows of the
// CUDA-core windows (too sparse for tiles) take a warp per row that streams
// the row of dY against the B rows of its nonzeros (L2-bound).
#include <cub/cub.cuh>
#include <vector>
#include "tca_internal.cuh"
#include "plan.cuh"

namespace tca {
namespace {

// Original row of each entry in sorted (plan) order, and the 64-bit key
// (col << 32 | original row) of each caller nonzero index.
__global__ void k_transpose_keys(const int *__restrict__ perm, const int *__restrict__ p_row_ptr,
                                 const int *__restrict__ p_col, const int *__restrict__ src, int M,
                                 unsigned long long *__restrict__ keys, int *__restrict__ vals)
{
    const int lane = threadIdx.x & 31;
    const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= M)
        return;
    const unsigned long long r = (unsigned)perm[i];
    for (int j = p_row_ptr[i] + lane; j < p_row_ptr[i + 1]; j += 32) {
        keys[j] = ((unsigned long long)(unsigned)p_col[j] << 32) | r;
        vals[j] = src[j];
    }
}

// A^T CSR from the sorted keys: column index = original row; row counts by
// atomics (order-free integer sums); values gathered from the caller's array.
__global__ void k_transpose_fill(const unsigned long long *__restrict__ keys, const int *__restrict__ order,
                                 const __half *__restrict__ vals, int nnz, int *__restrict__ t_count,
                                 int *__restrict__ t_col, __half *__restrict__ t_val, int *__restrict__ t_src)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnz)
        return;
    const unsigned long long k = keys[i];
    const int c = (int)(k >> 32);
    atomicAdd(&t_count[c], 1);
    t_col[i] = (int)(k & 0xffffffffull);
    t_src[i] = order[i];
    t_val[i] = vals[order[i]];
}

__global__ void k_scatter_half(const int *__restrict__ idx, const __half *__restrict__ src, __half *__restrict__ dst,
                               int n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[idx[i]] = src[i];
}

__global__ void k_gather_half(const int *__restrict__ idx, const __half *__restrict__ src, __half *__restrict__ dst,
                              int n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = src[idx[i]];
}

// Sorted row of warp w: w itself, or with a window list (the CUDA-core
// windows) row w % 128 of window windows[w / 128]; -1 past the rows.
__device__ __forceinline__ long long sddmm_row(long long w, const int *windows, long long n_rows, int M)
{
    if (w >= n_rows)
        return -1;
    if (!windows)
        return w;
    const long long i = (long long)windows[w >> 7] * 128 + (w & 127);
    return i < M ? i : -1;
}

// SDDMM, vectorised (N % 8 == 0, 16-byte aligned rows): one warp per sorted
// row; 8 nonzeros in flight per lane, each lane covering 8 columns of every
// 256-column slice; a warp-wide reduction per nonzero.
template <typename OutT>
__global__ void __launch_bounds__(256)
k_sddmm_vec(const int *__restrict__ perm, const int *__restrict__ p_row_ptr, const int *__restrict__ p_col,
            const int *__restrict__ src, int M, const int *__restrict__ windows, long long n_rows,
            const __half *__restrict__ dY, int ldy, const __half *__restrict__ B, int ldb, int N,
            OutT *__restrict__ out, float alpha)
{
    constexpr int U = 8;
    const int lane = threadIdx.x & 31;
    const long long i = sddmm_row(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, windows, n_rows, M);
    if (i < 0)
        return;
    const __half *y = dY + (size_t)perm[i] * ldy;
    const int j0 = p_row_ptr[i], j1 = p_row_ptr[i + 1];
    for (int jb = j0; jb < j1; jb += U) {
        float acc[U];
        int cols[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            acc[u] = 0.f;
            cols[u] = (jb + u < j1) ? __ldg(p_col + jb + u) : -1;
        }
        for (int n0 = lane * 8; n0 < N; n0 += 256) {
            const uint4 yv = __ldg(reinterpret_cast<const uint4 *>(y + n0));
            const __half2 *yh = reinterpret_cast<const __half2 *>(&yv);
            uint4 bv[U];
#pragma unroll
            for (int u = 0; u < U; u++)
                bv[u] = cols[u] >= 0 ? __ldg(reinterpret_cast<const uint4 *>(B + (size_t)cols[u] * ldb + n0))
                                     : make_uint4(0, 0, 0, 0);
#pragma unroll
            for (int u = 0; u < U; u++) {
                const __half2 *bh = reinterpret_cast<const __half2 *>(&bv[u]);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float2 a = __half22float2(yh[q]), b = __half22float2(bh[q]);
                    acc[u] = fmaf(a.x, b.x, acc[u]);
                    acc[u] = fmaf(a.y, b.y, acc[u]);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            float v = acc[u];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == u && jb + u < j1) {
                const float r = alpha * v;
                if constexpr (sizeof(OutT) == 2)
                    out[src[jb + u]] = __float2half_rn(r);
                else
                    out[src[jb + u]] = r;
            }
        }
    }
}

// SDDMM for any N / alignment: one warp per sorted row, one column per lane.
template <typename OutT>
__global__ void __launch_bounds__(256)
k_sddmm_scalar(const int *__restrict__ perm, const int *__restrict__ p_row_ptr, const int *__restrict__ p_col,
               const int *__restrict__ src, int M, const int *__restrict__ windows, long long n_rows,
               const __half *__restrict__ dY, int ldy, const __half *__restrict__ B, int ldb, int N,
               OutT *__restrict__ out, float alpha)
{
    const int lane = threadIdx.x & 31;
    const long long i = sddmm_row(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, windows, n_rows, M);
    if (i < 0)
        return;
    const __half *y = dY + (size_t)perm[i] * ldy;
    for (int j = p_row_ptr[i]; j < p_row_ptr[i + 1]; j++) {
        const __half *b = B + (size_t)p_col[j] * ldb;
        float v = 0.f;
        for (int n = lane; n < N; n += 32) v = fmaf(__half2float(y[n]), __half2float(b[n]), v);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) {
            if constexpr (sizeof(OutT) == 2)
                out[src[j]] = __float2half_rn(alpha * v);
            else
                out[src[j]] = alpha * v;
        }
    }
}

unsigned blocks_of(long long n, int per) { return (unsigned)((n + per - 1) / per); }

struct Tmp {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    ~Tmp() { if (p) dev_free(p, s); }
};

int build_transpose(tca_plan *p, cudaStream_t s)
{
    if (p->tplan)
        return TCA_OK;
    const int M = p->M, K = p->K, nnz = p->nnz;
    Tmp tk, tk2, tv, tv2, tcount, trp, tcol, tcub;
    for (Tmp *t : {&tk, &tk2, &tv, &tv2, &tcount, &trp, &tcol, &tcub}) t->s = s;
    unsigned long long *keys = nullptr, *keys2 = nullptr;
    int *order = nullptr, *order2 = nullptr, *count = nullptr, *t_rp = nullptr, *t_col = nullptr;
    const size_t n1 = nnz > 0 ? nnz : 1;
    TCA_TRY(dev_malloc((void **)&keys, sizeof(unsigned long long) * n1, s)); tk.p = keys;
    TCA_TRY(dev_malloc((void **)&keys2, sizeof(unsigned long long) * n1, s)); tk2.p = keys2;
    TCA_TRY(dev_malloc((void **)&order, sizeof(int) * n1, s)); tv.p = order;
    TCA_TRY(dev_malloc((void **)&order2, sizeof(int) * n1, s)); tv2.p = order2;
    TCA_TRY(dev_malloc((void **)&count, sizeof(int) * (size_t)(K + 1), s)); tcount.p = count;
    TCA_TRY(dev_malloc((void **)&t_rp, sizeof(int) * (size_t)(K + 1), s)); trp.p = t_rp;
    TCA_TRY(dev_malloc((void **)&t_col, sizeof(int) * n1, s)); tcol.p = t_col;
    TCA_TRY(dev_malloc((void **)&p->t_src, sizeof(int) * n1, s));
    TCA_TRY(dev_malloc((void **)&p->t_vals, sizeof(__half) * n1, s));
    TCA_CUDA_TRY(cudaMemsetAsync(count, 0, sizeof(int) * (size_t)(K + 1), s));
    if (M > 0)
        k_transpose_keys<<<blocks_of((long long)M * 32, 256), 256, 0, s>>>(p->perm, p->p_row_ptr, p->p_col, p->src,
                                                                          M, keys, order);
    if (nnz > 0) {
        size_t tmp = 0;
        TCA_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, keys2, order, order2, nnz, 0, 64, s));
        void *tb;
        TCA_TRY(dev_malloc((void **)&tb, tmp > 0 ? tmp : 1, s)); tcub.p = tb;
        TCA_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tb, tmp, keys, keys2, order, order2, nnz, 0, 64, s));
        // values in A^T order come from the plan's values mapped back to the caller's order
        __half *vals_caller;
        Tmp tvc;
        tvc.s = s;
        TCA_TRY(dev_malloc((void **)&vals_caller, sizeof(__half) * n1, s)); tvc.p = vals_caller;
        // p_val[k] is the value of caller index src[k]: scatter it back
        // (src is a permutation, so the scatter has no conflicts)
        k_scatter_half<<<blocks_of(nnz, 256), 256, 0, s>>>(p->src, p->p_val, vals_caller, nnz);
        k_transpose_fill<<<blocks_of(nnz, 256), 256, 0, s>>>(keys2, order2, vals_caller, nnz, count, t_col,
                                                            p->t_vals, p->t_src);
        TCA_CUDA_TRY(cudaGetLastError());
        TCA_CUDA_TRY(cudaStreamSynchronize(s)); // vals_caller freed at scope exit
    }
    {
        size_t tmp = 0;
        TCA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp, count, t_rp, K + 1, s));
        Tmp tb;
        tb.s = s;
        void *b;
        TCA_TRY(dev_malloc((void **)&b, tmp > 0 ? tmp : 1, s)); tb.p = b;
        TCA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(b, tmp, count, t_rp, K + 1, s));
        TCA_CUDA_TRY(cudaStreamSynchronize(s));
    }
    tca_plan_t tp = nullptr;
    TCA_TRY(tca_plan_create(t_rp, t_col, p->t_vals, K, M, nnz, &p->opts, (tca_stream_t)s, &tp));
    p->tplan = tp;
    return TCA_OK;
}

} // namespace
} // namespace tca

using namespace tca;

extern "C" {

int tca_plan_build_transpose(tca_plan_t plan, tca_stream_t stream)
{
    clear_error();
    if (!plan) return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    return build_transpose(plan, (cudaStream_t)stream);
}

int tca_spmm_t(tca_plan_t plan, const void *d_dY_f16, int ldy, int N, void *d_dB, int lddb, int dB_dtype,
               float alpha, float beta, tca_stream_t stream)
{
    clear_error();
    if (!plan) return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    TCA_TRY(build_transpose(plan, (cudaStream_t)stream));
    return tca_spmm(plan->tplan, d_dY_f16, ldy, N, d_dB, lddb, dB_dtype, alpha, beta, 0u, stream);
}

int tca_sddmm(tca_plan_t plan, const void *d_dY_f16, int ldy, const void *d_B_f16, int ldb, int N, void *d_out,
              int out_dtype, float alpha, tca_stream_t stream)
{
    clear_error();
    if (!plan) return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    if (out_dtype != TCA_DTYPE_F16 && out_dtype != TCA_DTYPE_F32)
        return set_error(TCA_ERR_INVALID_ARG, "out_dtype %d is not F16 or F32", out_dtype);
    if (N < 0 || (N > 0 && (ldy < N || ldb < N)))
        return set_error(TCA_ERR_INVALID_ARG, "invalid N / leading dimensions");
    if (plan->nnz == 0 || plan->M == 0)
        return TCA_OK;
    if (!d_out || (N > 0 && (!d_dY_f16 || !d_B_f16)))
        return set_error(TCA_ERR_INVALID_ARG, "NULL operand");
    cudaStream_t s = (cudaStream_t)stream;
    if (N == 0) {
        TCA_CUDA_TRY(cudaMemsetAsync(d_out, 0, (size_t)plan->nnz * (out_dtype == TCA_DTYPE_F16 ? 2 : 4), s));
        return TCA_OK;
    }
    const __half *y = (const __half *)d_dY_f16, *b = (const __half *)d_B_f16;
    // the tensor-core windows on the tensor cores (TMA needs 16-byte aligned
    // rows), then the rows the CUDA-core kernels cover: those of the
    // CUDA-core windows, or every row
    const bool tma_ok = ldy % 8 == 0 && ldb % 8 == 0 && aligned16(y) && aligned16(b);
    const int *windows = nullptr;
    long long n_rows = plan->M;
    if (plan->n_tc > 0 && tma_ok) {
        TCA_TRY(sddmm_tc(plan, y, ldy, b, ldb, N, d_out, out_dtype == TCA_DTYPE_F16, alpha, s));
        windows = plan->cc_windows;
        n_rows = (long long)plan->n_cc * kWindowRows;
    }
    if (n_rows == 0)
        return TCA_OK;
    const unsigned grid = blocks_of(n_rows * 32, 256);
    const bool vec = (N % 8 == 0) && (ldy % 8 == 0) && (ldb % 8 == 0) && aligned16(y) && aligned16(b);
#define TCA_SDDMM(KERN, T)                                                                                  \
    KERN<T><<<grid, 256, 0, s>>>(plan->perm, plan->p_row_ptr, plan->p_col, plan->src, plan->M, windows, n_rows, y, \
                                 ldy, b, ldb, N, (T *)d_out, alpha)
    if (vec) {
        if (out_dtype == TCA_DTYPE_F16) TCA_SDDMM(k_sddmm_vec, __half);
        else TCA_SDDMM(k_sddmm_vec, float);
    } else {
        if (out_dtype == TCA_DTYPE_F16) TCA_SDDMM(k_sddmm_scalar, __half);
        else TCA_SDDMM(k_sddmm_scalar, float);
    }
#undef TCA_SDDMM
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

} // extern "C"

namespace tca {
// Called by tca_plan_update_values / tca_plan_destroy (plan.cu).
int transpose_update_values(tca_plan *p, const __half *vals, cudaStream_t s)
{
    if (!p->tplan || p->nnz == 0)
        return TCA_OK;
    k_gather_half<<<blocks_of(p->nnz, 256), 256, 0, s>>>(p->t_src, vals, p->t_vals, p->nnz);
    TCA_CUDA_TRY(cudaGetLastError());
    return tca_plan_update_values(p->tplan, p->t_vals, (tca_stream_t)s);
}

void transpose_free(tca_plan *p)
{
    if (p->tplan) tca_plan_destroy(p->tplan);
    if (p->t_src) dev_free(p->t_src, nullptr);
    if (p->t_vals) dev_free(p->t_vals, nullptr);
    p->tplan = nullptr;
    p->t_src = nullptr;
    p->t_vals = nullptr;
}
} // namespace tca
