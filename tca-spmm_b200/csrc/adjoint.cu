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
// dA has two paths. Dense-masked: D = dY B^T (M x K, FP32) as one cuBLAS GEMM
// on the tensor cores (FP16 in, FP32 accumulation), then the nonzeros' entries
// gathered from D -- it computes 1/density times the useful products but
// reads dY and B once. Sparse: a warp per row streams the row of dY against
// the B rows of its nonzeros, reading B once per nonzero (L2-bound). The
// dense path is taken where its estimated time is lower (density above
// ~0.004 + 1.5 / N, from the tensor-core rate against the L2 rate of the
// sparse path) and D fits in kSddmmDenseMaxBytes of scratch.
#include <cub/cub.cuh>
#include <cublas_v2.h>
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

// out[src[j]] = alpha * D[perm[i], p_col[j]] for the nonzeros j of sorted row
// i: the dense-masked SDDMM's sampling step (one warp per row).
template <typename OutT>
__global__ void __launch_bounds__(256)
k_sddmm_gather(const int *__restrict__ perm, const int *__restrict__ p_row_ptr, const int *__restrict__ p_col,
               const int *__restrict__ src, int M, const float *__restrict__ D, int K, OutT *__restrict__ out,
               float alpha)
{
    const int lane = threadIdx.x & 31;
    const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= M)
        return;
    const float *d = D + (size_t)perm[i] * K;
    for (int j = p_row_ptr[i] + lane; j < p_row_ptr[i + 1]; j += 32) {
        const float r = alpha * d[p_col[j]];
        if constexpr (sizeof(OutT) == 2)
            out[src[j]] = __float2half_rn(r);
        else
            out[src[j]] = r;
    }
}

constexpr size_t kSddmmDenseMaxBytes = size_t(256) << 20; // D of the dense-masked SDDMM

// This host thread's cuBLAS handle on the current device.
int cublas_handle(cublasHandle_t *out)
{
    thread_local std::vector<std::pair<int, cublasHandle_t>> handles;
    int dev = 0;
    TCA_CUDA_TRY(cudaGetDevice(&dev));
    for (const auto &h : handles)
        if (h.first == dev) {
            *out = h.second;
            return TCA_OK;
        }
    cublasHandle_t h = nullptr;
    const cublasStatus_t st = cublasCreate(&h);
    if (st != CUBLAS_STATUS_SUCCESS)
        return set_error(TCA_ERR_CUDA, "cublasCreate failed: %s", cublasGetStatusString(st));
    handles.emplace_back(dev, h);
    *out = h;
    return TCA_OK;
}

__global__ void k_gather_half(const int *__restrict__ idx, const __half *__restrict__ src, __half *__restrict__ dst,
                              int n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = src[idx[i]];
}

// SDDMM, vectorised (N % 8 == 0, 16-byte aligned rows): one warp per sorted
// row; 8 nonzeros in flight per lane, each lane covering 8 columns of every
// 256-column slice; a warp-wide reduction per nonzero.
template <typename OutT>
__global__ void __launch_bounds__(256)
k_sddmm_vec(const int *__restrict__ perm, const int *__restrict__ p_row_ptr, const int *__restrict__ p_col,
            const int *__restrict__ src, int M, const __half *__restrict__ dY, int ldy,
            const __half *__restrict__ B, int ldb, int N, OutT *__restrict__ out, float alpha)
{
    constexpr int U = 8;
    const int lane = threadIdx.x & 31;
    const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= M)
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
               const int *__restrict__ src, int M, const __half *__restrict__ dY, int ldy,
               const __half *__restrict__ B, int ldb, int N, OutT *__restrict__ out, float alpha)
{
    const int lane = threadIdx.x & 31;
    const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= M)
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
    const unsigned grid = blocks_of((long long)plan->M * 32, 256);
    const double density = (double)plan->nnz / ((double)plan->M * (double)plan->K);
    const size_t d_bytes = sizeof(float) * (size_t)plan->M * (size_t)plan->K;
    if (density > 0.004 + 1.5 / N && d_bytes <= kSddmmDenseMaxBytes) {
        // D (row-major M x K) = dY B^T, i.e. column-major D^T = B dY^T:
        // B row-major K x N is column-major N x K (transposed: op T), dY
        // row-major M x N is column-major N x M (op N)
        cublasHandle_t h = nullptr;
        TCA_TRY(cublas_handle(&h));
        float *D = nullptr;
        TCA_TRY(dev_malloc((void **)&D, d_bytes, s));
        const float one = 1.f, zero = 0.f;
        cublasStatus_t cs = cublasSetStream(h, s);
        if (cs == CUBLAS_STATUS_SUCCESS)
            cs = cublasGemmEx(h, CUBLAS_OP_T, CUBLAS_OP_N, plan->K, plan->M, N, &one, b, CUDA_R_16F, ldb, y,
                              CUDA_R_16F, ldy, &zero, D, CUDA_R_32F, plan->K, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT);
        if (cs != CUBLAS_STATUS_SUCCESS) {
            dev_free(D, s);
            return set_error(TCA_ERR_CUDA, "cublasGemmEx (dY B^T) failed: %s", cublasGetStatusString(cs));
        }
        if (out_dtype == TCA_DTYPE_F16)
            k_sddmm_gather<__half><<<grid, 256, 0, s>>>(plan->perm, plan->p_row_ptr, plan->p_col, plan->src, plan->M,
                                                        D, plan->K, (__half *)d_out, alpha);
        else
            k_sddmm_gather<float><<<grid, 256, 0, s>>>(plan->perm, plan->p_row_ptr, plan->p_col, plan->src, plan->M,
                                                       D, plan->K, (float *)d_out, alpha);
        const cudaError_t e = cudaGetLastError();
        dev_free(D, s);
        if (e != cudaSuccess)
            return set_error(TCA_ERR_CUDA, "k_sddmm_gather launch failed: %s", cudaGetErrorString(e));
        return TCA_OK;
    }
    const bool vec = (N % 8 == 0) && (ldy % 8 == 0) && (ldb % 8 == 0) && aligned16(y) && aligned16(b);
#define TCA_SDDMM(KERN, T)                                                                                  \
    KERN<T><<<grid, 256, 0, s>>>(plan->perm, plan->p_row_ptr, plan->p_col, plan->src, plan->M, y, ldy, b, ldb, N, \
                                 (T *)d_out, alpha)
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
