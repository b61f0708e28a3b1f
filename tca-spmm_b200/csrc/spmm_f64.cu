// spmm_f64.cu -- the FP64 mode: CSR (FP64 values) x dense FP64 B -> FP64 C on
// CUDA cores, accumulated in FP64.
//
// The reference advertises an FP64 data type (src/arg_parse.h:102-105, the
// m8n8k4 FP64 MMA named in src/general.cuh:58,65) but never implements it;
// here it is a plan-free forward for callers that need full precision. SpMM in
// FP64 is bound by B-row traffic (8 bytes per element), not by FP64
// arithmetic, so it runs on CUDA cores: a warp per row, lanes over columns
// (coalesced), the row's nonzeros broadcast by shuffle, four B loads in
// flight per lane.
#include "tca_internal.cuh"

namespace tca {
namespace {

__global__ void __launch_bounds__(256)
spmm_csr_f64_kernel(const int *__restrict__ row_ptr, const int *__restrict__ col_idx,
                    const double *__restrict__ vals, int M, int K, int nnz, const double *__restrict__ B, int ldb,
                    int N, double *__restrict__ C, int ldc, double alpha, double beta, unsigned flags)
{
    const int lane = threadIdx.x & 31;
    const long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= M)
        return;
    int start = row_ptr[r], end = row_ptr[r + 1];
    start = max(0, min(start, nnz)); // malformed offsets never fault
    end = max(start, min(end, nnz));
    if (start == end && (flags & TCA_FLAG_KEEP_EMPTY_ROWS))
        return;
    double *Crow = C + (size_t)r * ldc;
    for (int nb = 0; nb < N; nb += 32) {
        const int n = nb + lane;
        double acc = 0.0;
        for (int base = start; base < end; base += 32) {
            const int j = base + lane;
            int c = -1;
            double a = 0.0;
            if (j < end) {
                c = __ldg(col_idx + j);
                a = __ldg(vals + j);
                if (c < 0 || c >= K) { c = -1; a = 0.0; }
            }
            const int cnt = min(32, end - base);
            int t = 0;
            for (; t + 4 <= cnt; t += 4) {
                double bv[4], av[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int cu = __shfl_sync(0xffffffffu, c, t + u);
                    av[u] = __shfl_sync(0xffffffffu, a, t + u);
                    bv[u] = (n < N && cu >= 0) ? __ldg(B + (size_t)cu * ldb + n) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) acc = fma(av[u], bv[u], acc);
            }
            for (; t < cnt; t++) {
                const int cu = __shfl_sync(0xffffffffu, c, t);
                const double au = __shfl_sync(0xffffffffu, a, t);
                if (n < N && cu >= 0)
                    acc = fma(au, __ldg(B + (size_t)cu * ldb + n), acc);
            }
        }
        if (n < N)
            Crow[n] = beta != 0.0 ? fma(alpha, acc, beta * Crow[n]) : alpha * acc;
    }
}

} // namespace
} // namespace tca

using namespace tca;

int tca_spmm_csr_f64(const int *d_row_ptr, const int *d_col_idx, const double *d_vals, int M, int K, int nnz,
                     const double *d_B, int ldb, int N, double *d_C, int ldc, double alpha, double beta,
                     unsigned flags, tca_stream_t stream)
{
    clear_error();
    if (M < 0 || K < 0 || N < 0 || nnz < 0)
        return set_error(TCA_ERR_INVALID_ARG, "negative size (M=%d, K=%d, N=%d, nnz=%d)", M, K, N, nnz);
    if (M == 0 || N == 0)
        return TCA_OK;
    if (!d_row_ptr || (nnz > 0 && (!d_col_idx || !d_vals)) || !d_C || (K > 0 && !d_B))
        return set_error(TCA_ERR_INVALID_ARG, "NULL buffer");
    if (ldb < N || ldc < N)
        return set_error(TCA_ERR_INVALID_ARG, "ldb (%d) and ldc (%d) must be >= N (%d)", ldb, ldc, N);
    const long long threads = (long long)M * 32;
    spmm_csr_f64_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        d_row_ptr, d_col_idx, d_vals, M, K, nnz, d_B, ldb, N, d_C, ldc, alpha, beta, flags);
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}
