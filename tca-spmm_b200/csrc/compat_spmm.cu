// compat_spmm.cu -- the reference's SpMM host entry points with their exact
// signatures (include/tca_spmm_compat.h): our_spmm_balanced on top of this
// library's C ABI, and the cuSPARSE / cuBLAS comparators called the way the
// reference calls them. Host buffers in, host buffers out, blocking, default
// stream, mean milliseconds per iteration through `elapsed`.
#include <cublas_v2.h>
#include <cusparse.h>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <vector>
#include "tca_internal.cuh"
#include "tca_spmm_compat.h"

namespace tca {
void compat_report(int st);
}

using tca::set_error;

#define COMPAT_CUDA(expr)                                                                        \
    do {                                                                                         \
        cudaError_t e_ = (expr);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            st = set_error(TCA_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));               \
            goto done;                                                                           \
        }                                                                                        \
    } while (0)
#define COMPAT_SPARSE(expr)                                                                      \
    do {                                                                                         \
        cusparseStatus_t e_ = (expr);                                                            \
        if (e_ != CUSPARSE_STATUS_SUCCESS) {                                                     \
            st = set_error(TCA_ERR_CUDA, "%s: %s", #expr, cusparseGetErrorString(e_));           \
            goto done;                                                                           \
        }                                                                                        \
    } while (0)
#define COMPAT_BLAS(expr)                                                                        \
    do {                                                                                         \
        cublasStatus_t e_ = (expr);                                                              \
        if (e_ != CUBLAS_STATUS_SUCCESS) {                                                       \
            st = set_error(TCA_ERR_CUDA, "%s: %s", #expr, cublasGetStatusString(e_));            \
            goto done;                                                                           \
        }                                                                                        \
    } while (0)

// src/our_spmm.cu:472-588. C is FP32 and in/out: rows of A without nonzeros
// keep the caller's values (the reference uploads C and never writes those
// rows). The plan (GPU-built tile format) replaces workload_manager; the
// reference's 5 untimed warm-up launches are not needed and not made.
void our_spmm_balanced(CSR *A_csr, half *B, float *C, int M, int N, int K, int n_iter, double *elapsed)
{
    int st = TCA_OK;
    if (!A_csr || A_csr->nRow != M || A_csr->nCol != K)
        st = set_error(TCA_ERR_INVALID_ARG, "our_spmm_balanced: CSR shape does not match M, K");
    else
        st = tca_spmm_host(A_csr->row_offset, A_csr->col_idx, A_csr->value, M, K, A_csr->nnz, B, N, C,
                           TCA_DTYPE_F32, TCA_FLAG_KEEP_EMPTY_ROWS, n_iter < 1 ? 1 : n_iter, elapsed);
    if (st != TCA_OK)
        tca::compat_report(st);
}

// src/spmm_cusparse.cu:446-580: dense A -> CSR on the host, cusparseSpMM with
// 32-bit indices, FP16 A and B, FP32 C and compute, CUSPARSE_SPMM_ALG_DEFAULT,
// num_iter untimed then num_iter timed calls. C is uploaded (beta = 0).
void perform_cuSPARSE_SpMM(half *A, half *B, float *C, int M, int N, int K, int num_iter, double *elapsed)
{
    int st = TCA_OK;
    int nnz = 0, *h_rp = nullptr, *h_ci = nullptr;
    void *h_v = nullptr;
    int *d_rp = nullptr, *d_ci = nullptr;
    half *d_v = nullptr, *d_B = nullptr;
    float *d_C = nullptr;
    void *d_buf = nullptr;
    size_t buf_bytes = 0;
    cusparseHandle_t h = nullptr;
    cusparseSpMatDescr_t mA = nullptr;
    cusparseDnMatDescr_t mB = nullptr, mC = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float alpha = 1.f, beta = 0.f, ms = 0.f;
    if (num_iter < 1)
        num_iter = 1;
    st = tca_dense_to_csr(A, M, K, &nnz, &h_rp, &h_ci, &h_v);
    if (st != TCA_OK)
        goto done;
    COMPAT_CUDA(cudaMalloc(&d_rp, sizeof(int) * (M + 1)));
    COMPAT_CUDA(cudaMalloc(&d_ci, sizeof(int) * (nnz > 0 ? nnz : 1)));
    COMPAT_CUDA(cudaMalloc(&d_v, sizeof(half) * (nnz > 0 ? nnz : 1)));
    COMPAT_CUDA(cudaMalloc(&d_B, sizeof(half) * (size_t)K * N));
    COMPAT_CUDA(cudaMalloc(&d_C, sizeof(float) * (size_t)M * N));
    COMPAT_CUDA(cudaMemcpy(d_rp, h_rp, sizeof(int) * (M + 1), cudaMemcpyHostToDevice));
    if (nnz > 0) {
        COMPAT_CUDA(cudaMemcpy(d_ci, h_ci, sizeof(int) * nnz, cudaMemcpyHostToDevice));
        COMPAT_CUDA(cudaMemcpy(d_v, h_v, sizeof(half) * nnz, cudaMemcpyHostToDevice));
    }
    COMPAT_CUDA(cudaMemcpy(d_B, B, sizeof(half) * (size_t)K * N, cudaMemcpyHostToDevice));
    COMPAT_CUDA(cudaMemcpy(d_C, C, sizeof(float) * (size_t)M * N, cudaMemcpyHostToDevice));
    COMPAT_SPARSE(cusparseCreate(&h));
    COMPAT_SPARSE(cusparseCreateCsr(&mA, M, K, nnz, d_rp, d_ci, d_v, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                                    CUSPARSE_INDEX_BASE_ZERO, CUDA_R_16F));
    COMPAT_SPARSE(cusparseCreateDnMat(&mB, K, N, N, d_B, CUDA_R_16F, CUSPARSE_ORDER_ROW));
    COMPAT_SPARSE(cusparseCreateDnMat(&mC, M, N, N, d_C, CUDA_R_32F, CUSPARSE_ORDER_ROW));
    COMPAT_SPARSE(cusparseSpMM_bufferSize(h, CUSPARSE_OPERATION_NON_TRANSPOSE, CUSPARSE_OPERATION_NON_TRANSPOSE,
                                          &alpha, mA, mB, &beta, mC, CUDA_R_32F, CUSPARSE_SPMM_ALG_DEFAULT,
                                          &buf_bytes));
    COMPAT_CUDA(cudaMalloc(&d_buf, buf_bytes > 0 ? buf_bytes : 1));
    for (int i = 0; i < num_iter; i++)
        COMPAT_SPARSE(cusparseSpMM(h, CUSPARSE_OPERATION_NON_TRANSPOSE, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha,
                                   mA, mB, &beta, mC, CUDA_R_32F, CUSPARSE_SPMM_ALG_DEFAULT, d_buf));
    COMPAT_CUDA(cudaEventCreate(&e0));
    COMPAT_CUDA(cudaEventCreate(&e1));
    COMPAT_CUDA(cudaEventRecord(e0));
    for (int i = 0; i < num_iter; i++)
        COMPAT_SPARSE(cusparseSpMM(h, CUSPARSE_OPERATION_NON_TRANSPOSE, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha,
                                   mA, mB, &beta, mC, CUDA_R_32F, CUSPARSE_SPMM_ALG_DEFAULT, d_buf));
    COMPAT_CUDA(cudaEventRecord(e1));
    COMPAT_CUDA(cudaEventSynchronize(e1));
    COMPAT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (elapsed)
        *elapsed = (double)ms / num_iter;
    COMPAT_CUDA(cudaMemcpy(C, d_C, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToHost));
done:
    if (mA) cusparseDestroySpMat(mA);
    if (mB) cusparseDestroyDnMat(mB);
    if (mC) cusparseDestroyDnMat(mC);
    if (h) cusparseDestroy(h);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_buf);
    cudaFree(d_rp);
    cudaFree(d_ci);
    cudaFree(d_v);
    cudaFree(d_B);
    cudaFree(d_C);
    tca_free(h_rp);
    tca_free(h_ci);
    tca_free(h_v);
    if (st != TCA_OK)
        tca::compat_report(st);
}

// src/gemm_cublas.cu:3-111: dense cuBLAS GemmEx gold, computed as
// C^T = B^T A^T in column-major so that C comes out row-major; FP16 A/B,
// FP32 C and compute, 5 untimed then n_iter timed calls.
void perform_GemmEx(half *A, half *B, float *C, int M, int N, int K, int n_iter, double *elapsed)
{
    int st = TCA_OK;
    half *dA = nullptr, *dB = nullptr;
    float *dC = nullptr;
    cublasHandle_t h = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float alpha = 1.f, beta = 0.f, ms = 0.f;
    if (n_iter < 1)
        n_iter = 1;
    COMPAT_CUDA(cudaMalloc(&dA, sizeof(half) * (size_t)M * K));
    COMPAT_CUDA(cudaMalloc(&dB, sizeof(half) * (size_t)K * N));
    COMPAT_CUDA(cudaMalloc(&dC, sizeof(float) * (size_t)M * N));
    COMPAT_CUDA(cudaMemcpy(dA, A, sizeof(half) * (size_t)M * K, cudaMemcpyHostToDevice));
    COMPAT_CUDA(cudaMemcpy(dB, B, sizeof(half) * (size_t)K * N, cudaMemcpyHostToDevice));
    COMPAT_CUDA(cudaMemcpy(dC, C, sizeof(float) * (size_t)M * N, cudaMemcpyHostToDevice));
    COMPAT_BLAS(cublasCreate(&h));
    for (int i = 0; i < 5; i++)
        COMPAT_BLAS(cublasGemmEx(h, CUBLAS_OP_N, CUBLAS_OP_N, N, M, K, &alpha, dB, CUDA_R_16F, N, dA, CUDA_R_16F, K,
                                 &beta, dC, CUDA_R_32F, N, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT_TENSOR_OP));
    COMPAT_CUDA(cudaEventCreate(&e0));
    COMPAT_CUDA(cudaEventCreate(&e1));
    COMPAT_CUDA(cudaEventRecord(e0));
    for (int i = 0; i < n_iter; i++)
        COMPAT_BLAS(cublasGemmEx(h, CUBLAS_OP_N, CUBLAS_OP_N, N, M, K, &alpha, dB, CUDA_R_16F, N, dA, CUDA_R_16F, K,
                                 &beta, dC, CUDA_R_32F, N, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT_TENSOR_OP));
    COMPAT_CUDA(cudaEventRecord(e1));
    COMPAT_CUDA(cudaEventSynchronize(e1));
    COMPAT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (elapsed)
        *elapsed = (double)ms / n_iter;
    COMPAT_CUDA(cudaMemcpy(C, dC, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToHost));
done:
    if (h) cublasDestroy(h);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    if (st != TCA_OK)
        tca::compat_report(st);
}

// src/spmm_cusparse.cu:181-445: the cuSPARSE Blocked-ELL comparator. A (dense,
// M x K) is cut into ell_block_size square blocks; every block row keeps the
// blocks that hold a nonzero, padded to the widest block row with empty
// slots (column index -1); cusparseSpMM on that Blocked-ELL matrix with FP16
// A and B, FP32 C and compute, CUSPARSE_SPMM_ALG_DEFAULT, num_iter timed calls
// after one untimed call. M and K are padded to multiples of the block size
// with zeros (the reference pads the shapes too, but reads the unpadded host
// A and B with the padded strides); C gets the first M rows back.
void perform_cuSPARSE_BlockSpMM(half *A, half *B, float *C, int M, int N, int K, int num_iter, int ell_block_size,
                                double *elapsed)
{
    int st = TCA_OK;
    const int bs = ell_block_size;
    int *d_cols = nullptr;
    half *d_vals = nullptr, *d_B = nullptr;
    float *d_C = nullptr;
    void *d_buf = nullptr;
    size_t buf_bytes = 0;
    cusparseHandle_t h = nullptr;
    cusparseSpMatDescr_t mA = nullptr;
    cusparseDnMatDescr_t mB = nullptr, mC = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float alpha = 1.f, beta = 0.f, ms = 0.f;
    std::vector<int> cols;
    std::vector<half> vals, Bp;
    int brows = 0, bcols = 0, width = 0, Mp = 0, Kp = 0;
    if (bs <= 0 || M <= 0 || K <= 0 || N <= 0 || !A || !B || !C) {
        st = set_error(TCA_ERR_INVALID_ARG, "perform_cuSPARSE_BlockSpMM: invalid sizes or buffers");
        goto done;
    }
    if (num_iter < 1)
        num_iter = 1;
    brows = (M + bs - 1) / bs;
    bcols = (K + bs - 1) / bs;
    Mp = brows * bs;
    Kp = bcols * bs;
    {
        // occupied blocks per block row, in column order
        std::vector<std::vector<int>> occ((size_t)brows);
        for (int bi = 0; bi < brows; bi++) {
            for (int bj = 0; bj < bcols; bj++) {
                bool any = false;
                for (int i = bi * bs; i < std::min(M, (bi + 1) * bs) && !any; i++)
                    for (int j = bj * bs; j < std::min(K, (bj + 1) * bs); j++)
                        if (__half2float(A[(size_t)i * K + j]) != 0.f) { any = true; break; }
                if (any) occ[bi].push_back(bj);
            }
            width = std::max(width, (int)occ[bi].size());
        }
        width = std::max(width, 1);
        cols.assign((size_t)brows * width, -1);
        vals.assign((size_t)Mp * width * bs, __float2half(0.f));
        for (int bi = 0; bi < brows; bi++)
            for (int s = 0; s < (int)occ[bi].size(); s++) {
                const int bj = occ[bi][s];
                cols[(size_t)bi * width + s] = bj;
                for (int r = 0; r < bs; r++) {
                    const int i = bi * bs + r;
                    if (i >= M) break;
                    for (int c = 0; c < bs; c++) {
                        const int j = bj * bs + c;
                        if (j < K) vals[(size_t)i * width * bs + (size_t)s * bs + c] = A[(size_t)i * K + j];
                    }
                }
            }
        Bp.assign((size_t)Kp * N, __float2half(0.f));
        std::copy(B, B + (size_t)K * N, Bp.begin());
    }
    COMPAT_CUDA(cudaMalloc(&d_cols, sizeof(int) * cols.size()));
    COMPAT_CUDA(cudaMalloc(&d_vals, sizeof(half) * vals.size()));
    COMPAT_CUDA(cudaMalloc(&d_B, sizeof(half) * Bp.size()));
    COMPAT_CUDA(cudaMalloc(&d_C, sizeof(float) * (size_t)Mp * N));
    COMPAT_CUDA(cudaMemcpy(d_cols, cols.data(), sizeof(int) * cols.size(), cudaMemcpyHostToDevice));
    COMPAT_CUDA(cudaMemcpy(d_vals, vals.data(), sizeof(half) * vals.size(), cudaMemcpyHostToDevice));
    COMPAT_CUDA(cudaMemcpy(d_B, Bp.data(), sizeof(half) * Bp.size(), cudaMemcpyHostToDevice));
    COMPAT_SPARSE(cusparseCreate(&h));
    COMPAT_SPARSE(cusparseCreateBlockedEll(&mA, Mp, Kp, bs, (int64_t)width * bs, d_cols, d_vals, CUSPARSE_INDEX_32I,
                                           CUSPARSE_INDEX_BASE_ZERO, CUDA_R_16F));
    COMPAT_SPARSE(cusparseCreateDnMat(&mB, Kp, N, N, d_B, CUDA_R_16F, CUSPARSE_ORDER_ROW));
    COMPAT_SPARSE(cusparseCreateDnMat(&mC, Mp, N, N, d_C, CUDA_R_32F, CUSPARSE_ORDER_ROW));
    COMPAT_SPARSE(cusparseSpMM_bufferSize(h, CUSPARSE_OPERATION_NON_TRANSPOSE, CUSPARSE_OPERATION_NON_TRANSPOSE,
                                          &alpha, mA, mB, &beta, mC, CUDA_R_32F, CUSPARSE_SPMM_ALG_DEFAULT,
                                          &buf_bytes));
    COMPAT_CUDA(cudaMalloc(&d_buf, buf_bytes > 0 ? buf_bytes : 1));
    COMPAT_SPARSE(cusparseSpMM(h, CUSPARSE_OPERATION_NON_TRANSPOSE, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha, mA, mB,
                               &beta, mC, CUDA_R_32F, CUSPARSE_SPMM_ALG_DEFAULT, d_buf));
    COMPAT_CUDA(cudaEventCreate(&e0));
    COMPAT_CUDA(cudaEventCreate(&e1));
    COMPAT_CUDA(cudaEventRecord(e0));
    for (int i = 0; i < num_iter; i++)
        COMPAT_SPARSE(cusparseSpMM(h, CUSPARSE_OPERATION_NON_TRANSPOSE, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha,
                                   mA, mB, &beta, mC, CUDA_R_32F, CUSPARSE_SPMM_ALG_DEFAULT, d_buf));
    COMPAT_CUDA(cudaEventRecord(e1));
    COMPAT_CUDA(cudaEventSynchronize(e1));
    COMPAT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (elapsed)
        *elapsed = (double)ms / num_iter;
    COMPAT_CUDA(cudaMemcpy(C, d_C, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToHost));
done:
    if (mA) cusparseDestroySpMat(mA);
    if (mB) cusparseDestroyDnMat(mB);
    if (mC) cusparseDestroyDnMat(mC);
    if (h) cusparseDestroy(h);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_buf);
    cudaFree(d_cols);
    cudaFree(d_vals);
    cudaFree(d_B);
    cudaFree(d_C);
    if (st != TCA_OK)
        tca::compat_report(st);
}
