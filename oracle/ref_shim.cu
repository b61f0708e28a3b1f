// ref_shim.cu -- TEST INFRASTRUCTURE ONLY (part of the oracle).
//
// A C-ABI shim over the reference's own, unmodified functions so that Python
// (ctypes) can call them. It is compiled together with the reference sources
// into oracle/_ref/libtcaref.so by oracle/Makefile and is used
//   * here, on the CPU, to generate the golden fixtures in tests/golden/
//     (smtx_input_to_Dense, mtx_input_to_CSR, mtx_input_to_Dense,
//     convert_dense_to_csr, convert_csr_to_dense, naive_gemm), and
//   * on a GPU, by the parity tests and by bench.py's reference arm
//     (our_spmm_balanced, perform_cuSPARSE_SpMM, perform_GemmEx), and by
//     bench.py's per-problem comparison, which times the reference's own
//     kernel with its own schedule (ref_tca_*) and the reference comparator's
//     cuSPARSE call (ref_cusparse_*) on device buffers, launched on a stream
//     the caller gives (so that they can be captured in a CUDA graph and timed
//     exactly like this project's forward).
// Every function forwards to the reference; none re-implements it. The
// reference's kernel and its schedule builder are file-local (static) in
// src/our_spmm.cu, so that file is compiled as part of this unit.
#include <fstream>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <cstdio>
#include <string>

#include "general.cuh"
#include "file_input.cuh"
#include "our_spmm.cu" // kernel_our_spmm_balanced and workload_manager (file-local there)
#include "spmm_cusparse.cuh"
#include "gemm_cublas.cuh"
#include "arg_parse.h"

extern "C" {

void ref_free(void *p) { free(p); }

// smtx_input_to_Dense (src/file_input.cu:135): returns a malloc'd M x K half matrix.
int ref_smtx_to_dense(const char *path, int *M, int *K, int *nnz, uint16_t **mat)
{
    std::ifstream fin;
    fin.open(path, std::ifstream::in);
    if (!fin.is_open())
        return -1;
    half *A = nullptr;
    smtx_input_to_Dense(fin, &A, const_cast<char *>(path), M, K, nnz);
    *mat = reinterpret_cast<uint16_t *>(A);
    return 0;
}

// The reference's run options with its defaults (no command-line options).
static Arguments *make_args(int zero_based, int pattern_only)
{
    static char name[] = "ref";
    char *argv[] = {name, nullptr};
    Arguments *a = new Arguments(1, argv); // prints its settings to stdout
    a->input_is_zero_based = zero_based != 0;
    a->pattern_only = pattern_only != 0;
    return a;
}

// mtx_input_to_CSR (src/file_input.cu:63). Arrays are malloc'd; free with ref_free.
int ref_mtx_to_csr(const char *path, int zero_based, int pattern_only, int *M, int *K, int *nnz, int **row_ptr,
                   int **col_idx, uint16_t **val)
{
    std::ifstream fin(path);
    if (!fin.is_open())
        return -1;
    Arguments *a = make_args(zero_based, pattern_only);
    CSR *c = nullptr;
    mtx_input_to_CSR(fin, &c, a);
    delete a;
    *M = c->nRow;
    *K = c->nCol;
    *nnz = c->nnz;
    *row_ptr = c->row_offset;
    *col_idx = c->col_idx;
    *val = reinterpret_cast<uint16_t *>(c->value);
    free(c);
    return 0;
}

// mtx_input_to_Dense (src/file_input.cu:8). The reference returns only the
// matrix; its shape is the file's "rows cols nnz" line, read here to size it.
int ref_mtx_to_dense(const char *path, int zero_based, int *M, int *K, uint16_t **mat)
{
    std::ifstream fin(path);
    if (!fin.is_open())
        return -1;
    std::ifstream hdr(path);
    std::string line;
    while (std::getline(hdr, line))
        if (!line.empty() && line[0] != '%')
            break;
    if (sscanf(line.c_str(), "%d %d", M, K) != 2)
        return -2;
    Arguments *a = make_args(zero_based, 0);
    half *A = nullptr;
    mtx_input_to_Dense(fin, &A, a);
    delete a;
    *mat = reinterpret_cast<uint16_t *>(A);
    return 0;
}

// convert_dense_to_csr (src/miscalleneous.cu:29). Arrays are malloc'd; free with ref_free.
int ref_dense_to_csr(const uint16_t *mat, int M, int K, int *nnz, int **row_ptr, int **col_idx, uint16_t **val)
{
    CSR *c = nullptr;
    convert_dense_to_csr(reinterpret_cast<half *>(const_cast<uint16_t *>(mat)), &c, M, K);
    *nnz = c->nnz;
    *row_ptr = c->row_offset;
    *col_idx = c->col_idx;
    *val = reinterpret_cast<uint16_t *>(c->value);
    free(c);
    return 0;
}

// convert_csr_to_dense (src/miscalleneous.cu:66).
int ref_csr_to_dense(int M, int K, int nnz, const int *row_ptr, const int *col_idx, const uint16_t *val, uint16_t **mat)
{
    CSR c;
    c.nRow = M;
    c.nCol = K;
    c.nnz = nnz;
    c.row_offset = const_cast<int *>(row_ptr);
    c.col_idx = const_cast<int *>(col_idx);
    c.value = reinterpret_cast<half *>(const_cast<uint16_t *>(val));
    half *out = nullptr;
    convert_csr_to_dense(&c, &out);
    *mat = reinterpret_cast<uint16_t *>(out);
    return 0;
}

// naive_gemm (src/miscalleneous.cu:114): dense fp32-accumulated GEMM on the CPU.
void ref_naive_gemm(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K)
{
    naive_gemm(reinterpret_cast<half *>(const_cast<uint16_t *>(A)),
               reinterpret_cast<half *>(const_cast<uint16_t *>(B)), C, M, N, K);
}

// our_spmm_balanced (src/our_spmm.cu:472): the reference TCA kernel, host buffers in/out.
void ref_our_spmm_balanced(int M, int N, int K, int nnz, const int *row_ptr, const int *col_idx,
                           const uint16_t *val, const uint16_t *B, float *C, int n_iter, double *elapsed)
{
    CSR c;
    c.nRow = M;
    c.nCol = K;
    c.nnz = nnz;
    c.row_offset = const_cast<int *>(row_ptr);
    c.col_idx = const_cast<int *>(col_idx);
    c.value = reinterpret_cast<half *>(const_cast<uint16_t *>(val));
    our_spmm_balanced(&c, reinterpret_cast<half *>(const_cast<uint16_t *>(B)), C, M, N, K, n_iter, elapsed);
}

// perform_cuSPARSE_SpMM (src/spmm_cusparse.cu:446): dense A in, converted internally.
void ref_cusparse_spmm(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K, int n_iter, double *elapsed)
{
    perform_cuSPARSE_SpMM(reinterpret_cast<half *>(const_cast<uint16_t *>(A)),
                          reinterpret_cast<half *>(const_cast<uint16_t *>(B)), C, M, N, K, n_iter, elapsed);
}

// perform_cuSPARSE_BlockSpMM (src/spmm_cusparse.cu:181): Blocked-ELL comparator.
void ref_cusparse_blockspmm(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K, int n_iter, int bs,
                            double *elapsed)
{
    perform_cuSPARSE_BlockSpMM(reinterpret_cast<half *>(const_cast<uint16_t *>(A)),
                               reinterpret_cast<half *>(const_cast<uint16_t *>(B)), C, M, N, K, n_iter, bs, elapsed);
}

// perform_cuSPARSELT_24sparsity (src/spmm_cusparse.cu:2): 2:4 comparator (A pruned).
void ref_cusparselt_24(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K, int n_iter,
                       double *elapsed)
{
    perform_cuSPARSELT_24sparsity(reinterpret_cast<half *>(const_cast<uint16_t *>(A)),
                                  reinterpret_cast<half *>(const_cast<uint16_t *>(B)), C, M, N, K, n_iter, elapsed);
}

// perform_GemmEx (src/gemm_cublas.cu:3): the reference test's dense gold.
void ref_gemmex(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K, int n_iter, double *elapsed)
{
    perform_GemmEx(reinterpret_cast<half *>(const_cast<uint16_t *>(A)),
                   reinterpret_cast<half *>(const_cast<uint16_t *>(B)), C, M, N, K, n_iter, elapsed);
}

// The reference TCA kernel on device buffers, as our_spmm_balanced launches it
// (src/our_spmm.cu:524-559): workload_manager's schedule for 8-warp blocks and
// 64-column output tiles, alpha = 1, beta = 0, FP32 C.
struct RefTcaSchedule {
    int M, N, K, num_block, blockdim;
    size_t shm;
    int *d_num_warps_per_row, *d_row_idx_for_each_warp, *d_warpid_within_row;
};

// Builds the schedule on the host from the CSR row offsets (the reference's
// workload_manager, src/our_spmm.cu:347-471); its arrays go to the device.
void *ref_tca_schedule(int M, int N, int K, int nnz, const int *row_ptr)
{
    CSR c;
    c.nRow = M;
    c.nCol = K;
    c.nnz = nnz;
    c.row_offset = const_cast<int *>(row_ptr);
    c.col_idx = nullptr;
    c.value = nullptr;
    RefTcaSchedule *s = new RefTcaSchedule{};
    s->M = M;
    s->N = N;
    s->K = K;
    workload_manager(&c, 8, N, &s->blockdim, &s->num_block, 64, &s->shm, &s->d_num_warps_per_row,
                     &s->d_row_idx_for_each_warp, &s->d_warpid_within_row);
    return s;
}

int ref_tca_launch(void *sched, const void *d_val, const int *d_row_ptr, const int *d_col, const void *d_B, float *d_C,
                   void *stream)
{
    const RefTcaSchedule *s = static_cast<const RefTcaSchedule *>(sched);
    if (s->num_block == 0)
        return 0;
    kernel_our_spmm_balanced<64><<<s->num_block, s->blockdim, s->shm, (cudaStream_t)stream>>>(
        (half *)d_val, d_row_ptr, const_cast<int *>(d_col), (half *)d_B, d_C, s->M, s->N, s->K, 1.0f, 0.0f,
        s->d_num_warps_per_row, s->d_row_idx_for_each_warp, s->d_warpid_within_row);
    return (int)cudaGetLastError();
}

void ref_tca_free(void *sched)
{
    RefTcaSchedule *s = static_cast<RefTcaSchedule *>(sched);
    if (!s)
        return;
    cudaFree(s->d_num_warps_per_row);
    cudaFree(s->d_row_idx_for_each_warp);
    cudaFree(s->d_warpid_within_row);
    delete s;
}

// The reference comparator's cuSPARSE call on device buffers, with its
// parameters (src/spmm_cusparse.cu:505-549): CSR with 32-bit indices and FP16
// values, row-major FP16 B and FP32 C, FP32 compute, CUSPARSE_SPMM_ALG_DEFAULT,
// alpha = 1, beta = 0.
struct RefSparse {
    cusparseHandle_t handle;
    cusparseSpMatDescr_t A;
    cusparseDnMatDescr_t B, C;
    void *buf;
};

void *ref_cusparse_setup(int M, int N, int K, int nnz, int *d_row_ptr, int *d_col, void *d_val, void *d_B,
                         float *d_C)
{
    RefSparse *r = new RefSparse{};
    size_t bytes = 0;
    const float alpha = 1.0f, beta = 0.0f;
    if (cusparseCreate(&r->handle) != CUSPARSE_STATUS_SUCCESS ||
        cusparseCreateCsr(&r->A, M, K, nnz, d_row_ptr, d_col, d_val, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                          CUSPARSE_INDEX_BASE_ZERO, CUDA_R_16F) != CUSPARSE_STATUS_SUCCESS ||
        cusparseCreateDnMat(&r->B, K, N, N, d_B, CUDA_R_16F, CUSPARSE_ORDER_ROW) != CUSPARSE_STATUS_SUCCESS ||
        cusparseCreateDnMat(&r->C, M, N, N, d_C, CUDA_R_32F, CUSPARSE_ORDER_ROW) != CUSPARSE_STATUS_SUCCESS ||
        cusparseSpMM_bufferSize(r->handle, CUSPARSE_OPERATION_NON_TRANSPOSE, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha,
                                r->A, r->B, &beta, r->C, CUDA_R_32F, CUSPARSE_SPMM_ALG_DEFAULT,
                                &bytes) != CUSPARSE_STATUS_SUCCESS ||
        cudaMalloc(&r->buf, bytes > 0 ? bytes : 16) != cudaSuccess) {
        delete r;
        return nullptr;
    }
    return r;
}

int ref_cusparse_run(void *h, void *stream)
{
    RefSparse *r = static_cast<RefSparse *>(h);
    const float alpha = 1.0f, beta = 0.0f;
    if (cusparseSetStream(r->handle, (cudaStream_t)stream) != CUSPARSE_STATUS_SUCCESS)
        return -1;
    return (int)cusparseSpMM(r->handle, CUSPARSE_OPERATION_NON_TRANSPOSE, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha,
                             r->A, r->B, &beta, r->C, CUDA_R_32F, CUSPARSE_SPMM_ALG_DEFAULT, r->buf);
}

void ref_cusparse_free(void *h)
{
    RefSparse *r = static_cast<RefSparse *>(h);
    if (!r)
        return;
    cusparseDestroySpMat(r->A);
    cusparseDestroyDnMat(r->B);
    cusparseDestroyDnMat(r->C);
    cusparseDestroy(r->handle);
    cudaFree(r->buf);
    delete r;
}

} // extern "C"
