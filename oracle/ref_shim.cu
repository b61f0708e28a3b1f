// ref_shim.cu -- TEST INFRASTRUCTURE ONLY (part of the oracle).
//
// A C-ABI shim over the reference's own, unmodified functions so that Python
// (ctypes) can call them. It is compiled together with the reference sources
// into oracle/_ref/libtcaref.so by oracle/Makefile and is used
//   * here, on the CPU, to generate the golden fixtures in tests/golden/
//     (smtx_input_to_Dense, mtx_input_to_CSR, mtx_input_to_Dense,
//     convert_dense_to_csr, convert_csr_to_dense, naive_gemm), and
//   * on a GPU, by the parity tests and by bench.py's reference arm
//     (our_spmm_balanced, perform_cuSPARSE_SpMM, perform_GemmEx).
// Every function forwards to the reference; none re-implements it.
#include <fstream>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <cstdio>
#include <string>

#include "general.cuh"
#include "file_input.cuh"
#include "our_spmm.cuh"
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

} // extern "C"
