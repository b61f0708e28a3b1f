/*
 * tca_spmm_compat.h -- C++ drop-in for the reference's host API.
 *
 * Same names, argument meaning and calling convention (host buffers,
 * blocking, default stream, ms/iteration through `elapsed`) as the reference
 * functions cited on each declaration (paths within the reference project),
 * implemented on top of libtca_spmm's C ABI (tca_spmm.h). A caller written
 * against the reference (e.g. its src/test.cu) compiles against this header
 * and links libtca_spmm.so instead of the reference objects.
 *
 * Error behaviour mirrors the reference, whose CHECK_CUDA / CHECK_CUSPARSE /
 * CHECK_CUBLAS macros print and exit(EXIT_FAILURE) (src/general.cuh:8-16):
 * the void functions below do the same on failure unless
 * tca_compat_set_exit_on_error(0) was called, in which case they print, set
 * tca_last_error_string() and return.
 */
#ifndef TCA_SPMM_COMPAT_H
#define TCA_SPMM_COMPAT_H

#include <cuda_fp16.h>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <fstream>
#include <random>
#include <type_traits>
#include "tca_spmm.h"

/* CSR, layout-identical to the reference's (src/general.cuh:125-134):
 * host memory, 0-based int32 indices, FP16 values. */
#ifndef TCA_NO_COMPAT_CSR
typedef struct CSR {
    int nRow;
    int nCol;
    int nnz;
    int *row_offset;
    int *col_idx;
    half *value;
} CSR;
#endif

/* src/mat_format.cuh:10-15 */
typedef enum _mat_format { dense, csr, coo } mat_format;

/* COO (row-major sorted) used by format_conversion. */
typedef struct COO {
    int nRow, nCol, nnz;
    int *row_idx;
    int *col_idx;
    half *value;
} COO;

extern "C" TCA_API void tca_compat_set_exit_on_error(int enabled);

/* src/our_spmm.cuh:4, src/our_spmm.cu:472 -- C (FP32, M x N) is in/out: rows
 * of A without nonzeros keep the caller's values. Any N >= 1 is accepted (the
 * reference needs N % 64 == 0). */
TCA_API void our_spmm_balanced(CSR *A_csr, half *B, float *C, int M, int N, int K, int n_iter,
                               double *elapsed = NULL);

/* src/spmm_cusparse.cuh:15, src/spmm_cusparse.cu:446 -- cuSPARSE CSR SpMM
 * comparator on a dense A: FP16 A/B, FP32 compute and C, ALG_DEFAULT,
 * num_iter warm-up then num_iter timed calls. */
TCA_API void perform_cuSPARSE_SpMM(half *A, half *B, float *C, int M, int N, int K, int num_iter,
                                   double *elapsed = NULL);

/* src/spmm_cusparse.cuh:14, src/spmm_cusparse.cu:181 -- cuSPARSE Blocked-ELL
 * SpMM comparator on a dense A cut into ell_block_size square blocks (block
 * rows keep their occupied blocks, padded to the widest): FP16 A/B, FP32
 * compute and C, ALG_DEFAULT, one untimed then num_iter timed calls. */
TCA_API void perform_cuSPARSE_BlockSpMM(half *A, half *B, float *C, int M, int N, int K, int num_iter,
                                        int ell_block_size, double *elapsed = NULL);

/* src/spmm_cusparse.cuh, src/spmm_cusparse.cu:2 -- cuSPARSELt 2:4 comparator
 * on a dense A: cuSPARSELt prunes A to the 2:4 pattern along its rows (STRIP),
 * compresses it and multiplies with B: FP16 A/B, FP32 compute, FP16 result
 * returned as FP32 C, num_iter timed calls. A different product (A pruned);
 * cuSPARSELt is loaded at the first call (an error is reported without it). */
TCA_API void perform_cuSPARSELT_24sparsity(half *A, half *B, float *C, int M, int N, int K, int num_iter,
                                           double *elapsed = NULL);

/* src/gemm_cublas.cuh:12, src/gemm_cublas.cu:3 -- dense cuBLAS GemmEx gold:
 * FP16 A/B, FP32 C and compute, 5 warm-up then n_iter timed calls. */
TCA_API void perform_GemmEx(half *A, half *B, float *C, int M, int N, int K, int n_iter,
                            double *elapsed = NULL);

/* src/file_input.cuh:8, src/file_input.cu:135 -- reads an .smtx file
 * ("rows, cols, nnz" / row_ptr line / col_idx lines) into a malloc'd dense
 * M x K FP16 matrix with 1.0 at every nonzero (or the values of the optional
 * values line, see tca_smtx_parse). `filename` is unused, as in the reference. */
TCA_API void smtx_input_to_Dense(std::ifstream &fin, half **mat, char *filename, int *nRow, int *nCol,
                                 int *nnz);

/* src/general.cuh:54-59 */
typedef enum entry_dtype { fp16, fp32, fp64 } entry_dtype;

/* src/arg_parse.h:15-161 -- the reference's run options, layout-identical (the
 * MatrixMarket readers take a pointer to it and read pattern_only and
 * input_is_zero_based). Both constructors start from the reference's defaults
 * (src/general.cuh:21-28, src/arg_parse.h:33-48: M = N = K = 1024, 10
 * iterations, sparsity 0.8, tolerance 1e-3, FP16 A/B, FP32 C, zero-based,
 * Blocked-ELL block 32).
 *
 * Arguments(argc, argv) then parses the reference's getopt options
 * (src/arg_parse.h:54-133), with the same meaning:
 *   -m M  -n N  -k K  -i num_iter  -t tolerance  -s target_sparsity
 *   -f input file (must exist; sets input_file_exists)
 *   -p 1: pattern_only    -b 0: input_is_zero_based, else one-based
 *   -e ell_block_size     -d 0 (FP16 A/B, FP32 C) or 2 (FP64 A, B, C)
 * Unknown options are reported by getopt and skipped, as in the reference.
 * A missing input file, a -d other than 0 or 2, or a malformed number prints
 * an error and exits with EXIT_FAILURE like the reference (whose std::stoi
 * throws on a malformed number); after tca_compat_set_exit_on_error(0) it
 * sets tca_last_error_string() and keeps the default for that option.
 * Differences: parsing restarts at argv[1] on every call (getopt's optind is
 * reset, so a second Arguments in one process parses its own argv), and
 * input_fname is a malloc'd copy with room for its terminator (the
 * reference's copy is one byte short). As in the reference, the destructor
 * does not free input_fname. The constructor prints nothing (the reference's
 * constructor calls print(), whose body is compiled out at its default
 * VERBOSE = false); print() writes the settings in the reference's layout. */
class TCA_API Arguments
{
public:
    int M;
    int N;
    int K;
    int num_iter;
    bool pattern_only;
    bool input_is_zero_based;
    bool input_file_exists;
    float target_sparsity;
    float tolerance;
    entry_dtype a_type, b_type, c_type;
    char *input_fname;
    int ell_block_size;
    Arguments();
    Arguments(int argc, char *argv[]);
    void ParseArgs(int argc, char *argv[]);
    void print();
};

/* src/file_input.cuh:6-7, src/file_input.cu:8-134 -- MatrixMarket coordinate
 * files ('%' comments, "rows cols nnz", then "r c [v]" lines, 1-based unless
 * arg->input_is_zero_based) into a malloc'd CSR (rows grouped, file order
 * within a row; missing values 0.0, or 1.0 with arg->pattern_only) or a
 * malloc'd dense FP16 matrix (missing values 1.0, later duplicates win). A
 * NULL arg means the defaults. Malformed text (count mismatch, indices out
 * of range) is an error (see tca_mtx_parse) where the reference asserts or
 * reads out of bounds. */
TCA_API void mtx_input_to_CSR(std::ifstream &fin, CSR **csr_mat, Arguments *arg);
TCA_API void mtx_input_to_Dense(std::ifstream &fin, half **mat, Arguments *arg);
/* src/file_input.cuh:9 declares this (its body, src/file_input.cu:194-196,
 * is empty): reads an .smtx file straight into a malloc'd CSR (values 1.0
 * unless a values line is present). `arg` is unused; NULL is accepted. */
TCA_API void smtx_input_to_CSR(std::ifstream &fin, CSR **csr_mat, Arguments *arg = NULL);

/* src/general.cuh:135-138, src/miscalleneous.cu:29-112 */
TCA_API void convert_dense_to_csr(half *mat, CSR **descr, int nRow, int nCol);
TCA_API void convert_csr_to_dense(CSR *descr, half **mat);
TCA_API void destroy_csr(CSR *descr);
TCA_API void print_csr(CSR *descr);

/* src/mat_format.cuh:17, src/mat_format.cu:2-37 -- the reference declares
 * format_conversion over {dense, csr, coo} with empty bodies; these are the
 * filled-in conversions. `dense` arguments are half* with the shape passed
 * alongside; the destination is allocated with malloc (free with
 * destroy_csr / destroy_coo / free). Returns a tca_status_t. */
TCA_API int format_conversion(mat_format in, mat_format out, const half *src_dense, int nRow, int nCol, CSR **dst);
TCA_API int format_conversion(mat_format in, mat_format out, const CSR *src, half **dst);
TCA_API int format_conversion(mat_format in, mat_format out, const CSR *src, COO **dst);
TCA_API int format_conversion(mat_format in, mat_format out, const COO *src, CSR **dst);
TCA_API int format_conversion(mat_format in, mat_format out, const half *src_dense, int nRow, int nCol, COO **dst);
TCA_API int format_conversion(mat_format in, mat_format out, const COO *src, half **dst);
TCA_API void destroy_coo(COO *descr);

/* src/general.cuh:71-123 -- element i fails only when both |gold-x|/|gold| >=
 * tolerance and |gold-x| >= tolerance; prints up to 10 failures. */
template <typename T>
bool compare_mat(T *gold, T *comparing, int num_elem, float tolerance)
{
    bool ok = true;
    int count = 0;
    for (int i = 0; i < num_elem; i++) {
        float v1, v2;
        if (std::is_same<T, half>::value) {
            v1 = __half2float(reinterpret_cast<const half *>(gold)[i]);
            v2 = __half2float(reinterpret_cast<const half *>(comparing)[i]);
        } else {
            v1 = (float)gold[i];
            v2 = (float)comparing[i];
        }
        const float d = std::fabs(v1 - v2);
        const float rel = std::fabs(d / v1);
        if (rel >= tolerance && d >= tolerance) {
            ok = false;
            std::printf("Discrepancy occured in %dth element :: %f vs %f ...abs_disc : %f, rel_disc : %f %%\n", i, v1,
                        v2, d, rel * 100.0);
            if (++count >= 10)
                return ok;
        }
    }
    return ok;
}

/* src/general.cuh:140-174 -- a malloc'd nRow x nCol matrix whose entries are
 * nonzero with probability 1 - target_sparsity, value U(0, 1); zero-filled
 * when leave_empty. Deterministic for a given seed (the reference seeds from
 * std::random_device). */
template <typename T>
void prepare_cpu_matrix(T **mat, size_t nRow, size_t nCol, float target_sparsity, bool leave_empty = false,
                        unsigned long long seed = 0)
{
    *mat = (T *)malloc(sizeof(T) * nRow * nCol);
    if (leave_empty) {
        std::memset(*mat, 0, nRow * nCol * sizeof(T));
        return;
    }
    std::mt19937_64 e2(seed);
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    for (size_t i = 0; i < nRow * nCol; i++) {
        double elem = 0.0;
        if (dist(e2) > target_sparsity)
            elem = dist(e2);
        if (std::is_same<T, half>::value)
            reinterpret_cast<half *>(*mat)[i] = __double2half(elem);
        else
            (*mat)[i] = (T)elem;
    }
}

#endif /* TCA_SPMM_COMPAT_H */
