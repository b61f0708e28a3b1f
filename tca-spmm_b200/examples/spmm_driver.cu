// spmm_driver.cu -- an end-to-end driver written against the reference's host
// API only (include/tca_spmm_compat.h), linked with libtca_spmm.so: read an
// .smtx matrix as dense A, make B, compute the dense cuBLAS GemmEx gold, the
// cuSPARSE result and our_spmm_balanced, and check both against the gold with
// compare_mat at tolerance 1e-3 -- the flow of the reference's harness
// (src/test.cu:29-88), here with a deterministic B and a non-zero exit status
// on mismatch.
//
//   nvcc -std=c++17 -I include spmm_driver.cu -L lib -ltca_spmm -o spmm_driver
//   ./spmm_driver matrix.smtx [N]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include "tca_spmm_compat.h"

int main(int argc, char **argv)
{
    if (argc < 2) {
        std::puts("Usage : spmm_driver {matrix.smtx} [N]");
        return 2;
    }
    const int N = argc > 2 ? std::atoi(argv[2]) : 256;
    std::ifstream fin(argv[1]);
    half *A = nullptr, *B = nullptr;
    int M = 0, K = 0, nnz = 0;
    smtx_input_to_Dense(fin, &A, argv[1], &M, &K, &nnz);
    prepare_cpu_matrix(&B, K, N, 0.1f, false, 1234);
    float *gold = nullptr, *C = nullptr;
    prepare_cpu_matrix(&gold, M, N, 1.f, true);
    prepare_cpu_matrix(&C, M, N, 1.f, true);
    double t_gemm = -1, t_sp = -1, t_our = -1;
    perform_GemmEx(A, B, gold, M, N, K, 10, &t_gemm);
    perform_cuSPARSE_SpMM(A, B, C, M, N, K, 10, &t_sp);
    bool ok = compare_mat(gold, C, M * N, 1e-3f);
    if (!ok)
        std::puts("validation failed (cuSPARSE)");
    CSR *csrA = nullptr;
    convert_dense_to_csr(A, &csrA, M, K);
    std::memset(C, 0, sizeof(float) * (size_t)M * N);
    our_spmm_balanced(csrA, B, C, M, N, K, 10, &t_our);
    const bool ok_our = compare_mat(gold, C, M * N, 1e-3f);
    if (!ok_our)
        std::puts("validation failed (our_spmm_balanced)");
    std::printf("M=%d K=%d nnz=%d N=%d\n", M, K, nnz, N);
    std::printf("GemmEx : [%lf] ms\ncuSPARSE: [%lf] ms\nour: [%lf] ms\n", t_gemm, t_sp, t_our);
    destroy_csr(csrA);
    std::free(A);
    std::free(B);
    std::free(gold);
    std::free(C);
    return (ok && ok_our) ? 0 : 1;
}
