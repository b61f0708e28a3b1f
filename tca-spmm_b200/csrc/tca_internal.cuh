// tca_internal.cuh -- shared helpers of libtca_spmm: status plumbing, FP16
// helpers and launch constants. Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <cstdio>
#include <cstdarg>
#include "tca_spmm.h"

namespace tca {

constexpr int kSMs = 148;          // B200: 2 dies x 74 SMs
constexpr int kWindowRows = 128;   // rows per window = tcgen05 M
constexpr int kChunkCols = 64;     // condensed columns per tile = one 128-byte swizzle atom of FP16

// Records a formatted error for tca_last_error_string() and returns `status`.
int set_error(int status, const char *fmt, ...);
void clear_error();

#define TCA_CUDA_TRY(expr)                                                              \
    do {                                                                                \
        cudaError_t e_ = (expr);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return ::tca::set_error(TCA_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,        \
                                    cudaGetErrorString(e_), __FILE__, __LINE__);        \
    } while (0)

#define TCA_TRY(expr)                    \
    do {                                 \
        int s_ = (expr);                 \
        if (s_ != TCA_OK)                \
            return s_;                   \
    } while (0)

inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

constexpr int kSmRegs = 65536; // registers of one SM

// Registers that one block of kernel `fn` with `threads` threads holds on an
// SM: per warp, its registers per thread x 32 rounded up to the allocation
// unit of 256.
inline int block_regs(const void *fn, int threads, int *out)
{
    cudaFuncAttributes a;
    TCA_CUDA_TRY(cudaFuncGetAttributes(&a, fn));
    *out = ((a.numRegs * 32 + 255) / 256) * 256 * ((threads + 31) / 32);
    return TCA_OK;
}

// Device memory of the library (api.cu): stream-ordered allocations from a
// per-device memory pool that keeps freed memory for reuse (plan builds and
// host-buffer calls allocate and free dozens of arrays per call; plain
// cudaMalloc / cudaFree cost ~60 us each and cudaFree synchronises the device).
int dev_malloc(void **ptr, size_t bytes, cudaStream_t s);
void dev_free(void *ptr, cudaStream_t s);

// Checks the dense operands of a forward (api.cu).
int check_dense_args(const void *B, int ldb, int N, const void *C, int ldc, int c_dtype, int M, int K);

// Launchers implemented in the .cu files.
int launch_spmm_csr_cc(const int *row_ptr, const int *col_idx, const __half *vals, int M, int K, int nnz,
                       const __half *B, int ldb, int N, void *C, int ldc, int c_dtype,
                       float alpha, float beta, unsigned flags, cudaStream_t stream);

} // namespace tca
