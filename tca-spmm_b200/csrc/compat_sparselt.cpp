// compat_sparselt.cpp -- the reference's cuSPARSELt 2:4 comparator
// (perform_cuSPARSELT_24sparsity, src/spmm_cusparse.cu:2-179) with its exact
// signature: A (dense, row-major M x K, host FP16) is pruned to the 2:4
// pattern by cuSPARSELt itself (CUSPARSELT_PRUNE_SPMMA_STRIP: two of every
// four consecutive elements of a row are zeroed), compressed, and multiplied
// with B (row-major K x N, FP16): FP32 compute, FP16 C, alpha 1, beta 0,
// the default algorithm, num_iter timed calls; C is returned as FP32. It is a
// different product from the SpMM (A is pruned) and a reference point only.
//
// cuSPARSELt is loaded at the first call (dlopen), so that the library loads
// and every other entry point works where cuSPARSELt is absent; the call then
// reports an error instead.
#include <dlfcn.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cusparseLt.h>
#include <mutex>
#include <vector>
#include "tca_internal.cuh"
#include "tca_spmm_compat.h"

namespace tca {
void compat_report(int st);
}

using tca::set_error;

namespace {

#ifndef TCA_CUSPARSELT_LIB
#define TCA_CUSPARSELT_LIB ""
#endif

struct SpLt {
    bool ok = false;
    decltype(&cusparseLtInit) init;
    decltype(&cusparseLtDestroy) destroy;
    decltype(&cusparseLtStructuredDescriptorInit) structured;
    decltype(&cusparseLtDenseDescriptorInit) dense;
    decltype(&cusparseLtMatDescriptorDestroy) mat_destroy;
    decltype(&cusparseLtMatmulDescriptorInit) matmul_desc;
    decltype(&cusparseLtMatmulAlgSelectionInit) alg_init;
    decltype(&cusparseLtMatmulPlanInit) plan_init;
    decltype(&cusparseLtMatmulPlanDestroy) plan_destroy;
    decltype(&cusparseLtSpMMAPrune) prune;
    decltype(&cusparseLtSpMMAPruneCheck) prune_check;
    decltype(&cusparseLtSpMMACompressedSize) compressed_size;
    decltype(&cusparseLtSpMMACompress) compress;
    decltype(&cusparseLtMatmulGetWorkspace) workspace;
    decltype(&cusparseLtMatmul) matmul;
};

// The library from the loader's search path, else from the directory found
// when this library was built.
const SpLt &sparselt()
{
    static SpLt s;
    static std::once_flag once;
    std::call_once(once, [] {
        void *h = dlopen("libcusparseLt.so.0", RTLD_NOW | RTLD_LOCAL);
        if (!h && TCA_CUSPARSELT_LIB[0])
            h = dlopen(TCA_CUSPARSELT_LIB, RTLD_NOW | RTLD_LOCAL);
        if (!h)
            return;
        bool all = true;
        auto sym = [&](auto &fn, const char *name) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
            all = all && fn != nullptr;
        };
        sym(s.init, "cusparseLtInit");
        sym(s.destroy, "cusparseLtDestroy");
        sym(s.structured, "cusparseLtStructuredDescriptorInit");
        sym(s.dense, "cusparseLtDenseDescriptorInit");
        sym(s.mat_destroy, "cusparseLtMatDescriptorDestroy");
        sym(s.matmul_desc, "cusparseLtMatmulDescriptorInit");
        sym(s.alg_init, "cusparseLtMatmulAlgSelectionInit");
        sym(s.plan_init, "cusparseLtMatmulPlanInit");
        sym(s.plan_destroy, "cusparseLtMatmulPlanDestroy");
        sym(s.prune, "cusparseLtSpMMAPrune");
        sym(s.prune_check, "cusparseLtSpMMAPruneCheck");
        sym(s.compressed_size, "cusparseLtSpMMACompressedSize");
        sym(s.compress, "cusparseLtSpMMACompress");
        sym(s.workspace, "cusparseLtMatmulGetWorkspace");
        sym(s.matmul, "cusparseLtMatmul");
        s.ok = all;
    });
    return s;
}

} // namespace

#define LT_CUDA(expr)                                                                            \
    do {                                                                                         \
        cudaError_t e_ = (expr);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            st = set_error(TCA_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));               \
            goto done;                                                                           \
        }                                                                                        \
    } while (0)
#define LT_CALL(expr)                                                                            \
    do {                                                                                         \
        cusparseStatus_t e_ = (expr);                                                            \
        if (e_ != CUSPARSE_STATUS_SUCCESS) {                                                     \
            st = set_error(TCA_ERR_CUDA, "%s: cuSPARSELt status %d", #expr, (int)e_);            \
            goto done;                                                                           \
        }                                                                                        \
    } while (0)

void perform_cuSPARSELT_24sparsity(half *A, half *B, float *C, int M, int N, int K, int num_iter, double *elapsed)
{
    int st = TCA_OK;
    const SpLt &lt = sparselt();
    half *dA = nullptr, *dB = nullptr, *dC = nullptr, *dAc = nullptr;
    void *dAcBuf = nullptr, *dWs = nullptr;
    int *d_valid = nullptr;
    int valid = 1;
    size_t c_size = 0, c_buf_size = 0, ws_size = 0;
    cusparseLtHandle_t handle;
    cusparseLtMatDescriptor_t mA, mB, mC;
    cusparseLtMatmulDescriptor_t mm;
    cusparseLtMatmulAlgSelection_t alg;
    cusparseLtMatmulPlan_t plan;
    bool have_handle = false, have_a = false, have_b = false, have_c = false, have_plan = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t s = nullptr; // the default stream, as the reference
    float alpha = 1.f, beta = 0.f, ms = 0.f;
    std::vector<half> Ch;
    if (!lt.ok) {
        st = set_error(TCA_ERR_UNSUPPORTED, "perform_cuSPARSELT_24sparsity: libcusparseLt.so.0 could not be loaded");
        goto done;
    }
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) {
        st = set_error(TCA_ERR_INVALID_ARG, "perform_cuSPARSELT_24sparsity: invalid sizes or buffers");
        goto done;
    }
    if (num_iter < 1)
        num_iter = 1;
    LT_CUDA(cudaMalloc(&dA, sizeof(half) * (size_t)M * K));
    LT_CUDA(cudaMalloc(&dB, sizeof(half) * (size_t)K * N));
    LT_CUDA(cudaMalloc(&dC, sizeof(half) * (size_t)M * N));
    LT_CUDA(cudaMalloc(&d_valid, sizeof(int)));
    LT_CUDA(cudaMemcpy(dA, A, sizeof(half) * (size_t)M * K, cudaMemcpyHostToDevice));
    LT_CUDA(cudaMemcpy(dB, B, sizeof(half) * (size_t)K * N, cudaMemcpyHostToDevice));
    LT_CUDA(cudaMemset(dC, 0, sizeof(half) * (size_t)M * N));

    LT_CALL(lt.init(&handle));
    have_handle = true;
    // row-major operands, 16-byte alignment, A 50 % structured
    LT_CALL(lt.structured(&handle, &mA, M, K, K, 16, CUDA_R_16F, CUSPARSE_ORDER_ROW, CUSPARSELT_SPARSITY_50_PERCENT));
    have_a = true;
    LT_CALL(lt.dense(&handle, &mB, K, N, N, 16, CUDA_R_16F, CUSPARSE_ORDER_ROW));
    have_b = true;
    LT_CALL(lt.dense(&handle, &mC, M, N, N, 16, CUDA_R_16F, CUSPARSE_ORDER_ROW));
    have_c = true;
    LT_CALL(lt.matmul_desc(&handle, &mm, CUSPARSE_OPERATION_NON_TRANSPOSE, CUSPARSE_OPERATION_NON_TRANSPOSE, &mA,
                           &mB, &mC, &mC, CUSPARSE_COMPUTE_32F));
    LT_CALL(lt.alg_init(&handle, &alg, &mm, CUSPARSELT_MATMUL_ALG_DEFAULT));
    LT_CALL(lt.plan_init(&handle, &plan, &mm, &alg));
    have_plan = true;

    LT_CALL(lt.prune(&handle, &mm, dA, dA, CUSPARSELT_PRUNE_SPMMA_STRIP, s));
    LT_CALL(lt.prune_check(&handle, &mm, dA, d_valid, s));
    LT_CUDA(cudaMemcpy(&valid, d_valid, sizeof(int), cudaMemcpyDeviceToHost));
    if (valid != 0) {
        st = set_error(TCA_ERR_CUDA, "perform_cuSPARSELT_24sparsity: A is not 2:4 after pruning");
        goto done;
    }
    LT_CALL(lt.compressed_size(&handle, &plan, &c_size, &c_buf_size));
    LT_CUDA(cudaMalloc(&dAc, c_size));
    LT_CUDA(cudaMalloc(&dAcBuf, c_buf_size > 0 ? c_buf_size : 1));
    LT_CALL(lt.compress(&handle, &plan, dA, dAc, dAcBuf, s));
    LT_CALL(lt.workspace(&handle, &plan, &ws_size));
    if (ws_size > 0)
        LT_CUDA(cudaMalloc(&dWs, ws_size));

    LT_CUDA(cudaEventCreate(&e0));
    LT_CUDA(cudaEventCreate(&e1));
    LT_CUDA(cudaEventRecord(e0, s));
    for (int i = 0; i < num_iter; i++)
        LT_CALL(lt.matmul(&handle, &plan, &alpha, dAc, dB, &beta, dC, dC, dWs, nullptr, 0));
    LT_CUDA(cudaEventRecord(e1, s));
    LT_CUDA(cudaEventSynchronize(e1));
    LT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (elapsed)
        *elapsed = (double)ms / num_iter;

    Ch.resize((size_t)M * N);
    LT_CUDA(cudaMemcpy(Ch.data(), dC, sizeof(half) * Ch.size(), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < Ch.size(); i++)
        C[i] = __half2float(Ch[i]);
done:
    if (have_plan) lt.plan_destroy(&plan);
    if (have_a) lt.mat_destroy(&mA);
    if (have_b) lt.mat_destroy(&mB);
    if (have_c) lt.mat_destroy(&mC);
    if (have_handle) lt.destroy(&handle);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    cudaFree(dAc);
    cudaFree(dAcBuf);
    cudaFree(dWs);
    cudaFree(d_valid);
    if (st != TCA_OK)
        tca::compat_report(st);
}
