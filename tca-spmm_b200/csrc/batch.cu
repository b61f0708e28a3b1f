// batch.cu -- the batched forward as a CUDA graph, and its autotuner.
//
// A batch (many layers of different shapes, sparsity and N) runs as a few
// persistent launches (tca_spmm_batched / tca_spmm_fp8_batched). The host
// side of such a call -- argument checks, one TMA descriptor pair per item,
// kernel-parameter blocks of up to 32 items -- costs more than the launches'
// device time for small layers, so the batch is captured once into a CUDA
// graph and replayed: a replay is one cudaGraphLaunch.
//
// The autotuner picks, per item, the tensor-core N-slice width (n_tile) and
// the CUDA-core columns per lane (cc_cols) by timing each candidate on the
// item alone with CUDA events (median of a few runs). Items with different
// picks run in different launches, and launches of a batch run one after the
// other, so the per-item picks are then weighed as a whole against every
// uniform (n_tile, cc_cols) -- one tensor-core and one CUDA-core launch --
// by replaying each as a captured graph; the fastest is written back into
// the items (measured on a 24-layer batch: per-item picks in 3 launches
// 157 us, one uniform configuration in 2 launches 123 us). The reference has
// neither (its launch geometry is fixed by workload_manager,
// src/our_spmm.cu:347-471).
#include <algorithm>
#include <vector>
#include "tca_internal.cuh"
#include "plan.cuh"

struct tca_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace tca {
namespace {

int run_batch(const tca_batch_item_t *items, int n, int c_dtype, float alpha, float beta, unsigned flags, int precision,
              cudaStream_t s, void *const *events = nullptr)
{
    return precision == TCA_PRECISION_E4M3
               ? tca_spmm_fp8_batched(items, n, c_dtype, alpha, beta, flags, s, events)
               : tca_spmm_batched(items, n, c_dtype, alpha, beta, flags, s, events);
}

struct StreamGuard {
    cudaStream_t s = nullptr;
    ~StreamGuard() { if (s) cudaStreamDestroy(s); }
};

} // namespace
} // namespace tca

using namespace tca;

int tca_batch_graph_create(const tca_batch_item_t *items, int n_items, int c_dtype, float alpha, float beta,
                           unsigned flags, int precision, tca_graph_t *out)
{
    return tca_batch_graph_create_events(items, n_items, c_dtype, alpha, beta, flags, precision, nullptr, out);
}

int tca_batch_graph_create_events(const tca_batch_item_t *items, int n_items, int c_dtype, float alpha, float beta,
                                  unsigned flags, int precision, void *const *events, tca_graph_t *out)
{
    clear_error();
    if (!out) return set_error(TCA_ERR_INVALID_ARG, "graph output pointer is NULL");
    *out = nullptr;
    if (precision != TCA_PRECISION_F16 && precision != TCA_PRECISION_E4M3)
        return set_error(TCA_ERR_INVALID_ARG, "unknown precision %d", precision);
    StreamGuard g;
    TCA_CUDA_TRY(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking));
    // One eager run first: it does the one-time work (kernel attributes, the
    // E4M3 form of the plans, workspaces) that must not happen inside capture,
    // and validates every item.
    TCA_TRY(run_batch(items, n_items, c_dtype, alpha, beta, flags, precision, g.s));
    TCA_CUDA_TRY(cudaStreamSynchronize(g.s));
    cudaGraph_t graph = nullptr;
    TCA_CUDA_TRY(cudaStreamBeginCapture(g.s, cudaStreamCaptureModeRelaxed));
    const int st = run_batch(items, n_items, c_dtype, alpha, beta, flags, precision, g.s, events);
    const cudaError_t ce = cudaStreamEndCapture(g.s, &graph);
    if (st != TCA_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (ce != cudaSuccess)
        return set_error(TCA_ERR_CUDA, "stream capture of the batch failed: %s", cudaGetErrorString(ce));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(graph);
        return set_error(TCA_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(ie));
    }
    tca_graph *h = new tca_graph;
    h->graph = graph;
    h->exec = exec;
    *out = h;
    return TCA_OK;
}

int tca_batch_graph_launch(tca_graph_t g, tca_stream_t stream)
{
    clear_error();
    if (!g) return set_error(TCA_ERR_INVALID_ARG, "graph is NULL");
    TCA_CUDA_TRY(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    return TCA_OK;
}

int tca_batch_graph_destroy(tca_graph_t g)
{
    clear_error();
    if (!g) return TCA_OK;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return TCA_OK;
}

int tca_batch_autotune(tca_batch_item_t *items, int n_items, int c_dtype, int precision, int reps,
                       tca_stream_t stream)
{
    clear_error();
    if (n_items < 0 || (n_items > 0 && !items))
        return set_error(TCA_ERR_INVALID_ARG, "invalid batch");
    if (precision != TCA_PRECISION_F16 && precision != TCA_PRECISION_E4M3)
        return set_error(TCA_ERR_INVALID_ARG, "unknown precision %d", precision);
    reps = std::max(1, std::min(reps, 50));
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TCA_CUDA_TRY(cudaEventCreate(&e0));
    const cudaError_t ee = cudaEventCreate(&e1);
    if (ee != cudaSuccess) {
        cudaEventDestroy(e0);
        return set_error(TCA_ERR_CUDA, "cudaEventCreate failed: %s", cudaGetErrorString(ee));
    }
    int status = TCA_OK;
    // time one candidate: warm-up, then the median of `reps` runs of the item alone
    auto time_item = [&](const tca_batch_item_t &it, float *us) -> int {
        TCA_TRY(run_batch(&it, 1, c_dtype, 1.f, 0.f, 0, precision, s));
        std::vector<float> t;
        for (int r = 0; r < reps; r++) {
            TCA_CUDA_TRY(cudaEventRecord(e0, s));
            TCA_TRY(run_batch(&it, 1, c_dtype, 1.f, 0.f, 0, precision, s));
            TCA_CUDA_TRY(cudaEventRecord(e1, s));
            TCA_CUDA_TRY(cudaEventSynchronize(e1));
            float ms = 0.f;
            TCA_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
            t.push_back(ms * 1000.f);
        }
        std::nth_element(t.begin(), t.begin() + t.size() / 2, t.end());
        *us = t[t.size() / 2];
        return TCA_OK;
    };
    for (int i = 0; i < n_items && status == TCA_OK; i++) {
        tca_batch_item_t best = items[i];
        float best_us = 3.4e38f;
        const int N = items[i].N;
        std::vector<int> tiles = precision == TCA_PRECISION_E4M3 ? std::vector<int>{128, 256}
                                                                : std::vector<int>{64, 128, 256};
        std::vector<int> cols = {2, 4, 8};
        if (precision == TCA_PRECISION_F16)
            cols.push_back(16); // the tensor-core item kernel
        for (int nt : tiles) {
            if (nt > 64 && nt / 2 >= N && !(precision == TCA_PRECISION_E4M3 && nt == 128))
                continue; // a slice at least twice as wide as N only adds zero columns
            for (int w : cols) {
                if (w > 2 && w < 16 && w * 16 > N)
                    continue; // fewer than half of the lanes would have columns
                tca_batch_item_t cand = items[i];
                cand.n_tile = nt;
                cand.cc_cols = w;
                float us = 0.f;
                status = time_item(cand, &us);
                if (status != TCA_OK)
                    break;
                if (us < best_us) {
                    best_us = us;
                    best = cand;
                }
            }
            if (status != TCA_OK)
                break;
        }
        if (status == TCA_OK)
            items[i] = best;
    }
    // the whole batch: the per-item picks against each uniform configuration
    auto time_batch = [&](const std::vector<tca_batch_item_t> &cand, float *us) -> int {
        tca_graph_t g = nullptr;
        TCA_TRY(tca_batch_graph_create(cand.data(), (int)cand.size(), c_dtype, 1.f, 0.f, 0, precision, &g));
        int st = TCA_OK;
        std::vector<float> t;
        for (int r = -1; r < reps && st == TCA_OK; r++) { // r = -1: warm-up
            cudaError_t e = cudaEventRecord(e0, s);
            if (e == cudaSuccess) e = cudaGraphLaunch(g->exec, s);
            if (e == cudaSuccess) e = cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess)
                st = set_error(TCA_ERR_CUDA, "timing a batch graph failed: %s", cudaGetErrorString(e));
            else if (r >= 0)
                t.push_back(ms * 1000.f);
        }
        tca_batch_graph_destroy(g);
        if (st != TCA_OK)
            return st;
        std::nth_element(t.begin(), t.begin() + t.size() / 2, t.end());
        *us = t[t.size() / 2];
        return TCA_OK;
    };
    if (status == TCA_OK && n_items > 1) {
        std::vector<tca_batch_item_t> best(items, items + n_items);
        float best_us = 0.f;
        status = time_batch(best, &best_us);
        const std::vector<int> tiles = precision == TCA_PRECISION_E4M3 ? std::vector<int>{128, 256}
                                                                       : std::vector<int>{64, 128, 256};
        std::vector<int> cols = {2, 4, 8};
        if (precision == TCA_PRECISION_F16)
            cols.push_back(16);
        for (int nt : tiles)
            for (int w : cols) {
                if (status != TCA_OK)
                    break;
                std::vector<tca_batch_item_t> cand(items, items + n_items);
                for (auto &it : cand) {
                    it.n_tile = nt;
                    it.cc_cols = w;
                }
                float us = 0.f;
                status = time_batch(cand, &us);
                if (status == TCA_OK && us < best_us) {
                    best_us = us;
                    best = cand;
                }
            }
        if (status == TCA_OK)
            std::copy(best.begin(), best.end(), items);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return status;
}
