// fp8.cu -- the FP8-E4M3 forward: quantization of A (per sorted row) and of
// B (per column), and the entry points that run the tensor-core and CUDA-core
// kernels on the quantized operands.
//
// Scales: s = max|x| / 448 over the row of A (or column of B); 1 when the row
// or column is all zero. Values: q = E4M3(x / s) for A and E4M3(x * r) with
// r = 1 / s rounded to FP32 for B (a multiply per element instead of a
// division), round to nearest even, saturating at +-448 (cvt.rn.satfinite). Products q_a * q_b are exact in
// FP32; sums accumulate in FP32; the result is multiplied by s_a[row] *
// s_b[col] before alpha / beta.
//
// The reference has no reduced-precision path; this is a new component of the
// rebuild, checked against a CPU restatement of the same quantization.
#include <cuda_fp8.h>
#include <algorithm>
#include <mutex>
#include <vector>
#include "tca_internal.cuh"
#include "plan.cuh"

namespace tca {
namespace {

__device__ __forceinline__ uint8_t to_e4m3(float x)
{
    return (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
}

__device__ __forceinline__ float scale_of(float amax) { return amax > 0.f ? amax / kE4M3Max : 1.f; }

// One warp per sorted row: the row's scale and its quantized values.
__global__ void k_quant_rows(const int *__restrict__ p_row_ptr, const __half *__restrict__ p_val, int M,
                             float *__restrict__ row_scale, uint8_t *__restrict__ p_val_f8)
{
    const int lane = threadIdx.x & 31;
    const long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= M)
        return;
    const int j0 = p_row_ptr[r], j1 = p_row_ptr[r + 1];
    float m = 0.f;
    for (int j = j0 + lane; j < j1; j += 32) m = fmaxf(m, fabsf(__half2float(p_val[j])));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    const float s = scale_of(m);
    if (lane == 0)
        row_scale[r] = s;
    for (int j = j0 + lane; j < j1; j += 32) p_val_f8[j] = to_e4m3(__half2float(p_val[j]) / s);
}

// Tile entries with their E4M3 value in the low byte (tile_src indexes p_val).
__global__ void k_entries_f8(const uint32_t *__restrict__ entries, const int *__restrict__ tile_src,
                             const uint8_t *__restrict__ p_val_f8, uint32_t *__restrict__ out, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = (entries[i] & 0xffff0000u) | (uint32_t)p_val_f8[tile_src[i]];
}

// Dense 128 x 64 E4M3 images in the 64-byte swizzled K-major layout.
__global__ void __launch_bounds__(256)
k_render_images_f8(const int *__restrict__ img_chunk, const int *__restrict__ tile_ptr,
                   const uint32_t *__restrict__ entries_f8, uint8_t *__restrict__ images)
{
    // rendered in shared memory, written out in 16-byte stores (as k_render_images)
    constexpr int kBytes = kWindowRows * kChunkCols;
    __shared__ __align__(16) uint8_t tile[kBytes];
    const int m = blockIdx.x;
    const int c = img_chunk[m];
    for (int k = threadIdx.x; k < kBytes / 16; k += blockDim.x)
        reinterpret_cast<uint4 *>(tile)[k] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    const int e0 = tile_ptr[c], e1 = tile_ptr[c + 1];
    for (int e = e0 + (int)threadIdx.x; e < e1; e += 8 * (int)blockDim.x) { // 8 loads in flight per thread
        uint32_t v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int eu = e + u * (int)blockDim.x;
            v[u] = eu < e1 ? entries_f8[eu] : 0xffffffffu;
        }
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (v[u] != 0xffffffffu)
                tile[swz64_offset(v[u] >> 22, (v[u] >> 16) & 63u)] = (uint8_t)(v[u] & 0xffu);
    }
    __syncthreads();
    uint4 *img = reinterpret_cast<uint4 *>(images + (size_t)m * kBytes);
    for (int k = threadIdx.x; k < kBytes / 16; k += blockDim.x)
        img[k] = reinterpret_cast<const uint4 *>(tile)[k];
}

// B quantization of up to kMaxQJobs matrices per launch (blockIdx.z = matrix).
constexpr int kMaxQJobs = 32;
struct QJob {
    const __half *B;
    uint8_t *Bq;
    unsigned *colmax; // column maxima as FP32 bit patterns, then the scales (in place)
    int ldb, ldq, K, N;
};
struct QBatch {
    int n;
    QJob job[kMaxQJobs];
};

__global__ void k_col_zero(const __grid_constant__ QBatch b)
{
    const QJob &q = b.job[blockIdx.z];
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < q.N; n += gridDim.x * blockDim.x) q.colmax[n] = 0u;
}

// B rows load 8 halves (16 bytes) at a time when B and its rows are 16-byte
// aligned; otherwise one half at a time.
__device__ __forceinline__ bool vec8_ok(const QJob &q)
{
    return (reinterpret_cast<uintptr_t>(q.B) & 15u) == 0 && (q.ldb & 7) == 0;
}

__device__ __forceinline__ void load8h(const QJob &q, int k, int n, bool vec, float *v)
{
    const __half *row = q.B + (size_t)k * q.ldb;
    if (vec && n + 8 <= q.N) {
        const uint4 u = __ldg(reinterpret_cast<const uint4 *>(row + n));
        const __half2 *h = reinterpret_cast<const __half2 *>(&u);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float2 f = __half22float2(h[i]);
            v[2 * i] = f.x;
            v[2 * i + 1] = f.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = n + i < q.N ? __half2float(row[n + i]) : 0.f;
    }
}

// The two B passes tile B into blocks of 64 rows x 256 columns: thread
// (x, y) of a 32 x 8 block takes the 8 consecutive columns (one 16-byte
// vector) 8 x of the block's columns in the 8 consecutive rows 8 y .. of its
// rows, so that a warp reads whole 512-byte row segments; all 8 loads of a
// thread are issued before the first is used (blockIdx.z = matrix).
constexpr int kQTileRows = 64, kQTileCols = 256, kQRows = kQTileRows / 8;

struct QTile {
    int n, k0, k1;
    bool fast; // full 16-byte vectors and all kQRows rows in range
};

__device__ __forceinline__ QTile q_tile(const QJob &q)
{
    QTile t;
    t.n = blockIdx.x * kQTileCols + threadIdx.x * 8;
    t.k0 = blockIdx.y * kQTileRows + threadIdx.y * kQRows;
    t.k1 = min(q.K, t.k0 + kQRows);
    t.fast = vec8_ok(q) && t.n + 8 <= q.N && t.k0 + kQRows <= q.K;
    return t;
}

__device__ __forceinline__ void load_rows8(const QJob &q, const QTile &t, uint4 *r)
{
#pragma unroll
    for (int j = 0; j < kQRows; j++)
        r[j] = __ldg(reinterpret_cast<const uint4 *>(q.B + (size_t)(t.k0 + j) * q.ldb + t.n));
    asm volatile("" ::: "memory"); // every load issued before the first use
}

// Column absolute maxima (FP32 bit patterns order like the non-negative
// values): per thread the maxima of its rows, per block the maxima over its
// 8 row slices (shared memory), then one atomicMax per column and block.
__global__ void __launch_bounds__(256) k_col_absmax(const __grid_constant__ QBatch b)
{
    const QJob &q = b.job[blockIdx.z];
    if ((int)blockIdx.x * kQTileCols >= q.N || (int)blockIdx.y * kQTileRows >= q.K)
        return; // whole block
    __shared__ float s_m[8][8][32]; // [row slice][column in vector][vector]
    const QTile t = q_tile(q);
    float m[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (t.fast) {
        uint4 r[kQRows];
        load_rows8(q, t, r);
#pragma unroll
        for (int j = 0; j < kQRows; j++) {
            const __half2 *h = reinterpret_cast<const __half2 *>(&r[j]);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float2 f = __half22float2(h[i]);
                m[2 * i] = fmaxf(m[2 * i], fabsf(f.x));
                m[2 * i + 1] = fmaxf(m[2 * i + 1], fabsf(f.y));
            }
        }
    } else if (t.n < q.N) {
        const bool vec = vec8_ok(q);
        for (int k = t.k0; k < t.k1; k++) {
            float v[8];
            load8h(q, k, t.n, vec, v);
#pragma unroll
            for (int i = 0; i < 8; i++) m[i] = fmaxf(m[i], fabsf(v[i]));
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) s_m[threadIdx.y][i][threadIdx.x] = m[i];
    __syncthreads();
    const int c = threadIdx.y * 32 + threadIdx.x; // column of the block: vector c / 8, element c % 8
    float v = 0.f;
#pragma unroll
    for (int y = 0; y < 8; y++) v = fmaxf(v, s_m[y][c & 7][c >> 3]);
    const int col = blockIdx.x * kQTileCols + c;
    if (col < q.N && v > 0.f) // the maxima start at 0
        atomicMax(q.colmax + col, __float_as_uint(v));
}

// Bq[k, n] = E4M3(B[k, n] / s[n]) over the thread's rows and columns.
__global__ void __launch_bounds__(256) k_quant_cols(const __grid_constant__ QBatch b)
{
    const QJob &q = b.job[blockIdx.z];
    const QTile t = q_tile(q);
    if (t.n >= q.N || t.k0 >= q.K)
        return;
    float s[8]; // reciprocals of the column scales (B is multiplied by them)
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] = 1.f / (t.n + i < q.N ? scale_of(__uint_as_float(q.colmax[t.n + i])) : 1.f);
    const bool st8 = (q.ldq & 7) == 0 && (reinterpret_cast<uintptr_t>(q.Bq) & 7u) == 0;
    if (t.fast && st8) {
        uint4 r[kQRows];
        load_rows8(q, t, r);
#pragma unroll
        for (int j = 0; j < kQRows; j++) {
            const __half2 *h = reinterpret_cast<const __half2 *>(&r[j]);
            uint32_t w[2];
#pragma unroll
            for (int p = 0; p < 2; p++) {
                const float2 f0 = __half22float2(h[2 * p]), f1 = __half22float2(h[2 * p + 1]);
                const uint32_t q0 = __nv_cvt_float2_to_fp8x2(make_float2(f0.x * s[4 * p], f0.y * s[4 * p + 1]),
                                                             __NV_SATFINITE, __NV_E4M3);
                const uint32_t q1 = __nv_cvt_float2_to_fp8x2(make_float2(f1.x * s[4 * p + 2], f1.y * s[4 * p + 3]),
                                                             __NV_SATFINITE, __NV_E4M3);
                w[p] = (q0 & 0xffffu) | (q1 << 16);
            }
            *reinterpret_cast<uint2 *>(q.Bq + (size_t)(t.k0 + j) * q.ldq + t.n) = make_uint2(w[0], w[1]);
        }
        return;
    }
    const bool vec = vec8_ok(q);
    for (int k = t.k0; k < t.k1; k++) {
        float v[8];
        load8h(q, k, t.n, vec, v);
        uint32_t lo = 0, hi = 0;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            lo |= (uint32_t)to_e4m3(v[i] * s[i]) << (8 * i);
            hi |= (uint32_t)to_e4m3(v[4 + i] * s[4 + i]) << (8 * i);
        }
        uint8_t *dst = q.Bq + (size_t)k * q.ldq + t.n;
        if (t.n + 8 <= q.N && (reinterpret_cast<uintptr_t>(dst) & 7u) == 0) {
            *reinterpret_cast<uint2 *>(dst) = make_uint2(lo, hi);
        } else {
            for (int i = 0; t.n + i < q.N && i < 8; i++) dst[i] = (uint8_t)((i < 4 ? lo : hi) >> (8 * (i & 3)));
        }
    }
}

// The whole quantization of B in one launch: one block per (matrix, strip of
// SW columns) reads the strip's K rows for the column maxima, reduces them
// (warp shuffles, then the block's 8 warps), writes the scales and reads the
// strip again (now from L2) to quantize it. Nothing is cleared beforehand
// and no block depends on another. A thread takes 8 consecutive columns
// (16 bytes) of every RPP-th row, four rows' loads in flight.
template <int SW>
__global__ void __launch_bounds__(256) k_quant_b_strip(const __grid_constant__ QBatch b)
{
    constexpr int TPR = SW / 8;    // threads per row
    constexpr int RPP = 256 / TPR; // rows per pass
    const QJob &q = b.job[blockIdx.y];
    const int n0 = blockIdx.x * SW;
    if (n0 >= q.N)
        return; // whole block
    __shared__ float s_m[8][SW];
    __shared__ float s_scale[SW];
    const int tx = threadIdx.x % TPR, ty = threadIdx.x / TPR;
    const int n = n0 + tx * 8;
    const bool vec = vec8_ok(q);
    float m[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (n < q.N) {
        for (int k = ty; k < q.K; k += 4 * RPP) {
            float v[4][8];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if (k + u * RPP < q.K)
                    load8h(q, k + u * RPP, n, vec, v[u]);
                else
#pragma unroll
                    for (int i = 0; i < 8; i++) v[u][i] = 0.f;
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int i = 0; i < 8; i++) m[i] = fmaxf(m[i], fabsf(v[u][i]));
        }
    }
    // lanes of a warp with the same columns differ by multiples of TPR
#pragma unroll
    for (int o = TPR; o < 32; o <<= 1)
#pragma unroll
        for (int i = 0; i < 8; i++) m[i] = fmaxf(m[i], __shfl_xor_sync(0xffffffffu, m[i], o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane < TPR)
#pragma unroll
        for (int i = 0; i < 8; i++) s_m[warp][lane * 8 + i] = m[i];
    __syncthreads();
    if ((int)threadIdx.x < SW) {
        float v = 0.f;
#pragma unroll
        for (int w = 0; w < 8; w++) v = fmaxf(v, s_m[w][threadIdx.x]);
        const float sc = scale_of(v);
        s_scale[threadIdx.x] = sc;
        if (n0 + (int)threadIdx.x < q.N)
            q.colmax[n0 + threadIdx.x] = __float_as_uint(sc);
    }
    __syncthreads();
    if (n >= q.N)
        return;
    float sc[8]; // reciprocals of the column scales (B is multiplied by them)
#pragma unroll
    for (int i = 0; i < 8; i++) sc[i] = 1.f / s_scale[tx * 8 + i];
    const bool st8 = n + 8 <= q.N && (q.ldq & 7) == 0 && (reinterpret_cast<uintptr_t>(q.Bq) & 7u) == 0;
    for (int k = ty; k < q.K; k += 4 * RPP) {
        float v[4][8];
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (k + u * RPP < q.K)
                load8h(q, k + u * RPP, n, vec, v[u]);
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (k + u * RPP >= q.K)
                break;
            uint32_t lo = 0, hi = 0;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                lo |= (uint32_t)to_e4m3(v[u][i] * sc[i]) << (8 * i);
                hi |= (uint32_t)to_e4m3(v[u][4 + i] * sc[4 + i]) << (8 * i);
            }
            uint8_t *dst = q.Bq + (size_t)(k + u * RPP) * q.ldq + n;
            if (st8)
                *reinterpret_cast<uint2 *>(dst) = make_uint2(lo, hi);
            else
                for (int i = 0; n + i < q.N && i < 8; i++) dst[i] = (uint8_t)((i < 4 ? lo : hi) >> (8 * (i & 3)));
        }
    }
}

// 8 halves of B row k from column n as raw FP16 bits (zeros past N).
__device__ __forceinline__ uint4 load8raw(const QJob &q, int k, int n, bool vec)
{
    const __half *row = q.B + (size_t)k * q.ldb;
    if (vec && n + 8 <= q.N)
        return __ldg(reinterpret_cast<const uint4 *>(row + n));
    unsigned short h[8];
#pragma unroll
    for (int i = 0; i < 8; i++) h[i] = n + i < q.N ? __half_as_ushort(row[n + i]) : (unsigned short)0;
    return make_uint4(h[0] | (unsigned)h[1] << 16, h[2] | (unsigned)h[3] << 16, h[4] | (unsigned)h[5] << 16,
                      h[6] | (unsigned)h[7] << 16);
}

// k_quant_b_strip with the strip kept in shared memory (K x SW halves, when
// that fits): every row of the strip is read from HBM once, with all of a
// thread's loads (K / RPP of them, at most kQStripLoads) in flight together,
// written to shared memory on arrival and folded into the column maxima; the
// quantization then reads shared memory. One HBM round trip per block instead
// of two passes of dependent loads (measured on the headline batch: 23 us for
// the two-pass kernel under the profiler).
constexpr int kQStripLoads = 8;             // rows a thread loads before the first use
constexpr size_t kQStripSmem = 96 * 1024;     // largest strip kept in shared memory (two blocks per SM)

template <int SW>
__global__ void __launch_bounds__(256) k_quant_b_smem(const __grid_constant__ QBatch b)
{
    constexpr int TPR = SW / 8;
    constexpr int RPP = 256 / TPR;
    extern __shared__ uint4 s_strip[]; // [K][TPR]
    __shared__ float s_m[8][SW];
    __shared__ float s_scale[SW];
    const QJob &q = b.job[blockIdx.y];
    const int n0 = blockIdx.x * SW;
    if (n0 >= q.N)
        return; // whole block
    const int tx = threadIdx.x % TPR, ty = threadIdx.x / TPR;
    const int n = n0 + tx * 8;
    const bool vec = vec8_ok(q);
    float m[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int k0 = ty; k0 < q.K; k0 += kQStripLoads * RPP) {
        uint4 r[kQStripLoads];
#pragma unroll
        for (int u = 0; u < kQStripLoads; u++) {
            const int k = k0 + u * RPP;
            r[u] = (k < q.K && n < q.N) ? load8raw(q, k, n, vec) : make_uint4(0, 0, 0, 0);
        }
#pragma unroll
        for (int u = 0; u < kQStripLoads; u++) {
            const int k = k0 + u * RPP;
            if (k < q.K)
                s_strip[k * TPR + tx] = r[u];
            const __half2 *h = reinterpret_cast<const __half2 *>(&r[u]);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float2 f = __half22float2(h[i]);
                m[2 * i] = fmaxf(m[2 * i], fabsf(f.x));
                m[2 * i + 1] = fmaxf(m[2 * i + 1], fabsf(f.y));
            }
        }
    }
#pragma unroll
    for (int o = TPR; o < 32; o <<= 1)
#pragma unroll
        for (int i = 0; i < 8; i++) m[i] = fmaxf(m[i], __shfl_xor_sync(0xffffffffu, m[i], o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane < TPR)
#pragma unroll
        for (int i = 0; i < 8; i++) s_m[warp][lane * 8 + i] = m[i];
    __syncthreads(); // also: the whole strip is in shared memory
    if ((int)threadIdx.x < SW) {
        float v = 0.f;
#pragma unroll
        for (int w = 0; w < 8; w++) v = fmaxf(v, s_m[w][threadIdx.x]);
        const float sc = scale_of(v);
        s_scale[threadIdx.x] = sc;
        if (n0 + (int)threadIdx.x < q.N)
            q.colmax[n0 + threadIdx.x] = __float_as_uint(sc);
    }
    __syncthreads();
    if (n >= q.N)
        return;
    float sc[8]; // reciprocals of the column scales (B is multiplied by them)
#pragma unroll
    for (int i = 0; i < 8; i++) sc[i] = 1.f / s_scale[tx * 8 + i];
    const bool st8 = n + 8 <= q.N && (q.ldq & 7) == 0 && (reinterpret_cast<uintptr_t>(q.Bq) & 7u) == 0;
    for (int k = ty; k < q.K; k += RPP) {
        const uint4 r = s_strip[k * TPR + tx];
        const __half2 *h = reinterpret_cast<const __half2 *>(&r);
        uint32_t w[2];
#pragma unroll
        for (int p = 0; p < 2; p++) {
            const float2 f0 = __half22float2(h[2 * p]), f1 = __half22float2(h[2 * p + 1]);
            const uint32_t lo = __nv_cvt_float2_to_fp8x2(make_float2(f0.x * sc[4 * p], f0.y * sc[4 * p + 1]),
                                                         __NV_SATFINITE, __NV_E4M3);
            const uint32_t hi = __nv_cvt_float2_to_fp8x2(make_float2(f1.x * sc[4 * p + 2], f1.y * sc[4 * p + 3]),
                                                         __NV_SATFINITE, __NV_E4M3);
            w[p] = lo | hi << 16;
        }
        uint8_t *dst = q.Bq + (size_t)k * q.ldq + n;
        if (st8)
            *reinterpret_cast<uint2 *>(dst) = make_uint2(w[0], w[1]);
        else
            for (int i = 0; n + i < q.N && i < 8; i++) dst[i] = (uint8_t)(w[i >> 2] >> (8 * (i & 3)));
    }
}

// column maxima -> scales, in place
__global__ void k_col_scale(const __grid_constant__ QBatch b)
{
    const QJob &q = b.job[blockIdx.z];
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < q.N; n += gridDim.x * blockDim.x)
        q.colmax[n] = __float_as_uint(scale_of(__uint_as_float(q.colmax[n])));
}

unsigned blocks(long long n, int per) { return (unsigned)((n + per - 1) / per); }

int quantize_b_batch(const QBatch &b, cudaStream_t s)
{
    int maxK = 0, maxN = 0;
    for (int i = 0; i < b.n; i++) {
        maxK = std::max(maxK, b.job[i].K);
        maxN = std::max(maxN, b.job[i].N);
    }
    if (b.n == 0 || maxK == 0 || maxN == 0)
        return TCA_OK;
    const unsigned z = (unsigned)b.n;
    // One launch, a block per column strip (k_quant_b_strip), when the strips
    // give about two blocks per SM; else (few, wide matrices) the column
    // maxima of 64-row tiles with one atomic per column and block, then the
    // quantization and the scales, in four launches.
    auto strips = [&](int sw) { return (long long)b.n * blocks(maxN, sw); };
    if (strips(8) >= kSMs) {
        const int sw = strips(64) >= 2 * kSMs ? 64 : strips(32) >= 2 * kSMs ? 32 : strips(16) >= 2 * kSMs ? 16 : 8;
        const dim3 grid(blocks(maxN, sw), z);
        const size_t strip_bytes = (size_t)maxK * sw * 2;
        if (strip_bytes <= kQStripSmem) {
            auto launch = [&](auto kernel) -> int {
                TCA_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kQStripSmem));
                kernel<<<grid, 256, strip_bytes, s>>>(b);
                TCA_CUDA_TRY(cudaGetLastError());
                return TCA_OK;
            };
            switch (sw) {
            case 64: return launch(k_quant_b_smem<64>);
            case 32: return launch(k_quant_b_smem<32>);
            case 16: return launch(k_quant_b_smem<16>);
            default: return launch(k_quant_b_smem<8>);
            }
        }
        switch (sw) {
        case 64: k_quant_b_strip<64><<<grid, 256, 0, s>>>(b); break;
        case 32: k_quant_b_strip<32><<<grid, 256, 0, s>>>(b); break;
        case 16: k_quant_b_strip<16><<<grid, 256, 0, s>>>(b); break;
        default: k_quant_b_strip<8><<<grid, 256, 0, s>>>(b); break;
        }
        TCA_CUDA_TRY(cudaGetLastError());
        return TCA_OK;
    }
    const dim3 tiles(blocks(maxN, kQTileCols), blocks(maxK, kQTileRows), z), tile_threads(32, 8);
    if (tiles.y > 65535u)
        return set_error(TCA_ERR_INVALID_ARG, "B has too many rows to quantize (K=%d)", maxK);
    k_col_zero<<<dim3(blocks(maxN, 256), 1, z), 256, 0, s>>>(b);
    k_col_absmax<<<tiles, tile_threads, 0, s>>>(b);
    k_quant_cols<<<tiles, tile_threads, 0, s>>>(b);
    k_col_scale<<<dim3(blocks(maxN, 256), 1, z), 256, 0, s>>>(b);
    TCA_CUDA_TRY(cudaGetLastError());
    return TCA_OK;
}

int quantize_b(const __half *B, int ldb, int K, int N, uint8_t *Bq, int ldq, float *scale, cudaStream_t s)
{
    QBatch b;
    b.n = 1;
    b.job[0] = QJob{B, Bq, reinterpret_cast<unsigned *>(scale), ldb, ldq, K, N};
    return quantize_b_batch(b, s);
}

int quantize_plan(tca_plan *p, cudaStream_t s)
{
    if (!p->row_scale) {
        auto alloc = [&](void **ptr, size_t b) -> int {
            TCA_TRY(dev_malloc(ptr, b, s));
            p->bytes += b;
            return TCA_OK;
        };
        TCA_TRY(alloc((void **)&p->row_scale, sizeof(float) * (size_t)p->M));
        TCA_TRY(alloc((void **)&p->p_val_f8, (size_t)p->nnz));
        TCA_TRY(alloc((void **)&p->tile_entries_f8, sizeof(uint32_t) * ((size_t)p->tc_nnz + kEntryPad)));
        TCA_TRY(alloc((void **)&p->images_f8, (size_t)p->n_images * kWindowRows * kChunkCols));
        TCA_CUDA_TRY(cudaMemsetAsync(p->tile_entries_f8, 0, sizeof(uint32_t) * ((size_t)p->tc_nnz + kEntryPad), s));
    }
    if (p->M > 0)
        k_quant_rows<<<blocks((long long)p->M * 32, 256), 256, 0, s>>>(p->p_row_ptr, p->p_val, p->M, p->row_scale,
                                                                       p->p_val_f8);
    if (p->tc_nnz > 0)
        k_entries_f8<<<blocks(p->tc_nnz, 256), 256, 0, s>>>(p->tile_entries, p->tile_src, p->p_val_f8,
                                                            p->tile_entries_f8, p->tc_nnz);
    if (p->n_images > 0)
        k_render_images_f8<<<p->n_images, 256, 0, s>>>(p->img_chunk, p->tile_ptr, p->tile_entries_f8, p->images_f8);
    TCA_CUDA_TRY(cudaGetLastError());
    p->has_fp8 = true;
    return TCA_OK;
}

// The plan's B workspace for E4M3 forwards: K x ldq bytes, then N scales.
int plan_workspace(tca_plan *p, int N, uint8_t **Bq, int *ldq, float **scale)
{
    const int q = (N + 15) & ~15;
    const size_t bq = ((size_t)p->K * q + 255) & ~(size_t)255;
    const size_t need = bq + sizeof(float) * (size_t)q;
    if (need > p->fp8_ws_bytes) {
        if (p->fp8_ws) {
            TCA_CUDA_TRY(cudaDeviceSynchronize()); // queued work on any stream may still read it
            dev_free(p->fp8_ws, nullptr);
            p->bytes -= p->fp8_ws_bytes;
            p->fp8_ws = nullptr;
            p->fp8_ws_bytes = 0;
        }
        TCA_TRY(dev_malloc(&p->fp8_ws, need, nullptr));
        TCA_CUDA_TRY(cudaStreamSynchronize(nullptr)); // usable from every stream
        p->fp8_ws_bytes = need;
        p->bytes += need;
    }
    *Bq = static_cast<uint8_t *>(p->fp8_ws);
    *ldq = q;
    *scale = reinterpret_cast<float *>(static_cast<uint8_t *>(p->fp8_ws) + bq);
    return TCA_OK;
}

// The E4M3 job of one forward; B's quantization is appended to `qb` (flushed
// by the caller) when given, else run here.
int make_fp8_job(tca_plan_t p, const void *B, int ldb, int N, void *C, int ldc, int c_dtype, bool batched,
                 cudaStream_t s, SpmmJob *job, QBatch *qb)
{
    if (!p) return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    TCA_TRY(check_dense_args(B, ldb, N, C, ldc, c_dtype, p->M, p->K));
    const size_t c_elem = c_dtype == TCA_DTYPE_F16 ? 2 : 4;
    if (p->M > 0 && N > 0 && (N % 8 != 0 || !aligned16(C) || ((size_t)ldc * c_elem) % 16 != 0))
        return set_error(TCA_ERR_UNSUPPORTED,
                         "the E4M3 forward needs N %% 8 == 0 and a 16-byte aligned C with 16-byte aligned rows");
    if (!p->has_fp8)
        TCA_TRY(quantize_plan(p, s));
    job->p = p;
    job->B = (const __half *)B;
    job->C = C;
    job->ldb = ldb;
    job->N = N;
    job->ldc = ldc;
    job->f8 = true;
    job->tc = p->n_tc > 0;
    job->n_tile = pick_tc_tile(p, N, batched, true);
    if (p->M == 0 || N == 0 || p->K == 0)
        return TCA_OK;
    uint8_t *Bq;
    float *scale;
    int ldq;
    TCA_TRY(plan_workspace(p, N, &Bq, &ldq, &scale));
    const QJob q{(const __half *)B, Bq, reinterpret_cast<unsigned *>(scale), ldb, ldq, p->K, N};
    if (qb) {
        if (qb->n == kMaxQJobs) {
            TCA_TRY(quantize_b_batch(*qb, s));
            qb->n = 0;
        }
        qb->job[qb->n++] = q;
    } else {
        TCA_TRY(quantize_b(q.B, ldb, p->K, N, Bq, ldq, scale, s));
    }
    job->Bq = Bq;
    job->ldq = ldq;
    job->col_scale = scale;
    return TCA_OK;
}

} // namespace

int plan_requantize_fp8(tca_plan *p, cudaStream_t s)
{
    return p->has_fp8 ? quantize_plan(p, s) : TCA_OK;
}

void plan_free_fp8(tca_plan *p)
{
    void *arrs[] = {p->row_scale, p->p_val_f8, p->tile_entries_f8, p->images_f8, p->fp8_ws};
    for (void *a : arrs)
        if (a) dev_free(a, nullptr);
    p->row_scale = nullptr;
    p->p_val_f8 = nullptr;
    p->tile_entries_f8 = nullptr;
    p->images_f8 = nullptr;
    p->fp8_ws = nullptr;
    p->fp8_ws_bytes = 0;
    p->has_fp8 = false;
}

} // namespace tca

using namespace tca;

int tca_plan_quantize_fp8(tca_plan_t p, tca_stream_t stream)
{
    clear_error();
    if (!p) return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    return quantize_plan(p, (cudaStream_t)stream);
}

int tca_quantize_b_fp8(const void *d_B_f16, int ldb, int K, int N, void *d_Bq, int ldq, float *d_scale,
                       tca_stream_t stream)
{
    clear_error();
    if (K < 0 || N < 0) return set_error(TCA_ERR_INVALID_ARG, "negative size (K=%d, N=%d)", K, N);
    if (K == 0 || N == 0) return TCA_OK;
    if (!d_B_f16 || !d_Bq || !d_scale) return set_error(TCA_ERR_INVALID_ARG, "NULL buffer");
    if (ldb < N || ldq < N) return set_error(TCA_ERR_INVALID_ARG, "ldb (%d) and ldq (%d) must be >= N (%d)", ldb, ldq, N);
    if (ldq % 4 != 0 || (reinterpret_cast<uintptr_t>(d_Bq) & 3u) || (reinterpret_cast<uintptr_t>(d_scale) & 3u))
        return set_error(TCA_ERR_INVALID_ARG, "Bq needs 4-byte aligned rows (ldq %% 4 == 0) and scale 4-byte alignment");
    return quantize_b((const __half *)d_B_f16, ldb, K, N, (uint8_t *)d_Bq, ldq, d_scale, (cudaStream_t)stream);
}

int tca_spmm_fp8(tca_plan_t p, const void *d_B_f16, int ldb, int N, void *d_C, int ldc, int c_dtype, float alpha,
                 float beta, unsigned flags, tca_stream_t stream)
{
    clear_error();
    cudaStream_t s = (cudaStream_t)stream;
    SpmmJob job;
    TCA_TRY(make_fp8_job(p, d_B_f16, ldb, N, d_C, ldc, c_dtype, false, s, &job, nullptr));
    if (p->M == 0 || N == 0) return TCA_OK;
    if (p->K == 0) // no nonzeros can exist: A B = 0
        return tca_spmm(p, d_B_f16, ldb, N, d_C, ldc, c_dtype, alpha, beta, flags, stream);
    return run_jobs_with_events(&job, 1, c_dtype, alpha, beta, flags, s, nullptr);
}

int tca_spmm_fp8_batched(const tca_batch_item_t *items, int n_items, int c_dtype, float alpha, float beta,
                         unsigned flags, tca_stream_t stream, void *const *events)
{
    clear_error();
    if (n_items < 0 || (n_items > 0 && !items))
        return set_error(TCA_ERR_INVALID_ARG, "invalid batch");
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<SpmmJob> jobs;
    jobs.reserve((size_t)n_items);
    QBatch qb;
    qb.n = 0;
    for (int i = 0; i < n_items; i++) {
        const tca_batch_item_t &it = items[i];
        for (int k = 0; k < i; k++)
            if (items[k].plan == it.plan)
                return set_error(TCA_ERR_INVALID_ARG,
                                 "batch items %d and %d share a plan: an E4M3 batch quantizes B into the plan", k, i);
        SpmmJob j;
        TCA_TRY(make_fp8_job(it.plan, it.d_B_f16, it.ldb, it.N, it.d_C, it.ldc, c_dtype, true, s, &j, &qb));
        if (it.n_tile == 128 || it.n_tile == 256)
            j.n_tile = it.n_tile;
        j.cc_w = it.cc_cols;
        if (it.plan->M > 0 && it.N > 0 && it.plan->K == 0) // no nonzeros can exist: A B = 0
            TCA_TRY(tca_spmm(it.plan, it.d_B_f16, it.ldb, it.N, it.d_C, it.ldc, c_dtype, alpha, beta, flags, stream));
        else if (it.plan->M > 0 && it.N > 0)
            jobs.push_back(j);
    }
    TCA_TRY(quantize_b_batch(qb, s));
    return run_jobs_with_events(jobs.data(), (int)jobs.size(), c_dtype, alpha, beta, flags, s, events);
}

// ---------------------------------------------------------------------------
// tca_spmm_fp8_static: the E4M3 forward with no allocation at all.
//
// tca_spmm_fp8 quantizes B into a workspace that it allocates on first use
// and grows when N grows. Some callers cannot let it: their device memory is
// handed out by someone else (a framework's own caching allocator, a fixed
// per-process budget), or they sit on a latency-critical path where a
// cudaMalloc / cudaFree -- which may synchronise the whole device -- is not
// allowed. This entry point quantizes B into a fixed scratch array instead:
// g_fp8_scratch, below, allocated with the library's module on every GPU that
// loads it and held until the process exits.
//
// Layout of the scratch for one call: Bq (K rows of ldq = N rounded up to 16
// bytes), rounded up to 256 bytes, then ldq FP32 words that first hold the
// column maxima (cleared by the call itself) and then the column scales.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_fp8_scratch[TCA_FP8_STATIC_SCRATCH_BYTES];

namespace tca {
namespace {

constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices]; // device address of g_fp8_scratch, per device ordinal
std::mutex g_scratch_mutex;

// Device address of the scratch on the current device. The array's name in
// host code is only a host-side handle of the symbol; the address a kernel
// can use comes from cudaGetSymbolAddress, asked once per device with that
// device current (the first call on each device). The cached address belongs
// to the device's primary context: after cudaDeviceReset the module is loaded
// anew and the cache is stale, so a process that resets a device must not
// call this entry point on it again.
int static_scratch(void **out)
{
    int dev = 0;
    TCA_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(TCA_ERR_UNSUPPORTED, "device ordinal %d beyond the %d this entry point tracks", dev, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_fp8_scratch);
        if (e != cudaSuccess || !p)
            return set_error(TCA_ERR_CUDA, "cudaGetSymbolAddress of the static E4M3 scratch failed: %s",
                             cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return TCA_OK;
}

} // namespace
} // namespace tca

int tca_spmm_fp8_static(tca_plan_t p, const void *d_B_f16, int ldb, int N, void *d_C, int ldc, int c_dtype,
                        float alpha, float beta, unsigned flags, tca_stream_t stream)
{
    clear_error();
    if (!p) return set_error(TCA_ERR_INVALID_ARG, "plan is NULL");
    TCA_TRY(check_dense_args(d_B_f16, ldb, N, d_C, ldc, c_dtype, p->M, p->K));
    if (p->M == 0 || N == 0) return TCA_OK;
    const size_t c_elem = c_dtype == TCA_DTYPE_F16 ? 2 : 4;
    if (N % 8 != 0 || !aligned16(d_C) || ((size_t)ldc * c_elem) % 16 != 0)
        return set_error(TCA_ERR_UNSUPPORTED,
                         "the E4M3 forward needs N %% 8 == 0 and a 16-byte aligned C with 16-byte aligned rows");
    if (p->K == 0) // no nonzeros can exist: A B = 0, so C = beta * C, which tca_spmm writes without allocating
        return tca_spmm(p, d_B_f16, ldb, N, d_C, ldc, c_dtype, alpha, beta, flags, stream);
    if (!p->has_fp8)
        return set_error(TCA_ERR_INVALID_ARG,
                         "the plan has no E4M3 form: call tca_plan_quantize_fp8 once first (it allocates)");
    const int ldq = (N + 15) & ~15;
    const size_t bq = ((size_t)p->K * ldq + 255) & ~(size_t)255;
    const size_t need = bq + sizeof(float) * (size_t)ldq;
    if (need > (size_t)TCA_FP8_STATIC_SCRATCH_BYTES)
        return set_error(TCA_ERR_INVALID_ARG,
                         "B of %d x %d needs %zu bytes of E4M3 scratch; the static scratch holds %u "
                         "(K * round_up(N, 16) + 4 * round_up(N, 16) bytes must fit): use tca_spmm_fp8",
                         p->K, N, need, (unsigned)TCA_FP8_STATIC_SCRATCH_BYTES);
    void *base = nullptr;
    TCA_TRY(static_scratch(&base));
    cudaStream_t s = (cudaStream_t)stream;
    uint8_t *Bq = static_cast<uint8_t *>(base);
    float *scale = reinterpret_cast<float *>(static_cast<uint8_t *>(base) + bq);
    TCA_TRY(quantize_b((const __half *)d_B_f16, ldb, p->K, N, Bq, ldq, scale, s));
    SpmmJob job;
    job.p = p;
    job.B = (const __half *)d_B_f16;
    job.C = d_C;
    job.ldb = ldb;
    job.N = N;
    job.ldc = ldc;
    job.f8 = true;
    job.tc = p->n_tc > 0;
    job.n_tile = pick_tc_tile(p, N, false, true);
    job.Bq = Bq;
    job.ldq = ldq;
    job.col_scale = scale;
    // the launches of tca_spmm_fp8 (the CUDA-core launch runs beside the
    // tensor-core launch as its programmatic dependent); they allocate nothing
    return run_jobs_with_events(&job, 1, c_dtype, alpha, beta, flags, s, nullptr);
}
