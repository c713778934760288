// Drop-in operator entries in the reference's feature-major layout:
//   cospdnn_layer          <- ftxj::cospdnn_single   (src/kernels/kernel.cu:240-379)
//   cospdnn_prune_compact  <- check_active_f_col + host compaction + matrix_reshape
//                             (src/kernels/kernel.cu:129-172, src/cospdnn.cu:236-276)
// These keep the reference's [feature][batch] activations so a harness can
// call them where the reference kernels are launched.  The whole-network
// engine (engine.cu) keeps its own layouts (row-major or MMA tiles).
#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace cospdnn {

namespace {

constexpr int kLayerThreads = 128;  // one thread per batch column of the tile
constexpr int kMaxBlockVals = 32 * 32;

// One CTA = 128 batch columns x one block column; each thread keeps the
// block column's outputs for its batch column in registers.  Block values are
// staged in shared memory and broadcast; activation loads are coalesced along
// the batch.
template <int BC, bool AF32, bool BF32, bool REF_ARITH>
__global__ void __launch_bounds__(kLayerThreads)
    k_layer_featmajor(const void *__restrict__ A, const void *__restrict__ B, float *__restrict__ C,
                      const int *__restrict__ fuse, const int *__restrict__ idx_ptr,
                      const int *__restrict__ index, float bias, int batch, int neuron, int br) {
    __shared__ float vs[kMaxBlockVals];
    const int bid = blockIdx.y;
    const int b = blockIdx.x * kLayerThreads + threadIdx.x;
    const bool live = b < batch;
    float acc[BC];
#pragma unroll
    for (int i = 0; i < BC; ++i) acc[i] = 0.0f;

    const int p0 = idx_ptr[bid];
    const int p1 = REF_ARITH ? p0 + 2 : idx_ptr[bid + 1];
    const int bsz = BC * br;
    for (int blk = p0; blk < p1; ++blk) {
        __syncthreads();
        for (int t = threadIdx.x; t < bsz; t += kLayerThreads) {
            int64_t g = (int64_t)blk * bsz + t;
            vs[t] = BF32 ? ((const float *)B)[g] : __half2float(((const __half *)B)[g]);
        }
        __syncthreads();
        const int rs = index[blk];
        for (int k = 0; k < br; ++k) {
            const int r = rs + k;
            if (r >= neuron || r < 0) continue;
            const int f = fuse ? fuse[r] : r;
            if (f < 0 || f >= neuron || !live) continue;
            float hi, lo = 0.0f;
            if (AF32) {
                hi = ((const float *)A)[(int64_t)f * batch + b];
            } else {
                hi = __half2float(((const __half *)A)[(int64_t)f * batch + b]);
                lo = __half2float(((const __half *)A)[(int64_t)(f + neuron) * batch + b]);
            }
#pragma unroll
            for (int o = 0; o < BC; ++o) {
                // REF_ARITH: value [k*16 + o] feeds output o from input start+k
                // (the reference's ldmatrix.trans pairing); otherwise value
                // [o*BC + k] is W[start+k][col_start+o].
                const float w = REF_ARITH ? vs[k * 16 + o] : vs[o * BC + k];
                acc[o] = fmaf(w, hi, acc[o]);
                if (!AF32) acc[o] = fmaf(w, lo, acc[o]);
            }
        }
    }
    if (!live) return;
#pragma unroll
    for (int o = 0; o < BC; ++o) {
        const int out = bid * BC + o;
        if (out < neuron) C[(int64_t)out * batch + b] = clamp32(acc[o] + bias);
    }
}

template <int BC>
void launch_layer(dim3 grid, cudaStream_t s, unsigned flags, const void *A, const void *B,
                  float *C, const int *fuse, const int *idx_ptr, const int *index, float bias,
                  int batch, int neuron, int br) {
    const bool af = flags & COSPDNN_LAYER_A_FLOAT, bf = flags & COSPDNN_LAYER_B_FLOAT;
    const bool ra = flags & COSPDNN_LAYER_REFERENCE_ARITH;
#define CSP_L(AF, BF, RA) \
    k_layer_featmajor<BC, AF, BF, RA><<<grid, kLayerThreads, 0, s>>>(A, B, C, fuse, idx_ptr, index, bias, batch, neuron, br)
    if (af) {
        if (bf) { if (ra) CSP_L(true, true, true); else CSP_L(true, true, false); }
        else { if (ra) CSP_L(true, false, true); else CSP_L(true, false, false); }
    } else {
        if (bf) { if (ra) CSP_L(false, true, true); else CSP_L(false, true, false); }
        else { if (ra) CSP_L(false, false, true); else CSP_L(false, false, false); }
    }
#undef CSP_L
}

// ---- pruning -----------------------------------------------------------
constexpr int kPruneCols = 128;
constexpr int kScanThreads = 1024;

// flags[k] |= 1 if any C[n][k] > thr for n in this CTA's row slice.
__global__ void k_prune_flags(const float *__restrict__ C, int neuron, int batch, float thr,
                              int rows_per_cta, int *__restrict__ flags) {
    const int k = blockIdx.x * kPruneCols + threadIdx.x;
    if (k >= batch) return;
    const int n0 = blockIdx.y * rows_per_cta;
    const int n1 = min(neuron, n0 + rows_per_cta);
    bool any = false;
    for (int n = n0; n < n1 && !any; ++n) any = C[(int64_t)n * batch + k] > thr;
    if (any && flags[k] == 0) atomicOr(&flags[k], 1);
}

// Stable compaction of the surviving columns (one CTA, any batch size).
__global__ void __launch_bounds__(kScanThreads)
    k_prune_scan(const int *__restrict__ flags, int batch, const int *__restrict__ map_in,
                 int *__restrict__ category, int *__restrict__ map_out, int *__restrict__ count) {
    __shared__ int warp_tot[kScanThreads / 32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int base = 0; base < batch; base += kScanThreads) {
        const int k = base + threadIdx.x;
        const int f = (k < batch && flags[k]) ? 1 : 0;
        const unsigned m = __ballot_sync(0xffffffffu, f);
        const int before = __popc(m & ((1u << lane) - 1u));
        if (lane == 31) warp_tot[wid] = __popc(m);
        __syncthreads();
        if (wid == 0) {
            int v = warp_tot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += t;
            }
            warp_tot[lane] = v;  // inclusive
        }
        __syncthreads();
        const int wbase = (wid ? warp_tot[wid - 1] : 0) + carry;
        if (f) {
            const int j = wbase + before;
            category[j] = k;
            map_out[j] = map_in ? map_in[k] : k;
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_tot[kScanThreads / 32 - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = carry;
}

// A_out[n][j] = C[n][category[j]] for j < count, 0 up to the 128-padded stride.
template <bool HILO>
__global__ void k_prune_gather(const float *__restrict__ C, int neuron, int batch,
                               const int *__restrict__ category, const int *__restrict__ count,
                               int rows_per_cta, void *__restrict__ A_out) {
    const int cnt = *count;
    const int stride = (cnt + 127) / 128 * 128;
    const int j = blockIdx.x * kPruneCols + threadIdx.x;
    if (j >= stride) return;
    const int src = j < cnt ? category[j] : -1;
    const int n0 = blockIdx.y * rows_per_cta;
    const int n1 = min(neuron, n0 + rows_per_cta);
    for (int n = n0; n < n1; ++n) {
        const float x = src >= 0 ? C[(int64_t)n * batch + src] : 0.0f;
        if (HILO) {
            // the split of floatTohalf2 (src/kernels/kernel.cu:147-148)
            __half *h = (__half *)A_out;
            const __half hi = __float2half(x);
            h[(int64_t)n * stride + j] = hi;
            h[(int64_t)(n + neuron) * stride + j] = __float2half(x - __half2float(hi));
        } else {
            ((float *)A_out)[(int64_t)n * stride + j] = x;
        }
    }
}

}  // namespace

int prune_compact_impl(const float *C, int neuron, int batch, float threshold, void *A_out,
                       int *category, const int *map_in, int *map_out, int *count_dev,
                       unsigned flags, int *flag_ws, cudaStream_t s) {
    const int col_ctas = (batch + kPruneCols - 1) / kPruneCols;
    const int rows_per_cta = 64;
    const int row_ctas = (neuron + rows_per_cta - 1) / rows_per_cta;
    CSP_CUDA(cudaMemsetAsync(flag_ws, 0, sizeof(int) * (size_t)batch, s));
    k_prune_flags<<<dim3(col_ctas, row_ctas), kPruneCols, 0, s>>>(C, neuron, batch, threshold,
                                                                 rows_per_cta, flag_ws);
    k_prune_scan<<<1, kScanThreads, 0, s>>>(flag_ws, batch, map_in, category, map_out, count_dev);
    const int grows = 16;
    const dim3 g2(col_ctas, (neuron + grows - 1) / grows);
    if (flags & COSPDNN_PRUNE_OUT_HALF_HILO)
        k_prune_gather<true><<<g2, kPruneCols, 0, s>>>(C, neuron, batch, category, count_dev, grows, A_out);
    else
        k_prune_gather<false><<<g2, kPruneCols, 0, s>>>(C, neuron, batch, category, count_dev, grows, A_out);
    CSP_CUDA(cudaGetLastError());
    return COSPDNN_OK;
}

}  // namespace cospdnn

using namespace cospdnn;

extern "C" int cospdnn_layer(const void *A, const void *B, float *C, const int *fuse,
                             const int *idx_ptr, const int *index, float bias, int batch,
                             int neuron, int blocksize_c, int blocksize_r, int nblockcols,
                             unsigned flags, void *stream) {
    CSP_CHECK(A && B && C && idx_ptr && index, COSPDNN_ERR_INVALID, "cospdnn_layer: null pointer");
    CSP_CHECK(batch > 0 && neuron > 0 && nblockcols > 0, COSPDNN_ERR_INVALID, "cospdnn_layer: bad sizes");
    CSP_CHECK(nblockcols <= 65535, COSPDNN_ERR_UNSUPPORTED, "cospdnn_layer: too many block columns");
    CSP_CHECK(blocksize_r > 0 && blocksize_c * blocksize_r <= kMaxBlockVals, COSPDNN_ERR_UNSUPPORTED,
              "cospdnn_layer: block larger than 32x32");
    CSP_CHECK(!(flags & ~7u), COSPDNN_ERR_INVALID, "cospdnn_layer: unknown flag");
    if (flags & COSPDNN_LAYER_REFERENCE_ARITH)
        CSP_CHECK(blocksize_c == 16 && blocksize_r == 16, COSPDNN_ERR_UNSUPPORTED,
                  "cospdnn_layer: reference arithmetic needs 16x16 blocks");
    const dim3 grid((batch + kLayerThreads - 1) / kLayerThreads, nblockcols);
    cudaStream_t s = (cudaStream_t)stream;
    switch (blocksize_c) {
        case 8: launch_layer<8>(grid, s, flags, A, B, C, fuse, idx_ptr, index, bias, batch, neuron, blocksize_r); break;
        case 16: launch_layer<16>(grid, s, flags, A, B, C, fuse, idx_ptr, index, bias, batch, neuron, blocksize_r); break;
        case 32: launch_layer<32>(grid, s, flags, A, B, C, fuse, idx_ptr, index, bias, batch, neuron, blocksize_r); break;
        default: return fail(COSPDNN_ERR_UNSUPPORTED, "cospdnn_layer: blocksize_c must be 8, 16 or 32");
    }
    CSP_CUDA(cudaGetLastError());
    return COSPDNN_OK;
}

extern "C" size_t cospdnn_prune_workspace_bytes(int batch) {
    if (batch <= 0) return 0;
    return ((size_t)batch * sizeof(int) + 255) / 256 * 256;
}

extern "C" int cospdnn_prune_compact(const float *C, int neuron, int batch, float threshold,
                                     void *A_out, int *category, const int *map_in, int *map_out,
                                     int *count_dev, unsigned flags, void *workspace,
                                     size_t workspace_bytes, void *stream) {
    CSP_CHECK(C && A_out && category && map_out && count_dev && workspace, COSPDNN_ERR_INVALID,
              "cospdnn_prune_compact: null pointer");
    CSP_CHECK(neuron > 0 && batch > 0, COSPDNN_ERR_INVALID, "cospdnn_prune_compact: bad sizes");
    CSP_CHECK(workspace_bytes >= cospdnn_prune_workspace_bytes(batch), COSPDNN_ERR_INVALID,
              "cospdnn_prune_compact: workspace too small");
    CSP_CHECK(!(flags & ~1u), COSPDNN_ERR_INVALID, "cospdnn_prune_compact: unknown flag");
    return prune_compact_impl(C, neuron, batch, threshold, A_out, category, map_in, map_out,
                              count_dev, flags, (int *)workspace, (cudaStream_t)stream);
}

// ---- allocation-free pruning entry ----------------------------------------
// Same computation as cospdnn_prune_compact, with the per-column flag
// scratch in a file-scope device array instead of caller-provided memory.
namespace cospdnn {
namespace {
constexpr int kNoAllocMaxBatch = 1 << 20;  // columns; 4 MiB of scratch on every GPU that loads the library
__device__ __align__(256) int g_prune_scratch[kNoAllocMaxBatch];
std::mutex g_scratch_mu;
int *g_scratch_addr[1024];  // device address of g_prune_scratch, per device ordinal

// Host code cannot use g_prune_scratch's name as a device address: ask the
// runtime for it once per device, with that device current.
int scratch_for_current_device(int **out) {
    int dev = 0;
    CSP_CUDA(cudaGetDevice(&dev));
    CSP_CHECK(dev >= 0 && dev < 1024, COSPDNN_ERR_UNSUPPORTED, "prune_compact_noalloc: device ordinal too large");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_prune_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "prune_compact_noalloc: cudaGetSymbolAddress");
        g_scratch_addr[dev] = (int *)p;
    }
    *out = g_scratch_addr[dev];
    return COSPDNN_OK;
}
}  // namespace
}  // namespace cospdnn

extern "C" int cospdnn_prune_compact_noalloc(const float *C, int neuron, int batch, float threshold,
                                             void *A_out, int *category, const int *map_in, int *map_out,
                                             int *count_dev, unsigned flags, void *stream) {
    CSP_CHECK(C && A_out && category && map_out && count_dev, COSPDNN_ERR_INVALID,
              "cospdnn_prune_compact_noalloc: null pointer");
    CSP_CHECK(neuron > 0 && batch > 0, COSPDNN_ERR_INVALID, "cospdnn_prune_compact_noalloc: bad sizes");
    CSP_CHECK(batch <= kNoAllocMaxBatch, COSPDNN_ERR_INVALID,
              "cospdnn_prune_compact_noalloc: batch exceeds the 1048576-column scratch");
    CSP_CHECK(!(flags & ~1u), COSPDNN_ERR_INVALID, "cospdnn_prune_compact_noalloc: unknown flag");
    int *ws = nullptr;
    const int rc = scratch_for_current_device(&ws);
    if (rc) return rc;
    // prune_compact_impl clears the flags it uses (an async memset, no allocation)
    return prune_compact_impl(C, neuron, batch, threshold, A_out, category, map_in, map_out, count_dev, flags, ws,
                              (cudaStream_t)stream);
}
