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

// 16x16 blocks, batch a multiple of 8.  One CTA = 256 batch columns x one
// block column.  The rows of up to two blocks (32 rows; hi and lo halves, or
// FP32) are copied into shared memory with cp.async (16-byte pieces,
// zero-filled past the matrix), one copy group per block so the second block
// lands while the first is computed; a CTA keeps 32 KB of loads in flight
// without holding them in registers (six CTAs per SM).  Each thread sums
// hi + lo for its 2 columns (exact in FP32: the pair spans at most 22
// significant bits) and does one packed two-lane FMA per weight
// (fma.rn.f32x2: two IEEE FMAs, identical to fmaf on each column), the
// block's weights staged transposed ([k][o]) for broadcast 16-byte shared
// loads.
constexpr int kFastThreads = 128;
constexpr int kFastCols = 2;                          // batch columns per thread
constexpr int kFastChunk = kFastThreads * kFastCols;  // 256 batch columns per CTA
constexpr int kFastRows = 32;                         // rows staged at once (two blocks)
constexpr size_t kFastSmem = (size_t)kFastRows * 2 * kFastChunk * 2;  // 32 KB: two 16-bit planes

// acc.x += w * a.x, acc.y += w * a.y in one sm_100 packed instruction
__device__ __forceinline__ void ffma2(float2 &acc, float w, float2 a) {
    asm("{\n\t.reg .b64 d, x, w;\n\t"
        "mov.b64 d, {%0, %1};\n\t"
        "mov.b64 x, {%2, %3};\n\t"
        "mov.b64 w, {%4, %4};\n\t"
        "fma.rn.f32x2 d, w, x, d;\n\t"
        "mov.b64 {%0, %1}, d;\n\t}"
        : "+f"(acc.x), "+f"(acc.y)
        : "f"(a.x), "f"(a.y), "f"(w));
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool pred) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
    const int n = pred ? 16 : 0;  // 0: fill with zeros, read nothing
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gmem), "r"(n) : "memory");
}

template <bool AF32, bool BF32, bool REF_ARITH>
__global__ void __launch_bounds__(kFastThreads)
    k_layer_fm16(const void *__restrict__ A, const void *__restrict__ B, float *__restrict__ C,
                 const int *__restrict__ fuse, const int *__restrict__ idx_ptr, const int *__restrict__ index,
                 float bias, int batch, int neuron) {
    extern __shared__ __align__(16) unsigned char fsm[];
    __shared__ __align__(16) float wT[2][16][16];
    __shared__ int s_row[kFastRows];
    // block column fastest in the grid: CTAs running together share batch
    // columns, so activation rows read by several block columns hit L2
    const int bid = blockIdx.x;
    const int c0 = blockIdx.y * kFastChunk;  // first batch column of the CTA
    const int b0 = threadIdx.x * kFastCols;  // this thread's columns within the chunk
    float2 acc[16];
#pragma unroll
    for (int o = 0; o < 16; ++o) acc[o] = make_float2(0.f, 0.f);
    const int p0 = idx_ptr[bid];
    const int p1 = REF_ARITH ? p0 + 2 : idx_ptr[bid + 1];
    // 16-bit input: plane 0 = hi rows, plane 1 = lo rows, each [32][512] halves;
    // FP32 input: one [32][512] float plane in the same bytes
    __half *hs = reinterpret_cast<__half *>(fsm);
    float *fs = reinterpret_cast<float *>(fsm);
    for (int q0 = p0; q0 < p1; q0 += 2) {
        const int nb = min(2, p1 - q0);
        __syncthreads();  // the previous stage's rows and weights are consumed
        if (threadIdx.x < kFastRows) {
            const int t = threadIdx.x, r = t < nb * 16 ? index[q0 + (t >> 4)] + (t & 15) : -1;
            int f = -1;
            if (r >= 0 && r < neuron) f = fuse ? fuse[r] : r;
            s_row[t] = (f >= 0 && f < neuron) ? f : -1;
        }
        for (int t = threadIdx.x; t < nb * 256; t += kFastThreads) {
            const int j = t >> 8, k = (t >> 4) & 15, o = t & 15;
            // REF_ARITH: value [k*16 + o] feeds output o from input start+k;
            // otherwise value [o*16 + k] is W[start+k][col_start+o]
            const int64_t g = (int64_t)(q0 + j) * 256 + (REF_ARITH ? k * 16 + o : o * 16 + k);
            wT[j][k][o] = BF32 ? ((const float *)B)[g] : __half2float(((const __half *)B)[g]);
        }
        __syncthreads();
        constexpr int kPiecesPerRow = AF32 ? kFastChunk * 4 / 16 : kFastChunk * 2 / 16;
        constexpr int kPlanes = AF32 ? 1 : 2;
        constexpr int kPerBlock = 16 * kPiecesPerRow * kPlanes;
        for (int j = 0; j < nb; ++j) {
            for (int i = threadIdx.x; i < kPerBlock; i += kFastThreads) {
                const int pc = i % kPiecesPerRow, rowp = i / kPiecesPerRow;
                const int t = j * 16 + (rowp & 15), plane = rowp >> 4;
                const int f = s_row[t];
                const int col = c0 + pc * (AF32 ? 4 : 8);
                const bool ok = f >= 0 && col < batch;
                if (AF32) {
                    const float *src = ok ? (const float *)A + (int64_t)f * batch + col : (const float *)A;
                    cp_async16(fs + (int64_t)t * kFastChunk + pc * 4, src, ok);
                } else {
                    const __half *src = ok ? (const __half *)A + (int64_t)(f + plane * neuron) * batch + col
                                           : (const __half *)A;
                    cp_async16(hs + ((int64_t)plane * kFastRows + t) * kFastChunk + pc * 8, src, ok);
                }
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
        for (int j = 0; j < nb; ++j) {
            if (j + 1 < nb)
                asm volatile("cp.async.wait_group 1;" ::: "memory");
            else
                asm volatile("cp.async.wait_group 0;" ::: "memory");
            __syncthreads();
#pragma unroll 4
            for (int k = 0; k < 16; ++k) {
                const int t = j * 16 + k;
                float2 a;
                if (AF32) {
                    a = *reinterpret_cast<const float2 *>(fs + (int64_t)t * kFastChunk + b0);
                } else {
                    const float2 h =
                        __half22float2(*reinterpret_cast<const __half2 *>(hs + (int64_t)t * kFastChunk + b0));
                    const float2 l = __half22float2(
                        *reinterpret_cast<const __half2 *>(hs + (int64_t)(kFastRows + t) * kFastChunk + b0));
                    a = make_float2(h.x + l.x, h.y + l.y);
                }
#pragma unroll
                for (int o4 = 0; o4 < 16; o4 += 4) {
                    const float4 w = *reinterpret_cast<const float4 *>(&wT[j][k][o4]);
                    ffma2(acc[o4], w.x, a);
                    ffma2(acc[o4 + 1], w.y, a);
                    ffma2(acc[o4 + 2], w.z, a);
                    ffma2(acc[o4 + 3], w.w, a);
                }
            }
        }
    }
    const int col = c0 + b0;
    if (col >= batch) return;  // batch % 8 == 0: the thread's two columns both exist
#pragma unroll
    for (int o = 0; o < 16; ++o) {
        const int out = bid * 16 + o;
        if (out < neuron)
            *reinterpret_cast<float2 *>(C + (int64_t)out * batch + col) =
                make_float2(clamp32(acc[o].x + bias), clamp32(acc[o].y + bias));
    }
}

void launch_layer_fast(dim3 grid, cudaStream_t s, unsigned flags, const void *A, const void *B, float *C,
                       const int *fuse, const int *idx_ptr, const int *index, float bias, int batch, int neuron) {
    const bool af = flags & COSPDNN_LAYER_A_FLOAT, bf = flags & COSPDNN_LAYER_B_FLOAT;
    const bool ra = flags & COSPDNN_LAYER_REFERENCE_ARITH;
#define CSP_F(AF, BF, RA)                                                                                     \
    do {                                                                                                      \
        cudaFuncSetAttribute(k_layer_fm16<AF, BF, RA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFastSmem); \
        k_layer_fm16<AF, BF, RA><<<grid, kFastThreads, kFastSmem, s>>>(A, B, C, fuse, idx_ptr, index, bias, batch, neuron); \
    } while (0)
    if (af) {
        if (bf) { if (ra) CSP_F(true, true, true); else CSP_F(true, true, false); }
        else { if (ra) CSP_F(true, false, true); else CSP_F(true, false, false); }
    } else {
        if (bf) { if (ra) CSP_F(false, true, true); else CSP_F(false, true, false); }
        else { if (ra) CSP_F(false, false, true); else CSP_F(false, false, false); }
    }
#undef CSP_F
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
    cudaStream_t s = (cudaStream_t)stream;
    const bool aligned = ((uintptr_t)A % 16 == 0) && ((uintptr_t)C % 16 == 0);
    if (blocksize_c == 16 && blocksize_r == 16 && batch % 8 == 0 && aligned) {
        const int per = kFastChunk;
        CSP_CHECK((batch + per - 1) / per <= 65535, COSPDNN_ERR_UNSUPPORTED, "cospdnn_layer: batch too large");
        launch_layer_fast(dim3(nblockcols, (batch + per - 1) / per), s, flags, A, B, C, fuse, idx_ptr, index, bias,
                          batch, neuron);
        CSP_CUDA(cudaGetLastError());
        return COSPDNN_OK;
    }
    const dim3 grid((batch + kLayerThreads - 1) / kLayerThreads, nblockcols);
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
