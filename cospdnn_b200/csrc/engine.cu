// Whole-network engine: host side (setup, graph capture, C ABI) plus the
// input conversion kernel.  Replaces the host layer loops of the reference
// (src/cospdnn.cu:3-369, src/cospdnn_double.cu:208-1214).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "bits_layer.cuh"
#include "cc_layer.cuh"
#include "cs_layer.cuh"
#include "engine_kernels.cuh"
#include "tc_layer.cuh"

namespace cospdnn {

namespace {

// ---- input conversion: any format -> compute type, per-row error and max --
template <typename T, int FMT>
__global__ void k_convert_input(const void *__restrict__ src, int rows, int N, int layout, T *__restrict__ y0,
                                float *__restrict__ y0_f32, float *__restrict__ err0,
                                float *__restrict__ mx0) {
    // one warp per row
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = w; r < rows; r += nw) {
        float e = 0.0f, m = 0.0f;
        for (int j = lane; j < N; j += 32) {
            float x;
            if (FMT == COSPDNN_INPUT_U8) x = (float)((const uint8_t *)src)[r * N + j];
            else if (FMT == COSPDNN_INPUT_F32) x = ((const float *)src)[r * N + j];
            else x = (float)((((const uint8_t *)src)[r * (N / 8) + (j >> 3)] >> (j & 7)) & 1u);
            const T v = act_traits<T>::from_f(x);
            y0[act_index(layout, N, r, j)] = v;
            if (y0_f32) y0_f32[r * N + j] = x;
            e = fmaxf(e, fabsf(act_traits<T>::to_f(v) - x));
            m = fmaxf(m, fabsf(x));
        }
        e = warp_max(e);
        m = warp_max(m);
        if (lane == 0) {
            err0[r] = e;
            mx0[r] = m;
        }
    }
}

// Integer inputs (bytes or bits) into row tiles (layout TR >= 2): one thread
// per (tile, run of up to 8 rows, 8 features); each feature's run of rows is
// written as one contiguous piece.  Values 0..255 are exact in every compute
// type, so the per-row error is 0 (k_row_max fills it and the row max).
// `skip_if_binary` (may be NULL): the net counts layer 0 on bit planes when
// the input is binary, and nothing reads this copy then, so the kernel
// returns when the flag (raised by k_row_max for a value above 1) is clear.
template <typename T, int FMT>
__global__ void k_convert_tile(const uint8_t *__restrict__ src, int rows, int N, int TR, T *__restrict__ y0,
                               const int *__restrict__ skip_if_binary) {
    if (skip_if_binary && *skip_if_binary == 0) return;
    const int RC = TR < 8 ? TR : 8, nrc = TR / RC, nfb = N / 8;
    const int64_t ntiles = (rows + TR - 1) / TR;
    const int64_t total = ntiles * nrc * nfb;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < total; u += (int64_t)gridDim.x * blockDim.x) {
        const int fb = (int)(u % nfb);
        const int64_t rest = u / nfb;
        const int rc = (int)(rest % nrc);
        const int64_t t = rest / nrc;
        uint8_t v[8][8];  // [row][feature]
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int64_t row = t * TR + rc * RC + r;
            uint2 b = make_uint2(0u, 0u);
            if (r < RC && row < rows) {
                if (FMT == COSPDNN_INPUT_U8) {
                    b = *reinterpret_cast<const uint2 *>(src + row * N + 8 * fb);
                } else {
                    const uint32_t bits = src[row * nfb + fb];
                    // byte k of the pair = bit k of the feature byte
                    b.x = (bits & 1u) | ((bits >> 1) & 1u) << 8 | ((bits >> 2) & 1u) << 16 | ((bits >> 3) & 1u) << 24;
                    b.y = ((bits >> 4) & 1u) | ((bits >> 5) & 1u) << 8 | ((bits >> 6) & 1u) << 16 | ((bits >> 7) & 1u) << 24;
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                v[r][k] = (uint8_t)(b.x >> (8 * k));
                v[r][k + 4] = (uint8_t)(b.y >> (8 * k));
            }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            T *dst = y0 + ((t * N + 8 * fb + k) * TR + rc * RC);
            __align__(16) T o[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) o[r] = act_traits<T>::from_f((float)v[r][k]);
            if (RC * (int)sizeof(T) == 16) {
                *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(o);
            } else if (RC * (int)sizeof(T) == 32) {
                reinterpret_cast<uint4 *>(dst)[0] = reinterpret_cast<const uint4 *>(o)[0];
                reinterpret_cast<uint4 *>(dst)[1] = reinterpret_cast<const uint4 *>(o)[1];
            } else if (RC * (int)sizeof(T) == 8) {
                *reinterpret_cast<uint2 *>(dst) = *reinterpret_cast<const uint2 *>(o);
            } else {
                for (int r = 0; r < RC; ++r) dst[r] = o[r];
            }
        }
    }
}

// Integer inputs (bytes or bits) into row-major buffers: one thread per
// (row, 8 features), one 16-byte piece (two for FP32) per thread.
template <typename T, int FMT>
__global__ void k_convert_pieces(const uint8_t *__restrict__ src, int rows, int N, int layout,
                                 T *__restrict__ y0) {
    const int nfb = N / 8;
    const int64_t total = (int64_t)rows * nfb;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < total; u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = u / nfb;
        const int fb = (int)(u - row * nfb);
        uint2 b;
        if (FMT == COSPDNN_INPUT_U8) {
            b = *reinterpret_cast<const uint2 *>(src + row * N + 8 * fb);
        } else {
            const uint32_t bits = src[row * nfb + fb];
            b.x = (bits & 1u) | ((bits >> 1) & 1u) << 8 | ((bits >> 2) & 1u) << 16 | ((bits >> 3) & 1u) << 24;
            b.y = ((bits >> 4) & 1u) | ((bits >> 5) & 1u) << 8 | ((bits >> 6) & 1u) << 16 | ((bits >> 7) & 1u) << 24;
        }
        __align__(16) T o[8];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            o[k] = act_traits<T>::from_f((float)((b.x >> (8 * k)) & 0xFFu));
            o[k + 4] = act_traits<T>::from_f((float)((b.y >> (8 * k)) & 0xFFu));
        }
        T *dst = y0 + act_index(layout, N, row, 8 * fb);
        reinterpret_cast<uint4 *>(dst)[0] = reinterpret_cast<const uint4 *>(o)[0];
        if (sizeof(T) == 4) reinterpret_cast<uint4 *>(dst)[1] = reinterpret_cast<const uint4 *>(o)[1];
    }
}

// Integer inputs into MMA tiles (layout 1): one CTA (256 threads) per
// (128-row tile, 64 features); the slab is staged in shared memory as bytes,
// then every 16-feature block is written as one contiguous 4 KB operand.
template <typename T, int FMT>
__global__ void __launch_bounds__(256) k_convert_mma(const uint8_t *__restrict__ src, int rows, int N,
                                                     T *__restrict__ y0, const int *__restrict__ skip_if_binary) {
    // as k_convert_tile: a net counting layer 0 does not read this copy
    if (skip_if_binary && *skip_if_binary == 0) return;
    __shared__ __align__(16) uint8_t slab[128][64];
    const int ng = (N + 63) / 64, nbk = N / 16;
    const int64_t units = (int64_t)((rows + 127) / 128) * ng;
    for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
        const int64_t t = u / ng;
        const int g = (int)(u - t * ng), fw = min(64, N - 64 * g);
        __syncthreads();  // the previous unit is done with the slab
        if (FMT == COSPDNN_INPUT_U8) {
            for (int i = threadIdx.x; i < 128 * 4; i += 256) {  // 16-byte pieces
                const int m = i >> 2, pc = i & 3;
                const int64_t row = t * 128 + m;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (row < rows && pc * 16 < fw) v = *reinterpret_cast<const uint4 *>(src + row * N + 64 * g + 16 * pc);
                *reinterpret_cast<uint4 *>(&slab[m][16 * pc]) = v;
            }
        } else {
            for (int i = threadIdx.x; i < 128 * 8; i += 256) {  // bytes of 8 features
                const int m = i >> 3, by = i & 7;
                const int64_t row = t * 128 + m;
                const uint32_t bits = (row < rows && by * 8 < fw) ? src[row * (N / 8) + 8 * g + by] : 0u;
#pragma unroll
                for (int k = 0; k < 8; ++k) slab[m][8 * by + k] = (uint8_t)((bits >> k) & 1u);
            }
        }
        __syncthreads();
        for (int b = 0; b < fw / 16; ++b) {
            // piece i of the block: rows m, 8-feature half kh (canonical order)
            const int i = threadIdx.x, m = ((i >> 4) << 3) + (i & 7), kh = (i >> 3) & 1;
            __align__(16) T o[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) o[k] = act_traits<T>::from_f((float)slab[m][16 * b + 8 * kh + k]);
            T *dst = y0 + ((t * nbk) + 4 * g + b) * 2048 + (int64_t)i * 8;
            *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(o);
        }
    }
}

// Stores a network descriptor passed by value (kernel arguments are copied at
// launch, so the update is asynchronous: a copy from pageable host memory
// would synchronize the stream first).
__global__ void k_store_netdev(NetDev *dst, NetDev v) { *dst = v; }

// Per-row max |input| (error 0) of integer inputs: one warp per row.
// `nonbin` (may be NULL) is raised when a value is above 1.
template <int FMT>
__global__ void k_row_max(const uint8_t *__restrict__ src, int rows, int N, float *__restrict__ err0,
                          float *__restrict__ mx0, int *__restrict__ nonbin) {
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int nb = FMT == COSPDNN_INPUT_U8 ? N : N / 8;  // bytes per row
    for (int64_t r = w; r < rows; r += nw) {
        uint32_t m = 0;
        const uint8_t *row = src + r * nb;
        if (FMT == COSPDNN_INPUT_U8) {
            // N is a multiple of 8, so every row starts 8-byte aligned
            for (int i = lane * 8; i < nb; i += 256) {
                const uint2 v = *reinterpret_cast<const uint2 *>(row + i);
                m = max(m, __vmaxu4(v.x, v.y));
            }
        } else {
            for (int i = lane; i < nb; i += 32) m |= row[i];  // rows of N/8 bytes: any alignment
        }
        if (FMT == COSPDNN_INPUT_U8) m = max(max(m & 0xFFu, (m >> 8) & 0xFFu), max((m >> 16) & 0xFFu, m >> 24));
        else m = m ? 1u : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) {
            err0[r] = 0.0f;
            mx0[r] = (float)m;
            if (nonbin && m > 1u) atomicOr(nonbin, 1);
        }
    }
}

// Gather of the current activations (rows 0..R-1 of the next input: the
// output of the last computed layer for the rows kept after it) and of their
// original ids, at most max_rows rows; for checks.
template <typename T>
__global__ void k_gather_rows(const NetDev *__restrict__ nd_p, float *__restrict__ out, int32_t *__restrict__ ids,
                              float *__restrict__ bounds, int64_t max_rows) {
    const NetDev &nd = *nd_p;
    const int R = nd.st->R, N = nd.N;
    const T *act = (const T *)nd.act[nd.st->in_buf];
    const int64_t rows = min((int64_t)R, max_rows), total = rows * N;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (int64_t)gridDim.x * blockDim.x;
    const bool gather = nd.st->gather != 0;  // row q is row cmap[q] of the buffer (compaction pending)
    for (int64_t i = tid; i < total; i += nth) {
        const int64_t q = i / N, j = i % N;
        const int64_t src = gather ? nd.cmap[q] : q;
        out[i] = act_traits<T>::to_f(act[act_index(nd.layout, N, src, (int)j)]);
    }
    // the row lists of the next layer: original ids, and the proven bound on
    // |Y(fast) - Y(FP64)| of these values
    if (ids)
        for (int64_t q = tid; q < rows; q += nth) ids[q] = nd.orig[nd.st->layer & 1][q];
    if (bounds)
        for (int64_t q = tid; q < rows; q += nth) bounds[q] = nd.err[nd.st->layer & 1][q];
}

size_t elem_size(int prec) { return prec == COSPDNN_PREC_FP32 ? 4 : 2; }

template <typename T>
T *dalloc(size_t n, std::vector<void *> &owned) {
    void *p = nullptr;
    if (n == 0) n = 1;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
    owned.push_back(p);
    return (T *)p;
}

float to_compute(float w, int prec) {
    if (prec == COSPDNN_PREC_FP16) return __half2float(__float2half_rn(w));
    if (prec == COSPDNN_PREC_BF16) return __bfloat162float(__float2bfloat16_rn(w));
    return w;
}

struct HostLayer {
    std::vector<int32_t> colptr, rowidx;
    std::vector<float> vals;
    bool set = false;
};

struct Net {
    cospdnn_net_desc d{};
    std::vector<HostLayer> layers;
    NetDev dev{};
    std::vector<LayerDev> ldev;
    LayerDev *d_layers = nullptr;
    // Inputs are double buffered: set_input fills the back buffers (staging
    // copy, Y0 in the compute type, per-row error and max, exact FP32 rows),
    // the next run makes them current.  So the copy and conversion of the
    // next batch can run on another stream while a run reads the current one.
    void *staging[2] = {nullptr, nullptr};
    size_t staging_bytes[2] = {0, 0};
    void *y0buf[2] = {nullptr, nullptr};
    float *err0buf[2] = {nullptr, nullptr}, *mx0buf[2] = {nullptr, nullptr};
    float *f32buf[2] = {nullptr, nullptr};  // exact rows of FP32 inputs (allocated on first use)
    bool f32used[2] = {false, false};       // the buffer's last input came as FP32
    uint32_t *bitsbuf[2] = {nullptr, nullptr};  // bit planes of binary inputs (layer 0 by counting)
    int *nbflag[2] = {nullptr, nullptr};        // raised when that input is not binary
    int front = 0;                          // buffers of the current input
    bool pending = false;                   // the back buffers hold a newer input
};

}  // namespace

thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }
int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}
int cuda_fail(cudaError_t err, const char *what) {
    g_err = std::string(what) + ": " + cudaGetErrorString(err);
    return err == cudaErrorMemoryAllocation ? COSPDNN_ERR_NOMEM : COSPDNN_ERR_CUDA;
}

}  // namespace cospdnn

using namespace cospdnn;

struct cospdnn_engine {
    int device = 0;
    std::vector<Net> nets;
    std::vector<void *> owned;
    bool built = false;
    NetDev *d_nets = nullptr;
    int max_n = 0, max_layers = 0;
    double *scratch = nullptr;
    int replay_ctas = 0;
    int compact_ctas = 0;  // compaction chunks of all nets at full size
    unsigned long long *launches = nullptr;
    unsigned int *finished = nullptr;
    int *loop_guard = nullptr;
    int *abort_flag = nullptr;  // raised by a layer kernel whose bounded wait expired
    DevLimits *limits = nullptr;  // wait and loop limits read by the kernels at launch
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle loop{};
    KSpec k0, k2, k3, k4_graph, k4_eager, k5;
    std::vector<KSpec> layer_specs;
    std::vector<KSpec> l0_specs;  // layer 0 by bit counting, once per run before the layer loop
    std::vector<long long *> packbuf;  // per net: device buffer for result_async
    ~cospdnn_engine() {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (void *p : owned) cudaFree(p);
        cudaSetDevice(cur);
    }
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// Fraction of the 16x16 aligned blocks of W that its nonzeros fill, over all
// layers (1 = every touched block dense; XOR-mask weights: 1/16).
double block_fill(const Net &net) {
    const int N = net.d.neuron, nb = (N + 15) / 16;
    double nnz = 0.0, blocks = 0.0;
    std::vector<int> mark(nb, -1);
    for (const HostLayer &h : net.layers) {
        nnz += h.colptr[N];
        for (int c = 0; c < nb; ++c) {  // block column c: distinct input blocks
            for (int j = c * 16; j < std::min(N, c * 16 + 16); ++j)
                for (int p = h.colptr[j]; p < h.colptr[j + 1]; ++p) {
                    const int b = h.rowidx[p] / 16;
                    if (mark[b] != c) {
                        mark[b] = c;
                        blocks += 1.0;
                    }
                }
        }
        std::fill(mark.begin(), mark.end(), -1);
    }
    return blocks > 0.0 ? nnz / (blocks * 256.0) : 0.0;
}

// Distinct aligned 16x16 blocks per block column of one layer, on average.
double blocks_per_column(const HostLayer &h, int N) {
    const int nb = (N + 15) / 16;
    std::vector<int> mark(nb, -1);
    double blocks = 0.0;
    for (int c = 0; c < nb; ++c)
        for (int j = c * 16; j < std::min(N, c * 16 + 16); ++j)
            for (int p = h.colptr[j]; p < h.colptr[j + 1]; ++p) {
                const int b = h.rowidx[p] / 16;
                if (mark[b] != c) {
                    mark[b] = c;
                    blocks += 1.0;
                }
            }
    return blocks / nb;
}

// Kernel for COSPDNN_KERNEL_AUTO.  The CUDA-core row-tile kernel costs about
// the same per nonzero whatever the sparsity pattern; a tcgen05 MMA costs a
// fixed 16x16 block whatever its fill.  Measured on one B200 (4096 neurons,
// 60000 rows, FP16): one layer takes 0.86 ms on CUDA cores for any pattern,
// 2.13 ms on tcgen05 at 29 blocks per block column (fill 1/16, XOR masks) and
// 0.39 ms at 2 (fill 1); the lines cross near 9.5 blocks, fill 0.21.  So
// tcgen05 when its blocks are at least a quarter full or when neither the
// row tile of the CUDA-core kernel nor half of a 2-row tile (feature-split
// kernel) fits; FP32 always on CUDA cores.
int auto_kernel(const Net &n) {
    const int N = n.d.neuron, prec = n.d.precision;
    if (prec == COSPDNN_PREC_FP32 || !tc_supported(N)) return COSPDNN_KERNEL_CUDA_CORE;
    if (cc_tile_rows(N, prec) == 0 && !cs_supported(N, prec)) return COSPDNN_KERNEL_TCGEN05;
    return block_fill(n) >= 0.25 ? COSPDNN_KERNEL_TCGEN05 : COSPDNN_KERNEL_CUDA_CORE;
}

int upload_layer(cospdnn_engine *e, Net &net, int l, LayerDev &ld) {
    const HostLayer &h = net.layers[l];
    const int N = net.d.neuron;
    int K = 1;
    for (int j = 0; j < N; ++j) K = std::max(K, h.colptr[j + 1] - h.colptr[j]);
    std::vector<int32_t> idx((size_t)K * N, 0);
    std::vector<float> val((size_t)K * N, 0.0f);
    double S = 0.0, dW = 0.0;
    for (int j = 0; j < N; ++j) {
        double s = 0.0, d = 0.0;
        for (int p = h.colptr[j], k = 0; p < h.colptr[j + 1]; ++p, ++k) {
            idx[(size_t)k * N + j] = h.rowidx[p];
            val[(size_t)k * N + j] = h.vals[p];
            const float wc = to_compute(h.vals[p], net.d.precision);
            s += std::max(std::fabs((double)h.vals[p]), std::fabs((double)wc));
            d += std::fabs((double)wc - (double)h.vals[p]);
        }
        S = std::max(S, s);
        dW = std::max(dW, d);
    }
    int32_t *didx = dalloc<int32_t>(idx.size(), e->owned);
    float *dval = dalloc<float>(val.size(), e->owned);
    CSP_CHECK(didx && dval, COSPDNN_ERR_NOMEM, "engine: weight allocation failed");
    CSP_CUDA(cudaMemcpy(didx, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice));
    CSP_CUDA(cudaMemcpy(dval, val.data(), val.size() * 4, cudaMemcpyHostToDevice));
    ld = LayerDev{};
    ld.ell_idx = didx;
    ld.ell_val = dval;
    ld.K = K;
    ld.S = (float)(S * (1.0 + 1e-7));
    ld.dW = (float)(dW * (1.0 + 1e-7));
    // entries for the FP64 replay in a quarter of the bytes when the layer
    // has one weight value: 16-bit indices, that value held once
    bool one = N <= 65536 && K <= 65535 && h.colptr[N] > 0;
    for (int64_t p = 1; one && p < h.colptr[N]; ++p) one = h.vals[p] == h.vals[0];
    if (one) {
        std::vector<uint16_t> ri((size_t)K * N, 0), rc(N);
        for (int j = 0; j < N; ++j) {
            rc[j] = (uint16_t)(h.colptr[j + 1] - h.colptr[j]);
            for (int p = h.colptr[j], k = 0; p < h.colptr[j + 1]; ++p, ++k) ri[(size_t)k * N + j] = (uint16_t)h.rowidx[p];
        }
        uint16_t *dri = dalloc<uint16_t>(ri.size(), e->owned), *drc = dalloc<uint16_t>(rc.size(), e->owned);
        CSP_CHECK(dri && drc, COSPDNN_ERR_NOMEM, "engine: weight allocation failed");
        CSP_CUDA(cudaMemcpy(dri, ri.data(), ri.size() * 2, cudaMemcpyHostToDevice));
        CSP_CUDA(cudaMemcpy(drc, rc.data(), rc.size() * 2, cudaMemcpyHostToDevice));
        ld.rp_idx = dri;
        ld.rp_cnt = drc;
        ld.rp_w = h.vals[0];
    }
    if (net.dev.kernel == COSPDNN_KERNEL_TCGEN05) {
        int rc = tc_build_blocks(h.colptr, h.rowidx, h.vals, N, net.d.precision, ld, e->owned);
        if (rc) return rc;
    } else if (net.dev.cc_split) {
        int rc = cs_build_entries(h.colptr, h.rowidx, h.vals, N, net.d.precision, net.dev.cc_compact != 0, ld,
                                  e->owned);
        if (rc) return rc;
    } else if (const int TR = cc_tile_rows(N, net.d.precision)) {
        int rc = cc_build_entries(h.colptr, h.rowidx, h.vals, N, net.d.precision, TR, net.dev.cc_compact != 0, ld,
                                  e->owned);
        if (rc) return rc;
    }
    return COSPDNN_OK;
}

// Precisions of the nets on each layer kernel.
struct KernelSets {
    std::vector<int> plain, tc;
    // row-tile kernel: (precision, lane bytes | compact entries << 8) -> largest row tile of those nets
    std::vector<std::pair<std::pair<int, int>, size_t>> cc;
    // feature-split kernel: (precision, compact entries) -> widest of those nets
    std::vector<std::pair<std::pair<int, int>, int>> cs;
};

int make_specs(cospdnn_engine *e, const KernelSets &ks) {
    int sms = 148;
    CSP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device));
    const int nn = (int)e->nets.size();
    NetDev *nets = e->d_nets;
    unsigned long long *launches = e->launches;
    int *guard = e->loop_guard;
    KSpec &k0 = e->k0;
    k0.fn = (void *)k_init_run;
    k0.grid = dim3(sms * 4);
    k0.block = dim3(256);
    k0.arg(nets).arg(nn).arg(launches).arg(guard).arg(e->abort_flag);
    for (int prec : ks.plain) {
        KSpec k;
        k.fn = prec == COSPDNN_PREC_FP32 ? (void *)k_layer_plain<float>
             : prec == COSPDNN_PREC_FP16 ? (void *)k_layer_plain<__half>
                                         : (void *)k_layer_plain<__nv_bfloat16>;
        int per_sm = 0;
        CSP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, kPlainThreads, 0));
        k.grid = dim3(sms * std::max(1, per_sm));
        k.block = dim3(kPlainThreads);
        k.arg(nets).arg(nn).arg(prec).arg(launches);
        e->layer_specs.push_back(std::move(k));
    }
    for (const auto &cc : ks.cc) {
        KSpec k;
        // key: precision, lane bytes | compact entries << 8
        int rc = cc_layer_spec(k, nets, nn, cc.first.first, cc.first.second & 0xff, (cc.first.second >> 8) != 0,
                               launches, sms, cc.second);
        if (rc) return rc;
        e->layer_specs.push_back(std::move(k));
    }
    for (int kind : {kL0Rows32, kL0Mma16, kL0Split16})
        for (int prec = 0; prec < 3; ++prec) {
            int max_n = 0;
            for (const Net &n : e->nets) {
                const int nk = n.dev.cc_split ? kL0Split16 : n.dev.layout == 1 ? kL0Mma16 : kL0Rows32;
                if (n.dev.l0_k > 0 && n.d.precision == prec && nk == kind) max_n = std::max(max_n, n.d.neuron);
            }
            if (!max_n) continue;
            KSpec k;
            int rc = l0_spec(k, nets, nn, prec, kind, launches, sms, max_n);
            if (rc) return rc;
            e->l0_specs.push_back(std::move(k));
        }
    for (const auto &c : ks.cs) {
        KSpec k;
        int rc = cs_layer_spec(k, nets, nn, c.first.first, c.first.second != 0, launches, e->abort_flag, e->limits, sms,
                               c.second);
        if (rc) return rc;
        e->layer_specs.push_back(std::move(k));
    }
    for (int prec : ks.tc) {
        KSpec k;
        int rc = tc_layer_spec(k, nets, nn, prec, launches, e->abort_flag, e->limits, sms);
        if (rc) return rc;
        e->layer_specs.push_back(std::move(k));
    }
    KSpec &k2 = e->k2;
    k2.fn = (void *)k_classify;
    k2.grid = dim3(sms * 4);
    k2.block = dim3(256);
    k2.arg(nets).arg(nn).arg(launches);
    KSpec &k3 = e->k3;
    k3.fn = (void *)k_replay;
    k3.grid = dim3(e->replay_ctas);
    k3.block = dim3(kReplayThreads);
    {
        int sd = 0;
        for (const Net &n : e->nets) sd = std::max(sd, replay_smem_doubles(n.d.neuron));
        k3.smem = sizeof(double) * (size_t)sd;
    }
    CSP_CUDA(cudaFuncSetAttribute(k3.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k3.smem));
    k3.arg(nets).arg(nn).arg(e->scratch).arg(e->max_n).arg(launches);
    KSpec &k5 = e->k5;
    k5.fn = (void *)k_copy_rows;
    k5.grid = dim3(sms * 8);
    k5.block = dim3(256);
    k5.arg(nets).arg(nn).arg(launches);
    for (int use_cond = 0; use_cond < 2; ++use_cond) {
        KSpec &k4 = use_cond ? e->k4_graph : e->k4_eager;
        k4.fn = (void *)k_compact;
        k4.grid = dim3(e->compact_ctas);
        k4.block = dim3(kCompactThreads);
        k4.arg(nets).arg(nn).arg(e->finished).arg(e->loop).arg(use_cond).arg(guard)
            .arg((const DevLimits *)e->limits).arg((const int *)e->abort_flag).arg(launches);
    }
    return COSPDNN_OK;
}

int add_node(cudaGraph_t g, cudaGraphNode_t *node, const cudaGraphNode_t *deps, int ndeps, KSpec &k) {
    cudaKernelNodeParams p{};
    p.func = k.fn;
    p.gridDim = k.grid;
    p.blockDim = k.block;
    p.sharedMemBytes = (unsigned)k.smem;
    p.kernelParams = k.params();
    CSP_CUDA(cudaGraphAddKernelNode(node, g, deps, ndeps, &p));
    return COSPDNN_OK;
}

int launch(KSpec &k, cudaStream_t s) {
    CSP_CUDA(cudaLaunchKernel(k.fn, k.grid, k.block, k.params(), k.smem, s));
    return COSPDNN_OK;
}

int build_graph(cospdnn_engine *e, const KernelSets &ks) {
    CSP_CUDA(cudaGraphCreate(&e->graph, 0));
    CSP_CUDA(cudaGraphConditionalHandleCreate(&e->loop, e->graph, 1, cudaGraphCondAssignDefault));
    int rc = make_specs(e, ks);
    if (rc) return rc;
    cudaGraphNode_t k0;
    if ((rc = add_node(e->graph, &k0, nullptr, 0, e->k0))) return rc;
    std::vector<cudaGraphNode_t> l0_nodes(e->l0_specs.size());
    for (size_t i = 0; i < e->l0_specs.size(); ++i)
        if ((rc = add_node(e->graph, &l0_nodes[i], &k0, 1, e->l0_specs[i]))) return rc;
    // while (any network live) { layer kernels; classify; FP64 replay; compact }
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = e->loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    if (l0_nodes.empty()) CSP_CUDA(cudaGraphAddNode(&cnode, e->graph, &k0, 1, &cp));
    else CSP_CUDA(cudaGraphAddNode(&cnode, e->graph, l0_nodes.data(), l0_nodes.size(), &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    std::vector<cudaGraphNode_t> layer_nodes(e->layer_specs.size());
    for (size_t i = 0; i < e->layer_specs.size(); ++i)
        if ((rc = add_node(body, &layer_nodes[i], nullptr, 0, e->layer_specs[i]))) return rc;
    cudaGraphNode_t k2, k3, k4, k5;
    if ((rc = add_node(body, &k2, layer_nodes.data(), (int)layer_nodes.size(), e->k2))) return rc;
    if ((rc = add_node(body, &k3, &k2, 1, e->k3))) return rc;
    if ((rc = add_node(body, &k4, &k3, 1, e->k4_graph))) return rc;
    if ((rc = add_node(body, &k5, &k4, 1, e->k5))) return rc;
    CSP_CUDA(cudaGraphInstantiate(&e->exec, e->graph, 0));
    return COSPDNN_OK;
}

}  // namespace

extern "C" const char *cospdnn_last_error(void) { return g_err.c_str(); }
extern "C" int cospdnn_version(void) { return 100; }

extern "C" int cospdnn_engine_create(cospdnn_engine **out, int device) {
    CSP_CHECK(out, COSPDNN_ERR_INVALID, "engine_create: null out");
    int ndev = 0;
    CSP_CUDA(cudaGetDeviceCount(&ndev));
    CSP_CHECK(device >= 0 && device < ndev, COSPDNN_ERR_INVALID, "engine_create: no such device");
    cudaDeviceProp prop;
    CSP_CUDA(cudaGetDeviceProperties(&prop, device));
    CSP_CHECK(prop.major == 10 && prop.minor == 0, COSPDNN_ERR_UNSUPPORTED,
              "engine_create: this library is built for sm_100a (B200) only");
    auto *e = new (std::nothrow) cospdnn_engine();
    CSP_CHECK(e, COSPDNN_ERR_NOMEM, "engine_create: out of host memory");
    e->device = device;
    *out = e;
    return COSPDNN_OK;
}

extern "C" void cospdnn_engine_destroy(cospdnn_engine *e) { delete e; }

extern "C" int cospdnn_engine_add_net(cospdnn_engine *e, const cospdnn_net_desc *d, int *net_id) {
    CSP_CHECK(e && d, COSPDNN_ERR_INVALID, "add_net: null argument");
    CSP_CHECK(!e->built, COSPDNN_ERR_STATE, "add_net: engine already built");
    CSP_CHECK(d->neuron > 0 && d->layers > 0 && d->rows >= 0, COSPDNN_ERR_INVALID, "add_net: bad sizes");
    CSP_CHECK(d->neuron % 8 == 0, COSPDNN_ERR_UNSUPPORTED, "add_net: neuron must be a multiple of 8");
    CSP_CHECK(d->precision >= 0 && d->precision <= 2, COSPDNN_ERR_INVALID, "add_net: bad precision");
    CSP_CHECK(d->kernel >= 0 && d->kernel <= 2, COSPDNN_ERR_INVALID, "add_net: bad kernel");
    CSP_CHECK(!(d->kernel == COSPDNN_KERNEL_TCGEN05 && d->precision == COSPDNN_PREC_FP32),
              COSPDNN_ERR_UNSUPPORTED, "add_net: tcgen05 kernel needs FP16 or BF16");
    CSP_CHECK(d->threshold >= 0.0f && d->threshold < 32.0f, COSPDNN_ERR_INVALID, "add_net: threshold outside [0,32)");
    CSP_CHECK(std::isfinite(d->bias), COSPDNN_ERR_INVALID, "add_net: non-finite bias");
    Net net;
    net.d = *d;
    net.layers.resize(d->layers);
    const int k = d->kernel;
    if (k == COSPDNN_KERNEL_TCGEN05)
        CSP_CHECK(tc_supported(d->neuron), COSPDNN_ERR_UNSUPPORTED, "add_net: tcgen05 kernel needs neuron % 16 == 0");
    net.dev.kernel = k;  // AUTO is resolved at build, from the weights
    e->nets.push_back(std::move(net));
    if (net_id) *net_id = (int)e->nets.size() - 1;
    return COSPDNN_OK;
}

extern "C" int cospdnn_engine_set_layer_csc(cospdnn_engine *e, int net, int layer,
                                            const int32_t *colptr, const int32_t *rowidx,
                                            const float *vals) {
    CSP_CHECK(e && colptr, COSPDNN_ERR_INVALID, "set_layer_csc: null argument");
    CSP_CHECK(!e->built, COSPDNN_ERR_STATE, "set_layer_csc: engine already built");
    CSP_CHECK(net >= 0 && net < (int)e->nets.size(), COSPDNN_ERR_INVALID, "set_layer_csc: bad net");
    Net &n = e->nets[net];
    CSP_CHECK(layer >= 0 && layer < n.d.layers, COSPDNN_ERR_INVALID, "set_layer_csc: bad layer");
    const int N = n.d.neuron;
    CSP_CHECK(colptr[0] == 0, COSPDNN_ERR_INVALID, "set_layer_csc: colptr[0] != 0");
    for (int j = 0; j < N; ++j)
        CSP_CHECK(colptr[j + 1] >= colptr[j], COSPDNN_ERR_INVALID, "set_layer_csc: colptr not monotone");
    const int64_t nnz = colptr[N];
    CSP_CHECK(nnz == 0 || (rowidx && vals), COSPDNN_ERR_INVALID, "set_layer_csc: null rowidx/vals");
    for (int j = 0; j < N; ++j)
        for (int p = colptr[j]; p < colptr[j + 1]; ++p) {
            CSP_CHECK(rowidx[p] >= 0 && rowidx[p] < N, COSPDNN_ERR_INVALID, "set_layer_csc: row index out of range");
            CSP_CHECK(p == colptr[j] || rowidx[p] > rowidx[p - 1], COSPDNN_ERR_INVALID,
                      "set_layer_csc: rows must be strictly ascending within a column");
            CSP_CHECK(std::isfinite(vals[p]), COSPDNN_ERR_INVALID, "set_layer_csc: non-finite weight");
        }
    HostLayer &h = n.layers[layer];
    h.colptr.assign(colptr, colptr + N + 1);
    h.rowidx.assign(rowidx, rowidx + nnz);
    h.vals.assign(vals, vals + nnz);
    h.set = true;
    return COSPDNN_OK;
}

extern "C" int cospdnn_engine_set_layer_bcsc(cospdnn_engine *e, int net, int layer,
                                             const int32_t *col_ptr, int n_col_ptr,
                                             const int32_t *row_index, int n_blocks,
                                             const float *values, int blocksize,
                                             const int32_t *fuse) {
    CSP_CHECK(e && col_ptr && row_index && values, COSPDNN_ERR_INVALID, "set_layer_bcsc: null argument");
    CSP_CHECK(net >= 0 && net < (int)e->nets.size(), COSPDNN_ERR_INVALID, "set_layer_bcsc: bad net");
    const int N = e->nets[net].d.neuron;
    CSP_CHECK(blocksize > 0 && n_col_ptr >= 1 && n_blocks >= 0, COSPDNN_ERR_INVALID, "set_layer_bcsc: bad sizes");
    CSP_CHECK(col_ptr[0] == 0 && col_ptr[n_col_ptr - 1] == n_blocks, COSPDNN_ERR_INVALID,
              "set_layer_bcsc: col_ptr does not span the blocks");
    // fold: W[fuse[start+ro]][bid*bs+co] += V[co*bs+ro]
    std::vector<std::vector<std::pair<int32_t, float>>> cols(N);
    const int64_t bsz = (int64_t)blocksize * blocksize;
    for (int bid = 0; bid + 1 < n_col_ptr; ++bid) {
        CSP_CHECK(col_ptr[bid + 1] >= col_ptr[bid], COSPDNN_ERR_INVALID, "set_layer_bcsc: col_ptr not monotone");
        for (int blk = col_ptr[bid]; blk < col_ptr[bid + 1]; ++blk) {
            for (int co = 0; co < blocksize; ++co) {
                const int o = bid * blocksize + co;
                for (int ro = 0; ro < blocksize; ++ro) {
                    const float v = values[blk * bsz + (int64_t)co * blocksize + ro];
                    if (v == 0.0f) continue;
                    const int r = row_index[blk] + ro;
                    CSP_CHECK(o < N && r >= 0 && r < N, COSPDNN_ERR_INVALID, "set_layer_bcsc: nonzero outside the matrix");
                    const int a = fuse ? fuse[r] : r;
                    CSP_CHECK(a >= 0 && a < N, COSPDNN_ERR_INVALID, "set_layer_bcsc: fuse entry out of range");
                    cols[o].push_back({a, v});
                }
            }
        }
    }
    std::vector<int32_t> cp(N + 1, 0), ri;
    std::vector<float> vv;
    for (int j = 0; j < N; ++j) {
        auto &c = cols[j];
        std::sort(c.begin(), c.end(), [](const std::pair<int32_t, float> &x, const std::pair<int32_t, float> &y) {
            return x.first < y.first;
        });
        for (size_t t = 0; t < c.size(); ++t) {
            if (!ri.empty() && (int)ri.size() > cp[j] && ri.back() == c[t].first) vv.back() += c[t].second;
            else { ri.push_back(c[t].first); vv.push_back(c[t].second); }
        }
        cp[j + 1] = (int32_t)ri.size();
    }
    return cospdnn_engine_set_layer_csc(e, net, layer, cp.data(), ri.data(), vv.data());
}

extern "C" int cospdnn_engine_build(cospdnn_engine *e) {
    CSP_CHECK(e, COSPDNN_ERR_INVALID, "build: null engine");
    CSP_CHECK(!e->built, COSPDNN_ERR_STATE, "build: already built");
    CSP_CHECK(!e->nets.empty(), COSPDNN_ERR_STATE, "build: no networks");
    DeviceGuard g(e->device);
    KernelSets ks;
    for (Net &n : e->nets) {
        for (int l = 0; l < n.d.layers; ++l)
            CSP_CHECK(n.layers[l].set, COSPDNN_ERR_STATE, "build: a layer's weights were not set");
        if (n.dev.kernel == COSPDNN_KERNEL_AUTO) n.dev.kernel = auto_kernel(n);
        e->max_n = std::max(e->max_n, n.d.neuron);
        e->max_layers = std::max(e->max_layers, n.d.layers);
        // activation layout: MMA tiles (tcgen05), row tiles (CUDA-core tile
        // kernel) or row-major (CUDA-core gather kernel, rows too wide for a tile)
        n.dev.layout = n.dev.kernel == COSPDNN_KERNEL_TCGEN05 ? 1 : cc_tile_rows(n.d.neuron, n.d.precision);
        n.dev.cc_split = 0;
        if (n.dev.kernel == COSPDNN_KERNEL_CUDA_CORE && n.dev.layout == 0 && cs_supported(n.d.neuron, n.d.precision)) {
            // 2-row tiles split by feature over the two CTAs of a cluster
            n.dev.layout = 2;
            n.dev.cc_split = 1;
        }
        if (n.dev.layout >= 2) {
            // compact entry lists when every layer has one weight value (the
            // Graph Challenge networks): 2 bytes per entry instead of 4 or 8
            bool compact = true;
            for (int l = 0; l < n.d.layers && compact; ++l)
                compact = cc_single_weight(n.layers[l].colptr, n.layers[l].vals, n.d.neuron, n.d.precision);
            n.dev.cc_compact = compact ? 1 : 0;
            if (n.dev.cc_split) {
                const std::pair<int, int> key(n.d.precision, n.dev.cc_compact);
                auto it = std::find_if(ks.cs.begin(), ks.cs.end(), [&](const auto &x) { return x.first == key; });
                if (it == ks.cs.end()) ks.cs.push_back({key, n.d.neuron});
                else it->second = std::max(it->second, n.d.neuron);
                continue;
            }
            const std::pair<int, int> key(n.d.precision,
                                          cc_lane_bytes(n.d.precision, n.dev.layout) | (n.dev.cc_compact << 8));
            const size_t tb = cc_tile_bytes(n.d.neuron, n.d.precision, n.dev.layout);
            auto it = std::find_if(ks.cc.begin(), ks.cc.end(), [&](const auto &x) { return x.first == key; });
            if (it == ks.cc.end()) ks.cc.push_back({key, tb});
            else it->second = std::max(it->second, tb);
        } else {
            auto &v = n.dev.kernel == COSPDNN_KERNEL_TCGEN05 ? ks.tc : ks.plain;
            if (std::find(v.begin(), v.end(), n.d.precision) == v.end()) v.push_back(n.d.precision);
        }
    }
    for (Net &n : e->nets) {
        const int N = n.d.neuron, R = std::max(1, n.d.rows);
        n.ldev.resize(n.d.layers);
        const bool l0_rows = n.dev.kernel == COSPDNN_KERNEL_CUDA_CORE && n.dev.layout >= 4;
        // tcgen05 nets: counting pays when layer 0's blocks are sparse (measured
        // on one B200 at 4096 neurons, 60000 rows: counting 0.58 ms, the MMA
        // kernel 0.26 + 0.064 ms per block per column; dense-block layers
        // such as R1's, 2 blocks per column, stay on tcgen05)
        const bool l0_mma = n.dev.kernel == COSPDNN_KERNEL_TCGEN05 && n.dev.layout == 1 &&
                            n.d.precision != COSPDNN_PREC_FP32 && n.d.layers > 0 &&
                            blocks_per_column(n.layers[0], N) >= 6.0;
        // feature-split nets: the 16-row counting kernel (a 32-row unit of
        // 65536 features does not fit shared memory), stores into 2-row tiles
        const bool l0_split = n.dev.cc_split != 0;
        if ((l0_rows || l0_mma || l0_split) && n.d.layers > 0) {
            const HostLayer &h0 = n.layers[0];
            int rc = l0_build(h0.colptr, h0.rowidx, h0.vals, N, n.d.precision, l0_split ? 1 : n.dev.layout, n.d.bias,
                              n.dev, e->owned);
            if (rc) return rc;
            if (n.dev.l0_k > 0) {
                for (int b = 0; b < 2; ++b) {
                    n.bitsbuf[b] = dalloc<uint32_t>(l0_bits_bytes(R, N) / 4, e->owned);
                    n.nbflag[b] = dalloc<int>(1, e->owned);
                    CSP_CHECK(n.bitsbuf[b] && n.nbflag[b], COSPDNN_ERR_NOMEM, "build: device allocation failed");
                    CSP_CUDA(cudaMemset(n.bitsbuf[b], 0, l0_bits_bytes(R, N)));
                    CSP_CUDA(cudaMemset(n.nbflag[b], 1, sizeof(int)));  // no input yet
                }
                n.dev.y0bits = n.bitsbuf[0];
                n.dev.y0nonbin = n.nbflag[0];
            }
        }
        for (int l = 0; l < n.d.layers; ++l) {
            int rc = upload_layer(e, n, l, n.ldev[l]);
            if (rc) return rc;
            n.layers[l] = HostLayer();  // host copy no longer needed
            n.layers[l].set = true;
        }
        n.d_layers = dalloc<LayerDev>(n.d.layers, e->owned);
        CSP_CHECK(n.d_layers, COSPDNN_ERR_NOMEM, "build: allocation failed");
        CSP_CUDA(cudaMemcpy(n.d_layers, n.ldev.data(), sizeof(LayerDev) * n.d.layers, cudaMemcpyHostToDevice));
        NetDev &d = n.dev;
        d.N = N;
        d.L = n.d.layers;
        d.rows = n.d.rows;
        d.prec = n.d.precision;
        d.bias = n.d.bias;
        d.tau = n.d.threshold;
        d.layers = n.d_layers;
        const size_t rows_pad = (size_t)(R + 127) / 128 * 128;
        const size_t es = elem_size(d.prec), act = rows_pad * N * es;
        for (int b = 0; b < 2; ++b) {
            n.y0buf[b] = dalloc<char>(act, e->owned);
            n.err0buf[b] = dalloc<float>(R, e->owned);
            n.mx0buf[b] = dalloc<float>(R, e->owned);
            CSP_CHECK(n.y0buf[b] && n.err0buf[b] && n.mx0buf[b], COSPDNN_ERR_NOMEM, "build: device allocation failed");
            CSP_CUDA(cudaMemset(n.y0buf[b], 0, act));
            CSP_CUDA(cudaMemset(n.err0buf[b], 0, sizeof(float) * R));
            CSP_CUDA(cudaMemset(n.mx0buf[b], 0, sizeof(float) * R));
        }
        n.front = 0;
        d.y0 = n.y0buf[0];
        d.act[0] = dalloc<char>(act, e->owned);
        d.act[1] = dalloc<char>(act, e->owned);
        float *err0 = n.err0buf[0], *mx0 = n.mx0buf[0];
        d.err0 = err0;
        d.mx0 = mx0;
        d.cmap = dalloc<int32_t>(R, e->owned);
        for (int b = 0; b < 2; ++b) {
            d.orig[b] = dalloc<int32_t>(R, e->owned);
            d.err[b] = dalloc<float>(R, e->owned);
            d.mx[b] = dalloc<float>(R, e->owned);
        }
        d.stat = dalloc<uint32_t>((size_t)3 * R, e->owned);
        d.cls = dalloc<int8_t>(R, e->owned);
        d.ulist = dalloc<int32_t>(R, e->owned);
        const int nchunks = (R + kCompactChunk - 1) / kCompactChunk;
        d.ccount = dalloc<int32_t>(nchunks, e->owned);
        CSP_CHECK(d.ccount, COSPDNN_ERR_NOMEM, "build: device allocation failed");
        CSP_CUDA(cudaMemset(d.ccount, 0, sizeof(int32_t) * nchunks));
        e->compact_ctas += nchunks;
        d.alive_count = dalloc<long long>(d.L, e->owned);
        d.recheck_count = dalloc<long long>(d.L, e->owned);
        d.st = dalloc<NetState>(1, e->owned);
        CSP_CHECK(d.y0 && d.act[0] && d.act[1] && err0 && mx0 && d.cmap && d.orig[0] &&
                      d.orig[1] && d.err[0] && d.err[1] && d.mx[0] && d.mx[1] && d.stat && d.cls &&
                      d.ulist && d.alive_count && d.recheck_count && d.st,
                  COSPDNN_ERR_NOMEM, "build: device allocation failed");
        CSP_CUDA(cudaMemset(d.act[0], 0, act));
        CSP_CUDA(cudaMemset(d.act[1], 0, act));
        CSP_CUDA(cudaMemset(d.st, 0, sizeof(NetState)));
    }
    for (Net &n : e->nets) {
        long long *pb = dalloc<long long>(1 + n.d.layers + (std::max(1, n.d.rows) + 1) / 2, e->owned);
        CSP_CHECK(pb, COSPDNN_ERR_NOMEM, "build: allocation failed");
        e->packbuf.push_back(pb);
    }
    e->d_nets = dalloc<NetDev>(e->nets.size(), e->owned);
    CSP_CHECK(e->d_nets, COSPDNN_ERR_NOMEM, "build: allocation failed");
    for (size_t i = 0; i < e->nets.size(); ++i)
        CSP_CUDA(cudaMemcpy(e->d_nets + i, &e->nets[i].dev, sizeof(NetDev), cudaMemcpyHostToDevice));
    int sms = 148;
    CSP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device));
    e->replay_ctas = 2 * sms;
    e->scratch = dalloc<double>((size_t)e->replay_ctas * 2 * e->max_n, e->owned);
    e->launches = dalloc<unsigned long long>(1, e->owned);
    e->finished = dalloc<unsigned int>(1, e->owned);
    e->loop_guard = dalloc<int>(1, e->owned);
    e->abort_flag = dalloc<int>(1, e->owned);
    e->limits = dalloc<DevLimits>(1, e->owned);
    CSP_CHECK(e->scratch && e->launches && e->finished && e->loop_guard && e->abort_flag && e->limits,
              COSPDNN_ERR_NOMEM, "build: allocation failed");
    CSP_CUDA(cudaMemset(e->abort_flag, 0, sizeof(int)));
    {
        const DevLimits lim{kDefaultWaitCycles, e->max_layers + 2, 0};
        CSP_CUDA(cudaMemcpy(e->limits, &lim, sizeof(lim), cudaMemcpyHostToDevice));
    }
    CSP_CUDA(cudaMemset(e->finished, 0, sizeof(unsigned int)));
    CSP_CUDA(cudaMemset(e->launches, 0, sizeof(unsigned long long)));
    int rc = build_graph(e, ks);
    if (rc) return rc;
    CSP_CUDA(cudaDeviceSynchronize());
    e->built = true;
    return COSPDNN_OK;
}

extern "C" int cospdnn_engine_set_input(cospdnn_engine *e, int net, const void *y0, int format,
                                        int on_device, void *stream) {
    CSP_CHECK(e && y0, COSPDNN_ERR_INVALID, "set_input: null argument");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "set_input: build first");
    CSP_CHECK(net >= 0 && net < (int)e->nets.size(), COSPDNN_ERR_INVALID, "set_input: bad net");
    CSP_CHECK(format >= 0 && format <= 2, COSPDNN_ERR_INVALID, "set_input: bad format");
    // the conversion kernels read device rows with 8- and 16-byte loads
    CSP_CHECK(!on_device || (uintptr_t)y0 % 16 == 0, COSPDNN_ERR_INVALID,
              "set_input: device input must be 16-byte aligned");
    DeviceGuard g(e->device);
    Net &n = e->nets[net];
    const int N = n.d.neuron, R = n.d.rows;
    if (R == 0) return COSPDNN_OK;
    CSP_CHECK(format != COSPDNN_INPUT_BITS || N % 8 == 0, COSPDNN_ERR_INVALID, "set_input: bit rows need neuron % 8 == 0");
    const size_t bytes = format == COSPDNN_INPUT_U8 ? (size_t)R * N
                       : format == COSPDNN_INPUT_F32 ? (size_t)R * N * 4 : (size_t)R * (N / 8);
    cudaStream_t s = (cudaStream_t)stream;
    const int back = n.front ^ 1;  // the current input stays untouched for a run in flight
    const void *src = y0;
    if (!on_device) {
        if (n.staging_bytes[back] < bytes) {
            if (n.staging[back]) {
                // the engine owns the old buffer: drop it from the list it frees at destruction
                e->owned.erase(std::remove(e->owned.begin(), e->owned.end(), n.staging[back]), e->owned.end());
                cudaFree(n.staging[back]);
            }
            n.staging[back] = nullptr;
            n.staging_bytes[back] = 0;
            CSP_CUDA(cudaMalloc(&n.staging[back], bytes));
            e->owned.push_back(n.staging[back]);
            n.staging_bytes[back] = bytes;
        }
        CSP_CUDA(cudaMemcpyAsync(n.staging[back], y0, bytes, cudaMemcpyHostToDevice, s));
        src = n.staging[back];
    }
    float *f32 = nullptr;
    if (format == COSPDNN_INPUT_F32 && n.d.precision != COSPDNN_PREC_FP32) {
        if (!n.f32buf[back]) {
            CSP_CUDA(cudaMalloc(&n.f32buf[back], (size_t)R * N * 4));
            e->owned.push_back(n.f32buf[back]);
        }
        f32 = n.f32buf[back];
    }
    n.f32used[back] = f32 != nullptr;
    n.pending = true;
    void *const y0dst = n.y0buf[back];
    const int blocks = std::min(65535, (R + 7) / 8);
    float *err0 = n.err0buf[back], *mx0 = n.mx0buf[back];
    if (n.nbflag[back]) {
        // binary unless the row maxima say otherwise (FP32 values: never counted)
        CSP_CUDA(cudaMemsetAsync(n.nbflag[back], format == COSPDNN_INPUT_F32 ? 1 : 0, sizeof(int), s));
    }
    if (n.dev.layout < 2 && format != COSPDNN_INPUT_F32) {
        // integer input into row-major or MMA-tile buffers
        const uint8_t *b = (const uint8_t *)src;
        const int64_t units = (int64_t)R * (N / 8);
        const int cb = (int)std::min<int64_t>((units + 255) / 256, 148 * 16);
        const int layout = n.dev.layout;
        const int mb = (int)std::min<int64_t>((int64_t)((R + 127) / 128) * ((N + 63) / 64), 148 * 8);
        // a net counting layer 0 (MMA tiles): bit planes with the row maxima
        // first, the compute-type copy only if the input is not binary
        const int *skip = n.nbflag[back];
        if (skip) l0_convert_bits(b, format, R, N, n.bitsbuf[back], err0, mx0, n.nbflag[back], s);
#define CSP_PIECES(T)                                                                                        \
    do {                                                                                                     \
        if (layout == 1) {                                                                                   \
            if (format == COSPDNN_INPUT_U8) k_convert_mma<T, COSPDNN_INPUT_U8><<<mb, 256, 0, s>>>(b, R, N, (T *)y0dst, skip); \
            else if (!skip) k_convert_mma<T, COSPDNN_INPUT_BITS><<<mb, 256, 0, s>>>(b, R, N, (T *)y0dst, nullptr); \
        } else if (format == COSPDNN_INPUT_U8) {                                                             \
            k_convert_pieces<T, COSPDNN_INPUT_U8><<<cb, 256, 0, s>>>(b, R, N, layout, (T *)y0dst);        \
        } else {                                                                                             \
            k_convert_pieces<T, COSPDNN_INPUT_BITS><<<cb, 256, 0, s>>>(b, R, N, layout, (T *)y0dst);      \
        }                                                                                                    \
    } while (0)
        if (n.d.precision == COSPDNN_PREC_FP32) CSP_PIECES(float);
        else if (n.d.precision == COSPDNN_PREC_FP16) CSP_PIECES(__half);
        else CSP_PIECES(__nv_bfloat16);
#undef CSP_PIECES
        if (!skip) {
            if (format == COSPDNN_INPUT_U8) k_row_max<COSPDNN_INPUT_U8><<<blocks, 256, 0, s>>>(b, R, N, err0, mx0, nullptr);
            else k_row_max<COSPDNN_INPUT_BITS><<<blocks, 256, 0, s>>>(b, R, N, err0, mx0, nullptr);
        }
        CSP_CUDA(cudaGetLastError());
        return COSPDNN_OK;
    }
    if (n.dev.layout >= 2 && format != COSPDNN_INPUT_F32) {
        // integer input into row tiles
        const uint8_t *b = (const uint8_t *)src;
        const int TR = n.dev.layout;
        const int64_t units = (int64_t)((R + TR - 1) / TR) * (TR / std::min(TR, 8)) * (N / 8);
        const int cb = (int)std::min<int64_t>((units + 255) / 256, 148 * 16);
        // row maxima first: their binary flag decides whether the compute-type
        // copy is needed (a net counting layer 0 reads the bit planes instead,
        // and packed bits are always binary); for such a net the bit-plane
        // conversion writes them
        if (n.nbflag[back])
            l0_convert_bits(b, format, R, N, n.bitsbuf[back], err0, mx0, n.nbflag[back], s);
        else if (format == COSPDNN_INPUT_U8)
            k_row_max<COSPDNN_INPUT_U8><<<blocks, 256, 0, s>>>(b, R, N, err0, mx0, nullptr);
        else k_row_max<COSPDNN_INPUT_BITS><<<blocks, 256, 0, s>>>(b, R, N, err0, mx0, nullptr);
        const int *skip = n.nbflag[back];
        if (!(skip && format == COSPDNN_INPUT_BITS)) {
#define CSP_TILE(T)                                                                                             \
    do {                                                                                                        \
        if (format == COSPDNN_INPUT_U8)                                                                         \
            k_convert_tile<T, COSPDNN_INPUT_U8><<<cb, 256, 0, s>>>(b, R, N, TR, (T *)y0dst, skip);             \
        else                                                                                                    \
            k_convert_tile<T, COSPDNN_INPUT_BITS><<<cb, 256, 0, s>>>(b, R, N, TR, (T *)y0dst, nullptr);        \
    } while (0)
            if (n.d.precision == COSPDNN_PREC_FP32) CSP_TILE(float);
            else if (n.d.precision == COSPDNN_PREC_FP16) CSP_TILE(__half);
            else CSP_TILE(__nv_bfloat16);
#undef CSP_TILE
        }
        CSP_CUDA(cudaGetLastError());
        return COSPDNN_OK;
    }
#define CSP_CONV(T)                                                                                      \
    do {                                                                                                 \
        T *dst = (T *)y0dst;                                                                          \
        if (format == COSPDNN_INPUT_U8) k_convert_input<T, COSPDNN_INPUT_U8><<<blocks, 256, 0, s>>>(src, R, N, n.dev.layout, dst, f32, err0, mx0); \
        else if (format == COSPDNN_INPUT_F32) k_convert_input<T, COSPDNN_INPUT_F32><<<blocks, 256, 0, s>>>(src, R, N, n.dev.layout, dst, f32, err0, mx0); \
        else k_convert_input<T, COSPDNN_INPUT_BITS><<<blocks, 256, 0, s>>>(src, R, N, n.dev.layout, dst, f32, err0, mx0); \
    } while (0)
    if (n.d.precision == COSPDNN_PREC_FP32) CSP_CONV(float);
    else if (n.d.precision == COSPDNN_PREC_FP16) CSP_CONV(__half);
    else CSP_CONV(__nv_bfloat16);
#undef CSP_CONV
    CSP_CUDA(cudaGetLastError());
    return COSPDNN_OK;
}

namespace {

// Makes the inputs set since the last run current: swaps each such net's
// input buffers and updates its device descriptor, ordered on `s` before
// the run that reads it.
int take_inputs(cospdnn_engine *e, cudaStream_t s) {
    for (size_t i = 0; i < e->nets.size(); ++i) {
        Net &n = e->nets[i];
        if (!n.pending) continue;
        n.front ^= 1;
        n.pending = false;
        n.dev.y0 = n.y0buf[n.front];
        n.dev.err0 = n.err0buf[n.front];
        n.dev.mx0 = n.mx0buf[n.front];
        n.dev.y0_f32 = n.f32used[n.front] ? n.f32buf[n.front] : nullptr;
        if (n.bitsbuf[n.front]) {
            n.dev.y0bits = n.bitsbuf[n.front];
            n.dev.y0nonbin = n.nbflag[n.front];
        }
        k_store_netdev<<<1, 1, 0, s>>>(e->d_nets + i, n.dev);
        CSP_CUDA(cudaGetLastError());
    }
    return COSPDNN_OK;
}

}  // namespace

extern "C" int cospdnn_engine_run(cospdnn_engine *e, void *stream) {
    CSP_CHECK(e, COSPDNN_ERR_INVALID, "run: null engine");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "run: build first");
    DeviceGuard g(e->device);
    int rc = take_inputs(e, (cudaStream_t)stream);
    if (rc) return rc;
    CSP_CUDA(cudaGraphLaunch(e->exec, (cudaStream_t)stream));
    return COSPDNN_OK;
}

extern "C" int cospdnn_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

extern "C" int cospdnn_engine_run_timed(cospdnn_engine *e, void *stream, float *ms) {
    CSP_CHECK(e && ms, COSPDNN_ERR_INVALID, "run_timed: null argument");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "run_timed: build first");
    DeviceGuard g(e->device);
    cudaStream_t s = (cudaStream_t)stream;
    int rc = take_inputs(e, s);
    if (rc) return rc;
    cudaEvent_t a, b;
    CSP_CUDA(cudaEventCreate(&a));
    cudaError_t err = cudaEventCreate(&b);
    if (err != cudaSuccess) {
        cudaEventDestroy(a);
        return cuda_fail(err, "run_timed: event");
    }
    err = cudaEventRecord(a, s);
    if (err == cudaSuccess) err = cudaGraphLaunch(e->exec, s);
    if (err == cudaSuccess) err = cudaEventRecord(b, s);
    if (err == cudaSuccess) err = cudaEventSynchronize(b);
    if (err == cudaSuccess) err = cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CSP_CUDA(err);
    return COSPDNN_OK;
}

extern "C" int cospdnn_engine_result(cospdnn_engine *e, int net, int32_t *categories, int64_t *count,
                                     int64_t *alive_per_layer, int64_t *rechecked_per_layer,
                                     void *stream) {
    CSP_CHECK(e && count, COSPDNN_ERR_INVALID, "result: null argument");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "result: build first");
    CSP_CHECK(net >= 0 && net < (int)e->nets.size(), COSPDNN_ERR_INVALID, "result: bad net");
    DeviceGuard g(e->device);
    cudaStream_t s = (cudaStream_t)stream;
    Net &n = e->nets[net];
    NetState st;
    CSP_CUDA(cudaMemcpyAsync(&st, n.dev.st, sizeof(st), cudaMemcpyDeviceToHost, s));
    CSP_CUDA(cudaStreamSynchronize(s));
    CSP_CHECK(st.err == 0, COSPDNN_ERR_DEVICE, "result: device-side loop guard tripped");
    CSP_CHECK(st.done, COSPDNN_ERR_STATE, "result: network has not finished (run first)");
    const int64_t cnt = (st.layer >= n.d.layers) ? st.R : 0;
    *count = cnt;
    if (categories && cnt > 0)
        CSP_CUDA(cudaMemcpyAsync(categories, n.dev.orig[st.layer & 1], sizeof(int32_t) * cnt, cudaMemcpyDeviceToHost, s));
    std::vector<long long> tmp(n.d.layers);
    if (alive_per_layer) {
        CSP_CUDA(cudaMemcpyAsync(tmp.data(), n.dev.alive_count, sizeof(long long) * n.d.layers, cudaMemcpyDeviceToHost, s));
        CSP_CUDA(cudaStreamSynchronize(s));
        for (int l = 0; l < n.d.layers; ++l) alive_per_layer[l] = tmp[l];
    }
    if (rechecked_per_layer) {
        CSP_CUDA(cudaMemcpyAsync(tmp.data(), n.dev.recheck_count, sizeof(long long) * n.d.layers, cudaMemcpyDeviceToHost, s));
        CSP_CUDA(cudaStreamSynchronize(s));
        for (int l = 0; l < n.d.layers; ++l) rechecked_per_layer[l] = tmp[l];
    }
    CSP_CUDA(cudaStreamSynchronize(s));
    return COSPDNN_OK;
}

namespace {

// Copies rows 0..min(R, max_rows)-1 of network `net`'s current activations
// (as floats) and their original ids (ids may be NULL) to host memory;
// *count gets the rows copied.  Synchronizes `s`.
int copy_current_rows(cospdnn_engine *e, int net, float *out, int32_t *ids, float *bounds, int64_t max_rows,
                      int64_t *count, cudaStream_t s) {
    Net &n = e->nets[net];
    NetState st;
    CSP_CUDA(cudaMemcpyAsync(&st, n.dev.st, sizeof(st), cudaMemcpyDeviceToHost, s));
    CSP_CUDA(cudaStreamSynchronize(s));
    const int64_t rows = std::min<int64_t>(st.R, max_rows);
    *count = rows;
    if (rows <= 0) {
        *count = 0;
        return COSPDNN_OK;
    }
    const size_t bytes = (size_t)rows * n.d.neuron * 4;
    float *tmp = nullptr;
    CSP_CUDA(cudaMalloc(&tmp, bytes + 8 * rows));
    int32_t *tids = reinterpret_cast<int32_t *>(reinterpret_cast<char *>(tmp) + bytes);
    float *tb = reinterpret_cast<float *>(tids + rows);
    if (n.d.precision == COSPDNN_PREC_FP32) k_gather_rows<float><<<592, 256, 0, s>>>(e->d_nets + net, tmp, tids, tb, rows);
    else if (n.d.precision == COSPDNN_PREC_FP16) k_gather_rows<__half><<<592, 256, 0, s>>>(e->d_nets + net, tmp, tids, tb, rows);
    else k_gather_rows<__nv_bfloat16><<<592, 256, 0, s>>>(e->d_nets + net, tmp, tids, tb, rows);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaMemcpyAsync(out, tmp, bytes, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess && ids) err = cudaMemcpyAsync(ids, tids, sizeof(int32_t) * rows, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess && bounds) err = cudaMemcpyAsync(bounds, tb, sizeof(float) * rows, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    cudaFree(tmp);
    CSP_CUDA(err);
    return COSPDNN_OK;
}

}  // namespace

extern "C" int cospdnn_engine_final_values(cospdnn_engine *e, int net, float *out, int64_t max_rows,
                                           void *stream) {
    CSP_CHECK(e && out, COSPDNN_ERR_INVALID, "final_values: null argument");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "final_values: build first");
    CSP_CHECK(net >= 0 && net < (int)e->nets.size(), COSPDNN_ERR_INVALID, "final_values: bad net");
    CSP_CHECK(max_rows >= 0, COSPDNN_ERR_INVALID, "final_values: negative max_rows");
    DeviceGuard g(e->device);
    int64_t cnt = 0;
    return copy_current_rows(e, net, out, nullptr, nullptr, max_rows, &cnt, (cudaStream_t)stream);
}

extern "C" int cospdnn_engine_net_info(cospdnn_engine *e, int net, int *kernel, int *row_tile,
                                       int *layer0_counted, void *stream) {
    CSP_CHECK(e && kernel && row_tile && layer0_counted, COSPDNN_ERR_INVALID, "net_info: null argument");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "net_info: build first");
    CSP_CHECK(net >= 0 && net < (int)e->nets.size(), COSPDNN_ERR_INVALID, "net_info: bad net");
    DeviceGuard g(e->device);
    const Net &n = e->nets[net];
    NetState st;
    CSP_CUDA(cudaMemcpyAsync(&st, n.dev.st, sizeof(st), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CSP_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    *kernel = n.dev.kernel;
    *row_tile = n.dev.layout >= 2 ? n.dev.layout : 0;
    *layer0_counted = st.l0_bits;
    return COSPDNN_OK;
}

extern "C" int cospdnn_engine_final_bound(cospdnn_engine *e, int net, float *max_bound, void *stream) {
    CSP_CHECK(e && max_bound, COSPDNN_ERR_INVALID, "final_bound: null argument");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "final_bound: build first");
    CSP_CHECK(net >= 0 && net < (int)e->nets.size(), COSPDNN_ERR_INVALID, "final_bound: bad net");
    DeviceGuard g(e->device);
    cudaStream_t s = (cudaStream_t)stream;
    const Net &n = e->nets[net];
    NetState st;
    CSP_CUDA(cudaMemcpyAsync(&st, n.dev.st, sizeof(st), cudaMemcpyDeviceToHost, s));
    CSP_CUDA(cudaStreamSynchronize(s));
    *max_bound = 0.0f;
    if (st.R <= 0) return COSPDNN_OK;
    std::vector<float> b((size_t)st.R);
    CSP_CUDA(cudaMemcpyAsync(b.data(), n.dev.err[st.layer & 1], sizeof(float) * st.R, cudaMemcpyDeviceToHost, s));
    CSP_CUDA(cudaStreamSynchronize(s));
    for (float x : b) *max_bound = std::max(*max_bound, x);
    return COSPDNN_OK;
}

extern "C" int cospdnn_engine_set_test_limits(cospdnn_engine *e, long long wait_cycles, int max_iters,
                                              int withhold_stage) {
    CSP_CHECK(e, COSPDNN_ERR_INVALID, "set_test_limits: null engine");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "set_test_limits: build first");
    CSP_CHECK(wait_cycles >= 0 && max_iters >= 0 && (withhold_stage == 0 || withhold_stage == 1), COSPDNN_ERR_INVALID,
              "set_test_limits: bad argument");
    CSP_CHECK(wait_cycles == 0 || wait_cycles >= 1000000, COSPDNN_ERR_INVALID,
              "set_test_limits: a wait limit below 1e6 cycles would fail correct runs");
    DeviceGuard g(e->device);
    const DevLimits lim{wait_cycles ? wait_cycles : kDefaultWaitCycles, max_iters ? max_iters : e->max_layers + 2,
                        withhold_stage};
    CSP_CUDA(cudaDeviceSynchronize());  // no run in flight reads the old limits
    CSP_CUDA(cudaMemcpy(e->limits, &lim, sizeof(lim), cudaMemcpyHostToDevice));
    return COSPDNN_OK;
}

extern "C" int cospdnn_engine_launch_count(cospdnn_engine *e, int64_t *launches, void *stream) {
    CSP_CHECK(e && launches, COSPDNN_ERR_INVALID, "launch_count: null argument");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "launch_count: build first");
    DeviceGuard g(e->device);
    unsigned long long v = 0;
    CSP_CUDA(cudaMemcpyAsync(&v, e->launches, sizeof(v), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CSP_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    *launches = (int64_t)v;
    return COSPDNN_OK;
}

extern "C" int cospdnn_engine_result_async(cospdnn_engine *e, int net, void *host_buf, size_t bytes,
                                           void *stream) {
    CSP_CHECK(e && host_buf, COSPDNN_ERR_INVALID, "result_async: null argument");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "result_async: build first");
    CSP_CHECK(net >= 0 && net < (int)e->nets.size(), COSPDNN_ERR_INVALID, "result_async: bad net");
    const Net &n = e->nets[net];
    const size_t need = 8 * (size_t)(1 + n.d.layers) + 4 * (size_t)n.d.rows;
    CSP_CHECK(bytes >= need, COSPDNN_ERR_INVALID, "result_async: buffer too small");
    DeviceGuard g(e->device);
    cudaStream_t s = (cudaStream_t)stream;
    k_result_pack<<<8, 256, 0, s>>>(e->d_nets + net, e->packbuf[net]);
    CSP_CUDA(cudaGetLastError());
    CSP_CUDA(cudaMemcpyAsync(host_buf, e->packbuf[net], need, cudaMemcpyDeviceToHost, s));
    return COSPDNN_OK;
}

extern "C" int cospdnn_run_networks(const cospdnn_network *nets, int n, int device, float *ms) {
    CSP_CHECK(nets && n > 0, COSPDNN_ERR_INVALID, "run_networks: no networks");
    for (int i = 0; i < n; ++i) {
        const cospdnn_network &w = nets[i];
        CSP_CHECK(w.count && w.y0, COSPDNN_ERR_INVALID, "run_networks: null input or count");
        CSP_CHECK(w.desc.layers <= 0 || (w.colptr && w.rowidx && w.vals), COSPDNN_ERR_INVALID,
                  "run_networks: null layer arrays");
        CSP_CHECK(w.desc.rows <= 0 || w.categories, COSPDNN_ERR_INVALID, "run_networks: null categories");
    }
    cospdnn_engine *e = nullptr;
    int rc = cospdnn_engine_create(&e, device);
    if (rc) return rc;
    std::unique_ptr<cospdnn_engine, void (*)(cospdnn_engine *)> guard(e, cospdnn_engine_destroy);
    std::vector<int> ids(n);
    for (int i = 0; i < n && !rc; ++i) {
        rc = cospdnn_engine_add_net(e, &nets[i].desc, &ids[i]);
        for (int l = 0; l < nets[i].desc.layers && !rc; ++l)
            rc = cospdnn_engine_set_layer_csc(e, ids[i], l, nets[i].colptr[l], nets[i].rowidx[l], nets[i].vals[l]);
    }
    if (!rc) rc = cospdnn_engine_build(e);
    for (int i = 0; i < n && !rc; ++i) rc = cospdnn_engine_set_input(e, ids[i], nets[i].y0, nets[i].format, 0, nullptr);
    float t = 0.0f;
    if (!rc) rc = cospdnn_engine_run_timed(e, nullptr, &t);
    for (int i = 0; i < n && !rc; ++i)
        rc = cospdnn_engine_result(e, ids[i], nets[i].categories, nets[i].count, nets[i].alive_per_layer, nullptr,
                                   nullptr);
    if (!rc && ms) *ms = t;
    return rc;
}

namespace {

// The layer loop of the graph run from the host, one iteration (every live
// network advances one layer) at a time, synchronizing after each.  With
// layer_ms the layer kernels of iteration i are timed into layer_ms[i].
// Stops after max_iters iterations, when every network is done, or (stop_net
// >= 0) once network stop_net has computed layer stop_layer or finished.
// With start false the loop resumes a stopped pass at iteration it0 (no new
// inputs, no reset of the states).
int eager_run(cospdnn_engine *e, cudaStream_t s, int max_iters, float *layer_ms, int *iters, int stop_net,
              int stop_layer, bool start = true, int it0 = 0) {
    int rc = start ? take_inputs(e, s) : COSPDNN_OK;
    if (rc) return rc;
    cudaEvent_t a, b;
    CSP_CUDA(cudaEventCreate(&a));
    {
        const cudaError_t err = cudaEventCreate(&b);
        if (err != cudaSuccess) {
            cudaEventDestroy(a);
            return cuda_fail(err, "eager run: event");
        }
    }
    if (start) rc = launch(e->k0, s);
    int it = it0;
    std::vector<NetState> st(e->nets.size());
    while (!rc && it < max_iters) {
        bool live = false;
        for (size_t i = 0; i < e->nets.size() && !rc; ++i) {
            cudaError_t err = cudaMemcpyAsync(&st[i], e->nets[i].dev.st, sizeof(NetState), cudaMemcpyDeviceToHost, s);
            if (err != cudaSuccess) rc = cuda_fail(err, "eager run: state copy");
        }
        if (rc) break;
        cudaError_t err = cudaStreamSynchronize(s);
        if (err != cudaSuccess) { rc = cuda_fail(err, "eager run: sync"); break; }
        bool failed = false;
        for (auto &x : st) {
            live |= !x.done;
            failed |= x.err != 0;  // a device-side check stopped the run (as the graph's loop stops)
        }
        if (!live || failed) break;
        if (stop_net >= 0 && (st[stop_net].done || st[stop_net].layer > stop_layer)) break;
        if (layer_ms) cudaEventRecord(a, s);
        if (it == 0)
            for (KSpec &k : e->l0_specs) if (!rc) rc = launch(k, s);
        for (KSpec &k : e->layer_specs) if (!rc) rc = launch(k, s);
        if (layer_ms) cudaEventRecord(b, s);
        if (!rc) rc = launch(e->k2, s);
        if (!rc) rc = launch(e->k3, s);
        if (!rc) rc = launch(e->k4_eager, s);
        if (!rc) rc = launch(e->k5, s);
        if (rc) break;
        if (layer_ms) {
            err = cudaEventSynchronize(b);
            if (err != cudaSuccess) { rc = cuda_fail(err, "eager run: event"); break; }
            cudaEventElapsedTime(&layer_ms[it], a, b);
        }
        ++it;
    }
    if (iters) *iters = it;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (!rc) {
        cudaError_t err = cudaStreamSynchronize(s);
        if (err != cudaSuccess) rc = cuda_fail(err, "eager run: final sync");
    }
    return rc;
}

}  // namespace

extern "C" int cospdnn_engine_profile_layers(cospdnn_engine *e, void *stream, int max_iters,
                                             float *layer_ms, int *iters) {
    CSP_CHECK(e && layer_ms && iters && max_iters > 0, COSPDNN_ERR_INVALID, "profile_layers: bad argument");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "profile_layers: build first");
    DeviceGuard g(e->device);
    return eager_run(e, (cudaStream_t)stream, max_iters, layer_ms, iters, -1, 0);
}

extern "C" int cospdnn_engine_layer_values(cospdnn_engine *e, int net, int layer, float *out, int32_t *ids,
                                           float *bounds, int64_t max_rows, int64_t *count, void *stream) {
    CSP_CHECK(e && out && count, COSPDNN_ERR_INVALID, "layer_values: null argument");
    CSP_CHECK(e->built, COSPDNN_ERR_STATE, "layer_values: build first");
    CSP_CHECK(net >= 0 && net < (int)e->nets.size(), COSPDNN_ERR_INVALID, "layer_values: bad net");
    CSP_CHECK(layer >= 0 && layer < e->nets[net].d.layers, COSPDNN_ERR_INVALID, "layer_values: bad layer");
    CSP_CHECK(max_rows >= 0, COSPDNN_ERR_INVALID, "layer_values: negative max_rows");
    DeviceGuard g(e->device);
    cudaStream_t s = (cudaStream_t)stream;
    *count = 0;
    int it = 0;
    int rc = eager_run(e, s, e->max_layers + 1, nullptr, &it, net, layer);
    if (rc) return rc;
    NetState st;
    CSP_CUDA(cudaMemcpyAsync(&st, e->nets[net].dev.st, sizeof(st), cudaMemcpyDeviceToHost, s));
    CSP_CUDA(cudaStreamSynchronize(s));
    CSP_CHECK(st.err == 0, COSPDNN_ERR_DEVICE, "layer_values: device-side check failed");
    // rows of `layer` (none when every row was pruned before it)
    if (st.layer == layer + 1) rc = copy_current_rows(e, net, out, ids, bounds, max_rows, count, s);
    if (rc) return rc;
    // the pass runs on to the end, so that every network's result is again
    // that of a complete run
    return eager_run(e, s, e->max_layers + 1, nullptr, nullptr, -1, 0, false, it);
}
