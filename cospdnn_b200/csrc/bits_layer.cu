// Layer 0 by bit counting.  The inputs of the sparse-DNN benchmarks are binary
// images and every output's weights are one value (1/16 in the Graph
// Challenge networks), so an output of layer 0 is
//     z = bias + w_j * (number of its inputs that are 1),
// an exact integer count.  The inputs are stored as bit planes (one 32-bit
// word per feature and 32 rows, made by the input conversion, which then
// skips the compute-type copy).  A CTA stages one unit of rows in shared
// memory and lane j of a warp adds the words of output j's inputs into six
// bit-sliced counters (carry-save adders, Harley-Seal: about 2.4 logic
// instructions per word); the counters are turned into one byte per row by
// an 8x8 bit transpose across the planes (three rounds of delta swaps) and
// into floats exactly by a byte permute.  Bias, clamp and the store in the
// compute type follow the epilogue of the kernel the net uses otherwise, with
// its per-row statistics for the keep/prune decision, so the stored values
// and the rows sent to the FP64 recheck are the same as without counting.
//   k_layer0_bits    row-tile nets: units of 32 rows (4 bytes per feature);
//                    shared-memory traffic per output and 32 rows is 32
//                    words against 32 x 32 16-bit values in the row-tile
//                    kernel.
//   k_layer0_bits16  MMA-tile (tcgen05) nets: units of 16 rows (2 bytes per
//                    feature, so 65536 features fit in shared memory), two
//                    entries' words packed per 32-bit word, values stored into
//                    the MMA operand tiles.
// Entry schedule: per warp of 32 outputs, either an edge colouring of
// outputs x banks (the lanes of a step read 32 distinct banks; padding reads
// zero words placed in free banks) or ascending input order, whichever costs
// fewer shared-memory wavefronts (ascending order is conflict-free for XOR
// masks and broadcast-friendly for dense blocks).  Binary inputs are checked
// per input (U8 maxima; the packed-bit format is binary); other inputs, FP32
// values, and layers whose outputs mix weight values take the general kernels.
#include <algorithm>
#include <cmath>
#include <type_traits>

#include "bit_count.cuh"
#include "bits_layer.cuh"
#include "cc_layer.cuh"

namespace cospdnn {

namespace {

constexpr int kBitsThreads = 256;
constexpr int kBitsWarps = kBitsThreads / 32;
constexpr int kBitsMaxK = 63;  // real entries per output: six bit-sliced counters

// byte g of a counts word as the float 2^23 + count (the byte as its mantissa)
__device__ __forceinline__ uint32_t count_bits(uint32_t c, int g) { return __byte_perm(c, 0x4B000000u, 0x7440u | g); }

// z = count * w + bias for two counts given as 2^23 + count: the count is
// recovered exactly by subtracting 2^23, in two sm_100 packed instructions
// (add.rn.f32x2, fma.rn.f32x2: each half one IEEE operation, identical to
// the scalar subtraction and fmaf)
__device__ __forceinline__ void z_pair(uint32_t c0, uint32_t c1, float w, float bias, float &z0, float &z1) {
    asm("{\n\t.reg .b64 x, m, w, b;\n\t"
        "mov.b64 x, {%2, %3};\n\t"
        "mov.b64 m, {%6, %6};\n\t"
        "add.rn.f32x2 x, x, m;\n\t"
        "mov.b64 w, {%4, %4};\n\t"
        "mov.b64 b, {%5, %5};\n\t"
        "fma.rn.f32x2 x, x, w, b;\n\t"
        "mov.b64 {%0, %1}, x;\n\t}"
        : "=f"(z0), "=f"(z1)
        : "r"(c0), "r"(c1), "f"(w), "f"(bias), "f"(-8388608.0f));
}

// Two values as the 16-bit pair word {lo, hi} of type T, each max(v, 0)
// rounded to nearest (one cvt.rn.relu: the same values as from_f(fmaxf(v, 0))).
__device__ __forceinline__ uint32_t relu_pack(float lo, float hi, __half) {
    uint32_t d;
    asm("cvt.rn.relu.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}
__device__ __forceinline__ uint32_t relu_pack(float lo, float hi, __nv_bfloat16) {
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

template <typename T>
struct Pack;
template <>
struct Pack<float> {
    static constexpr int kPer16 = 4;
};
template <>
struct Pack<__half> {
    static constexpr int kPer16 = 8;
};
template <>
struct Pack<__nv_bfloat16> {
    static constexpr int kPer16 = 8;
};

__device__ __forceinline__ bool l0_net(const NetDev &nd, int prec) {
    return nd.l0_k > 0 && nd.kernel == COSPDNN_KERNEL_CUDA_CORE && nd.layout >= 4 && nd.prec == prec &&
           !nd.st->done && nd.st->layer == 0 && nd.y0bits != nullptr && *nd.y0nonbin == 0;
}

// One unit of 32 rows for the warp's groups of 32 outputs: counts, outputs
// stored, and the warp's row max z (and, unless SMALL, min |z - 16|) merged
// into the CTA's row statistics.  SMALL: |z| <= 16, so min |z - 16| is
// |max z - 16| (rounding of z - 16 is monotone), taken from the row max, and
// there is no clamp at 32.
template <typename T, bool SMALL>
__device__ __forceinline__ void count_unit(const NetDev &nd, const uint32_t *s_bits, uint32_t *s_zmax,
                                           uint32_t *s_zdist, int u, int N, int TR, int K8, int ngroups, T *out,
                                           float bias) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float zmx[32], zds[SMALL ? 1 : 32];
#pragma unroll
    for (int r = 0; r < 32; ++r) {
        zmx[r] = -INFINITY;
        if constexpr (!SMALL) zds[r] = INFINITY;
    }
    for (int g = warp; g < ngroups; g += kBitsWarps) {
        const int j = g * 32 + lane;
        uint32_t p[6] = {0u, 0u, 0u, 0u, 0u, 0u};
        const uint4 *ent = nd.l0_idx + (int64_t)g * K8 * 32 + lane;
        for (int t = 0; t < K8; ++t) {
            const uint4 q = __ldg(ent + (int64_t)t * 32);
            const uint32_t x[8] = {s_bits[q.x & 0xFFFFu], s_bits[q.x >> 16], s_bits[q.y & 0xFFFFu],
                                   s_bits[q.y >> 16],     s_bits[q.z & 0xFFFFu], s_bits[q.z >> 16],
                                   s_bits[q.w & 0xFFFFu], s_bits[q.w >> 16]};
            add8(p, x);
        }
        const float w = nd.l0_w[j];
        // rows 8b .. 8b+7 (byte b of counts words 0..7), each group of 8 stored at once
        constexpr int V = Pack<T>::kPer16;  // values per 16-byte piece
        uint32_t c[8];
        counts8(p, c);
        const int64_t row0 = (int64_t)u * 32;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            __align__(16) T ov[8];
#pragma unroll
            for (int k = 0; k < 8; k += 2) {
                float z[2];
                z_pair(count_bits(c[k], b), count_bits(c[k + 1], b), w, bias, z[0], z[1]);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int r = 8 * b + k + h;
                    zmx[r] = fmaxf(zmx[r], z[h]);
                    if constexpr (SMALL) {
                        ov[k + h] = act_traits<T>::from_f(fmaxf(z[h], 0.0f));
                    } else {
                        zds[r] = fminf(zds[r], fabsf(z[h] - 16.0f));
                        ov[k + h] = act_traits<T>::from_f(clamp32(z[h]));
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 8; k += V) {
                if (TR >= V) {  // a 16-byte piece lies inside one tile
                    *reinterpret_cast<uint4 *>(out + act_index(TR, N, row0 + 8 * b + k, j)) =
                        *reinterpret_cast<const uint4 *>(ov + k);
                } else {  // 16-bit values, tiles of 4 rows: two 8-byte pieces
                    *reinterpret_cast<uint2 *>(out + act_index(TR, N, row0 + 8 * b + k, j)) =
                        *reinterpret_cast<const uint2 *>(ov + k);
                    *reinterpret_cast<uint2 *>(out + act_index(TR, N, row0 + 8 * b + k + 4, j)) =
                        *reinterpret_cast<const uint2 *>(ov + k + 4);
                }
            }
        }
    }
    // row max z and min |z - 16| over the warp's outputs, then over the CTA
#pragma unroll
    for (int r = 0; r < 32; ++r) {
        const uint32_t m = __reduce_max_sync(0xffffffffu, f2ord(zmx[r]));
        if (lane == r) atomicMax(&s_zmax[r], m);
        if constexpr (!SMALL) {
            const uint32_t d = __reduce_min_sync(0xffffffffu, __float_as_uint(zds[r]));  // >= 0
            if (lane == r) atomicMin(&s_zdist[r], d);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kBitsThreads, 2)
    k_layer0_bits(const NetDev *__restrict__ nets, int nnets, int prec, unsigned long long *launches) {
    count_launch(launches);
    extern __shared__ uint4 l0_smem[];
    uint32_t *s_bits = reinterpret_cast<uint32_t *>(l0_smem);
    __shared__ uint32_t s_zmax[32], s_zdist[32];
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (!l0_net(nd, prec)) continue;
        if (blockIdx.x == 0 && threadIdx.x == 0) nd.st->l0_bits = 1;  // the row-tile kernel skips layer 0
        const int N = nd.N, R = nd.st->R, TR = nd.layout, K8 = nd.l0_k / 8;
        const int units = (R + 31) / 32, ngroups = N / 32;
        const bool small = nd.l0_small != 0;
        const LayerDev &lw = nd.layers[0];
        T *out = (T *)nd.act[nd.st->in_buf ^ 1];
        const float bias = nd.bias;
        for (int u = blockIdx.x; u < units; u += gridDim.x) {
            __syncthreads();  // the previous unit is done with the words and the row statistics
            {
                const uint4 *src = reinterpret_cast<const uint4 *>(nd.y0bits + (int64_t)u * N);
                for (int i = threadIdx.x; i < N / 4; i += kBitsThreads) l0_smem[i] = __ldg(src + i);
                if (threadIdx.x < 32) {
                    s_bits[N + threadIdx.x] = 0u;  // padding words, one per bank
                    s_zmax[threadIdx.x] = 0u;
                    s_zdist[threadIdx.x] = 0x7F800000u;
                }
            }
            __syncthreads();
            if (small)
                count_unit<T, true>(nd, s_bits, s_zmax, s_zdist, u, N, TR, K8, ngroups, out, bias);
            else
                count_unit<T, false>(nd, s_bits, s_zmax, s_zdist, u, N, TR, K8, ngroups, out, bias);
            __syncthreads();
            if (threadIdx.x < 32) {
                const int p = u * 32 + threadIdx.x;
                if (p < R) {
                    const double steps = fast_steps(nd, lw);
                    const float ez = z_error_bound(nd.err[0][p], nd.mx[0][p], lw.S, lw.dW, bias, steps);
                    // the row-tile kernel's statistics (row_stats): max output, and the
                    // bound plus the storage rounding when some output is within
                    // 16 + ez of 16
                    const float zm = ord2f(s_zmax[threadIdx.x]);
                    const float zd = small ? fabsf(zm - 16.0f) : __uint_as_float(s_zdist[threadIdx.x]);
                    const float c = clamp32(zm);
                    const float ym = act_traits<T>::to_f(act_traits<T>::from_f(c));
                    float se = 0.0f;
                    if constexpr (sizeof(T) == 2) {
                        se = std::is_same<T, __half>::value ? __fmaf_ru(c, 4.8828125e-04f, 2.98023224e-08f)
                                                            : __fmaf_ru(c, 3.90625e-03f, 1.17549435e-38f);
                    }
                    const float em = zd < 16.0f + ez ? __fadd_ru(ez, se) : 0.0f;
                    atomicMax(&nd.stat[3 * p], s_zmax[threadIdx.x]);
                    atomicMax(&nd.stat[3 * p + 1], __float_as_uint(em));
                    atomicMax(&nd.stat[3 * p + 2], __float_as_uint(ym));
                }
            }
        }
    }
}

// MMA-tile (tcgen05) nets: units of 16 rows, so that the words of a unit
// (16 bits per feature) fit in shared memory up to 65536 features; a lane
// packs two entries' 16-bit words into one 32-bit word (the even entry in
// the low half), counts them as above and adds the two halves' counts; each
// output value is stored into its MMA operand tile (act_index layout 1), or
// (feature-split nets) into its 2-row tile word (layout 2).
constexpr int kBits16Threads = 512;
constexpr int kBits16Warps = kBits16Threads / 32;

// RT: feature-split nets (2-row tiles, the row-tile kernels' statistics);
// else MMA-tile (tcgen05) nets.
template <bool RT>
__device__ __forceinline__ bool l0_net16(const NetDev &nd, int prec) {
    const bool kind = RT ? nd.cc_split != 0 : (nd.kernel == COSPDNN_KERNEL_TCGEN05 && nd.layout == 1);
    return nd.l0_k > 0 && kind && nd.prec == prec && !nd.st->done && nd.st->layer == 0 && nd.y0bits != nullptr &&
           *nd.y0nonbin == 0;
}

template <typename T, bool RT>
__global__ void __launch_bounds__(kBits16Threads, 1)
    k_layer0_bits16(const NetDev *__restrict__ nets, int nnets, int prec, unsigned long long *launches) {
    count_launch(launches);
    extern __shared__ uint4 l0_smem[];
    uint16_t *s_w = reinterpret_cast<uint16_t *>(l0_smem);
    // per row: max z; RT: min |z - 16| (bits of a value >= 0), else the
    // tcgen05 epilogue's output error
    __shared__ uint32_t s_zmax[16], s_zx[16];
    __shared__ float s_ez[16];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (!l0_net16<RT>(nd, prec)) continue;
        if (blockIdx.x == 0 && threadIdx.x == 0) nd.st->l0_bits = 1;  // the layer kernel skips layer 0
        const int N = nd.N, R = nd.st->R, K4 = nd.l0_k / 4;
        const int units = (R + 15) / 16, ngroups = N / 32;
        const LayerDev &lw = nd.layers[0];
        T *out = (T *)nd.act[nd.st->in_buf ^ 1];
        const float bias = nd.bias;
        for (int u = blockIdx.x; u < units; u += gridDim.x) {
            __syncthreads();  // the previous unit is done with the words and the row statistics
            {
                // half (u & 1) of the 32-row words of unit u / 2
                const int sh = (u & 1) * 16;
                const uint4 *src = reinterpret_cast<const uint4 *>(nd.y0bits + (int64_t)(u >> 1) * N);
                for (int i = threadIdx.x; i < N / 4; i += kBits16Threads) {
                    const uint4 v = __ldg(src + i);
                    reinterpret_cast<uint2 *>(s_w)[i] =
                        make_uint2(((v.x >> sh) & 0xFFFFu) | (((v.y >> sh) & 0xFFFFu) << 16),
                                   ((v.z >> sh) & 0xFFFFu) | (((v.w >> sh) & 0xFFFFu) << 16));
                }
                if (threadIdx.x < 32) reinterpret_cast<uint32_t *>(s_w + N)[threadIdx.x] = 0u;  // padding
                if (threadIdx.x < 16) {
                    s_zmax[threadIdx.x] = 0u;
                    s_zx[threadIdx.x] = RT ? 0x7F800000u : 0u;  // +inf / 0
                    if (!RT) {
                        const int p = min(u * 16 + (int)threadIdx.x, R - 1);
                        s_ez[threadIdx.x] =
                            z_error_bound(nd.err[0][p], nd.mx[0][p], lw.S, lw.dW, bias, fast_steps(nd, lw));
                    }
                }
            }
            __syncthreads();
            float zmx[16], zx[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                zmx[r] = -INFINITY;
                zx[r] = RT ? INFINITY : 0.0f;
            }
            // blocks of 16 entries (4 x 16 bytes per lane) of the warp's groups in
            // turn, the next block loaded while one is counted
            uint32_t p[6] = {0u, 0u, 0u, 0u, 0u, 0u};
            uint4 qa[4], qb[4];
            auto load = [&](uint4 *q, int g, int t) {
                const uint4 *ent = nd.l0_idx + ((int64_t)g * K4 + t) * 32 + lane;
#pragma unroll
                for (int v = 0; v < 4; ++v) q[v] = __ldg(ent + v * 32);
            };
            auto count = [&](const uint4 *q) {
                uint32_t x[8];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    x[2 * v] = (uint32_t)s_w[q[v].x] | ((uint32_t)s_w[q[v].y] << 16);
                    x[2 * v + 1] = (uint32_t)s_w[q[v].z] | ((uint32_t)s_w[q[v].w] << 16);
                }
                add8(p, x);
            };
            const bool small = RT && nd.l0_small != 0;
            int g = warp, t = 0, par = 0;
            float w = 0.0f, wn = 0.0f;  // weight of the group being counted, of the next one
            if (g < ngroups) {
                load(qa, g, 0);
                w = __ldg(nd.l0_w + g * 32 + lane);
            }
            while (g < ngroups) {
                int gn = g, tn = t + 4;
                if (tn >= K4) {
                    tn = 0;
                    gn += kBits16Warps;
                }
                if (tn == 0 && gn < ngroups) wn = __ldg(nd.l0_w + gn * 32 + lane);
                if (par == 0) {
                    if (gn < ngroups) load(qb, gn, tn);
                    count(qa);
                } else {
                    if (gn < ngroups) load(qa, gn, tn);
                    count(qb);
                }
                par ^= 1;
                if (tn == 0 && small) {
                    // every output |z| <= 16: no clamp at 32, min |z - 16| from the
                    // row max; row pairs (r, r + 1) converted and packed at once
                    const int j = g * 32 + lane;
                    uint32_t c[8];
                    counts8(p, c);
#pragma unroll
                    for (int k = 0; k < 6; ++k) p[k] = 0u;
#pragma unroll
                    for (int k = 0; k < 8; k += 2) {
                        const uint32_t sa = c[k] + (c[k] >> 16), sb = c[k + 1] + (c[k + 1] >> 16);
                        float za[2], zb[2];  // rows (k, 8 + k), (k + 1, 9 + k)
                        z_pair(count_bits(sa, 0), count_bits(sa, 1), w, bias, za[0], za[1]);
                        z_pair(count_bits(sb, 0), count_bits(sb, 1), w, bias, zb[0], zb[1]);
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int r = 8 * h + k;
                            zmx[r] = fmaxf(zmx[r], za[h]);
                            zmx[r + 1] = fmaxf(zmx[r + 1], zb[h]);
                            *reinterpret_cast<uint32_t *>(out + act_index(2, N, (int64_t)u * 16 + r, j)) =
                                relu_pack(za[h], zb[h], T());
                        }
                    }
                } else if (tn == 0) {
                    // group g counted: outputs of its 16 rows
                    const int j = g * 32 + lane;
                    uint32_t c[8];
                    counts8(p, c);
#pragma unroll
                    for (int k = 0; k < 6; ++k) p[k] = 0u;
                    T ov[16];
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        const uint32_t s2 = c[k] + (c[k] >> 16);  // even + odd entries' counts (each <= 32)
                        float zz[2];
                        z_pair(count_bits(s2, 0), count_bits(s2, 1), w, bias, zz[0], zz[1]);
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int r = 8 * h + k;
                            const float z = zz[h];
                            const float cz = clamp32(z);
                            ov[r] = act_traits<T>::from_f(cz);
                            zmx[r] = fmaxf(zmx[r], z);
                            if constexpr (RT) {
                                zx[r] = fminf(zx[r], fabsf(z - 16.0f));
                            } else {
                                // the tcgen05 epilogue's error of an output near the clamp range
                                const float ez = s_ez[r];
                                if (z > -ez && z < 32.0f + ez)
                                    zx[r] = fmaxf(zx[r], __fadd_ru(ez, fabsf(act_traits<T>::to_f(ov[r]) - cz)));
                            }
                        }
                    }
                    if constexpr (RT) {
                        // 2-row tiles: one 4-byte word per row pair, consecutive outputs adjacent
#pragma unroll
                        for (int r = 0; r < 16; r += 2)
                            *reinterpret_cast<uint32_t *>(out + act_index(2, N, (int64_t)u * 16 + r, j)) =
                                (uint32_t)*reinterpret_cast<const uint16_t *>(&ov[r]) |
                                ((uint32_t)*reinterpret_cast<const uint16_t *>(&ov[r + 1]) << 16);
                    } else {
#pragma unroll
                        for (int r = 0; r < 16; ++r) out[act_index(1, N, (int64_t)u * 16 + r, j)] = ov[r];
                    }
                }
                if (tn == 0) w = wn;
                g = gn;
                t = tn;
            }
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const uint32_t m = __reduce_max_sync(0xffffffffu, f2ord(zmx[r]));
                if constexpr (RT) {
                    const uint32_t d = small ? 0x7F800000u : __reduce_min_sync(0xffffffffu, __float_as_uint(zx[r]));
                    if (lane == r) {
                        atomicMax(&s_zmax[r], m);
                        if (!small) atomicMin(&s_zx[r], d);  // >= 0: bit order = value order
                    }
                } else {
                    const uint32_t e = __reduce_max_sync(0xffffffffu, __float_as_uint(zx[r]));  // >= 0
                    if (lane == r) {
                        atomicMax(&s_zmax[r], m);
                        atomicMax(&s_zx[r], e);
                    }
                }
            }
            __syncthreads();
            if (threadIdx.x < 16) {
                const int pr = u * 16 + threadIdx.x;
                if (pr < R) {
                    float em, ym;
                    if constexpr (RT) {
                        const float ez = z_error_bound(nd.err[0][pr], nd.mx[0][pr], lw.S, lw.dW, bias,
                                                       fast_steps(nd, lw));
                        const float zm = ord2f(s_zmax[threadIdx.x]);
                        // |z| <= 16: min |z - 16| is |max z - 16| (rounding of z - 16 is monotone)
                        const float zd = small ? fabsf(zm - 16.0f) : __uint_as_float(s_zx[threadIdx.x]);
                        row_stats<T>(zm, zd, ez, em, ym);
                    } else {
                        const float c = clamp32(ord2f(s_zmax[threadIdx.x]));
                        ym = act_traits<T>::to_f(act_traits<T>::from_f(c));  // the max stored output
                        em = __uint_as_float(s_zx[threadIdx.x]);
                    }
                    atomicMax(&nd.stat[3 * pr], s_zmax[threadIdx.x]);
                    atomicMax(&nd.stat[3 * pr + 1], __float_as_uint(em));
                    atomicMax(&nd.stat[3 * pr + 2], __float_as_uint(ym));
                }
            }
        }
    }
}

// A 32x32 bit matrix held one row per lane (bit k of lane r = element (r, k))
// transposed in place: afterwards bit r of lane k = the old element (r, k).
// Five rounds swap the off-diagonal blocks of size j between lanes r and r^j.
__device__ __forceinline__ uint32_t transpose32(uint32_t x, int lane) {
#pragma unroll
    for (int j = 16; j >= 1; j >>= 1) {
        const uint32_t m = j == 16 ? 0x0000FFFFu : j == 8 ? 0x00FF00FFu : j == 4 ? 0x0F0F0F0Fu
                         : j == 2 ? 0x33333333u : 0x55555555u;  // bits k with (k & j) == 0
        const uint32_t y = __shfl_xor_sync(0xffffffffu, x, j);
        if (lane & j) x = (x & ~m) | ((y >> j) & m);
        else x = (x & m) | ((y << j) & ~m);
    }
    return x;
}

// Bit planes of U8 (FMT 0) or packed-bit (FMT 2) rows, with the row maxima
// (error 0) and, for bytes, the flag raised by a value above 1: one warp per
// unit of 32 rows, lane r reading row 32*unit + r 32 features at a time and
// the warp transposing each 32x32 block (coalesced 128-byte stores).
template <int FMT>
__global__ void k_convert_bits(const uint8_t *__restrict__ src, int rows, int N, uint32_t *__restrict__ bits,
                               float *__restrict__ err0, float *__restrict__ mx0, int *__restrict__ nonbin) {
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int units = (rows + 31) / 32, nfb = N / 32;
    for (int64_t u = w; u < units; u += nw) {
        const int64_t row = u * 32 + lane;
        const bool valid = row < rows;
        uint32_t rmax = 0;
        for (int fb = 0; fb < nfb; ++fb) {
            uint32_t x = 0;  // bit k = feature 32*fb + k of this lane's row
            if (valid) {
                if (FMT == COSPDNN_INPUT_BITS) {
                    const uint8_t *b = src + row * (N / 8) + fb * 4;  // rows of N/8 bytes: any alignment
                    x = (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
                    rmax |= x;
                } else {
                    const uint8_t *b = src + row * N + fb * 32;
#pragma unroll
                    for (int k = 0; k < 32; k += 8) {
                        const uint2 v = *reinterpret_cast<const uint2 *>(b + k);  // N % 32 == 0: 8-byte aligned
                        rmax = max(rmax, __vmaxu4(v.x, v.y));
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            x |= (((v.x >> (8 * i)) & 0xFFu) ? 1u : 0u) << (k + i);
                            x |= (((v.y >> (8 * i)) & 0xFFu) ? 1u : 0u) << (k + 4 + i);
                        }
                    }
                }
            }
            bits[u * N + fb * 32 + lane] = transpose32(x, lane);
        }
        if (valid) {
            uint32_t m;
            if (FMT == COSPDNN_INPUT_BITS) {
                m = rmax ? 1u : 0u;
            } else {
                m = max(max(rmax & 0xFFu, (rmax >> 8) & 0xFFu), max((rmax >> 16) & 0xFFu, rmax >> 24));
                if (m > 1u) atomicOr(nonbin, 1);
            }
            err0[row] = 0.0f;
            mx0[row] = (float)m;
        }
    }
}

// Bit planes of packed-bit rows (COSPDNN_INPUT_BITS) with the row maxima:
// one CTA per unit of 32 rows.  The unit's rows are read a slice of up to
// kConvSlice 32-feature words at a time with coalesced 4-byte loads into
// shared memory (row stride padded by one word, so that lane r reading row
// r of a column hits bank r); each warp then takes word columns of the
// slice: lane r reads row r's word, the warp transposes the 32x32 bit block
// and writes one 128-byte line of bit planes.  A row's maximum is 1 when any
// of its bits is set.
constexpr int kConvThreads = 256;
constexpr int kConvSlice = 256;  // words per row staged at once (32 KB of shared memory)

__global__ void __launch_bounds__(kConvThreads)
    k_convert_packed(const uint8_t *__restrict__ src, int rows, int N, uint32_t *__restrict__ bits,
                     float *__restrict__ err0, float *__restrict__ mx0) {
    __shared__ uint32_t cs[32 * (kConvSlice + 1)];
    __shared__ uint32_t s_any[32];
    const int wpr = N / 32;  // 32-feature words per row
    const int units = (rows + 31) / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        const int r0 = u * 32, nr = min(32, rows - r0);
        __syncthreads();  // the previous unit is done with s_any
        if (threadIdx.x < 32) s_any[threadIdx.x] = 0u;
        // N % 32 == 0, so rows of N/8 bytes are whole words and every row
        // starts on a word boundary (the input is 16-byte aligned)
        const uint32_t *w = reinterpret_cast<const uint32_t *>(src + (int64_t)r0 * (N / 8));
        uint32_t any = 0u;
        for (int c0 = 0; c0 < wpr; c0 += kConvSlice) {
            const int sw = min(kConvSlice, wpr - c0), stride = sw + 1;
            __syncthreads();  // the previous slice is done with cs
            for (int i = threadIdx.x; i < 32 * sw; i += kConvThreads) {
                const int r = i / sw, c = i - r * sw;
                cs[r * stride + c] = r < nr ? __ldg(w + (int64_t)r * wpr + c0 + c) : 0u;
            }
            __syncthreads();
            for (int c = warp; c < sw; c += kConvThreads / 32) {
                const uint32_t x = cs[lane * stride + c];
                any |= x;
                bits[(int64_t)u * N + (int64_t)(c0 + c) * 32 + lane] = transpose32(x, lane);
            }
        }
        if (any) atomicOr(&s_any[lane], 1u);
        __syncthreads();
        if (threadIdx.x < nr) {
            err0[r0 + threadIdx.x] = 0.0f;
            mx0[r0 + threadIdx.x] = s_any[threadIdx.x] ? 1.0f : 0.0f;
        }
    }
}

}  // namespace

int l0_build(const std::vector<int32_t> &colptr, const std::vector<int32_t> &rowidx, const std::vector<float> &vals,
             int N, int prec, int layout, float bias, NetDev &nd, std::vector<void *> &owned) {
    nd.l0_k = 0;
    nd.l0_small = 0;
    nd.l0_idx = nullptr;
    nd.l0_w = nullptr;
    // row-tile nets: 32-bit words (32 rows), 16-bit indices, steps in 8s;
    // MMA-tile nets: 16-bit words (16 rows), 32-bit indices, steps in 16s
    const bool half = layout == 1;
    if (N % 32 != 0 || (!half && (layout < 4 || N + 32 > 65535))) return 0;
    // one weight value per output, at most 63 non-zero entries
    std::vector<float> w(N, 0.0f);
    std::vector<std::vector<int>> ent(N);
    for (int j = 0; j < N; ++j) {
        bool first = true;
        for (int p = colptr[j]; p < colptr[j + 1]; ++p) {
            if (vals[p] == 0.0f) continue;
            if (first) {
                w[j] = vals[p];
                first = false;
            } else if (vals[p] != w[j]) {
                return 0;
            }
            ent[j].push_back(rowidx[p]);
        }
        if ((int)ent[j].size() > kBitsMaxK) return 0;
    }
    // weights in the compute type (what the error bound's dW assumes)
    for (int j = 0; j < N; ++j) {
        if (prec == COSPDNN_PREC_FP16) w[j] = __half2float(__float2half_rn(w[j]));
        else if (prec == COSPDNN_PREC_BF16) w[j] = __bfloat162float(__float2bfloat16_rn(w[j]));
    }
    // per warp of 32 outputs: edge colouring outputs x banks, so that the
    // lanes of a step read distinct banks, or ascending input order when that
    // costs fewer wavefronts (outputs sharing their inputs, as in dense
    // blocks: lanes reading the same word are served by one broadcast)
    const int ngroups = N / 32;
    int Knat = 1;
    for (int j = 0; j < N; ++j) Knat = std::max(Knat, (int)ent[j].size());
    std::vector<std::vector<int>> order(N);
    int K = 1;
    std::vector<int> eu, es, colour;
    for (int g = 0; g < ngroups; ++g) {
        eu.clear();
        es.clear();
        std::vector<int> ei;
        for (int l = 0; l < 32; ++l)
            for (int i : ent[g * 32 + l]) {
                eu.push_back(l);
                es.push_back(half ? (i >> 1) % 32 : i % 32);  // shared-memory bank of the input's word
                ei.push_back(i);
            }
        const int D = ei.empty() ? 0 : colour_group(32, eu, es, colour);
        K = std::max(K, D);
        for (int l = 0; l < 32; ++l) order[g * 32 + l].assign(D, -1);
        for (size_t e = 0; e < ei.size(); ++e) order[g * 32 + eu[e]][colour[e]] = ei[e];
    }
    // shared-memory wavefronts of both orders: the coloured one costs one per
    // step; ascending order costs, per step, the largest number of distinct
    // words one bank serves (lanes reading the same word share a broadcast)
    double cost_col = (double)ngroups * K, cost_nat = 0.0;
    {
        std::vector<int> seen(32 * 32);
        for (int g = 0; g < ngroups; ++g)
            for (int t = 0; t < Knat; ++t) {
                int nb[32] = {0}, worst = 1;
                int ns = 0;
                for (int l = 0; l < 32; ++l) {
                    const auto &e = ent[g * 32 + l];
                    if (t >= (int)e.size()) continue;
                    const int word = half ? e[t] >> 1 : e[t], bank = word % 32;
                    bool dup = false;
                    for (int q = 0; q < ns; ++q) dup |= seen[q] == word;
                    if (dup) continue;
                    seen[ns++] = word;
                    worst = std::max(worst, ++nb[bank]);
                }
                cost_nat += worst;
            }
    }
    if (cost_nat < cost_col) {
        K = Knat;
        for (int j = 0; j < N; ++j) order[j] = ent[j];  // rows ascending within each column (CSC)
    }
    // padding words are zero, so only the real entries (<= 63 per output)
    // reach the six counters; the number of steps is not limited
    const int Kp = half ? (K + 15) / 16 * 16 : (K + 7) / 8 * 8;
    // [group][step/8][lane] uint4 = 8 indices of 16 bits (row tiles) or
    // [group][step/4][lane] uint4 = 4 indices of 32 bits (MMA tiles)
    std::vector<uint16_t> idx(half ? 0 : (size_t)ngroups * Kp * 32);
    std::vector<uint32_t> idx32(half ? (size_t)ngroups * Kp * 32 : 0);
    for (int g = 0; g < ngroups; ++g)
        for (int t = 0; t < Kp; ++t) {
            uint32_t used = 0;
            for (int l = 0; l < 32; ++l) {
                const auto &o = order[g * 32 + l];
                if (t < (int)o.size() && o[t] >= 0) used |= 1u << (half ? (o[t] >> 1) % 32 : o[t] % 32);
            }
            for (int l = 0; l < 32; ++l) {
                const auto &o = order[g * 32 + l];
                int i;
                if (t < (int)o.size() && o[t] >= 0) {
                    i = o[t];
                } else {
                    int b = 0;  // a zero word in a bank no real entry of this step uses
                    while (used & (1u << b)) ++b;
                    used |= 1u << b;
                    i = half ? N + 2 * (((b - (N / 2) % 32) + 32) % 32) : N + ((b - N % 32) + 32) % 32;
                }
                if (half) idx32[(((size_t)g * (Kp / 4) + t / 4) * 32 + l) * 4 + t % 4] = (uint32_t)i;
                else idx[(((size_t)g * (Kp / 8) + t / 8) * 32 + l) * 8 + t % 8] = (uint16_t)i;
            }
        }
    void *d_idx = nullptr, *d_w = nullptr;
    const size_t ibytes = half ? idx32.size() * sizeof(uint32_t) : idx.size() * sizeof(uint16_t);
    CSP_CUDA(cudaMalloc(&d_idx, ibytes));
    owned.push_back(d_idx);
    CSP_CUDA(cudaMalloc(&d_w, (size_t)N * sizeof(float)));
    owned.push_back(d_w);
    CSP_CUDA(cudaMemcpy(d_idx, half ? (const void *)idx32.data() : (const void *)idx.data(), ibytes,
                        cudaMemcpyHostToDevice));
    CSP_CUDA(cudaMemcpy(d_w, w.data(), (size_t)N * sizeof(float), cudaMemcpyHostToDevice));
    nd.l0_idx = (const uint4 *)d_idx;
    nd.l0_w = (const float *)d_w;
    nd.l0_k = Kp;
    double zb = 0.0;  // bound on |z| of every output
    for (int j = 0; j < N; ++j) zb = std::max(zb, std::fabs((double)w[j]) * (double)ent[j].size());
    nd.l0_small = zb + std::fabs((double)bias) <= 16.0 ? 1 : 0;
    return 0;
}

int l0_spec(KSpec &k, NetDev *nets, int nnets, int prec, int kind, unsigned long long *launches, int sms,
            int max_n) {
    using F = void (*)(const NetDev *, int, int, unsigned long long *);
    static const F fns[3] = {k_layer0_bits<float>, k_layer0_bits<__half>, k_layer0_bits<__nv_bfloat16>};
    static const F fns16[2][3] = {{nullptr, k_layer0_bits16<__half, false>, k_layer0_bits16<__nv_bfloat16, false>},
                                  {nullptr, k_layer0_bits16<__half, true>, k_layer0_bits16<__nv_bfloat16, true>}};
    const bool sixteen = kind != kL0Rows32;
    CSP_CHECK(!sixteen || prec != COSPDNN_PREC_FP32, COSPDNN_ERR_UNSUPPORTED, "l0_spec: FP32 16-row net");
    k.fn = (void *)(sixteen ? fns16[kind == kL0Split16 ? 1 : 0][prec] : fns[prec]);
    k.smem = sixteen ? (size_t)(max_n + 64) * 2 : (size_t)(max_n + 32) * 4;
    CSP_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem));
    k.grid = dim3(sixteen ? sms : 2 * sms);
    k.block = dim3(sixteen ? kBits16Threads : kBitsThreads);
    k.arg(nets).arg(nnets).arg(prec).arg(launches);
    return COSPDNN_OK;
}

void l0_convert_bits(const uint8_t *src, int format, int rows, int N, uint32_t *bits, float *err0, float *mx0,
                     int *nonbin, cudaStream_t s) {
    const int64_t warps = (rows + 31) / 32;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((warps + 7) / 8, 148 * 16));
    if (format == COSPDNN_INPUT_BITS) {
        // packed bits are binary by construction: the flag stays clear
        const int units = (rows + 31) / 32;
        k_convert_packed<<<(int)std::max(1, std::min(units, 148 * 8)), kConvThreads, 0, s>>>(src, rows, N, bits,
                                                                                            err0, mx0);
    } else {
        k_convert_bits<COSPDNN_INPUT_U8><<<blocks, 256, 0, s>>>(src, rows, N, bits, err0, mx0, nonbin);
    }
}

}  // namespace cospdnn
