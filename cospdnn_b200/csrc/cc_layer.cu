// CUDA-core row-tile layer kernel: FP32 / FP16 / BF16 activations, FP32
// accumulation, any sparsity pattern.
//
// Activations of these nets are stored in row tiles of TR rows, feature-major
// inside a tile (act_index layout TR), so one tile is a contiguous block of
// N*TR values and the TR values of one input feature are 16*G adjacent bytes
// (G = TR*elem/16 >= 1).  A CTA (one per SM, 16 warps) copies a whole tile
// into shared memory, then computes every output of it: a group of G lanes
// owns one output j, lane c of the group owns rows c*V..c*V+V-1 of the tile
// (V = 16 bytes of values: 8 for 16-bit types, 4 for FP32), and for each of
// the output's entries (input i, weight w) the lane reads the 16 bytes of
// input i for its rows (one 128-bit shared load) and does V FMAs.  FP16/BF16
// use the sm_100 mixed-precision FMA (f16/bf16 operands, f32 accumulator), so
// no conversion instructions are needed.
//
// Shared-memory banks: 128-bit loads are served a quarter warp (8 lanes) at a
// time; those lanes hold P = 8/G outputs (P = 1 when G >= 8) whose current
// entries sit in the 16*G-byte column of their input, i.e. in bank group
// (input mod P).  The host orders each aligned group of P outputs' entries so
// that at every step their inputs have distinct residues mod P (a proper edge
// colouring of the bipartite multigraph outputs x residues, König's theorem:
// max-degree many steps, padded with zero-weight entries that keep the
// residues distinct), so every quarter warp is one conflict-free wavefront.
//
// Entries come from global memory (16-byte groups, [group][j]: adjacent
// outputs adjacent, so a warp's load is contiguous), 16 entries per block,
// with the next block's loads issued before the current block is used.
// Epilogue per output: bias, clamp to [0,32], store in the compute type (one
// 16-byte store per lane), per-row statistics for the keep/prune decision.
// Small layers are split into output slices so that the grid stays busy.
#include <algorithm>
#include <cmath>

#include "cc_layer.cuh"

namespace cospdnn {
namespace {

constexpr int kCcThreads = 512;
constexpr int kCcWarps = kCcThreads / 32;
constexpr size_t kCcTileBudget = 200 * 1024;  // shared memory for one tile
constexpr int kCcMaxTR = 128;

template <typename T>
struct cc_traits;
template <>
struct cc_traits<float> {
    static constexpr int V = 4, EPV = 2;  // rows per lane, entries per 16-byte group
};
template <>
struct cc_traits<__half> {
    static constexpr int V = 8, EPV = 4;
};
template <>
struct cc_traits<__nv_bfloat16> {
    static constexpr int V = 8, EPV = 4;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint4 lds128(uint32_t addr) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(addr));
    return v;
}

// a0 += w * y.lo, a1 += w * y.hi with w = the high half of `ent`; one
// rounding each, identical to fmaf on the widened operands.
__device__ __forceinline__ void fma2(float &a0, float &a1, uint32_t ent, uint32_t y, __half) {
    asm("{\n\t.reg .b16 wl, wh, y0, y1;\n\t"
        "mov.b32 {wl, wh}, %2;\n\t"
        "mov.b32 {y0, y1}, %3;\n\t"
        "fma.rn.f32.f16 %0, wh, y0, %0;\n\t"
        "fma.rn.f32.f16 %1, wh, y1, %1;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "r"(ent), "r"(y));
}
__device__ __forceinline__ void fma2(float &a0, float &a1, uint32_t ent, uint32_t y, __nv_bfloat16) {
    asm("{\n\t.reg .b16 wl, wh, y0, y1;\n\t"
        "mov.b32 {wl, wh}, %2;\n\t"
        "mov.b32 {y0, y1}, %3;\n\t"
        "fma.rn.f32.bf16 %0, wh, y0, %0;\n\t"
        "fma.rn.f32.bf16 %1, wh, y1, %1;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "r"(ent), "r"(y));
}

// One block of 16 entries into the V accumulators.
template <typename T>
__device__ __forceinline__ void cc_block(float *acc, const uint4 *q, uint32_t sbase, int lgs) {
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint4 e = q[i];
            const uint4 y0 = lds128(sbase + (e.x << lgs));
            const uint4 y1 = lds128(sbase + (e.z << lgs));
            const float w0 = __uint_as_float(e.y), w1 = __uint_as_float(e.w);
            acc[0] = fmaf(w0, __uint_as_float(y0.x), acc[0]);
            acc[1] = fmaf(w0, __uint_as_float(y0.y), acc[1]);
            acc[2] = fmaf(w0, __uint_as_float(y0.z), acc[2]);
            acc[3] = fmaf(w0, __uint_as_float(y0.w), acc[3]);
            acc[0] = fmaf(w1, __uint_as_float(y1.x), acc[0]);
            acc[1] = fmaf(w1, __uint_as_float(y1.y), acc[1]);
            acc[2] = fmaf(w1, __uint_as_float(y1.z), acc[2]);
            acc[3] = fmaf(w1, __uint_as_float(y1.w), acc[3]);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t ent[4] = {q[i].x, q[i].y, q[i].z, q[i].w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const uint4 y = lds128(sbase + ((ent[e] & 0xFFFFu) << lgs));
                fma2(acc[0], acc[1], ent[e], y.x, T());
                fma2(acc[2], acc[3], ent[e], y.y, T());
                fma2(acc[4], acc[5], ent[e], y.z, T());
                fma2(acc[6], acc[7], ent[e], y.w, T());
            }
        }
    }
}

template <typename T>
__device__ __forceinline__ void cc_load(uint4 *q, const uint4 *__restrict__ W, int N, int j, int b) {
    constexpr int NQ = 16 / cc_traits<T>::EPV;
#pragma unroll
    for (int i = 0; i < NQ; ++i) q[i] = __ldg(W + (int64_t)(b * NQ + i) * N + j);
}

__device__ __forceinline__ bool cc_net(const NetDev &nd, int prec) {
    return nd.kernel == COSPDNN_KERNEL_CUDA_CORE && nd.layout >= 2 && nd.prec == prec && !nd.st->done;
}

// Output slices per tile: the split (1, 2, 4, ... up to one CTA round of
// outputs per slice) whose last wave of items wastes the least of the grid,
// charging each extra slice for re-reading the tile.
__device__ __forceinline__ int cc_slices(const NetDev &nd, int es, int grid) {
    const int TR = nd.layout;
    const int ntiles = (nd.st->R + TR - 1) / TR;
    const int step = kCcWarps * (32 / (TR * es / 16));
    const int rounds = (nd.N + step - 1) / step;
    int best = 1;
    double best_cost = 1e30;
    for (int s = 1; s <= rounds && s <= 64; s <<= 1) {
        const double items = (double)ntiles * s;
        const double waves = ceil(items / grid);
        const double cost = waves / s * (1.0 + 0.03 * (s - 1));  // in tile-times
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best = s;
        }
    }
    return best;
}

struct CcItem {
    int net, tile, slice, slices;
};

__device__ __forceinline__ bool cc_locate(const NetDev *nets, int nnets, int prec, int es, int grid, int64_t u,
                                          CcItem &it) {
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (!cc_net(nd, prec)) continue;
        const int S = cc_slices(nd, es, grid);
        const int64_t cnt = (int64_t)((nd.st->R + nd.layout - 1) / nd.layout) * S;
        if (u < cnt) {
            it.net = n;
            it.tile = (int)(u / S);
            it.slice = (int)(u % S);
            it.slices = S;
            return true;
        }
        u -= cnt;
    }
    return false;
}

template <typename T>
__global__ void __launch_bounds__(kCcThreads, 1)
    k_layer_cc(const NetDev *__restrict__ nets, int nnets, int prec, unsigned long long *launches) {
    count_launch(launches);
    using tr = cc_traits<T>;
    constexpr int ES = (int)sizeof(T), V = tr::V, NQ = 16 / tr::EPV;
    extern __shared__ uint4 cc_smem[];
    __shared__ uint32_t s_stat[kCcMaxTR * 3];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grid = (int)gridDim.x;
    int64_t total = 0;
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (!cc_net(nd, prec)) continue;
        total += (int64_t)((nd.st->R + nd.layout - 1) / nd.layout) * cc_slices(nd, ES, grid);
    }
    for (int64_t item = blockIdx.x; item < total; item += grid) {
        CcItem it;
        cc_locate(nets, nnets, prec, ES, grid, item, it);
        const NetDev &nd = nets[it.net];
        const int N = nd.N, TR = nd.layout, l = nd.st->layer, R = nd.st->R, par = l & 1, ib = nd.st->in_buf;
        const LayerDev &lw = nd.layers[l];
        const T *in = (const T *)(l == 0 ? nd.y0 : nd.act[ib]);
        T *out = (T *)nd.act[ib ^ 1];
        const int G = TR * ES / 16, lg = __ffs(G) - 1, lgs = __ffs(TR * ES) - 1;
        const int opw = 32 >> lg;  // outputs per warp and round
        const int c = lane & (G - 1), o = lane >> lg;

        // ---- stage the tile (and the statistics) in shared memory
        __syncthreads();  // the previous item is done with both
        {
            const uint4 *src = reinterpret_cast<const uint4 *>(in + (int64_t)it.tile * N * TR);
            const int nvec = N * G;
            int i = threadIdx.x;
            for (; i + 7 * kCcThreads < nvec; i += 8 * kCcThreads) {
                uint4 v[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = __ldg(src + i + k * kCcThreads);
#pragma unroll
                for (int k = 0; k < 8; ++k) cc_smem[i + k * kCcThreads] = v[k];
            }
            for (; i < nvec; i += kCcThreads) cc_smem[i] = __ldg(src + i);
            for (int r = threadIdx.x; r < TR * 3; r += kCcThreads) s_stat[r] = 0u;
        }
        if (threadIdx.x == 0 && item + grid < total) {
            // the next tile of this CTA into L2 while this one is computed
            CcItem nx;
            if (cc_locate(nets, nnets, prec, ES, grid, item + grid, nx) && (nx.net != it.net || nx.tile != it.tile)) {
                const NetDev &nn = nets[nx.net];
                const T *nin = (const T *)(nn.st->layer == 0 ? nn.y0 : nn.act[nn.st->in_buf]);
                const uint32_t bytes = (uint32_t)((size_t)nn.N * nn.layout * ES);
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(nin + (int64_t)nx.tile * nn.N * nn.layout),
                             "r"(bytes)
                             : "memory");
            }
        }
        __syncthreads();

        // ---- per-row error bounds of this lane's rows
        const double steps = fast_steps(nd, lw);
        const int row0 = it.tile * TR + c * V;
        float ez[V], zmax[V], emax[V], ymax[V];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int p = row0 + v;
            ez[v] = p < R ? z_error_bound(nd.err[par][p], nd.mx[par][p], lw.S, lw.dW, nd.bias, steps) : 0.0f;
            zmax[v] = -INFINITY;
            emax[v] = 0.0f;
            ymax[v] = 0.0f;
        }

        // ---- outputs of this slice
        const int step = kCcWarps * opw;
        const int rounds = (N + step - 1) / step;
        const int j_lo = (it.slice * rounds / it.slices) * step;
        const int j_hi = min(N, ((it.slice + 1) * rounds / it.slices) * step);
        const int nb = lw.cc_k / 16;
        const uint4 *__restrict__ W = lw.cc_w;
        const uint32_t sbase = smem_u32(cc_smem) + c * 16;
        const float bias = nd.bias;
        int j = j_lo + warp * opw + o, b = 0;
        bool have = j < j_hi;
        uint4 cur[NQ], nxt[NQ];
        if (have) cc_load<T>(cur, W, N, j, 0);
        float acc[V];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = 0.0f;
        while (have) {
            int jn = j, bn = b + 1;
            if (bn == nb) {
                bn = 0;
                jn += step;
            }
            const bool hn = jn < j_hi;
            if (hn) cc_load<T>(nxt, W, N, jn, bn);
            cc_block<T>(acc, cur, sbase, lgs);
            if (bn == 0) {
                __align__(16) T ov[V];
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const float z = acc[v] + bias;
                    const float cl = clamp32(z);
                    const T ys = act_traits<T>::from_f(cl);
                    const float yf = act_traits<T>::to_f(ys);
                    ov[v] = ys;
                    zmax[v] = fmaxf(zmax[v], z);
                    ymax[v] = fmaxf(ymax[v], yf);
                    if (z > -ez[v] && z < 32.0f + ez[v]) emax[v] = fmaxf(emax[v], __fadd_ru(ez[v], fabsf(yf - cl)));
                    acc[v] = 0.0f;
                }
                *reinterpret_cast<uint4 *>(out + ((int64_t)it.tile * N + j) * TR + c * V) =
                    *reinterpret_cast<const uint4 *>(ov);
            }
#pragma unroll
            for (int i = 0; i < NQ; ++i) cur[i] = nxt[i];
            j = jn;
            b = bn;
            have = hn;
        }

        // ---- row statistics: lanes of equal c, then warps, then global
#pragma unroll
        for (int v = 0; v < V; ++v) {
            for (int off = G; off < 32; off <<= 1) {
                zmax[v] = fmaxf(zmax[v], __shfl_xor_sync(0xffffffffu, zmax[v], off));
                emax[v] = fmaxf(emax[v], __shfl_xor_sync(0xffffffffu, emax[v], off));
                ymax[v] = fmaxf(ymax[v], __shfl_xor_sync(0xffffffffu, ymax[v], off));
            }
        }
        if (o == 0) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int r = c * V + v;
                atomicMax(&s_stat[3 * r], f2ord(zmax[v]));
                atomicMax(&s_stat[3 * r + 1], __float_as_uint(emax[v]));
                atomicMax(&s_stat[3 * r + 2], __float_as_uint(ymax[v]));
            }
        }
        __syncthreads();
        for (int r = threadIdx.x; r < TR; r += kCcThreads) {
            const int p = it.tile * TR + r;
            if (p < R) {
                atomicMax(&nd.stat[3 * p], s_stat[3 * r]);
                atomicMax(&nd.stat[3 * p + 1], s_stat[3 * r + 1]);
                atomicMax(&nd.stat[3 * p + 2], s_stat[3 * r + 2]);
            }
        }
    }
}

template <typename T>
uint32_t weight_bits(float w);
template <>
uint32_t weight_bits<__half>(float w) {
    const __half h = __float2half_rn(w);
    return (uint32_t)*reinterpret_cast<const uint16_t *>(&h);
}
template <>
uint32_t weight_bits<__nv_bfloat16>(float w) {
    const __nv_bfloat16 h = __float2bfloat16_rn(w);
    return (uint32_t)*reinterpret_cast<const uint16_t *>(&h);
}

// Edge colouring of one group's bipartite multigraph (P outputs x P
// residues): colour[e] in [0, D), D = max degree, no two edges of a colour
// share a vertex.  Alternating-path recolouring (König's constructive proof).
int colour_group(int P, const std::vector<int> &eu, const std::vector<int> &es, std::vector<int> &colour) {
    const int E = (int)eu.size();
    std::vector<int> du(P, 0), ds(P, 0);
    for (int e = 0; e < E; ++e) {
        ++du[eu[e]];
        ++ds[es[e]];
    }
    int D = 0;
    for (int v = 0; v < P; ++v) D = std::max(D, std::max(du[v], ds[v]));
    std::vector<int> atU((size_t)P * D, -1), atS((size_t)P * D, -1);
    colour.assign(E, -1);
    std::vector<int> path;
    for (int e = 0; e < E; ++e) {
        const int u = eu[e], s = es[e];
        int a = 0, b = 0;
        while (atU[(size_t)u * D + a] >= 0) ++a;
        while (atS[(size_t)s * D + b] >= 0) ++b;
        if (atS[(size_t)s * D + a] >= 0) {
            // a/b path from s, starting with the edge of colour a
            path.clear();
            int v = s, cc = a;
            bool onS = true;
            for (;;) {
                const int f = onS ? atS[(size_t)v * D + cc] : atU[(size_t)v * D + cc];
                if (f < 0) break;
                path.push_back(f);
                v = onS ? eu[f] : es[f];
                onS = !onS;
                cc = cc == a ? b : a;
            }
            for (int f : path) {
                atU[(size_t)eu[f] * D + colour[f]] = -1;
                atS[(size_t)es[f] * D + colour[f]] = -1;
            }
            for (int f : path) {
                colour[f] = colour[f] == a ? b : a;
                atU[(size_t)eu[f] * D + colour[f]] = f;
                atS[(size_t)es[f] * D + colour[f]] = f;
            }
        }
        colour[e] = a;
        atU[(size_t)u * D + a] = e;
        atS[(size_t)s * D + a] = e;
    }
    return D;
}

}  // namespace

int cc_tile_rows(int N, int prec) {
    const int es = prec == COSPDNN_PREC_FP32 ? 4 : 2;
    if (N > 65536) return 0;  // 16-bit input indices
    for (int TR = kCcMaxTR; TR >= 2; TR >>= 1)
        if (TR * es >= 16 && (size_t)N * TR * es <= kCcTileBudget) return TR;
    return 0;
}

int cc_build_entries(const std::vector<int32_t> &colptr, const std::vector<int32_t> &rowidx,
                     const std::vector<float> &vals, int N, int prec, int TR, LayerDev &ld,
                     std::vector<void *> &owned) {
    const int es = prec == COSPDNN_PREC_FP32 ? 4 : 2;
    const int G = TR * es / 16;
    const int P = G >= 8 ? 1 : 8 / G;  // outputs per quarter warp
    CSP_CHECK(G >= 1 && N % P == 0, COSPDNN_ERR_UNSUPPORTED, "cc_build_entries: bad tile");
    // per output: the entries (CSC positions, -1 = padding) in step order
    std::vector<std::vector<int>> order(N);
    std::vector<std::vector<int>> pad_idx(N);
    int Kmax = 1;
    std::vector<int> eu, esl, ep, colour;
    for (int g0 = 0; g0 < N; g0 += P) {
        eu.clear();
        esl.clear();
        ep.clear();
        for (int u = 0; u < P; ++u)
            for (int p = colptr[g0 + u]; p < colptr[g0 + u + 1]; ++p) {
                eu.push_back(u);
                esl.push_back(rowidx[p] % P);
                ep.push_back(p);
            }
        const int D = P == 1 ? (int)eu.size() : colour_group(P, eu, esl, colour);
        Kmax = std::max(Kmax, D);
        for (int u = 0; u < P; ++u) order[g0 + u].assign(D, -1);
        if (P == 1) {
            for (int e = 0; e < (int)ep.size(); ++e) order[g0][e] = ep[e];
        } else {
            for (int e = 0; e < (int)ep.size(); ++e) order[g0 + eu[e]][colour[e]] = ep[e];
        }
    }
    const int Kc = (Kmax + 15) / 16 * 16;
    // padding at step t of a group: a residue unused by the group at t
    const int epv = es == 4 ? 2 : 4;
    const size_t ngroups = (size_t)Kc / epv;
    std::vector<uint32_t> packed(ngroups * N * 4, 0u);
    for (int g0 = 0; g0 < N; g0 += P) {
        for (int t = 0; t < Kc; ++t) {
            uint32_t used = 0;
            for (int u = 0; u < P; ++u) {
                const auto &ord = order[g0 + u];
                if (t < (int)ord.size() && ord[t] >= 0) used |= 1u << (rowidx[ord[t]] % P);
            }
            for (int u = 0; u < P; ++u) {
                const int j = g0 + u;
                const auto &ord = order[j];
                int idx;
                float w;
                if (t < (int)ord.size() && ord[t] >= 0) {
                    idx = rowidx[ord[t]];
                    w = vals[ord[t]];
                } else {
                    int r = 0;
                    if (P > 1) {
                        while (used & (1u << r)) ++r;  // fewer than P residues are taken
                        used |= 1u << r;
                    }
                    idx = r;  // residue r (N >= P)
                    w = 0.0f;
                }
                const size_t grp = (size_t)(t / epv), slot = (size_t)(t % epv);
                uint32_t *dst = &packed[(grp * N + j) * 4];
                if (es == 4) {
                    dst[2 * slot] = (uint32_t)idx;
                    uint32_t wb;
                    std::memcpy(&wb, &w, 4);
                    dst[2 * slot + 1] = wb;
                } else {
                    const uint32_t wb = prec == COSPDNN_PREC_FP16 ? weight_bits<__half>(w)
                                                                  : weight_bits<__nv_bfloat16>(w);
                    dst[slot] = (uint32_t)idx | (wb << 16);
                }
            }
        }
    }
    void *d = nullptr;
    CSP_CUDA(cudaMalloc(&d, packed.size() * 4));
    owned.push_back(d);
    CSP_CUDA(cudaMemcpy(d, packed.data(), packed.size() * 4, cudaMemcpyHostToDevice));
    ld.cc_w = (const uint4 *)d;
    ld.cc_k = Kc;
    return COSPDNN_OK;
}

int cc_layer_spec(KSpec &k, NetDev *nets, int nnets, int prec, unsigned long long *launches, int sms,
                  size_t max_tile_bytes) {
    k.fn = prec == COSPDNN_PREC_FP32   ? (void *)k_layer_cc<float>
         : prec == COSPDNN_PREC_FP16 ? (void *)k_layer_cc<__half>
                                     : (void *)k_layer_cc<__nv_bfloat16>;
    CSP_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_tile_bytes));
    k.grid = dim3(sms);  // one CTA per SM (the tile fills shared memory)
    k.block = dim3(kCcThreads);
    k.smem = max_tile_bytes;
    k.arg(nets).arg(nnets).arg(prec).arg(launches);
    return COSPDNN_OK;
}

}  // namespace cospdnn
