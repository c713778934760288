// CUDA-core row-tile layer kernel: FP32 / FP16 / BF16 activations, FP32
// accumulation, any sparsity pattern.
//
// Activations of these nets are stored in row tiles of TR rows, feature-major
// inside a tile (act_index layout TR), so one tile is a contiguous block of
// N*TR values and the TR values of one input feature are 16*G adjacent bytes
// (G = TR*elem/16 >= 1).  A CTA (two of 8 warps per SM when the tile fits
// 96 KB, else one of 16 warps) copies a whole tile into shared memory, then
// computes every output of it: a group of G lanes
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
#include <type_traits>

#include "cc_layer.cuh"

namespace cospdnn {
namespace {

// Two CTAs of 256 threads per SM when the tile fits half of shared memory
// (one CTA stages its next tile while the other computes), else one CTA of
// 512 threads with a tile of up to 200 KB.
constexpr size_t kCcPairBudget = 96 * 1024;
constexpr size_t kCcTileBudget = 200 * 1024;
constexpr int kCcMaxTR = 128;
constexpr int kQB = 4;   // 16-byte entry groups per block
constexpr int kQBc = 2;  // the same for compact entry lists (16 entries per block, as 16-bit nets)

// Entry blocks held in registers (the load of block s+ring-1 overlaps block
// s): measured on one B200, two for 16-bit types (3% faster than three at
// 4096/FP16), three for FP32 (5% faster than two at 1024/FP32, whose blocks
// of 8 entries are consumed twice as fast).
template <typename T>
constexpr int cc_ring() {
    return sizeof(T) == 4 ? 3 : 2;
}

// Entries per 16-byte group of the entry list.
template <typename T>
constexpr int cc_epv() {
    return sizeof(T) == 4 ? 2 : 4;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint2 lds64(uint32_t addr) {
    uint2 v;
    asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(addr));
    return v;
}
__device__ __forceinline__ uint4 lds128(uint32_t addr) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(addr));
    return v;
}

// a0 += w * y.lo, a1 += w * y.hi with w = the low half of `ent`; one
// rounding each, identical to fmaf on the widened operands.
__device__ __forceinline__ void fma2(float &a0, float &a1, uint32_t ent, uint32_t y, __half) {
    asm("{\n\t.reg .b16 wl, wh, y0, y1;\n\t"
        "mov.b32 {wl, wh}, %2;\n\t"
        "mov.b32 {y0, y1}, %3;\n\t"
        "fma.rn.f32.f16 %0, wl, y0, %0;\n\t"
        "fma.rn.f32.f16 %1, wl, y1, %1;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "r"(ent), "r"(y));
}
__device__ __forceinline__ void fma2(float &a0, float &a1, uint32_t ent, uint32_t y, __nv_bfloat16) {
    asm("{\n\t.reg .b16 wl, wh, y0, y1;\n\t"
        "mov.b32 {wl, wh}, %2;\n\t"
        "mov.b32 {y0, y1}, %3;\n\t"
        "fma.rn.f32.bf16 %0, wl, y0, %0;\n\t"
        "fma.rn.f32.bf16 %1, wl, y1, %1;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "r"(ent), "r"(y));
}

// a0 += w * y0, a1 += w * y1 in one sm_100 packed instruction (fma.rn.f32x2:
// two IEEE FMAs, bit-identical to fmaf on each lane).
__device__ __forceinline__ void ffma2(float &a0, float &a1, float w, uint32_t y0, uint32_t y1) {
    asm("{\n\t.reg .b64 d, x, w;\n\t"
        "mov.b64 d, {%0, %1};\n\t"
        "mov.b64 x, {%2, %3};\n\t"
        "mov.b64 w, {%4, %4};\n\t"
        "fma.rn.f32x2 d, w, x, d;\n\t"
        "mov.b64 {%0, %1}, d;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "r"(y0), "r"(y1), "f"(w));
}

// V = LB / elem FMAs of one entry on one LB-byte shared load (V rows of one
// input).
template <typename T, int LB>
__device__ __forceinline__ void cc_entry(float *acc, uint32_t w, uint32_t addr) {
    if constexpr (LB == 8) {
        const uint2 y = lds64(addr);
        if constexpr (sizeof(T) == 4) {
            ffma2(acc[0], acc[1], __uint_as_float(w), y.x, y.y);
        } else {
            fma2(acc[0], acc[1], w, y.x, T());
            fma2(acc[2], acc[3], w, y.y, T());
        }
        return;
    }
    const uint4 y = lds128(addr);
    if constexpr (sizeof(T) == 4) {
        const float wf = __uint_as_float(w);
        ffma2(acc[0], acc[1], wf, y.x, y.y);
        ffma2(acc[2], acc[3], wf, y.z, y.w);
    } else {
        fma2(acc[0], acc[1], w, y.x, T());
        fma2(acc[2], acc[3], w, y.y, T());
        fma2(acc[4], acc[5], w, y.z, T());
        fma2(acc[6], acc[7], w, y.w, T());
    }
}

// One block of four 16-byte groups of entries into the V accumulators: 16
// entries of a 16-bit net ((column << 16) | weight bits, 4 per group) or 8 of
// an FP32 net ({column, weight bits}, 2 per group); column = the input's
// LB-byte column in the tile (input * G).
template <typename T, int LB, bool CMP>
__device__ __forceinline__ void cc_block(float *acc, const uint4 *q, uint32_t sbase, uint32_t wconst) {
    constexpr int SH = LB == 16 ? 4 : 3;
    if constexpr (CMP) {
        // compact entries: eight 16-bit columns per group, one weight value
#pragma unroll
        for (int i = 0; i < kQBc; ++i) {
            const uint32_t ent[4] = {q[i].x, q[i].y, q[i].z, q[i].w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                cc_entry<T, LB>(acc, wconst, sbase + ((ent[e] & 0xFFFFu) << SH));
                cc_entry<T, LB>(acc, wconst, sbase + ((ent[e] >> 16) << SH));
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < kQB; ++i) {
            if constexpr (sizeof(T) == 4) {
                cc_entry<T, LB>(acc, q[i].y, sbase + (q[i].x << SH));
                cc_entry<T, LB>(acc, q[i].w, sbase + (q[i].z << SH));
            } else {
                const uint32_t ent[4] = {q[i].x, q[i].y, q[i].z, q[i].w};
#pragma unroll
                for (int e = 0; e < 4; ++e) cc_entry<T, LB>(acc, ent[e], sbase + ((ent[e] >> 16) << SH));
            }
        }
    }
}

template <int QB>
__device__ __forceinline__ void cc_load(uint4 *q, const uint4 *__restrict__ W, int N, int j, int b) {
#pragma unroll
    for (int i = 0; i < QB; ++i) q[i] = __ldg(W + (int64_t)(b * QB + i) * N + j);
}

// Bytes of a feature column a lane owns: 16 when the tile's column has 16 or
// more, else 8.
__host__ __device__ __forceinline__ int cc_lane_bytes_of(int prec, int TR) {
    return TR * (prec == COSPDNN_PREC_FP32 ? 4 : 2) >= 16 ? 16 : 8;
}

__device__ __forceinline__ bool cc_net(const NetDev &nd, int prec, int lb, bool cmp) {
    return nd.kernel == COSPDNN_KERNEL_CUDA_CORE && nd.layout >= 2 && !nd.cc_split && nd.prec == prec && !nd.st->done &&
           cc_lane_bytes_of(nd.prec, nd.layout) == lb && (nd.cc_compact != 0) == cmp &&
           !(nd.st->layer == 0 && nd.st->l0_bits);
}

// Output slices per tile: the split (1, 2, 4, ... up to one CTA round of
// outputs per slice) whose last wave of items wastes the least of the grid,
// charging each extra slice for re-reading the tile.
__device__ __forceinline__ int cc_slices(const NetDev &nd, int grid, int warps) {
    const int TR = nd.layout, es = nd.prec == COSPDNN_PREC_FP32 ? 4 : 2;
    const int ntiles = (nd.st->R + TR - 1) / TR;
    const int step = warps * (32 / (TR * es / cc_lane_bytes_of(nd.prec, TR)));
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

__device__ __forceinline__ bool cc_locate(const NetDev *nets, int nnets, int prec, int lb, bool cmp, int grid, int warps,
                                          int64_t u, CcItem &it) {
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (!cc_net(nd, prec, lb, cmp)) continue;
        const int S = cc_slices(nd, grid, warps);
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

// Bias, clamp, store of V accumulators as one LB-byte piece; per row the max
// z and the min |z - 16|.
template <typename T, int LB>
__device__ __forceinline__ void cc_store(float *acc, float *zmax, float *zdist, float bias, T *dst) {
    constexpr int V = LB / (int)sizeof(T);
    __align__(16) T ov[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const float z = acc[v] + bias;
        zmax[v] = fmaxf(zmax[v], z);
        zdist[v] = fminf(zdist[v], fabsf(z - 16.0f));
        ov[v] = act_traits<T>::from_f(clamp32(z));
        acc[v] = 0.0f;
    }
    if constexpr (LB == 16) *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(ov);
    else *reinterpret_cast<uint2 *>(dst) = *reinterpret_cast<const uint2 *>(ov);
}

// Staging of a row tile whose rows come through the compaction map (the
// previous layer pruned rows and left the copy to this kernel): row r of the
// tile <- row s_map[r] of the whole buffer `src` (-1: zero).  Kept rows are
// increasing, so a tile's rows come from a few consecutive source tiles: for
// 8- and 16-byte feature columns each row's source column is loaded (the
// loads independent, repeats served by L1) and its value picked out; wider
// columns are built one 16-byte piece at a time from single values.
template <typename E, int NT>
__device__ __forceinline__ void cc_stage_gather(const E *__restrict__ src, int N, int TR, const int *s_map,
                                                uint4 *smem) {
    constexpr int kV = 16 / (int)sizeof(E);  // values of a 16-byte piece
    const int lg = __ffs(TR) - 1;            // TR is a power of two
    const int colb = TR * (int)sizeof(E);
    if (colb == 16 || colb == 8) {
        int pm[kV];
#pragma unroll
        for (int i = 0; i < kV; ++i) pm[i] = i < TR ? s_map[i] : -1;
        for (int f = threadIdx.x; f < N; f += NT) {
            // every row's source column loaded independently (repeats of a
            // column hit L1), then the values picked out
            uint4 col[kV];
#pragma unroll
            for (int i = 0; i < kV; ++i) {
                const int p = pm[i];
                col[i] = make_uint4(0u, 0u, 0u, 0u);
                if (p < 0) continue;
                const E *c = src + (((int64_t)(p >> lg) * N + f) << lg);
                if (colb == 16) {
                    col[i] = __ldg(reinterpret_cast<const uint4 *>(c));
                } else {
                    const uint2 h = __ldg(reinterpret_cast<const uint2 *>(c));
                    col[i] = make_uint4(h.x, h.y, 0u, 0u);
                }
            }
            __align__(16) E v[kV];
#pragma unroll
            for (int i = 0; i < kV; ++i) {
                const int p = pm[i];
                const int off = (p & (TR - 1)) * (int)sizeof(E);  // byte offset in the column
                const uint32_t w = off < 8 ? (off < 4 ? col[i].x : col[i].y) : (off < 12 ? col[i].z : col[i].w);
                if constexpr (sizeof(E) == 4) {
                    v[i] = p < 0 ? E(0) : __uint_as_float(w);
                } else {
                    v[i] = p < 0 ? E(0) : (E)(w >> (8 * (off & 3)));
                }
            }
            if (colb == 16) smem[f] = *reinterpret_cast<const uint4 *>(v);
            else reinterpret_cast<uint2 *>(smem)[f] = *reinterpret_cast<const uint2 *>(v);
        }
        return;
    }
    const int lp = lg - (__ffs(kV) - 1);  // log2 of 16-byte pieces per column
    const int total = N << lp;
    for (int u = threadIdx.x; u < total; u += NT) {
        const int f = u >> lp, pc = u & ((1 << lp) - 1);
        __align__(16) E v[kV];
#pragma unroll
        for (int i = 0; i < kV; ++i) {
            const int p = s_map[pc * kV + i];
            v[i] = p < 0 ? E(0) : src[(((int64_t)(p >> lg) * N + f) << lg) + (p & (TR - 1))];
        }
        smem[u] = *reinterpret_cast<const uint4 *>(v);
    }
}

template <typename T, int NT, int LB, bool CMP>
__global__ void __launch_bounds__(NT, 512 / NT)
    k_layer_cc(const NetDev *__restrict__ nets, int nnets, int prec, unsigned long long *launches) {
    count_launch(launches);
    constexpr int ES = (int)sizeof(T), V = LB / ES, kWarps = NT / 32;
    constexpr int QB = CMP ? kQBc : kQB;                 // 16-byte groups per block
    constexpr int EB = QB * (CMP ? 8 : cc_epv<T>());      // entries per block
    constexpr int kRing = cc_ring<T>();
    extern __shared__ uint4 cc_smem[];
    __shared__ uint32_t s_zmax[kCcMaxTR], s_zdist[kCcMaxTR];
    __shared__ int s_map[kCcMaxTR];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grid = (int)gridDim.x;
    int64_t total = 0;
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (!cc_net(nd, prec, LB, CMP)) continue;
        total += (int64_t)((nd.st->R + nd.layout - 1) / nd.layout) * cc_slices(nd, grid, kWarps);
    }
    for (int64_t item = blockIdx.x; item < total; item += grid) {
        CcItem it;
        cc_locate(nets, nnets, prec, LB, CMP, grid, kWarps, item, it);
        const NetDev &nd = nets[it.net];
        const int N = nd.N, TR = nd.layout, l = nd.st->layer, R = nd.st->R, par = l & 1, ib = nd.st->in_buf;
        const LayerDev &lw = nd.layers[l];
        const T *in = (const T *)(l == 0 ? nd.y0 : nd.act[ib]);
        T *out = (T *)nd.act[ib ^ 1];
        const int G = TR * ES / LB, lg = __ffs(G) - 1;  // lanes per output
        const int opw = 32 >> lg;                        // outputs per warp and round
        const int c = lane & (G - 1), o = lane >> lg;

        // ---- stage the tile in shared memory
        __syncthreads();  // the previous item is done with the tile and s_zmax
        if (nd.st->gather) {
            for (int r = threadIdx.x; r < TR; r += NT) {
                const int q = it.tile * TR + r;
                s_map[r] = q < R ? nd.cmap[q] : -1;
            }
            __syncthreads();
            if constexpr (ES == 4) cc_stage_gather<float, NT>((const float *)in, N, TR, s_map, cc_smem);
            else cc_stage_gather<uint16_t, NT>((const uint16_t *)in, N, TR, s_map, cc_smem);
        } else {
            const uint4 *src = reinterpret_cast<const uint4 *>(in + (int64_t)it.tile * N * TR);
            const int nvec = N * TR * ES / 16;
            int i = threadIdx.x;
            for (; i + 7 * NT < nvec; i += 8 * NT) {
                uint4 v[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = __ldg(src + i + k * NT);
#pragma unroll
                for (int k = 0; k < 8; ++k) cc_smem[i + k * NT] = v[k];
            }
            for (; i < nvec; i += NT) cc_smem[i] = __ldg(src + i);
        }
        {
            // the zero columns after the N inputs (read by padding entries)
            const int nvec = N * TR * ES / 16;
            for (int z = threadIdx.x; z < kCcZeroCols * TR * ES / 16; z += NT)
                cc_smem[nvec + z] = make_uint4(0u, 0u, 0u, 0u);
            for (int r = threadIdx.x; r < TR; r += NT) {
                s_zmax[r] = 0u;
                s_zdist[r] = 0x7F800000u;  // +inf
            }
        }
        if (threadIdx.x == 0 && item + grid < total) {
            // the next tile of this CTA into L2 while this one is computed
            CcItem nx;
            if (cc_locate(nets, nnets, prec, LB, CMP, grid, kWarps, item + grid, nx) &&
                (nx.net != it.net || nx.tile != it.tile) && !nets[nx.net].st->gather) {
                const NetDev &nn = nets[nx.net];
                const T *nin = (const T *)(nn.st->layer == 0 ? nn.y0 : nn.act[nn.st->in_buf]);
                const uint32_t bytes = (uint32_t)((size_t)nn.N * nn.layout * ES);
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(nin + (int64_t)nx.tile * nn.N * nn.layout),
                             "r"(bytes)
                             : "memory");
            }
        }
        __syncthreads();

        // ---- outputs of this slice: step s = (output jc, block bc), entries
        // of step s+kRing-1 loaded while step s is computed
        const int step = kWarps * opw;
        const int rounds = (N + step - 1) / step;
        const int j_lo = (it.slice * rounds / it.slices) * step;
        const int j_hi = min(N, ((it.slice + 1) * rounds / it.slices) * step);
        const int nb = lw.cc_k / EB;
        const uint4 *__restrict__ W = lw.cc_w;
        const uint32_t sbase = smem_u32(cc_smem) + c * LB;
        const float bias = nd.bias;
        const int j0 = j_lo + warp * opw + o;
        const int nout = j0 < j_hi ? (j_hi - j0 + step - 1) / step : 0;
        const int nsteps = nout * nb;
        float acc[V], zmax[V], zdist[V];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            acc[v] = 0.0f;
            zmax[v] = -INFINITY;
            zdist[v] = INFINITY;
        }
        int jl = j0, bl = 0, jc = j0, bc = 0;
        const uint32_t wconst = lw.cc_wconst;
        uint4 q[kRing][QB];
        auto next_load = [&](uint4 *q) {
            cc_load<QB>(q, W, N, jl, bl);
            if (++bl == nb) {
                bl = 0;
                jl += step;
            }
        };
        auto finish_step = [&]() {
            if (++bc == nb) {
                cc_store<T, LB>(acc, zmax, zdist, bias, out + ((int64_t)it.tile * N + jc) * TR + c * V);
                bc = 0;
                jc += step;
            }
        };
#pragma unroll
        for (int r = 0; r < kRing - 1; ++r)
            if (r < nsteps) next_load(q[r]);
        for (int s = 0; s < nsteps; s += kRing) {
#pragma unroll
            for (int r = 0; r < kRing; ++r) {  // buffer indices are compile-time
                if (s + r >= nsteps) break;
                if (s + r + kRing - 1 < nsteps) next_load(q[(r + kRing - 1) % kRing]);
                cc_block<T, LB, CMP>(acc, q[r], sbase, wconst);
                finish_step();
            }
        }

        // ---- row statistics: max z over lanes of equal c, then warps, then
        // the row's error bound, max output and output error
#pragma unroll
        for (int v = 0; v < V; ++v)
            for (int off = G; off < 32; off <<= 1) {
                zmax[v] = fmaxf(zmax[v], __shfl_xor_sync(0xffffffffu, zmax[v], off));
                zdist[v] = fminf(zdist[v], __shfl_xor_sync(0xffffffffu, zdist[v], off));
            }
        if (o == 0) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
                atomicMax(&s_zmax[c * V + v], f2ord(zmax[v]));
                atomicMin(&s_zdist[c * V + v], __float_as_uint(zdist[v]));  // >= 0: bit order = value order
            }
        }
        __syncthreads();
        const double steps = fast_steps(nd, lw);
        for (int r = threadIdx.x; r < TR; r += NT) {
            const int p = it.tile * TR + r;
            if (p < R) {
                const float ez = z_error_bound(nd.err[par][p], nd.mx[par][p], lw.S, lw.dW, bias, steps);
                float em, ym;
                row_stats<T>(ord2f(s_zmax[r]), __uint_as_float(s_zdist[r]), ez, em, ym);
                atomicMax(&nd.stat[3 * p], s_zmax[r]);
                atomicMax(&nd.stat[3 * p + 1], __float_as_uint(em));
                atomicMax(&nd.stat[3 * p + 2], __float_as_uint(ym));
            }
        }
    }
}

// A weight as the compute type holds it.
float to_compute_weight(float w, int prec) {
    if (prec == COSPDNN_PREC_FP16) return __half2float(__float2half_rn(w));
    if (prec == COSPDNN_PREC_BF16) return __bfloat162float(__float2bfloat16_rn(w));
    return w;
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

}  // namespace

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
    // edge of each (vertex, colour) and, per vertex, a bit mask of its used
    // colours (the lowest free colour is the lowest clear bit)
    const int W = (D + 63) / 64;
    std::vector<int> atU((size_t)P * D, -1), atS((size_t)P * D, -1);
    std::vector<uint64_t> mU((size_t)P * W, 0), mS((size_t)P * W, 0);
    auto put = [&](int f, int c) {
        atU[(size_t)eu[f] * D + c] = f;
        atS[(size_t)es[f] * D + c] = f;
        mU[(size_t)eu[f] * W + c / 64] |= 1ull << (c % 64);
        mS[(size_t)es[f] * W + c / 64] |= 1ull << (c % 64);
    };
    auto take = [&](int f, int c) {
        atU[(size_t)eu[f] * D + c] = -1;
        atS[(size_t)es[f] * D + c] = -1;
        mU[(size_t)eu[f] * W + c / 64] &= ~(1ull << (c % 64));
        mS[(size_t)es[f] * W + c / 64] &= ~(1ull << (c % 64));
    };
    // a vertex with an uncoloured edge has a free colour below D
    auto lowest_free = [&](const std::vector<uint64_t> &m, int v) {
        int w = 0;
        while (m[(size_t)v * W + w] == ~0ull) ++w;
        return w * 64 + __builtin_ctzll(~m[(size_t)v * W + w]);
    };
    colour.assign(E, -1);
    std::vector<int> path;
    for (int e = 0; e < E; ++e) {
        const int u = eu[e], s = es[e];
        const int a = lowest_free(mU, u), b = lowest_free(mS, s);
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
            for (int f : path) take(f, colour[f]);
            for (int f : path) {
                colour[f] = colour[f] == a ? b : a;
                put(f, colour[f]);
            }
        }
        colour[e] = a;
        put(e, a);
    }
    return D;
}


int cc_tile_rows(int N, int prec) {
    const int es = prec == COSPDNN_PREC_FP32 ? 4 : 2;
    if (N > 65536) return 0;  // 16-bit input indices
    // 16-byte lane columns (two CTAs per SM, then one), then 8-byte ones
    for (int lb : {16, 8})
        for (size_t budget : {kCcPairBudget, kCcTileBudget})
            for (int TR = kCcMaxTR; TR >= 1; TR >>= 1)
                if (TR * es >= lb && cc_tile_bytes(N, prec, TR) <= budget) return TR;
    return 0;
}

bool cc_single_weight(const std::vector<int32_t> &colptr, const std::vector<float> &vals, int N, int prec) {
    const int64_t nnz = colptr[N];
    if (nnz == 0) return false;
    const float w0 = to_compute_weight(vals[0], prec);
    if (w0 == 0.0f) return false;
    for (int64_t p = 1; p < nnz; ++p)
        if (to_compute_weight(vals[p], prec) != w0) return false;
    return true;
}

int cc_build_entries(const std::vector<int32_t> &colptr, const std::vector<int32_t> &rowidx,
                     const std::vector<float> &vals, int N, int prec, int TR, bool compact, LayerDev &ld,
                     std::vector<void *> &owned) {
    const int es = prec == COSPDNN_PREC_FP32 ? 4 : 2;
    // A lane owns an LB-byte piece of a feature column; shared loads are served
    // 128 bytes at a time, i.e. by 128/LB lanes (a quarter warp for 16-byte,
    // a half warp for 8-byte loads).
    const int LB = cc_lane_bytes_of(prec, TR);
    const int colw = TR * es / LB;                         // lanes per output
    const int phase = 128 / LB;                            // lanes per wavefront
    const int B = colw >= phase ? 1 : phase / colw;        // outputs per wavefront
    const int P = B;                                       // residues that must differ
    CSP_CHECK(colw >= 1 && N % B == 0, COSPDNN_ERR_UNSUPPORTED, "cc_build_entries: bad tile");
    CSP_CHECK((size_t)(N + kCcZeroCols) * colw <= 65536, COSPDNN_ERR_UNSUPPORTED, "cc_build_entries: tile too large");
    CSP_CHECK(P <= kCcZeroCols, COSPDNN_ERR_UNSUPPORTED, "cc_build_entries: too many residues");
    // groups of outputs whose entries must have distinct residues mod P at
    // every step: the B outputs of a wavefront
    std::vector<std::vector<int>> groups;
    for (int g0 = 0; g0 < N; g0 += B) {
        groups.emplace_back();
        for (int u = 0; u < B; ++u) groups.back().push_back(g0 + u);
    }
    // per output: the entries (CSC positions, -1 = padding) in step order
    std::vector<std::vector<int>> order(N);
    int Kmax = 1;
    std::vector<int> eu, esl, ep, colour;
    for (const auto &grp : groups) {
        eu.clear();
        esl.clear();
        ep.clear();
        for (int u = 0; u < (int)grp.size(); ++u)
            for (int p = colptr[grp[u]]; p < colptr[grp[u] + 1]; ++p) {
                eu.push_back(u);
                esl.push_back(rowidx[p] % P);
                ep.push_back(p);
            }
        const int D = P == 1 ? (int)ep.size() : colour_group(P, eu, esl, colour);
        for (int u = 0; u < (int)grp.size(); ++u) order[grp[u]].assign(D, -1);
        if (P == 1) {
            // no constraint: each output's entries in ascending input order
            for (int u = 0; u < (int)grp.size(); ++u) {
                const int j = grp[u], k = colptr[j + 1] - colptr[j];
                order[j].assign(k, -1);
                for (int t = 0; t < k; ++t) order[j][t] = colptr[j] + t;
                Kmax = std::max(Kmax, k);
            }
        } else {
            Kmax = std::max(Kmax, D);
            for (int e = 0; e < (int)ep.size(); ++e) order[grp[eu[e]]][colour[e]] = ep[e];
        }
    }
    const int Kc = (Kmax + 15) / 16 * 16;
    const int epv = compact ? 8 : (es == 4 ? 2 : 4);  // entries per 16-byte group
    const size_t ngroups = (size_t)Kc / epv;
    std::vector<uint32_t> packed(ngroups * N * 4, 0u);
    for (const auto &grp : groups) {
        for (int t = 0; t < Kc; ++t) {
            // padding at step t: a residue unused by the group at t
            uint32_t used = 0;
            for (int j : grp)
                if (t < (int)order[j].size() && order[j][t] >= 0) used |= 1u << (rowidx[order[j][t]] % P);
            for (int j : grp) {
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
                    // residue r: input r with weight 0 (N >= P), or for a
                    // compact list the zero column of residue r after the N inputs
                    idx = compact ? N + ((r - N % P) % P + P) % P : r;
                    w = 0.0f;
                }
                const size_t g = (size_t)(t / epv), slot = (size_t)(t % epv);
                uint32_t *dst = &packed[(g * N + j) * 4];
                const uint32_t col = (uint32_t)idx * colw;  // first LB-byte column of the input
                if (compact) {
                    // entry 2k in the low half of word k, entry 2k+1 in its high half
                    dst[slot / 2] |= col << (16 * (slot % 2));
                } else if (es == 4) {
                    dst[2 * slot] = col;
                    uint32_t wb;
                    std::memcpy(&wb, &w, 4);
                    dst[2 * slot + 1] = wb;
                } else {
                    const uint32_t wb = prec == COSPDNN_PREC_FP16 ? weight_bits<__half>(w)
                                                                  : weight_bits<__nv_bfloat16>(w);
                    dst[slot] = (col << 16) | wb;
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
    ld.cc_wconst = 0u;
    if (compact) {
        const float w = to_compute_weight(vals[0], prec);
        if (es == 4) std::memcpy(&ld.cc_wconst, &w, 4);
        else ld.cc_wconst = prec == COSPDNN_PREC_FP16 ? weight_bits<__half>(w) : weight_bits<__nv_bfloat16>(w);
    }
    return COSPDNN_OK;
}

int cc_layer_spec(KSpec &k, NetDev *nets, int nnets, int prec, int lane_bytes, bool compact,
                  unsigned long long *launches, int sms, size_t max_tile_bytes) {
    using F = void (*)(const NetDev *, int, int, unsigned long long *);
#define CSP_CC(T, NT)                                                                     \
    {{k_layer_cc<T, NT, 16, false>, k_layer_cc<T, NT, 16, true>},                         \
     {k_layer_cc<T, NT, 8, false>, k_layer_cc<T, NT, 8, true>}}
    // [precision][one CTA of 512 / two of 256 per SM][lane bytes 16 / 8][compact entries]
    static const F fns[3][2][2][2] = {{CSP_CC(float, 512), CSP_CC(float, 256)},
                                      {CSP_CC(__half, 512), CSP_CC(__half, 256)},
                                      {CSP_CC(__nv_bfloat16, 512), CSP_CC(__nv_bfloat16, 256)}};
#undef CSP_CC
    const bool pair = max_tile_bytes <= kCcPairBudget;
    k.fn = (void *)fns[prec][pair ? 1 : 0][lane_bytes == 16 ? 0 : 1][compact ? 1 : 0];
    CSP_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_tile_bytes));
    k.grid = dim3(pair ? 2 * sms : sms);
    k.block = dim3(pair ? 256 : 512);
    k.smem = max_tile_bytes;
    k.arg(nets).arg(nnets).arg(prec).arg(launches);
    return COSPDNN_OK;
}

}  // namespace cospdnn
