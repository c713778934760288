// CUDA-core feature-split tile kernel: 16-bit activations (FP16 / BF16) of
// nets too wide for a row tile of the one-CTA kernel (65536 features: even
// 4 rows x 2 bytes x 65536 is 512 KB), FP32 accumulation, any sparsity.
//
// Activations are stored in row tiles of 2 rows (act_index layout 2): the two
// rows of a feature are one 4-byte word.  A tile is computed by a cluster of
// two CTAs (one per SM): the features are split in two halves by one bit of
// the feature index, chosen per layer (CTA h stages the words of the features
// whose bit is h, N/2 words, 128 KB at 65536), and each CTA forms, for every
// output of the tile, the partial sum over the output's entries in its half.
// The two partial sums of an output meet in the CTA that owns it: the other
// CTA sends its partial through distributed shared memory (st.async into the
// owner's receive buffer, completing on the owner's mbarrier), the owner adds
// them, adds the bias, clamps, stores the 2-row word and folds the output
// into its row statistics.  The sum is order-free (a + b == b + a in IEEE
// arithmetic) and the bound on its rounding error covers the split.
//
// Work per round (512 threads, 16 warps): warp w takes four groups of 32
// outputs, one from each quarter of the outputs (slot s: group s*Q + 16k + w
// in round k, Q = groups per quarter); lane l owns output l of each group and
// gathers, per 16-byte entry group, four (compact lists) or two entries: one
// 4-byte shared load (the input's two rows, at the byte offset the entry
// holds) and two FMAs per entry.  Slots 0
// and 2 are owned by CTA 0, 1 and 3 by CTA 1: every round each thread sends
// one 16-byte message (its two non-owned partial pairs) to the thread of the
// same index in the other CTA and receives one.  Receive buffers are double
// buffered: a thread sends round k, then finishes round k - 1 (waits for the
// peer's message, whose mbarrier phase completes with its bytes), so the
// peer's round k is computed meanwhile.  Each receiver warp hands its buffer
// slot back to the sender with one remote mbarrier arrive.
//
// Shared-memory banks: a warp's 32 loads of one step are one wavefront when
// their words lie in 32 distinct banks; the host orders each group's entries
// per half by an edge colouring of outputs x banks (local word index mod 32)
// and pads with zero words placed after the N/2 inputs, one per bank.
//
// Every wait is bounded (DevLimits::wait_cycles); on timeout the CTA stops
// sending, raises the engine's abort flag (the layer loop then stops with
// COSPDNN_ERR_DEVICE) and both CTAs meet at the cluster barrier before
// exiting, so no CTA exits while its peer may still write into its shared
// memory.  Neither CTA waits for the other anywhere else.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "cc_layer.cuh"
#include "cs_layer.cuh"

namespace cospdnn {
namespace {

constexpr int kCsThreads = 512;
constexpr int kCsWarps = kCsThreads / 32;
constexpr int kCsSlots = 4;     // groups of 32 outputs per warp and round
constexpr int kCsDepth = 2;     // receive buffers
constexpr int kCsCols = 2;      // entry columns (one 16-byte group per slot) held per lane: one loaded ahead
constexpr int kCsZero = 32;     // zero words after the N/2 inputs (one per bank)
constexpr int kCsMsgBytes = 16; // one message: two partial pairs

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_id() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_count() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}
// The shared::cluster address of the same variable in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t peer_addr(uint32_t local, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
    return r;
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
// Completion of a phase by this CTA's own arrive plus the bytes of remote
// st.async writes; the arrive also raises the phase's expected bytes.
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Arrive on an mbarrier of the peer CTA (release: this thread's earlier
// shared-memory reads are done before the peer sees the arrive).
__device__ __forceinline__ void mbar_arrive_remote(uint32_t peer_bar) {
    asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(peer_bar) : "memory");
}
// A phase completed by the peer's st.async bytes makes those bytes visible
// to the waiting thread; a phase completed by the peer's arrives orders the
// peer's reads of this CTA's messages before it (the buffer may be reused).
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// 16 bytes into the peer's shared memory, counted on the peer's mbarrier.
__device__ __forceinline__ void st_async16(uint32_t peer_dst, uint4 v, uint32_t peer_bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(
                     peer_dst),
                 "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(peer_bar)
                 : "memory");
}
__device__ __forceinline__ uint32_t lds32(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}

// a0 += w * y.lo, a1 += w * y.hi: the input's two rows (row 0 in the low
// half of its word) times w = the low half of `ent`; one rounding each,
// identical to fmaf on the widened operands.
__device__ __forceinline__ void fma_pair(float &a0, float &a1, uint32_t ent, uint32_t y, __half) {
    asm("{\n\t.reg .b16 wl, wh, y0, y1;\n\t"
        "mov.b32 {wl, wh}, %2;\n\t"
        "mov.b32 {y0, y1}, %3;\n\t"
        "fma.rn.f32.f16 %0, wl, y0, %0;\n\t"
        "fma.rn.f32.f16 %1, wl, y1, %1;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "r"(ent), "r"(y));
}
__device__ __forceinline__ void fma_pair(float &a0, float &a1, uint32_t ent, uint32_t y, __nv_bfloat16) {
    asm("{\n\t.reg .b16 wl, wh, y0, y1;\n\t"
        "mov.b32 {wl, wh}, %2;\n\t"
        "mov.b32 {y0, y1}, %3;\n\t"
        "fma.rn.f32.bf16 %0, wl, y0, %0;\n\t"
        "fma.rn.f32.bf16 %1, wl, y1, %1;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "r"(ent), "r"(y));
}

// One 16-byte entry group of one output into its two accumulators: four
// compact entries (byte offsets of the inputs' words in the tile; the weight
// is the layer's one value) or two {offset, weight bits} entries.
template <typename T, bool CMP>
__device__ __forceinline__ void cs_group(float &a0, float &a1, uint4 q, uint32_t sbase, uint32_t wconst) {
    if constexpr (CMP) {
        fma_pair(a0, a1, wconst, lds32(sbase + q.x), T());
        fma_pair(a0, a1, wconst, lds32(sbase + q.y), T());
        fma_pair(a0, a1, wconst, lds32(sbase + q.z), T());
        fma_pair(a0, a1, wconst, lds32(sbase + q.w), T());
    } else {
        fma_pair(a0, a1, q.y, lds32(sbase + q.x), T());
        fma_pair(a0, a1, q.w, lds32(sbase + q.z), T());
    }
}

// Bounded wait on a phase of one of this CTA's mbarriers.  False when this
// CTA has aborted: the limit ran out here or in another thread of the CTA.
__device__ __forceinline__ bool cs_wait(uint32_t bar, uint32_t parity, const volatile long long *limit,
                                        volatile int *abort) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    for (;;) {
        if (*abort) return false;
        if (mbar_try_wait(bar, parity)) return true;
        if (clock64() - t0 > *limit) {
            *abort = 1;
            return false;
        }
    }
}

__device__ __forceinline__ bool cs_net(const NetDev &nd, int prec, bool cmp) {
    return nd.cc_split && nd.kernel == COSPDNN_KERNEL_CUDA_CORE && nd.prec == prec && !nd.st->done &&
           (nd.cc_compact != 0) == cmp && !(nd.st->layer == 0 && nd.st->l0_bits);
}

// Groups of 32 outputs of a split layer, padded to a multiple of 64 (four
// slots x 16 warps per round).
__host__ __device__ __forceinline__ int cs_groups(int N) { return (N / 32 + 63) / 64 * 64; }

template <typename T, bool CMP>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kCsThreads, 1)
    k_layer_cs(const NetDev *__restrict__ nets, int nnets, int prec, unsigned long long *launches, int *abort_flag,
               const DevLimits *__restrict__ limits, uint32_t recv_off) {
    count_launch(launches);
    extern __shared__ uint4 cs_smem[];
    __shared__ __align__(8) unsigned long long s_full[kCsDepth], s_empty[kCsDepth];
    __shared__ uint32_t s_zmax[2], s_zdist[2];
    __shared__ int s_abort;
    __shared__ long long s_limit;
    __shared__ int s_withhold;  // test hook: CTA 0 of cluster 0 does not send its first message
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = cluster_rank(), peer = rank ^ 1u;
    if (tid == 0) {
        for (int d = 0; d < kCsDepth; ++d) {
            mbar_init(smem_addr(&s_full[d]), 1);
            mbar_init(smem_addr(&s_empty[d]), kCsWarps);
        }
        s_abort = 0;
        s_limit = limits->wait_cycles;
        s_withhold = limits->withhold_stage && rank == 0 && cluster_id() == 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        // the first phase of each receive buffer: this CTA's arrive plus the
        // peer's messages
        for (int d = 0; d < kCsDepth; ++d) mbar_expect_tx(smem_addr(&s_full[d]), kCsThreads * kCsMsgBytes);
    }
    cluster_sync_all();  // both CTAs' barriers are initialised before any remote access
    const uint32_t tile_base = smem_addr(cs_smem);
    const uint32_t recv_base = tile_base + recv_off;  // [kCsDepth][kCsThreads] messages
    const uint32_t peer_recv = peer_addr(recv_base, peer);
    volatile int *abort_p = &s_abort;
    bool ok = true;
    uint32_t rc = 0;  // rounds of this CTA so far (the two CTAs of a cluster count alike)

    int64_t total = 0;
    for (int n = 0; n < nnets; ++n)
        if (cs_net(nets[n], prec, CMP)) total += (nets[n].st->R + 1) / 2;
    for (int64_t item = cluster_id(); item < total; item += cluster_count()) {
        int n = 0;
        int64_t u = item;
        for (; n < nnets; ++n) {
            if (!cs_net(nets[n], prec, CMP)) continue;
            const int64_t cnt = (nets[n].st->R + 1) / 2;
            if (u < cnt) break;
            u -= cnt;
        }
        const NetDev &nd = nets[n];
        const int tile = (int)u;
        const int N = nd.N, l = nd.st->layer, R = nd.st->R, par = l & 1, ib = nd.st->in_buf;
        const LayerDev &lw = nd.layers[l];
        const uint32_t *in = (const uint32_t *)(l == 0 ? nd.y0 : nd.act[ib]) + (int64_t)tile * N;  // 2-row words
        uint32_t *out = (uint32_t *)nd.act[ib ^ 1] + (int64_t)tile * N;
        const int half = N >> 1, b = lw.cs_bit, cnt = lw.cs_cnt;
        const int NGp = cs_groups(N), Q = NGp / kCsSlots, rounds = Q / kCsWarps, C = rounds * cnt;

        // ---- stage this CTA's half of the tile: local word i <- feature
        // f(i) = i with bit b inserted as `rank` (b >= 4: runs of 16 words)
        __syncthreads();  // the previous item is done with the tile and the row statistics
        {
            const int nv = half / 4, lowm = (1 << b) - 1;
            int i = tid;
            for (; i + 7 * kCsThreads < nv; i += 8 * kCsThreads) {
                uint4 v[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int w4 = 4 * (i + k * kCsThreads);
                    const int f = ((w4 >> b) << (b + 1)) | ((int)rank << b) | (w4 & lowm);
                    v[k] = __ldg(reinterpret_cast<const uint4 *>(in + f));
                }
#pragma unroll
                for (int k = 0; k < 8; ++k) cs_smem[i + k * kCsThreads] = v[k];
            }
            for (; i < nv; i += kCsThreads) {
                const int w4 = 4 * i;
                const int f = ((w4 >> b) << (b + 1)) | ((int)rank << b) | (w4 & lowm);
                cs_smem[i] = __ldg(reinterpret_cast<const uint4 *>(in + f));
            }
            if (tid < kCsZero) reinterpret_cast<uint32_t *>(cs_smem)[half + tid] = 0u;
            if (tid < 2) {
                s_zmax[tid] = 0u;
                s_zdist[tid] = 0x7F800000u;  // +inf
            }
        }
        if (tid == 0 && rank == 0 && item + cluster_count() < total) {
            // the next tile of this cluster into L2 while this one is computed
            int64_t v = item + cluster_count();
            int m = 0;
            for (; m < nnets; ++m) {
                if (!cs_net(nets[m], prec, CMP)) continue;
                const int64_t c2 = (nets[m].st->R + 1) / 2;
                if (v < c2) break;
                v -= c2;
            }
            if (m < nnets) {
                const NetDev &nn = nets[m];
                const uint32_t *nin = (const uint32_t *)(nn.st->layer == 0 ? nn.y0 : nn.act[nn.st->in_buf]);
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(nin + v * nn.N),
                             "r"((uint32_t)nn.N * 4u)
                             : "memory");
            }
        }
        __syncthreads();

        // ---- rounds of four groups per warp (slot s: group s*Q + 16k + warp in
        // round k); the entry groups of column t of round k, slot s, are at
        // E[(((16k + warp)*cnt + t)*4 + s)*32]
        const uint4 *__restrict__ E = lw.cs_w + (int64_t)rank * rounds * kCsWarps * cnt * (kCsSlots * 32) + lane;
        const uint32_t wconst = lw.cc_wconst;
        const float bias = nd.bias;
        float zmax[2] = {-INFINITY, -INFINITY}, zdist[2] = {INFINITY, INFINITY};
        float acc[kCsSlots][2];
#pragma unroll
        for (int s = 0; s < kCsSlots; ++s) acc[s][0] = acc[s][1] = 0.0f;
        float own[4] = {0.0f, 0.0f, 0.0f, 0.0f};  // owned partials of the round awaiting the peer's message
        int own_k = -1;                            // that round (-1: none)
        uint32_t own_rc = 0;
        // this CTA's slot s' is slot s' ^ rank: its own slots are always 0 and
        // 2, the ones it sends 1 and 3
        const int sw = rank ? 32 : 0;
        auto load_col = [&](uint4 *q, int k, int t) {
            const uint4 *p = E + (int64_t)((kCsWarps * k + warp) * cnt + t) * (kCsSlots * 32);
            q[0] = __ldg(p + sw);
            q[1] = __ldg(p + 32 - sw);
            q[2] = __ldg(p + 64 + sw);
            q[3] = __ldg(p + 96 - sw);
        };
        // the owner's half of a round: wait for the peer's message, add, bias,
        // clamp, store, row statistics; then hand the buffer back
        auto finish = [&]() {
            const uint32_t d = own_rc & 1u;
            uint4 m = make_uint4(0u, 0u, 0u, 0u);
            if (ok) ok = cs_wait(smem_addr(&s_full[d]), (own_rc >> 1) & 1u, &s_limit, abort_p);
            if (ok) {
                asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                             : "=r"(m.x), "=r"(m.y), "=r"(m.z), "=r"(m.w)
                             : "r"(recv_base + (d * kCsThreads + tid) * kCsMsgBytes));
                // the next phase of this buffer (its round + 2): this CTA's arrive
                if (tid == 0) mbar_expect_tx(smem_addr(&s_full[d]), kCsThreads * kCsMsgBytes);
            }
            const float pm[4] = {__uint_as_float(m.x), __uint_as_float(m.y), __uint_as_float(m.z),
                                 __uint_as_float(m.w)};
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int j = 32 * (((int)rank + 2 * i) * Q + kCsWarps * own_k + warp) + lane;
                const float z0 = (own[2 * i] + pm[2 * i]) + bias;
                const float z1 = (own[2 * i + 1] + pm[2 * i + 1]) + bias;
                if (j < N) {
                    zmax[0] = fmaxf(zmax[0], z0);
                    zmax[1] = fmaxf(zmax[1], z1);
                    zdist[0] = fminf(zdist[0], fabsf(z0 - 16.0f));
                    zdist[1] = fminf(zdist[1], fabsf(z1 - 16.0f));
                    const T o0 = act_traits<T>::from_f(clamp32(z0)), o1 = act_traits<T>::from_f(clamp32(z1));
                    out[j] = (uint32_t)*reinterpret_cast<const uint16_t *>(&o0) |
                             ((uint32_t)*reinterpret_cast<const uint16_t *>(&o1) << 16);
                }
            }
            __syncwarp();  // every lane of the warp has read its message
            if (ok && lane == 0) mbar_arrive_remote(peer_addr(smem_addr(&s_empty[d]), peer));
        };
        // end of round k: send the peer's two partial pairs, finish the
        // previous round, keep this round's owned pairs
        auto round_end = [&](int k) {
            const uint32_t d = rc & 1u;
            const uint4 msg = make_uint4(__float_as_uint(acc[1][0]), __float_as_uint(acc[1][1]),
                                         __float_as_uint(acc[3][0]), __float_as_uint(acc[3][1]));
            if (ok && rc >= (uint32_t)kCsDepth)  // the peer has read this buffer's previous message
                ok = cs_wait(smem_addr(&s_empty[d]), ((rc >> 1) - 1u) & 1u, &s_limit, abort_p);
            if (ok && !(rc == 0 && s_withhold))
                st_async16(peer_recv + (d * kCsThreads + tid) * kCsMsgBytes, msg,
                           peer_addr(smem_addr(&s_full[d]), peer));
            if (own_k >= 0) finish();
            own[0] = acc[0][0];
            own[1] = acc[0][1];
            own[2] = acc[2][0];
            own[3] = acc[2][1];
            own_k = k;
            own_rc = rc++;
#pragma unroll
            for (int s = 0; s < kCsSlots; ++s) acc[s][0] = acc[s][1] = 0.0f;
        };
        uint4 q[kCsCols][kCsSlots];
        int kl = 0, tl = 0;  // next column to load
        int kc = 0, tc = 0;  // column being computed
#pragma unroll
        for (int r = 0; r < kCsCols - 1; ++r)
            if (kl < rounds) {
                load_col(q[r], kl, tl);
                if (++tl == cnt) { tl = 0; ++kl; }
            }
        for (int c = 0; c < C; c += kCsCols) {
#pragma unroll
            for (int r = 0; r < kCsCols; ++r) {  // ring indices are compile-time
                if (c + r >= C) break;
                if (kl < rounds) {
                    load_col(q[(r + kCsCols - 1) % kCsCols], kl, tl);
                    if (++tl == cnt) { tl = 0; ++kl; }
                }
#pragma unroll
                for (int s = 0; s < kCsSlots; ++s) cs_group<T, CMP>(acc[s][0], acc[s][1], q[r][s], tile_base, wconst);
                if (tc == cnt - 1) round_end(kc);
                if (++tc == cnt) { tc = 0; ++kc; }
            }
        }
        if (own_k >= 0) finish();

        // ---- row statistics of this CTA's outputs (the peer adds its own)
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            const uint32_t m = __reduce_max_sync(0xffffffffu, f2ord(zmax[v]));
            const uint32_t dd = __reduce_min_sync(0xffffffffu, __float_as_uint(zdist[v]));  // >= 0
            if (lane == 0) {
                atomicMax(&s_zmax[v], m);
                atomicMin(&s_zdist[v], dd);
            }
        }
        __syncthreads();
        if (tid < 2) {
            const int p = tile * 2 + tid;
            if (p < R) {
                const float ez = z_error_bound(nd.err[par][p], nd.mx[par][p], lw.S, lw.dW, bias, fast_steps(nd, lw));
                float em, ym;
                row_stats<T>(ord2f(s_zmax[tid]), __uint_as_float(s_zdist[tid]), ez, em, ym);
                atomicMax(&nd.stat[3 * p], s_zmax[tid]);
                atomicMax(&nd.stat[3 * p + 1], __float_as_uint(em));
                atomicMax(&nd.stat[3 * p + 2], __float_as_uint(ym));
            }
        }
    }
    __syncthreads();
    if (tid == 0 && s_abort) atomicExch(abort_flag, 1);
    // no CTA leaves while its peer may still access its shared memory
    cluster_sync_all();
}

}  // namespace

namespace {

constexpr size_t kCsRecvBytes = (size_t)kCsDepth * kCsThreads * kCsMsgBytes;
constexpr size_t kCsSmemLimit = 227 * 1024 - 1024;  // dynamic shared memory of one CTA (static part below 1 KB)

size_t cs_recv_off(int N) { return ((size_t)(N / 2 + kCsZero) * 4 + 15) / 16 * 16; }

// Local word index of feature f in its half (bit b removed).
inline int cs_local(int f, int b) { return ((f >> (b + 1)) << b) | (f & ((1 << b) - 1)); }

// A weight's bits in the 16-bit compute type.
uint32_t bits16_of(float w, int prec) {
    uint16_t u;
    if (prec == COSPDNN_PREC_FP16) {
        const __half h = __float2half_rn(w);
        std::memcpy(&u, &h, 2);
    } else {
        const __nv_bfloat16 h = __float2bfloat16_rn(w);
        std::memcpy(&u, &h, 2);
    }
    return u;
}

}  // namespace

bool cs_supported(int N, int prec) {
    if (prec == COSPDNN_PREC_FP32 || N % 64 != 0 || cc_tile_rows(N, prec) != 0) return false;
    if (N / 2 + kCsZero > 65535) return false;  // 16-bit local word indices
    return cs_recv_off(N) + kCsRecvBytes <= kCsSmemLimit;
}

int cs_build_entries(const std::vector<int32_t> &colptr, const std::vector<int32_t> &rowidx,
                     const std::vector<float> &vals, int N, int prec, bool compact, LayerDev &ld,
                     std::vector<void *> &owned) {
    CSP_CHECK(cs_supported(N, prec), COSPDNN_ERR_UNSUPPORTED, "cs_build_entries: width not supported");
    const int half = N / 2, NG = N / 32, NGp = cs_groups(N), epl = compact ? 4 : 2;
    int kmax = 0;
    for (int j = 0; j < N; ++j) kmax = std::max(kmax, colptr[j + 1] - colptr[j]);
    // split bit: the one (highest first: longer staging runs) whose largest
    // degree of a group's bipartite graph in either half (outputs or banks),
    // in 16-byte entry groups, is least; an output of K entries has at least K/2 in one
    // half, so the search stops at that bound
    const int lower = std::max(1, ((kmax + 1) / 2 + epl - 1) / epl);
    int best_b = -1, best_cnt = 1 << 30;
    std::vector<int> deg(4 * 32);
    for (int b = 30; b >= 4 && best_cnt > lower; --b) {
        if ((1LL << (b + 1)) > (long long)N || N % (1 << (b + 1)) != 0) continue;
        int cnt = 1;
        for (int g = 0; g < NG && cnt < best_cnt; ++g) {
            std::fill(deg.begin(), deg.end(), 0);  // [half][output], then [half][bank]
            for (int u = 0; u < 32; ++u)
                for (int p = colptr[32 * g + u]; p < colptr[32 * g + u + 1]; ++p) {
                    const int f = rowidx[p], h = (f >> b) & 1;
                    ++deg[h * 32 + u];
                    ++deg[64 + h * 32 + (cs_local(f, b) & 31)];
                }
            const int D = *std::max_element(deg.begin(), deg.end());
            cnt = std::max(cnt, (D + epl - 1) / epl);
        }
        if (cnt < best_cnt) {
            best_cnt = cnt;
            best_b = b;
        }
    }
    CSP_CHECK(best_b >= 4, COSPDNN_ERR_UNSUPPORTED, "cs_build_entries: no split bit");
    const int b = best_b, cnt = best_cnt, steps = cnt * epl;
    // per half and group: a conflict-free step for every entry (edge colouring
    // of outputs x banks), padding on the zero word of a bank free at its step
    const int Q = NGp / kCsSlots, rounds = Q / kCsWarps;
    std::vector<uint32_t> words((size_t)2 * NGp * cnt * 32 * 4, 0u);
    std::vector<int> eu, es, ep, colour, slot((size_t)32 * steps);
    for (int h = 0; h < 2; ++h)
        for (int g = 0; g < NGp; ++g) {
            std::fill(slot.begin(), slot.end(), -1);
            if (g < NG) {
                eu.clear();
                es.clear();
                ep.clear();
                for (int u = 0; u < 32; ++u)
                    for (int p = colptr[32 * g + u]; p < colptr[32 * g + u + 1]; ++p) {
                        const int f = rowidx[p];
                        if (((f >> b) & 1) != h) continue;
                        eu.push_back(u);
                        es.push_back(cs_local(f, b) & 31);
                        ep.push_back(p);
                    }
                if (!ep.empty()) {
                    const int D = colour_group(32, eu, es, colour);
                    CSP_CHECK(D <= steps, COSPDNN_ERR_UNSUPPORTED, "cs_build_entries: colouring exceeds the word count");
                    for (size_t e = 0; e < ep.size(); ++e) slot[(size_t)eu[e] * steps + colour[e]] = ep[e];
                }
            }
            for (int t = 0; t < steps; ++t) {
                uint32_t used = 0;
                for (int u = 0; u < 32; ++u) {
                    const int p = slot[(size_t)u * steps + t];
                    if (p >= 0) used |= 1u << (cs_local(rowidx[p], b) & 31);
                }
                for (int u = 0; u < 32; ++u) {
                    const int p = slot[(size_t)u * steps + t];
                    uint32_t idx, wb = 0;
                    if (p >= 0) {
                        idx = (uint32_t)cs_local(rowidx[p], b);
                        wb = bits16_of(vals[p], prec);
                    } else {
                        int r = 0;
                        while (used & (1u << r)) ++r;  // fewer than 32 banks are taken
                        used |= 1u << r;
                        idx = (uint32_t)(half + r);  // half % 32 == 0: the zero word of bank r
                    }
                    // group g = s*Q + 16k + w; column t / epl, entry t % epl of its 16 bytes
                    const int sl = g / Q, k = (g % Q) / kCsWarps, w = (g % Q) % kCsWarps;
                    const size_t wi =
                        (((((size_t)h * rounds + k) * kCsWarps + w) * cnt + t / epl) * kCsSlots + sl) * 32 + u;
                    const int e = t % epl;
                    if (compact) {
                        words[wi * 4 + e] = idx * 4u;  // byte offset of the input's word
                    } else {
                        words[wi * 4 + 2 * e] = idx * 4u;
                        words[wi * 4 + 2 * e + 1] = wb;
                    }
                }
            }
        }
    void *d = nullptr;
    CSP_CUDA(cudaMalloc(&d, words.size() * 4));
    owned.push_back(d);
    CSP_CUDA(cudaMemcpy(d, words.data(), words.size() * 4, cudaMemcpyHostToDevice));
    ld.cs_w = (const uint4 *)d;
    ld.cs_cnt = cnt;
    ld.cs_bit = b;
    ld.cc_wconst = compact ? bits16_of(vals[0], prec) : 0u;
    return COSPDNN_OK;
}

int cs_layer_spec(KSpec &k, NetDev *nets, int nnets, int prec, bool compact, unsigned long long *launches,
                  int *abort_flag, const DevLimits *limits, int sms, int max_n) {
    using F = void (*)(const NetDev *, int, int, unsigned long long *, int *, const DevLimits *, uint32_t);
    static const F fns[2][2] = {{k_layer_cs<__half, false>, k_layer_cs<__half, true>},
                                {k_layer_cs<__nv_bfloat16, false>, k_layer_cs<__nv_bfloat16, true>}};
    CSP_CHECK(prec == COSPDNN_PREC_FP16 || prec == COSPDNN_PREC_BF16, COSPDNN_ERR_UNSUPPORTED,
              "cs_layer_spec: 16-bit nets only");
    k.fn = (void *)fns[prec == COSPDNN_PREC_FP16 ? 0 : 1][compact ? 1 : 0];
    const uint32_t recv_off = (uint32_t)cs_recv_off(max_n);
    k.smem = recv_off + kCsRecvBytes;
    CSP_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem));
    // clusters of two CTAs that fit at once (one CTA per SM)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * sms);
    cfg.blockDim = dim3(kCsThreads);
    cfg.dynamicSmemBytes = k.smem;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k.fn, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        clusters = sms / 2;
    }
    k.grid = dim3(2 * clusters);
    k.block = dim3(kCsThreads);
    k.arg(nets).arg(nnets).arg(prec).arg(launches).arg(abort_flag).arg(limits).arg(recv_off);
    return COSPDNN_OK;
}

}  // namespace cospdnn
