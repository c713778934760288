// tcgen05 layer kernel: FP16 / BF16 activations, FP32 accumulation in TMEM.
//
// W_l is cut into 16x16 aligned blocks.  Work item = (network, tile of 128
// active rows, chunk of up to 32 output block columns); the chunk's 32
// accumulators (128 rows x 16 outputs, FP32) fill the 512 TMEM columns.  For
// every block b (input block i -> output block column c) one MMA
//     D_c[128 x 16] (+)= A_i[128 rows x 16 inputs] * B_b[16 x 16]
// (M=128, N=16, K=16, kind::f16).  The MMAs of a chunk run input-stationary:
// ordered by input block, so each A tile is fetched once per chunk and feeds
// every accumulator of the chunk that needs it, and consecutive MMAs write
// different accumulators (no serialising dependence).  The host-built
// schedule (tc_build_blocks) groups them into stages: one contiguous run of
// up to 8 input blocks (one bulk copy of the A tiles; activations of tcgen05
// nets are stored as MMA tiles, see act_index) plus the stage's B operands
// and MMA codes (one bulk copy each, stored in stage order).
// Roles (6 warps):
//   warp 0     producer: one thread issues the stage's bulk copies
//              (cp.async.bulk, no multicast) on the stage's `full` mbarrier;
//   warp 1     MMA issuer: one thread waits `full`, issues the stage's
//              tcgen05.mma and one tcgen05.commit to the stage's `empty`;
//              after the last stage of an item it commits to `tfull`;
//   warps 2-5  epilogue: tcgen05.ld of the accumulators (TMEM lane = row),
//              bias + clamp(0,32), store in the compute type (32 bytes per
//              row and output block of the output tile), per-row statistics
//              for the keep/prune decision (atomicMax); then `tempty`.
// While the epilogue drains TMEM the producer keeps prefetching the next
// item's stages.  Every wait is bounded; on timeout the CTA raises `abort`,
// drains its copies and MMAs, frees TMEM and returns, and the engine reports
// COSPDNN_ERR_DEVICE.
#include <algorithm>
#include <map>

#include "tc_layer.cuh"

namespace cospdnn {
namespace {

constexpr int kTileRows = 128;
constexpr int kChunk = 32;                   // output block columns per item
constexpr int kMaxA = 8;                     // A tiles (input blocks) per stage
constexpr int kMaxMma = 64;                  // MMAs per stage
constexpr int kTileBytes = kTileRows * 32;   // one A tile: 128 rows x 16 inputs x 2 bytes
constexpr int kBBytes = 512;                 // one B operand: 16 x 16 x 2 bytes
constexpr int kStageA = kMaxA * kTileBytes;
constexpr int kStageB = kMaxMma * kBBytes;
constexpr int kStageCode = kMaxMma * 2;
constexpr int kStageBytes = kStageA + kStageB + kStageCode;
constexpr int kStages = 3;
constexpr int kMaxGap = 1;                   // unused input blocks a stage may span
constexpr int kProducerWarp = 0;
constexpr int kMmaWarp = 1;
constexpr int kEpiWarps = 4;  // warps 2..5: (warp & 3) covers the four TMEM lane quarters
constexpr int kThreads = (2 + kEpiWarps) * 32;
constexpr int kTmemCols = kChunk * 16;      // 512: one accumulator per chunk column

struct __align__(128) TcSmem {
    uint8_t stage[kStages][kStageBytes];
    unsigned long long full[kStages];
    unsigned long long empty[kStages];
    unsigned long long tfull;
    unsigned long long tempty;
    unsigned long long fin;
    int nmma[kStages];  // MMAs of the stage in each slot, written by the producer before its copies
    uint32_t tmem_base;
    volatile int abort;
    long long wait_cycles;  // limit of every wait of this launch (DevLimits)
};
constexpr size_t kSmemBytes = sizeof(TcSmem) + 128;
static_assert(kSmemBytes <= 227 * 1024, "tcgen05 layer kernel shared memory");

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false if this CTA aborted (timeout here or elsewhere).
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, uint32_t parity, TcSmem &sm) {
    const long long t0 = clock64();
    while (!mbar_try_wait(b, parity)) {
        if (sm.abort) return false;
        if (clock64() - t0 > sm.wait_cycles) {
            sm.abort = 1;
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
// (release: the producer's shared-memory writes before it are seen by a
// thread whose wait on the barrier completes)
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
// Bulk copy global -> this CTA's shared memory, completing on `bar` (no multicast).
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar)));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of
// 8 rows x 16 bytes, the two 8-element K halves 128 bytes apart (leading
// byte offset), 8-row groups 256 bytes apart (stride byte offset), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
           (1ull << 46);
}
// Instruction descriptor: D f32, A/B f16 (fmt 0) or bf16 (fmt 1), both
// K-major, N = 16, M = 128.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t fmt) {
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void mma_commit(unsigned long long *b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(b)));
}
// 32 lanes x 32 columns (two accumulators) of TMEM into registers.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

struct Item {
    int net, tile, chunk;
};

__device__ __forceinline__ bool tc_net(const NetDev &nd, int prec) {
    // layer 0 of a net whose inputs were counted (bits_layer.cu) is done
    return nd.kernel == COSPDNN_KERNEL_TCGEN05 && nd.prec == prec && !nd.st->done &&
           !(nd.st->layer == 0 && nd.st->l0_bits);
}
// Work items of this layer (tile-major, so CTAs running at the same time share
// the row tile's A operands in L2).
__device__ __forceinline__ int64_t tc_items(const NetDev *nets, int nnets, int prec) {
    int64_t total = 0;
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (!tc_net(nd, prec)) continue;
        total += (int64_t)((nd.st->R + kTileRows - 1) / kTileRows) * nd.layers[nd.st->layer].tc_nchunks;
    }
    return total;
}
__device__ __forceinline__ Item tc_item(const NetDev *nets, int nnets, int prec, int64_t idx) {
    Item it{0, 0, 0};
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (!tc_net(nd, prec)) continue;
        const int nch = nd.layers[nd.st->layer].tc_nchunks;
        const int64_t cnt = (int64_t)((nd.st->R + kTileRows - 1) / kTileRows) * nch;
        if (idx < cnt) {
            it.net = n;
            it.tile = (int)(idx / nch);
            it.chunk = (int)(idx % nch);
            return it;
        }
        idx -= cnt;
    }
    return it;
}

// Epilogue of ncol (1 or 2) accumulators of one row: bias, clamp, store in
// the compute type, row statistics.  dst0 = the row's 32 bytes of the first
// output block in the output tile; the next block is 2048 elements further.
template <typename T>
__device__ __forceinline__ void epilogue_cols(const float *v, int ncol, float bias, float ez, T *dst0,
                                              bool valid, float &zmax, float &emax, float &ymax) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        if (q >= ncol) break;
        __align__(16) T o[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const float z = v[q * 16 + i] + bias;
            const float cz = clamp32(z);
            o[i] = act_traits<T>::from_f(cz);
            const float yf = act_traits<T>::to_f(o[i]);
            zmax = fmaxf(zmax, z);
            ymax = fmaxf(ymax, yf);
            if (z > -ez && z < 32.0f + ez) emax = fmaxf(emax, __fadd_ru(ez, fabsf(yf - cz)));
        }
        if (valid) {
            T *dst = dst0 + q * 2048;
            *reinterpret_cast<uint4 *>(dst) = reinterpret_cast<const uint4 *>(o)[0];
            *reinterpret_cast<uint4 *>(dst + 64) = reinterpret_cast<const uint4 *>(o)[1];
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 1)
    k_layer_tc(const NetDev *__restrict__ nets, int nnets, int prec, unsigned long long *launches,
               int *abort_flag, const DevLimits *__restrict__ limits) {
    count_launch(launches);
    const int64_t total = tc_items(nets, nnets, prec);
    if (total == 0 || blockIdx.x >= total) return;  // uniform across the CTA
    extern __shared__ uint8_t smem_raw[];
    TcSmem &sm = *reinterpret_cast<TcSmem *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 1);
        }
        mbar_init(&sm.tfull, 1);
        mbar_init(&sm.tempty, kEpiWarps * 32);
        mbar_init(&sm.fin, 1);
        sm.abort = 0;
        sm.wait_cycles = limits->wait_cycles;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem_base;

    if (warp == kProducerWarp) {
        // ---------------- producer: three bulk copies per stage ------------
        if (lane == 0) {
            uint32_t fill = 0;
            bool ok = true;
            // test hook: CTA 0 issues nothing for its first stage, so the MMA
            // issuer's bounded wait on it runs out (the error path of a lost copy)
            const bool withhold = limits->withhold_stage != 0 && blockIdx.x == 0;
            for (int64_t idx = blockIdx.x; idx < total && ok; idx += gridDim.x) {
                const Item it = tc_item(nets, nnets, prec, idx);
                const NetDev &nd = nets[it.net];
                const int l = nd.st->layer, N = nd.N;
                const LayerDev &lw = nd.layers[l];
                const char *in = (const char *)(l == 0 ? nd.y0 : nd.act[nd.st->in_buf]);
                const char *tile = in + (int64_t)it.tile * (N / 16) * kTileBytes;
                const int s0 = lw.tc_chunk_ptr[it.chunk], s1 = lw.tc_chunk_ptr[it.chunk + 1];
                // stage descriptors a_first, a_count, b_first, n_mma; the next
                // one is loaded before this one's slot is waited for, so its
                // latency overlaps the wait and the copies
                int4 next = s0 < s1 ? lw.tc_stage[s0] : make_int4(0, 0, 0, 0);
                for (int q = s0; q < s1; ++q) {
                    const int4 st = next;
                    if (q + 1 < s1) next = lw.tc_stage[q + 1];
                    const uint32_t s = fill % kStages, u = fill / kStages;
                    if (u > 0 && !mbar_wait(&sm.empty[s], (u - 1) & 1, sm)) { ok = false; break; }
                    if (withhold && fill == 0) {
                        ++fill;
                        continue;
                    }
                    sm.nmma[s] = st.w;  // read by the MMA issuer after its wait on full[s]
                    const uint32_t base = smem_u32(sm.stage[s]);
                    const uint32_t code_bytes = (uint32_t)((st.w + 7) & ~7) * 2;
                    mbar_expect_tx(&sm.full[s], (uint32_t)st.y * kTileBytes + (uint32_t)st.w * kBBytes + code_bytes);
                    bulk_load(base, tile + (int64_t)st.x * kTileBytes, (uint32_t)st.y * kTileBytes, &sm.full[s]);
                    bulk_load(base + kStageA, (const char *)lw.tc_b + (int64_t)st.z * kBBytes, (uint32_t)st.w * kBBytes,
                              &sm.full[s]);
                    bulk_load(base + kStageA + kStageB, lw.tc_code + st.z, code_bytes, &sm.full[s]);
                    ++fill;
                }
            }
            // no bulk copy may still be writing shared memory when the CTA exits:
            // wait (bounded) for the last fill of every stage
            const uint32_t first = fill > (uint32_t)kStages ? fill - kStages : 0u;
            for (uint32_t f = first; f < fill; ++f) {
                if (withhold && f == 0) continue;  // nothing was issued for it
                const long long t0 = clock64();
                while (!mbar_try_wait(&sm.full[f % kStages], (f / kStages) & 1) && clock64() - t0 < sm.wait_cycles) {
                }
            }
        }
        __syncwarp();
    } else if (warp == kMmaWarp) {
        // ---------------- MMA issuer ---------------------------------------
        if (lane == 0) {
            const uint32_t idesc = instr_desc(prec == COSPDNN_PREC_BF16 ? 1u : 0u);
            uint32_t fill = 0, iter = 0;
            bool ok = true;
            for (int64_t idx = blockIdx.x; idx < total && ok; idx += gridDim.x, ++iter) {
                const Item it = tc_item(nets, nnets, prec, idx);
                const NetDev &nd = nets[it.net];
                const LayerDev &lw = nd.layers[nd.st->layer];
                if (iter >= 1 && !mbar_wait(&sm.tempty, (iter - 1) & 1, sm)) { ok = false; break; }
                tc_fence_after();
                const int s0 = lw.tc_chunk_ptr[it.chunk], s1 = lw.tc_chunk_ptr[it.chunk + 1];
                for (int q = s0; q < s1; ++q) {
                    const uint32_t s = fill % kStages, u = fill / kStages;
                    if (!mbar_wait(&sm.full[s], u & 1, sm)) { ok = false; break; }
                    const int n_mma = sm.nmma[s];
                    const uint32_t base = smem_u32(sm.stage[s]);
                    const uint64_t adesc0 = smem_desc(base), bdesc0 = smem_desc(base + kStageA);
                    const uint4 *code8 = reinterpret_cast<const uint4 *>(sm.stage[s] + kStageA + kStageB);
                    // 8 MMAs per step, each with its own operand registers, so an MMA
                    // still reading its descriptors never holds up the next one
                    for (int j0 = 0; j0 < n_mma; j0 += 8) {
                        const uint4 cv = code8[j0 >> 3];
                        const uint32_t cw[4] = {cv.x, cv.y, cv.z, cv.w};
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            if (j0 + q < n_mma) {
                                const uint32_t c = (cw[q >> 1] >> ((q & 1) * 16)) & 0xFFFFu;
                                mma_f16(tmem + ((c >> 3) & 31u) * 16u, adesc0 + (uint64_t)((c & 7u) * (kTileBytes >> 4)),
                                        bdesc0 + (uint64_t)((j0 + q) * (kBBytes >> 4)), idesc, (c >> 8) ? 0u : 1u);
                            }
                        }
                    }
                    mma_commit(&sm.empty[s]);
                    ++fill;
                }
                if (ok) mma_commit(&sm.tfull);
            }
            // every MMA this thread issued has completed before TMEM is freed
            mma_commit(&sm.fin);
            const long long t0 = clock64();
            while (!mbar_try_wait(&sm.fin, 0) && clock64() - t0 < sm.wait_cycles) {
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue: TMEM lane = row ---------------------------
        const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31
        const int r = quarter * 32 + lane;
        const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
        uint32_t iter = 0;
        for (int64_t idx = blockIdx.x; idx < total; idx += gridDim.x, ++iter) {
            const Item it = tc_item(nets, nnets, prec, idx);
            const NetDev &nd = nets[it.net];
            const int l = nd.st->layer, R = nd.st->R, par = l & 1, N = nd.N;
            const LayerDev &lw = nd.layers[l];
            if (!mbar_wait(&sm.tfull, iter & 1, sm)) break;
            tc_fence_after();
            const int p = it.tile * kTileRows + r;
            const bool valid = p < R;
            const float ez = valid ? z_error_bound(nd.err[par][p], nd.mx[par][p], lw.S, lw.dW, nd.bias,
                                                   fast_steps(nd, lw))
                                   : 0.0f;
            float zmax = -INFINITY, emax = 0.0f, ymax = 0.0f;
            T *out = (T *)nd.act[nd.st->in_buf ^ 1];
            const uint32_t used = lw.tc_used[it.chunk];
            const int c0 = it.chunk * kChunk, ncol = min(kChunk, N / 16 - c0);
            for (int j = 0; j < ncol; j += 2) {
                float v[32];
                tmem_ld32(tmem + lane_addr + (uint32_t)j * 16u, v);
#pragma unroll
                for (int q = 0; q < 2; ++q)
                    if (!((used >> (j + q)) & 1u)) {
#pragma unroll
                        for (int i = 0; i < 16; ++i) v[q * 16 + i] = 0.0f;
                    }
                epilogue_cols<T>(v, min(2, ncol - j), nd.bias, ez, out + act_index(1, N, valid ? p : 0, (c0 + j) * 16),
                                 valid, zmax, emax, ymax);
            }
            tc_fence_before();
            mbar_arrive(&sm.tempty);
            if (valid) {
                atomicMax(&nd.stat[3 * p], f2ord(zmax));
                atomicMax(&nd.stat[3 * p + 1], __float_as_uint(emax));
                atomicMax(&nd.stat[3 * p + 2], __float_as_uint(ymax));
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == kMmaWarp)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    if (threadIdx.x == 0 && sm.abort) atomicExch(abort_flag, 1);
}

template <typename D>
int upload(const std::vector<D> &h, const D **dptr, std::vector<void *> &owned) {
    void *p = nullptr;
    CSP_CUDA(cudaMalloc(&p, std::max<size_t>(16, h.size() * sizeof(D))));
    owned.push_back(p);
    if (!h.empty()) CSP_CUDA(cudaMemcpy(p, h.data(), h.size() * sizeof(D), cudaMemcpyHostToDevice));
    *dptr = (const D *)p;
    return COSPDNN_OK;
}

}  // namespace

bool tc_supported(int neuron) { return neuron > 0 && neuron % 16 == 0; }

// Builds the chunked, input-stationary MMA schedule of one layer (see LayerDev).
int tc_build_blocks(const std::vector<int32_t> &colptr, const std::vector<int32_t> &rowidx,
                    const std::vector<float> &vals, int N, int prec, LayerDev &ld, std::vector<void *> &owned) {
    const int nb = N / 16, nchunks = (nb + kChunk - 1) / kChunk;
    std::vector<int32_t> chunk_ptr(nchunks + 1, 0);
    std::vector<int4> stages;
    std::vector<uint16_t> codes;
    std::vector<uint16_t> bvals;
    std::vector<uint32_t> used(nchunks, 0u);
    int maxb = 0;
    auto to_bits = [prec](float v) {
        uint16_t bits;
        if (prec == COSPDNN_PREC_BF16) {
            __nv_bfloat16 h = __float2bfloat16_rn(v);
            std::memcpy(&bits, &h, 2);
        } else {
            __half h = __float2half_rn(v);
            std::memcpy(&bits, &h, 2);
        }
        return bits;
    };
    for (int h = 0; h < nchunks; ++h) {
        // (input block, column in chunk) -> dense 16x16 block, ordered by input block
        std::map<std::pair<int, int>, std::vector<uint16_t>> blocks;
        for (int jc = 0; jc < kChunk && h * kChunk + jc < nb; ++jc) {
            const int c = h * kChunk + jc;
            int nblk = 0;
            for (int n = 0; n < 16; ++n) {
                const int j = c * 16 + n;
                for (int p = colptr[j]; p < colptr[j + 1]; ++p) {
                    const int i = rowidx[p], k = i % 16;
                    auto key = std::make_pair(i / 16, jc);
                    auto itb = blocks.find(key);
                    if (itb == blocks.end()) {
                        itb = blocks.emplace(key, std::vector<uint16_t>(256, 0)).first;
                        ++nblk;
                    }
                    // element (n, k) of the K-major B operand: 8x16-byte core matrices,
                    // K halves 128 bytes apart, 8-row groups 256 bytes apart
                    const size_t off = (size_t)(n / 8) * 128 + (size_t)(k / 8) * 64 + (size_t)(n % 8) * 8 + (size_t)(k % 8);
                    itb->second[off] = to_bits(vals[p]);
                }
            }
            maxb = std::max(maxb, nblk);
            if (nblk) used[h] |= 1u << jc;
        }
        // stages: runs of input blocks (<= kMaxA wide, gaps <= kMaxGap), <= kMaxMma MMAs
        uint32_t seen = 0u;
        auto it = blocks.begin();
        while (it != blocks.end()) {
            const int a_first = it->first.first;
            int a_last = a_first;
            std::vector<decltype(it)> members;
            while (it != blocks.end()) {
                const int i = it->first.first;
                auto jt = it;
                int cnt = 0;
                while (jt != blocks.end() && jt->first.first == i) { ++jt; ++cnt; }
                const bool fits = (i - a_first + 1 <= kMaxA) && (i - a_last <= kMaxGap + 1) &&
                                  ((int)members.size() + cnt <= kMaxMma);
                if (!members.empty() && !fits) break;
                for (auto kt = it; kt != jt; ++kt) members.push_back(kt);
                a_last = i;
                it = jt;
            }
            // round-robin over accumulators: the k-th MMA of every column before
            // any (k+1)-th, so MMAs into the same accumulator are far apart
            {
                std::map<int, int> occ;
                std::vector<std::pair<int, int>> key(members.size());
                for (size_t q = 0; q < members.size(); ++q) key[q] = {occ[members[q]->first.second]++, (int)q};
                std::stable_sort(key.begin(), key.end());
                std::vector<decltype(it)> ordered;
                for (auto &kq : key) ordered.push_back(members[kq.second]);
                members.swap(ordered);
            }
            const int b_first = (int)((codes.size() + 7) / 8 * 8);  // code copies start 16-byte aligned
            codes.resize(b_first, 0);
            bvals.resize((size_t)b_first * 256, 0);
            for (auto &m : members) {
                const int i = m->first.first, jc = m->first.second;
                const bool first = !((seen >> jc) & 1u);
                seen |= 1u << jc;
                codes.push_back((uint16_t)((i - a_first) | (jc << 3) | (first ? 256 : 0)));
                bvals.insert(bvals.end(), m->second.begin(), m->second.end());
            }
            stages.push_back(make_int4(a_first, a_last - a_first + 1, b_first, (int)members.size()));
        }
        chunk_ptr[h + 1] = (int32_t)stages.size();
    }
    codes.resize((codes.size() + 7) / 8 * 8 + 8, 0);  // room for the last aligned code copy
    bvals.resize(std::max<size_t>(bvals.size(), codes.size() * 256), 0);
    int rc;
    if ((rc = upload(chunk_ptr, &ld.tc_chunk_ptr, owned))) return rc;
    if ((rc = upload(stages, &ld.tc_stage, owned))) return rc;
    if ((rc = upload(codes, &ld.tc_code, owned))) return rc;
    if ((rc = upload(used, &ld.tc_used, owned))) return rc;
    const uint16_t *bptr = nullptr;
    if ((rc = upload(bvals, &bptr, owned))) return rc;
    ld.tc_b = bptr;
    ld.tc_nchunks = nchunks;
    ld.max_blocks = maxb;
    return COSPDNN_OK;
}

int tc_layer_spec(KSpec &k, NetDev *nets, int nnets, int prec, unsigned long long *launches, int *abort_flag,
                  const DevLimits *limits, int sms) {
    k.fn = prec == COSPDNN_PREC_BF16 ? (void *)k_layer_tc<__nv_bfloat16> : (void *)k_layer_tc<__half>;
    CSP_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
    k.grid = dim3(sms);  // one CTA (all of TMEM) per SM
    k.block = dim3(kThreads);
    k.smem = kSmemBytes;
    k.arg(nets).arg(nnets).arg(prec).arg(launches).arg(abort_flag).arg(limits);
    return COSPDNN_OK;
}

}  // namespace cospdnn
