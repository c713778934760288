// tcgen05 layer kernel: FP16 / BF16 activations, FP32 accumulation in TMEM.
//
// Work item = (network, tile of 128 active rows, group of kGroup output block
// columns of 16 outputs).  For every 16x16 weight block b of an output block
// column c the kernel issues one MMA
//     D_c[128 x 16] (+)= A[128 rows x 16 inputs of block b] * B_b[16 x 16]
// (M=128, N=16, K=16, kind::f16).  A is gathered from the active rows of the
// layer's input (row list = the previous layer's compaction), so pruned rows
// are never read.  Roles (9 warps):
//   warps 0-3  loaders: cp.async of each row's 32 bytes + the 512-byte B
//              block into a stage of the shared-memory ring (canonical
//              K-major, no-swizzle core-matrix layout), completion signalled
//              by cp.async.mbarrier.arrive on the stage's `full` barrier;
//   warp 4     MMA issuer: one thread waits `full`, issues tcgen05.mma and
//              tcgen05.commit to the stage's `empty` barrier; after the last
//              block of an item it commits to the item's `tfull` barrier;
//   warps 5-8  epilogue: tcgen05.ld of the accumulators (TMEM lane = row),
//              bias + clamp(0,32), store in the compute type, per-row
//              statistics for the keep/prune decision (atomicMax).
// Accumulators are double-buffered in TMEM (2 x kGroup x 16 columns) so the
// epilogue of one item overlaps the MMAs of the next.  Every wait is bounded;
// on timeout the CTA raises `abort`, drains its copies and MMAs, frees TMEM
// and returns, and the engine reports COSPDNN_ERR_DEVICE.
#include <algorithm>

#include "tc_layer.cuh"

namespace cospdnn {
namespace {

constexpr int kTileRows = 128;
constexpr int kGroup = 8;                 // output block columns per work item
constexpr int kStages = 20;  // ~92 KB of stages: at most two CTAs (2 x 256 TMEM columns) per SM
constexpr int kStageA = kTileRows * 32;   // 128 rows x 16 inputs x 2 bytes
constexpr int kStageB = 512;              // 16 x 16 x 2 bytes
constexpr int kStageBytes = kStageA + kStageB;
constexpr int kLoaderWarps = 4;
constexpr int kMmaWarp = 4;
constexpr int kEpiWarp0 = 5;
constexpr int kEpiWarps = 4;
constexpr int kThreads = (kLoaderWarps + 1 + kEpiWarps) * 32;
constexpr int kTmemCols = 2 * kGroup * 16;  // two accumulator buffers
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz

struct __align__(16) TcSmem {
    uint8_t stage[kStages][kStageBytes];
    unsigned long long full[kStages];
    unsigned long long empty[kStages];
    unsigned long long tfull[2];
    unsigned long long tempty[2];
    unsigned long long fin;
    uint32_t tmem_base;
    volatile int abort;
};
constexpr size_t kSmemBytes = sizeof(TcSmem) + 128;

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
        if (clock64() - t0 > kWaitCycles) {
            sm.abort = 1;
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_arrive_noinc(unsigned long long *b) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(b)) : "memory");
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
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_commit(unsigned long long *b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(b))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct Item {
    int net, tile, c0, c1;
};

// Work items of this layer for tcgen05 nets of precision `prec`.
__device__ __forceinline__ bool tc_net(const NetDev &nd, int prec) {
    return nd.kernel == COSPDNN_KERNEL_TCGEN05 && nd.prec == prec && !nd.st->done;
}
__device__ __forceinline__ int64_t tc_items(const NetDev *nets, int nnets, int prec) {
    int64_t total = 0;
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (!tc_net(nd, prec)) continue;
        const int nb = nd.N / 16;
        total += (int64_t)((nd.st->R + kTileRows - 1) / kTileRows) * ((nb + kGroup - 1) / kGroup);
    }
    return total;
}
__device__ __forceinline__ Item tc_item(const NetDev *nets, int nnets, int prec, int64_t idx) {
    Item it{0, 0, 0, 0};
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (!tc_net(nd, prec)) continue;
        const int nb = nd.N / 16, groups = (nb + kGroup - 1) / kGroup;
        const int64_t cnt = (int64_t)((nd.st->R + kTileRows - 1) / kTileRows) * groups;
        if (idx < cnt) {
            it.net = n;
            it.tile = (int)(idx / groups);
            it.c0 = (int)(idx % groups) * kGroup;
            it.c1 = min(nb, it.c0 + kGroup);
            return it;
        }
        idx -= cnt;
    }
    return it;
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 2)
    k_layer_tc(const NetDev *__restrict__ nets, int nnets, int prec, unsigned long long *launches,
               int *abort_flag) {
    count_launch(launches);
    const int64_t total = tc_items(nets, nnets, prec);
    if (total == 0 || blockIdx.x >= total) return;  // uniform across the CTA
    extern __shared__ uint8_t smem_raw[];
    TcSmem &sm = *reinterpret_cast<TcSmem *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&sm.full[s], kLoaderWarps * 32);
            mbar_init(&sm.empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&sm.tfull[b], 1);
            mbar_init(&sm.tempty[b], kEpiWarps * 32);
        }
        mbar_init(&sm.fin, 1);
        sm.abort = 0;
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

    if (warp < kLoaderWarps) {
        // ---------------- loaders: one row per thread -------------------
        const int t = threadIdx.x;  // row within the tile, 0..127
        const uint32_t a_off = (uint32_t)((t >> 3) * 256 + (t & 7) * 16);
        uint32_t fill = 0;
        bool ok = true;
        for (int64_t idx = blockIdx.x; idx < total && ok; idx += gridDim.x) {
            const Item it = tc_item(nets, nnets, prec, idx);
            const NetDev &nd = nets[it.net];
            const int l = nd.st->layer, R = nd.st->R, par = l & 1, N = nd.N;
            const LayerDev &lw = nd.layers[l];
            const T *in = (const T *)(l == 0 ? nd.y0 : nd.act[par]);
            const int p = it.tile * kTileRows + t;
            const char *row = p < R ? (const char *)(in + (int64_t)nd.pos[par][p] * N) : nullptr;
            const char *bsrc = (const char *)lw.blk_b;
            for (int c = it.c0; c < it.c1 && ok; ++c) {
                const int b1 = lw.blk_ptr[c + 1];
                for (int b = lw.blk_ptr[c]; b < b1; ++b) {
                    const uint32_t s = fill % kStages, u = fill / kStages;
                    if (u > 0 && !mbar_wait(&sm.empty[s], (u - 1) & 1, sm)) { ok = false; break; }
                    const uint32_t st = smem_u32(sm.stage[s]);
                    if (row) {
                        const char *src = row + (int64_t)lw.blk_row[b] * 32;
                        cp_async16(st + a_off, src);
                        cp_async16(st + a_off + 128, src + 16);
                    }
                    if (t < 32) cp_async16(st + kStageA + t * 16, bsrc + (int64_t)b * kStageB + t * 16);
                    cp_async_arrive_noinc(&sm.full[s]);
                    ++fill;
                }
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (warp == kMmaWarp) {
        // ---------------- MMA issuer ---------------------------------------
        if (lane == 0) {
            const uint32_t idesc = instr_desc(sizeof(T) == 2 && prec == COSPDNN_PREC_BF16 ? 1u : 0u);
            uint32_t fill = 0, iter = 0;
            bool ok = true;
            for (int64_t idx = blockIdx.x; idx < total && ok; idx += gridDim.x, ++iter) {
                const Item it = tc_item(nets, nnets, prec, idx);
                const NetDev &nd = nets[it.net];
                const LayerDev &lw = nd.layers[nd.st->layer];
                const uint32_t buf = iter & 1;
                if (iter >= 2 && !mbar_wait(&sm.tempty[buf], ((iter >> 1) - 1) & 1, sm)) { ok = false; break; }
                tc_fence_after();
                for (int c = it.c0; c < it.c1 && ok; ++c) {
                    const uint32_t d = tmem + buf * (kGroup * 16) + (uint32_t)(c - it.c0) * 16;
                    uint32_t acc = 0;
                    const int b1 = lw.blk_ptr[c + 1];
                    for (int b = lw.blk_ptr[c]; b < b1; ++b) {
                        const uint32_t s = fill % kStages, u = fill / kStages;
                        if (!mbar_wait(&sm.full[s], u & 1, sm)) { ok = false; break; }
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        tc_fence_after();
                        const uint32_t st = smem_u32(sm.stage[s]);
                        mma_f16(d, smem_desc(st), smem_desc(st + kStageA), idesc, acc);
                        mma_commit(&sm.empty[s]);
                        acc = 1;
                        ++fill;
                    }
                }
                if (ok) mma_commit(&sm.tfull[buf]);
            }
            // every MMA this thread issued has completed before TMEM is freed
            mma_commit(&sm.fin);
            const long long t0 = clock64();
            while (!mbar_try_wait(&sm.fin, 0) && clock64() - t0 < kWaitCycles) {
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue: TMEM lane = row ---------------------------
        const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31
        const int r = quarter * 32 + lane;
        uint32_t iter = 0;
        for (int64_t idx = blockIdx.x; idx < total; idx += gridDim.x, ++iter) {
            const Item it = tc_item(nets, nnets, prec, idx);
            const NetDev &nd = nets[it.net];
            const int l = nd.st->layer, R = nd.st->R, par = l & 1, N = nd.N;
            const LayerDev &lw = nd.layers[l];
            const uint32_t buf = iter & 1;
            if (!mbar_wait(&sm.tfull[buf], (iter >> 1) & 1, sm)) break;
            tc_fence_after();
            const int p = it.tile * kTileRows + r;
            const bool valid = p < R;
            const float ez = valid ? z_error_bound(nd.err[par][p], nd.mx[par][p], lw.S, lw.dW, nd.bias,
                                                   fast_steps(nd, lw))
                                   : 0.0f;
            float zmax = -INFINITY, emax = 0.0f, ymax = 0.0f;
            T *out = (T *)nd.act[par ^ 1] + (int64_t)(valid ? p : 0) * N;
            for (int c = it.c0; c < it.c1; ++c) {
                float v[16];
                if (lw.blk_ptr[c + 1] > lw.blk_ptr[c]) {
                    tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + buf * (kGroup * 16) + (uint32_t)(c - it.c0) * 16, v);
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] = 0.0f;
                }
                __align__(16) T o[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const float z = v[i] + nd.bias;
                    const float cz = clamp32(z);
                    o[i] = act_traits<T>::from_f(cz);
                    const float yf = act_traits<T>::to_f(o[i]);
                    zmax = fmaxf(zmax, z);
                    ymax = fmaxf(ymax, yf);
                    if (z > -ez && z < 32.0f + ez) emax = fmaxf(emax, __fadd_ru(ez, fabsf(yf - cz)));
                }
                if (valid) {
                    uint4 *dst = reinterpret_cast<uint4 *>(out + c * 16);
                    dst[0] = reinterpret_cast<const uint4 *>(o)[0];
                    dst[1] = reinterpret_cast<const uint4 *>(o)[1];
                }
            }
            tc_fence_before();
            mbar_arrive(&sm.tempty[buf]);
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

}  // namespace

bool tc_supported(int neuron) { return neuron > 0 && neuron % 16 == 0; }

int tc_build_blocks(const std::vector<int32_t> &colptr, const std::vector<int32_t> &rowidx,
                    const std::vector<float> &vals, int N, int prec, LayerDev &ld, std::vector<void *> &owned) {
    const int nb = N / 16;
    std::vector<int32_t> ptr(nb + 1, 0), brow;
    std::vector<uint16_t> bvals;
    int maxb = 0;
    std::vector<int> slot(nb, -1);
    for (int c = 0; c < nb; ++c) {
        std::vector<int> used;
        for (int n = 0; n < 16; ++n) {
            const int j = c * 16 + n;
            for (int p = colptr[j]; p < colptr[j + 1]; ++p) {
                const int ib = rowidx[p] / 16;
                if (slot[ib] < 0) { slot[ib] = 0; used.push_back(ib); }
            }
        }
        std::sort(used.begin(), used.end());
        const size_t base = brow.size();
        for (size_t q = 0; q < used.size(); ++q) slot[used[q]] = (int)(base + q);
        brow.insert(brow.end(), used.begin(), used.end());
        bvals.resize(brow.size() * 256, 0);
        for (int n = 0; n < 16; ++n) {
            const int j = c * 16 + n;
            for (int p = colptr[j]; p < colptr[j + 1]; ++p) {
                const int i = rowidx[p], k = i % 16;
                const size_t blk = (size_t)slot[i / 16];
                // element (n, k) of the K-major B operand: 8x16-byte core matrices,
                // K halves 128 bytes apart, 8-row groups 256 bytes apart
                const size_t off = (size_t)(n / 8) * 128 + (size_t)(k / 8) * 64 + (size_t)(n % 8) * 8 + (size_t)(k % 8);
                uint16_t bits;
                if (prec == COSPDNN_PREC_BF16) {
                    __nv_bfloat16 h = __float2bfloat16_rn(vals[p]);
                    std::memcpy(&bits, &h, 2);
                } else {
                    __half h = __float2half_rn(vals[p]);
                    std::memcpy(&bits, &h, 2);
                }
                bvals[blk * 256 + off] = bits;
            }
        }
        for (int ib : used) slot[ib] = -1;
        ptr[c + 1] = (int32_t)brow.size();
        maxb = std::max(maxb, (int)used.size());
    }
    int32_t *dptr = nullptr, *drow = nullptr;
    void *dvals = nullptr;
    CSP_CUDA(cudaMalloc(&dptr, sizeof(int32_t) * ptr.size()));
    owned.push_back(dptr);
    CSP_CUDA(cudaMalloc(&drow, sizeof(int32_t) * std::max<size_t>(1, brow.size())));
    owned.push_back(drow);
    CSP_CUDA(cudaMalloc(&dvals, 2 * std::max<size_t>(256, bvals.size())));
    owned.push_back(dvals);
    CSP_CUDA(cudaMemcpy(dptr, ptr.data(), sizeof(int32_t) * ptr.size(), cudaMemcpyHostToDevice));
    if (!brow.empty()) {
        CSP_CUDA(cudaMemcpy(drow, brow.data(), sizeof(int32_t) * brow.size(), cudaMemcpyHostToDevice));
        CSP_CUDA(cudaMemcpy(dvals, bvals.data(), 2 * bvals.size(), cudaMemcpyHostToDevice));
    }
    ld.blk_ptr = dptr;
    ld.blk_row = drow;
    ld.blk_b = dvals;
    ld.max_blocks = maxb;
    return COSPDNN_OK;
}

int tc_layer_spec(KSpec &k, NetDev *nets, int nnets, int prec, unsigned long long *launches, int *abort_flag,
                  int sms) {
    k.fn = prec == COSPDNN_PREC_BF16 ? (void *)k_layer_tc<__nv_bfloat16> : (void *)k_layer_tc<__half>;
    CSP_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
    int per_sm = 0;
    CSP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, kThreads, kSmemBytes));
    per_sm = std::max(1, std::min(per_sm, 512 / kTmemCols));
    k.grid = dim3(sms * per_sm);
    k.block = dim3(kThreads);
    k.smem = kSmemBytes;
    k.arg(nets).arg(nnets).arg(prec).arg(launches).arg(abort_flag);
    return COSPDNN_OK;
}

}  // namespace cospdnn
