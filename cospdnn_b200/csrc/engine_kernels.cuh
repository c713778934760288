// Kernels of the device-driven layer loop.  Every kernel reads the per-net
// state (current layer, active rows, buffer roles) from device memory, so one
// captured graph serves every layer and every network; grids are fixed and
// loop over the work that the state describes.
//
// Per iteration (every live network advances one layer):
//   layer kernel(s)  rows 0..R-1 of IN -> OUT, per-row statistics
//   k_classify       keep / prune / uncertain from the statistics and the
//                    row's error bound
//   k_replay         exact FP64 replay of the uncertain rows
//   k_compact        stable compaction of the kept rows: new lists, state
//   k_copy_rows      kept rows of OUT -> rows 0..R'-1 of the next input
// IN = y0 for layer 0, else act[in_buf]; OUT = act[in_buf ^ 1].
#pragma once

#include "engine.cuh"

namespace cospdnn {

// ---- K0: start of a run --------------------------------------------------
__global__ void k_init_run(const NetDev *__restrict__ nets, int nnets, unsigned long long *launches,
                           int *loop_guard, int *abort_flag) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (launches) *launches = 1ull;
        *loop_guard = 0;
        *abort_flag = 0;
    }
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (tid == 0) {
            nd.st->layer = 0;
            nd.st->R = nd.rows;
            nd.st->done = (nd.rows == 0 || nd.L == 0);
            nd.st->nunc = 0;
            nd.st->err = 0;
            nd.st->in_buf = 0;
            nd.st->copy_R = 0;
            nd.st->l0_bits = 0;
            nd.st->gather = 0;
        }
        for (int64_t l = tid; l < nd.L; l += nth) {
            nd.alive_count[l] = 0;
            nd.recheck_count[l] = 0;
        }
        for (int64_t c = tid; c < (nd.rows + kCompactChunk - 1) / kCompactChunk; c += nth) nd.ccount[c] = 0;
        for (int64_t p = tid; p < nd.rows; p += nth) {
            nd.orig[0][p] = (int32_t)p;
            nd.err[0][p] = nd.err0[p];
            nd.mx[0][p] = nd.mx0[p];
            nd.stat[3 * p] = 0u;
            nd.stat[3 * p + 1] = 0u;
            nd.stat[3 * p + 2] = 0u;
        }
    }
}

// ---- K1 (CUDA cores): one warp = 4 rows x all outputs ---------------------
// Lane j of a 32-output segment accumulates output j of 4 rows over the ELL
// entries of column j (index and weight loaded once, used for 4 rows), then
// applies bias + clamp, stores the compute-type value and folds the output into
// the row statistics (max z, error bound of the stored outputs, max output).
constexpr int kPlainRows = 4;
constexpr int kPlainThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kPlainThreads)
    k_layer_plain(const NetDev *__restrict__ nets, int nnets, int prec, unsigned long long *launches) {
    count_launch(launches);
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int64_t total = 0;
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (nd.kernel != COSPDNN_KERNEL_CUDA_CORE || nd.layout != 0 || nd.prec != prec || nd.st->done) continue;
        total += (nd.st->R + kPlainRows - 1) / kPlainRows;
    }
    for (int64_t unit = gwarp; unit < total; unit += nwarps) {
        int64_t u = unit;
        int n = 0;
        for (; n < nnets; ++n) {
            const NetDev &nd = nets[n];
            if (nd.kernel != COSPDNN_KERNEL_CUDA_CORE || nd.layout != 0 || nd.prec != prec || nd.st->done) continue;
            const int64_t cnt = (nd.st->R + kPlainRows - 1) / kPlainRows;
            if (u < cnt) break;
            u -= cnt;
        }
        const NetDev &nd = nets[n];
        const int N = nd.N, l = nd.st->layer, R = nd.st->R, par = l & 1, ib = nd.st->in_buf;
        const LayerDev lw = nd.layers[l];
        const T *in = (const T *)(l == 0 ? nd.y0 : nd.act[ib]);
        T *out = (T *)nd.act[ib ^ 1];
        const double steps = fast_steps(nd, lw);
        const T *inrow[kPlainRows];
        T *outrow[kPlainRows];
        float ez[kPlainRows], zmax[kPlainRows], emax[kPlainRows], ymax[kPlainRows];
        bool valid[kPlainRows];
#pragma unroll
        for (int r = 0; r < kPlainRows; ++r) {
            const int p = (int)(u * kPlainRows) + r;
            valid[r] = p < R;
            const int pp = valid[r] ? p : (int)(u * kPlainRows);
            inrow[r] = in + (int64_t)pp * N;
            outrow[r] = out + (int64_t)pp * N;
            ez[r] = z_error_bound(nd.err[par][pp], nd.mx[par][pp], lw.S, lw.dW, nd.bias, steps);
            zmax[r] = -INFINITY;
            emax[r] = 0.0f;
            ymax[r] = 0.0f;
        }
        for (int j0 = 0; j0 < N; j0 += 32) {
            const int j = j0 + lane;
            if (j < N) {
                float acc[kPlainRows];
#pragma unroll
                for (int r = 0; r < kPlainRows; ++r) acc[r] = 0.0f;
                const int32_t *ip = lw.ell_idx + j;
                const float *wp = lw.ell_val + j;
                for (int k = 0; k < lw.K; ++k) {
                    const int32_t i = __ldg(ip + (int64_t)k * N);
                    const float w = __ldg(wp + (int64_t)k * N);
#pragma unroll
                    for (int r = 0; r < kPlainRows; ++r)
                        acc[r] = fmaf(w, act_traits<T>::to_f(inrow[r][i]), acc[r]);
                }
#pragma unroll
                for (int r = 0; r < kPlainRows; ++r) {
                    const float z = acc[r] + nd.bias;
                    const float c = clamp32(z);
                    const T ys = act_traits<T>::from_f(c);
                    const float yf = act_traits<T>::to_f(ys);
                    if (valid[r]) outrow[r][j] = ys;
                    zmax[r] = fmaxf(zmax[r], z);
                    ymax[r] = fmaxf(ymax[r], yf);
                    if (z > -ez[r] && z < 32.0f + ez[r]) emax[r] = fmaxf(emax[r], __fadd_ru(ez[r], fabsf(yf - c)));
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kPlainRows; ++r) {
            const float zm = warp_max(zmax[r]), em = warp_max(emax[r]), ym = warp_max(ymax[r]);
            if (lane == 0 && valid[r]) {
                const int p = (int)(u * kPlainRows) + r;
                nd.stat[3 * p] = f2ord(zm);
                nd.stat[3 * p + 1] = __float_as_uint(em);
                nd.stat[3 * p + 2] = __float_as_uint(ym);
            }
        }
    }
}

// ---- K2: keep / prune / uncertain per row ---------------------------------
// A warp takes 32 consecutive rows (all in one compaction chunk) and adds its
// sure keeps to the chunk's count; k_replay adds the re-decided ones.
__global__ void k_classify(const NetDev *__restrict__ nets, int nnets, unsigned long long *launches) {
    count_launch(launches);
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int n = 0; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        if (nd.st->done) continue;
        const int l = nd.st->layer, R = nd.st->R, par = l & 1;
        const LayerDev &lw = nd.layers[l];
        const double steps = fast_steps(nd, lw);
        for (int64_t base = warp * 32; base < R; base += nwarps * 32) {
            const int64_t p = base + lane;
            int8_t c = CLS_PRUNE;
            if (p < R) {
                const float zm = ord2f(nd.stat[3 * p]);
                const float ez = z_error_bound(nd.err[par][p], nd.mx[par][p], lw.S, lw.dW, nd.bias, steps);
                const double lo = (double)zm - (double)ez, hi = (double)zm + (double)ez;
                if (lo > (double)nd.tau) c = CLS_KEEP;
                else if (hi <= (double)nd.tau) c = CLS_PRUNE;
                else c = CLS_UNCERTAIN;
                nd.cls[p] = c;
                if (c == CLS_UNCERTAIN) nd.ulist[atomicAdd(&nd.st->nunc, 1)] = (int32_t)p;
            }
            const unsigned keep = __ballot_sync(0xffffffffu, c == CLS_KEEP);
            if (lane == 0 && keep) atomicAdd(&nd.ccount[base / kCompactChunk], __popc(keep));
        }
    }
}

// ---- K3: exact FP64 replay of uncertain rows ------------------------------
// One CTA per uncertain row: recompute the row from its exact input through
// the current layer in the oracle's order (for each output, ascending input
// index, separately rounded multiply and add, bias last, clamp), decide
// keep/prune exactly, and for kept rows overwrite the fast output with the
// FP64 values rounded to the compute type.  The layer's input row is held
// in shared memory (the gathers read it) and its output row too when both
// fit in kReplaySmemDoubles; when only the input fits, the output goes to
// global scratch and is copied into shared memory for the next layer; wider
// rows stay in global scratch.
constexpr int kReplayThreads = 1024;
constexpr int kReplaySmemDoubles = 26624;  // 208 KB

// Doubles of shared memory a net of width N replays in (0: global scratch).
__host__ __device__ __forceinline__ int replay_smem_doubles(int N) {
    return 2 * N <= kReplaySmemDoubles ? 2 * N : N <= kReplaySmemDoubles ? N : 0;
}

__device__ __forceinline__ float block_max(float v, float *red) {
    v = warp_max(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = lane < (int)(blockDim.x >> 5) ? red[lane] : -INFINITY;
        v = warp_max(v);
        if (lane == 0) red[0] = v;
    }
    __syncthreads();
    return red[0];
}

template <typename T>
__device__ void replay_row(const NetDev &nd, int p, double *buf0, double *buf1, bool copy_back, float *red) {
    const int N = nd.N, l = nd.st->layer, par = l & 1, ib = nd.st->in_buf;
    const int orow = nd.orig[par][p];
    double *y = buf0, *z = buf1;
    // the input row: exact FP32 values, the bit planes when layer 0 of this
    // run was counted (the compute-type copy is not made then), else the
    // compute-type copy (integer inputs are exact in it)
    const bool counted = nd.st->l0_bits != 0;
    for (int j = threadIdx.x; j < N; j += blockDim.x)
        y[j] = nd.y0_f32 ? (double)nd.y0_f32[(int64_t)orow * N + j]
             : counted   ? (double)((nd.y0bits[(int64_t)(orow >> 5) * N + j] >> (orow & 31)) & 1u)
                         : act_traits<T>::to_d(((const T *)nd.y0)[act_index(nd.layout, N, orow, j)]);
    __syncthreads();
    const double b = (double)nd.bias;
    for (int ll = 0; ll <= l; ++ll) {
        const LayerDev &lw = nd.layers[ll];
        for (int j = threadIdx.x; j < N; j += blockDim.x) {
            double acc = 0.0;
            if (lw.rp_idx) {
                // one weight value: 16-bit indices of the real entries only
                const double w = (double)lw.rp_w;
                const int c = lw.rp_cnt[j];
                const uint16_t *ip = lw.rp_idx + j;
                int k = 0;
                for (; k + 32 <= c; k += 32) {
                    uint32_t ii[32];
#pragma unroll
                    for (int t = 0; t < 32; ++t) ii[t] = __ldg(ip + (int64_t)(k + t) * N);
#pragma unroll
                    for (int t = 0; t < 32; ++t) {
                        const double yi = y[ii[t]];
                        if (yi != 0.0) acc = __dadd_rn(acc, __dmul_rn(w, yi));
                    }
                }
                for (; k < c; ++k) {
                    const double yi = y[__ldg(ip + (int64_t)k * N)];
                    if (yi != 0.0) acc = __dadd_rn(acc, __dmul_rn(w, yi));
                }
                z[j] = clamp32d(__dadd_rn(acc, b));
                continue;
            }
            // entries in ascending input order, loads issued 8 ahead of the
            // (strictly sequential) accumulation
            const int32_t *ip = lw.ell_idx + j;
            const float *wp = lw.ell_val + j;
            int k = 0;
            for (; k + 32 <= lw.K; k += 32) {
                int32_t ii[32];
                float ww[32];
#pragma unroll
                for (int t = 0; t < 32; ++t) {
                    ii[t] = __ldg(ip + (int64_t)(k + t) * N);
                    ww[t] = __ldg(wp + (int64_t)(k + t) * N);
                }
#pragma unroll
                for (int t = 0; t < 32; ++t) {
                    const double yi = y[ii[t]];
                    if (yi != 0.0) acc = __dadd_rn(acc, __dmul_rn((double)ww[t], yi));
                }
            }
            for (; k < lw.K; ++k) {
                const double yi = y[__ldg(ip + (int64_t)k * N)];
                if (yi != 0.0) acc = __dadd_rn(acc, __dmul_rn((double)__ldg(wp + (int64_t)k * N), yi));
            }
            z[j] = clamp32d(__dadd_rn(acc, b));
        }
        __syncthreads();
        if (copy_back) {
            // the output row (global) becomes the next input row (shared)
            for (int j = threadIdx.x; j < N; j += blockDim.x) y[j] = z[j];
            __syncthreads();
        } else {
            double *t = y;
            y = z;
            z = t;
        }
    }
    // y holds the layer-l outputs; exact keep decision on the FP64 values
    double dmax = 0.0;
    for (int j = threadIdx.x; j < N; j += blockDim.x) dmax = fmax(dmax, y[j]);
    const bool keep = block_max(dmax > (double)nd.tau ? 1.0f : 0.0f, red) > 0.5f;
    float emax = 0.0f, ymax = 0.0f;
    if (keep) {
        T *out = (T *)nd.act[ib ^ 1];
        for (int j = threadIdx.x; j < N; j += blockDim.x) {
            const T v = act_traits<T>::from_d(y[j]);
            out[act_index(nd.layout, N, p, j)] = v;
            const double vd = act_traits<T>::to_d(v);
            emax = fmaxf(emax, __double2float_ru(fabs(vd - y[j])));
            ymax = fmaxf(ymax, (float)vd);
        }
        emax = block_max(emax, red);
        ymax = block_max(ymax, red);
    }
    if (threadIdx.x == 0) {
        nd.cls[p] = keep ? CLS_KEEP : CLS_PRUNE;
        if (keep) {
            atomicAdd(&nd.ccount[p / kCompactChunk], 1);
            nd.stat[3 * p + 1] = __float_as_uint(emax);
            nd.stat[3 * p + 2] = __float_as_uint(ymax);
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kReplayThreads)
    k_replay(const NetDev *__restrict__ nets, int nnets, double *__restrict__ scratch, int max_n,
             unsigned long long *launches) {
    count_launch(launches);
    __shared__ float red[32];
    extern __shared__ double ysm[];
    int64_t total = 0;
    for (int n = 0; n < nnets; ++n)
        if (!nets[n].st->done) total += nets[n].st->nunc;
    for (int64_t q = blockIdx.x; q < total; q += gridDim.x) {
        int64_t u = q;
        int n = 0;
        for (; n < nnets; ++n) {
            if (nets[n].st->done) continue;
            if (u < nets[n].st->nunc) break;
            u -= nets[n].st->nunc;
        }
        const NetDev &nd = nets[n];
        // the launch has replay_smem_doubles(N) of shared memory for every net
        const int sd = replay_smem_doubles(nd.N);
        double *const g0 = scratch + (int64_t)blockIdx.x * 2 * max_n;
        double *b0, *b1;
        if (sd == 2 * nd.N) {
            b0 = ysm;
            b1 = ysm + nd.N;
        } else if (sd == nd.N) {
            b0 = ysm;
            b1 = g0;
        } else {
            b0 = g0;
            b1 = g0 + max_n;
        }
        const bool copy_back = sd == nd.N;
        const int p = nd.ulist[u];
        if (nd.prec == COSPDNN_PREC_FP32) replay_row<float>(nd, p, b0, b1, copy_back, red);
        else if (nd.prec == COSPDNN_PREC_FP16) replay_row<__half>(nd, p, b0, b1, copy_back, red);
        else replay_row<__nv_bfloat16>(nd, p, b0, b1, copy_back, red);
    }
}

// Nets whose layer kernel can stage its row tiles through the compaction map
// (the one-CTA row-tile kernel, k_layer_cc): kept rows need no copy.
__device__ __forceinline__ bool gathers_rows(const NetDev &nd) {
    return nd.kernel == COSPDNN_KERNEL_CUDA_CORE && nd.layout >= 2 && !nd.cc_split;
}

// ---- K4: stable compaction + state advance + loop condition ---------------
// One CTA per chunk of kCompactChunk rows (grid = chunks of all nets at full
// size; chunks past a net's current rows are idle).  A chunk's first output
// position is the sum of the keep counts of the chunks before it.  The last
// CTA to finish advances every net's state and decides whether the graph
// loop runs again.
constexpr int kCompactThreads = kCompactChunk;

__global__ void __launch_bounds__(kCompactThreads)
    k_compact(const NetDev *__restrict__ nets, int nnets, unsigned int *finished_ctas,
              cudaGraphConditionalHandle loop, int use_cond, int *loop_guard, const DevLimits *__restrict__ limits,
              const int *abort_flag, unsigned long long *launches) {
    count_launch(launches);
    __shared__ int red[kCompactThreads / 32];
    __shared__ int s_base;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // locate this CTA's chunk
    int64_t u = blockIdx.x;
    int n = 0;
    for (; n < nnets; ++n) {
        const NetDev &nd = nets[n];
        const int64_t cnt = nd.st->done ? 0 : (nd.st->R + kCompactChunk - 1) / kCompactChunk;
        if (u < cnt) break;
        u -= cnt;
    }
    if (n < nnets) {
        const NetDev &nd = nets[n];
        const int l = nd.st->layer, R = nd.st->R, par = l & 1, b = (int)u;
        // kept rows of the chunks before this one
        int v = 0;
        for (int t = threadIdx.x; t < b; t += kCompactThreads) v += nd.ccount[t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[wid] = v;
        __syncthreads();
        if (wid == 0) {
            int w = red[lane];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
            if (lane == 0) s_base = w;
        }
        __syncthreads();
        // stable scan of this chunk's keeps
        const int p = b * kCompactChunk + threadIdx.x;
        const int keep = (p < R && nd.cls[p] == CLS_KEEP) ? 1 : 0;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) red[wid] = __popc(m);
        __syncthreads();
        if (wid == 0) {
            int w = red[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += t;
            }
            red[lane] = w;
        }
        __syncthreads();
        if (keep) {
            const int q = s_base + (wid ? red[wid - 1] : 0) + __popc(m & ((1u << lane) - 1u));
            nd.cmap[q] = p;
            nd.orig[par ^ 1][q] = nd.orig[par][p];
            nd.err[par ^ 1][q] = __uint_as_float(nd.stat[3 * p + 1]);
            nd.mx[par ^ 1][q] = __uint_as_float(nd.stat[3 * p + 2]);
        }
        if (p < R) {
            nd.stat[3 * p] = 0u;
            nd.stat[3 * p + 1] = 0u;
            nd.stat[3 * p + 2] = 0u;
        }
    }
    // the last CTA to finish advances the states and sets the loop condition
    __syncthreads();
    __shared__ int s_last;
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(finished_ctas, 1u) + 1u == gridDim.x;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int i = 0; i < nnets; ++i) {
        const NetDev &nd = nets[i];
        if (*(volatile int *)&nd.st->done) {
            if (threadIdx.x == 0) nd.st->copy_R = 0;
            continue;
        }
        const int l = nd.st->layer, R = nd.st->R, nch = (R + kCompactChunk - 1) / kCompactChunk;
        int v = 0;
        for (int t = threadIdx.x; t < nch; t += kCompactThreads) {
            v += *(volatile int32_t *)&nd.ccount[t];
            nd.ccount[t] = 0;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        __syncthreads();
        if (lane == 0) red[wid] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            int kept = 0;
            for (int w = 0; w < kCompactThreads / 32; ++w) kept += red[w];
            nd.alive_count[l] = kept;
            nd.recheck_count[l] = nd.st->nunc;
            nd.st->nunc = 0;
            nd.st->R = kept;
            nd.st->layer = l + 1;
            nd.st->done = (kept == 0 || l + 1 >= nd.L);
            if (kept == R) {
                // nothing pruned: the output buffer is the next input as it is
                nd.st->in_buf ^= 1;
                nd.st->copy_R = 0;
                nd.st->gather = 0;
            } else if (!nd.st->done && gathers_rows(nd) && 2 * kept >= R) {
                // the next layer's tile kernel reads the kept rows through cmap:
                // when most rows are kept, a tile's rows come from one or two
                // source tiles (measured on one B200: S1, 1024 neurons with
                // 90% kept per layer, 23.7 -> 22.5 ms per run; with a quarter
                // kept, C2's layer 2, the staging costs more than the copy)
                nd.st->in_buf ^= 1;
                nd.st->copy_R = 0;
                nd.st->gather = 1;
            } else {
                nd.st->copy_R = kept;  // k_copy_rows moves the kept rows
                nd.st->gather = 0;
            }
        }
    }
    if (threadIdx.x == 0) {
        *finished_ctas = 0u;
        __threadfence();
        int live = 0;
        for (int i = 0; i < nnets; ++i) live |= !(*(volatile int *)&nets[i].st->done);
        const int it = ++*loop_guard;
        if (it > limits->max_iters || *(volatile const int *)abort_flag) {
            for (int i = 0; i < nnets; ++i) nets[i].st->err = COSPDNN_ERR_DEVICE;
            live = 0;
        }
        if (use_cond) cudaGraphSetConditional(loop, live ? 1u : 0u);
    }
}

// ---- K5: move the kept rows to the front of the next input buffer ---------
// Row q of act[in_buf] <- row cmap[q] of act[in_buf ^ 1].
// Row-major and MMA-tile nets: 16-byte pieces (row-major: consecutive; MMA
// tiles: the two 8-feature halves of each block).  Row-tile nets: one CTA
// per destination tile, see copy_tile.
constexpr int kCopyThreads = 256;

// Row-tile copy of destination tile q of one net (a CTA's work item): rows
// q*TR .. q*TR+TR-1 of the next input <- the kept output rows cmap[...],
// rows past the kept count zero.  The tile's row map is read once into
// shared memory; threads then take the tile's feature columns in turn.
// Kept rows are increasing, so a tile's rows come from a few consecutive
// source tiles: when a feature column is one 4-, 8- or 16-byte piece, each
// distinct source column is loaded once (one vector load, coalesced across
// the threads of consecutive features) and the values are picked out of it;
// wider columns move 16-byte destination pieces whose values are loaded one
// by one (repeats hit L1).
constexpr int kCopyMaxTR = 128;

template <typename E>
__device__ __forceinline__ void copy_tile(const NetDev &nd, int q, int *s_map) {
    constexpr int kV = 16 / (int)sizeof(E);  // values of a 16-byte piece
    const int TR = nd.layout, N = nd.N, R = nd.st->copy_R, ib = nd.st->in_buf;
    const int lg = __ffs(TR) - 1;            // TR is a power of two
    const int colb = TR * (int)sizeof(E);    // bytes of a feature column
    const E *src = (const E *)nd.act[ib ^ 1];
    E *dst = (E *)nd.act[ib] + ((int64_t)q * N << lg);
    __syncthreads();  // the previous tile is done with s_map
    for (int r = threadIdx.x; r < TR; r += blockDim.x) {
        const int row = q * TR + r;
        s_map[r] = row < R ? nd.cmap[row] : -1;
    }
    __syncthreads();
    if (colb == 16 || colb == 8 || colb == 4) {
        // TR <= 8 values per column: the map in registers
        int pm[kV];
#pragma unroll
        for (int i = 0; i < kV; ++i) pm[i] = i < TR ? s_map[i] : -1;
        for (int f = threadIdx.x; f < N; f += blockDim.x) {
            __align__(16) E v[kV];
            int64_t cur = -1;
            uint4 col = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
            for (int i = 0; i < kV; ++i) {
                v[i] = E(0);
                const int p = pm[i];
                if (p < 0) continue;
                const int64_t t = p >> lg;
                if (t != cur) {
                    cur = t;
                    const E *c = src + ((t * N + f) << lg);
                    if (colb == 16) {
                        col = __ldg(reinterpret_cast<const uint4 *>(c));
                    } else if (colb == 8) {
                        const uint2 h = __ldg(reinterpret_cast<const uint2 *>(c));
                        col = make_uint4(h.x, h.y, 0u, 0u);
                    } else {
                        col = make_uint4(__ldg(reinterpret_cast<const uint32_t *>(c)), 0u, 0u, 0u);
                    }
                }
                const int off = (p & (TR - 1)) * (int)sizeof(E);  // byte offset in the column
                const uint32_t w = off < 8 ? (off < 4 ? col.x : col.y) : (off < 12 ? col.z : col.w);
                if (sizeof(E) == 4) {
                    v[i] = *reinterpret_cast<const E *>(&w);
                } else {
                    const uint16_t h = (uint16_t)(w >> (8 * (off & 3)));
                    v[i] = *reinterpret_cast<const E *>(&h);
                }
            }
            if (colb == 16) *reinterpret_cast<uint4 *>(dst + ((int64_t)f << lg)) = *reinterpret_cast<const uint4 *>(v);
            else if (colb == 8) *reinterpret_cast<uint2 *>(dst + ((int64_t)f << lg)) = *reinterpret_cast<const uint2 *>(v);
            else *reinterpret_cast<uint32_t *>(dst + ((int64_t)f << lg)) = *reinterpret_cast<const uint32_t *>(v);
        }
        return;
    }
    // wider columns: 16-byte destination pieces, P per column (a power of two)
    const int lp = lg - (__ffs(kV) - 1);  // log2 of pieces per column
    const int total = N << lp;
    for (int u = threadIdx.x; u < total; u += blockDim.x) {
        const int f = u >> lp, pc = u & ((1 << lp) - 1);
        __align__(16) E v[kV];
#pragma unroll
        for (int i = 0; i < kV; ++i) {
            const int p = s_map[pc * kV + i];
            v[i] = p < 0 ? E(0) : src[(((int64_t)(p >> lg) * N + f) << lg) + (p & (TR - 1))];
        }
        *reinterpret_cast<uint4 *>(dst + ((int64_t)f << lg) + pc * kV) = *reinterpret_cast<const uint4 *>(v);
    }
}

__global__ void __launch_bounds__(kCopyThreads)
    k_copy_rows(const NetDev *__restrict__ nets, int nnets, unsigned long long *launches) {
    count_launch(launches);
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    int64_t rows_total = 0;
    for (int n = 0; n < nnets; ++n)
        if (nets[n].layout < 2) rows_total += nets[n].st->copy_R;
    // row-major and MMA-tile nets: one warp per kept row, lanes over its
    // 16-byte pieces (8 features for 16-bit types, 4 for FP32)
    const int lane = threadIdx.x & 31;
    const int64_t gw = tid >> 5, nw = nth >> 5;
    for (int64_t w = gw; w < rows_total; w += nw) {
        int64_t u = w;
        int n = 0;
        for (; n < nnets; ++n) {
            if (nets[n].layout >= 2) continue;
            if (u < nets[n].st->copy_R) break;
            u -= nets[n].st->copy_R;
        }
        const NetDev &nd = nets[n];
        const int N = nd.N, ib = nd.st->in_buf, q = (int)u;
        const int es = nd.prec == COSPDNN_PREC_FP32 ? 4 : 2, per = 16 / es;
        const int p = nd.cmap[q];
        const char *src = (const char *)nd.act[ib ^ 1];
        char *dst = (char *)nd.act[ib];
        for (int f = lane * per; f < N; f += 32 * per) {
            const uint4 v = *reinterpret_cast<const uint4 *>(src + act_index(nd.layout, N, p, f) * es);
            *reinterpret_cast<uint4 *>(dst + act_index(nd.layout, N, q, f) * es) = v;
        }
    }
    // row-tile nets: one CTA per destination tile (copy_tile)
    __shared__ int s_map[kCopyMaxTR];
    int64_t tiles = 0;
    for (int n = 0; n < nnets; ++n)
        if (nets[n].layout >= 2) tiles += (nets[n].st->copy_R + nets[n].layout - 1) / nets[n].layout;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        int64_t u = t;
        int n = 0;
        for (; n < nnets; ++n) {
            const NetDev &nd = nets[n];
            if (nd.layout < 2) continue;
            const int64_t cnt = (nd.st->copy_R + nd.layout - 1) / nd.layout;
            if (u < cnt) break;
            u -= cnt;
        }
        if (nets[n].prec == COSPDNN_PREC_FP32) copy_tile<float>(nets[n], (int)u, s_map);
        else copy_tile<uint16_t>(nets[n], (int)u, s_map);
    }
}

// ---- packed result for asynchronous copies --------------------------------
// buf: int64 count, int64 alive[L], int32 categories[rows]
__global__ void k_result_pack(const NetDev *__restrict__ nd_p, long long *__restrict__ buf) {
    const NetDev &nd = *nd_p;
    const int layer = nd.st->layer, R = nd.st->R;
    const int cnt = (nd.st->done && layer >= nd.L) ? R : 0;
    int32_t *cats = (int32_t *)(buf + 1 + nd.L);
    const int32_t *src = nd.orig[layer & 1];
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    if (tid == 0) buf[0] = cnt;
    for (int l = tid; l < nd.L; l += nth) buf[1 + l] = nd.alive_count[l];
    for (int q = tid; q < cnt; q += nth) cats[q] = src[q];
}

}  // namespace cospdnn
