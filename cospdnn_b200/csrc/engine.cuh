// Device-side data of the whole-network engine (shared by engine.cu and the
// layer kernels).
#pragma once

#include <cstring>
#include <vector>

#include "common.cuh"

namespace cospdnn {

// A kernel launch described once and used both as a graph node and as an
// eager launch (argument values are owned by the spec).
struct KSpec {
    void *fn = nullptr;
    dim3 grid, block;
    size_t smem = 0;
    std::vector<std::vector<char>> vals;
    std::vector<void *> args;
    template <typename T>
    KSpec &arg(const T &v) {
        vals.emplace_back(sizeof(T));
        std::memcpy(vals.back().data(), &v, sizeof(T));
        return *this;
    }
    void **params() {
        args.clear();
        for (auto &v : vals) args.push_back(v.data());
        return args.data();
    }
};

// One layer of one network, device pointers.
struct LayerDev {
    // ELL-by-output view of W (used by the CUDA-core kernel and the FP64
    // replay): for output j, entries k < K at [k*N + j], ascending input
    // index, zero-weight padding at the end (index 0).
    const int32_t *ell_idx;
    const float *ell_val;
    int K;
    // 16x16 aligned block view (tcgen05 kernel): output block column c has
    // blocks blk_ptr[c]..blk_ptr[c+1]; blk_row[b] is the input block (rows
    // 16*blk_row .. +16); blk_b holds each block as the MMA B operand
    // (16 outputs x 16 inputs, K-major, 512 bytes per block).
    const int32_t *blk_ptr;
    const int32_t *blk_row;
    const void *blk_b;
    int max_blocks;  // max blocks in one output block column
    float S;         // max_j sum_i |W_ij|
    float dW;        // max_j sum_i |W'_ij - W_ij|, W' = weights in the compute type
};

struct NetState {
    int layer;  // next layer to compute
    int R;      // rows entering `layer`
    int done;   // finished (all rows pruned or all layers computed)
    int nunc;   // rows of this layer whose keep/prune decision needs the FP64 replay
    int err;    // device-side error code (0 = ok)
    int pad[3];
};

struct NetDev {
    int N, L, rows, prec;  // prec: COSPDNN_PREC_*
    int kernel;            // resolved COSPDNN_KERNEL_* (never AUTO here)
    float bias, tau;
    const LayerDev *layers;  // [L]
    const void *y0;          // [rows][N] in the compute type
    const float *y0_f32;     // exact input when the compute type cannot hold it (else NULL)
    const float *err0;       // [rows] bound on |y0(compute) - y0(exact)|
    const float *mx0;        // [rows] max |y0|
    void *act[2];            // [rows][N] ping-pong activations
    int32_t *pos[2];         // list: row position in the layer's input buffer
    int32_t *orig[2];        // list: original row id
    float *err[2];           // list: bound on |Y(fast) - Y(FP64)| of the row's inputs
    float *mx[2];            // list: max |Y(fast)| of the row's inputs
    uint32_t *stat;          // [rows][3]: ordered max z, e_out bits, m_out bits
    int8_t *cls;             // [rows] 0 prune, 1 keep, 2 uncertain
    int32_t *ulist;          // [rows] uncertain positions
    long long *alive_count;  // [L] rows kept after layer l
    long long *recheck_count;// [L] rows re-decided in FP64 at layer l
    NetState *st;
};

enum { CLS_PRUNE = 0, CLS_KEEP = 1, CLS_UNCERTAIN = 2 };

// Counts kernel launches of a run (one atomic per launch, block 0 thread 0).
__device__ __forceinline__ void count_launch(unsigned long long *launches) {
    if (launches && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(launches, 1ull);
}

// Bound on |z_fast - z_FP64| for one row of layer `lw` (z = pre-activation).
//   e_in  bound on the row's input error, m_in max |input| (fast values)
//   steps number of roundings in the fast accumulation of one output
// |sum_fast - sum_exact| <= steps * 2^-24 * (sum |w||y| + |b|) with
// sum |w||y| <= S * m_in; the FP64 recurrence itself is within
// 40 * 2^-53 * (S*(m_in+e_in) + |b|) of exact; input and weight errors add
// S*e_in and dW*(m_in+e_in).  Rounded up.
__device__ __forceinline__ float z_error_bound(float e_in, float m_in, float S, float dW, float bias,
                                               double steps) {
    const double u32 = 5.9604644775390625e-08;       // 2^-24
    const double u64 = 1.1102230246251565e-16;       // 2^-53
    const double ab = fabs((double)bias);
    const double T = (double)S * (double)m_in;
    const double eacc = steps * u32 * (T + ab);
    const double e64 = 40.0 * u64 * ((double)S * ((double)m_in + (double)e_in) + ab);
    const double ez = (double)S * e_in + (double)dW * ((double)m_in + (double)e_in) + eacc + e64;
    return __double2float_ru(ez * (1.0 + 1e-9));
}

// Roundings per output of each fast kernel (see z_error_bound).
__device__ __forceinline__ double fast_steps(const NetDev &n, const LayerDev &lw) {
    // CUDA-core: one FMA rounding per term and one for the bias.  tcgen05:
    // accumulation order inside the MMA is not specified, so allow two
    // roundings for every product of every block plus the bias.
    return n.kernel == COSPDNN_KERNEL_TCGEN05 ? 2.0 * (16.0 * lw.max_blocks + 2.0) : (double)(lw.K + 2);
}

}  // namespace cospdnn
