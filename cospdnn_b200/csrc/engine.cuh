// Device-side data of the whole-network engine (shared by engine.cu and the
// layer kernels).
#pragma once

#include <cstring>
#include <type_traits>
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
    // The same entries for the FP64 replay when every weight of the layer
    // has one FP32 value and N <= 65536: 16-bit input indices [K][N] (real
    // entries only, ascending, rp_cnt[j] of them) and that value.
    const uint16_t *rp_idx;
    const uint16_t *rp_cnt;
    float rp_w;
    // tcgen05 schedule (16x16 aligned blocks of W, built by tc_build_blocks):
    // output block columns are taken in chunks of up to 32 (one TMEM
    // accumulator of 16 columns each); within a chunk the MMAs are ordered by
    // input block and split into stages, each stage = one contiguous run of
    // input blocks (a_count <= 8, one bulk copy of the A tiles) + its MMAs'
    // B operands (contiguous in tc_b, one bulk copy).
    //   tc_chunk_ptr[h]..[h+1]  stages of chunk h
    //   tc_stage[s]             {a_first, a_count, b_first, n_mma}
    //   tc_code[b]              MMA b: bits 0-2 A block within the run,
    //                           bits 3-7 accumulator (column within the chunk),
    //                           bit 8 first MMA into that accumulator
    //   tc_b                    B operands, 512 bytes each, in stage order
    //   tc_used[h]              bit j: column j of chunk h has any weight
    const int32_t *tc_chunk_ptr;
    const int4 *tc_stage;
    const uint16_t *tc_code;
    const void *tc_b;
    const uint32_t *tc_used;
    int tc_nchunks;
    int max_blocks;  // max 16x16 blocks in one output block column (error bound)
    // CUDA-core tile kernel (k_layer_cc): per output j, cc_k entries (input
    // column, weight in the compute type) in a build-time order, padding
    // included; 16-byte groups of entries stored group-major, [group][j]
    // (16-bit nets: 4 entries of col << 16 | w; FP32 nets: 2 entries of
    // {col, w bits}; compact nets: 8 entries of a 16-bit col, the weight being
    // cc_wconst and padding pointing at a zero column), so consecutive
    // outputs are adjacent.
    const uint4 *cc_w;
    int cc_k;
    uint32_t cc_wconst;  // compact entry lists (NetDev::cc_compact): the layer's one weight value, its
                         // bits in the compute type (16-bit types in the low half)
    // Feature-split tile kernel (k_layer_cs, NetDev::cc_split): the inputs
    // are split in two halves by bit cs_bit of the feature index (CTA h of a
    // cluster holds the features whose bit is h, in ascending order).  Per
    // half h, round k, warp w, column t < cs_cnt, slot s and lane, one 16-byte
    // entry group at cs_w[((((h * rounds + k) * 16 + w) * cs_cnt + t) * 4 + s)
    // * 32 + lane] for output lane of group s * rounds * 16 + 16 k + w (groups
    // of 32 outputs, padded to a multiple of 64): compact lists four byte
    // offsets of the inputs' 2-row words in the CTA's tile, else two
    // {offset, weight bits} pairs.
    const uint4 *cs_w;
    int cs_cnt;
    int cs_bit;
    float S;         // max_j sum_i |W_ij|
    float dW;        // max_j sum_i |W'_ij - W_ij|, W' = weights in the compute type
};

struct NetState {
    int layer;   // next layer to compute
    int R;       // rows entering `layer` (rows 0..R-1 of its input buffer)
    int done;    // finished (all rows pruned or all layers computed)
    int nunc;    // rows of this layer whose keep/prune decision needs the FP64 replay
    int err;     // device-side error code (0 = ok)
    int in_buf;  // act[in_buf] is the input of `layer` (layer 0 reads y0)
    int copy_R;  // rows the pending compaction copies (0 = none pending)
    int l0_bits; // layer 0 of this run was computed by the bit-count kernel
    int gather;  // input row q of `layer` is row cmap[q] of act[in_buf] (row-tile nets: the
                 // layer kernel's staging does the compaction, no copy)
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
    int layout;              // activation layout: 0 row-major, 1 MMA tiles, >= 2 row tiles (see act_index)
    int cc_compact;          // row-tile nets: 16-bit entries (input column only), every layer one weight value
    int cc_split;            // row tiles of 2 rows split over the two CTAs of a cluster by feature (k_layer_cs)
    void *act[2];            // ping-pong activations, rows padded to a multiple of 128
    int32_t *cmap;           // [rows] compaction map: new row q <- output row cmap[q]
    int32_t *orig[2];        // list: original row id
    float *err[2];           // list: bound on |Y(fast) - Y(FP64)| of the row's inputs
    float *mx[2];            // list: max |Y(fast)| of the row's inputs
    uint32_t *stat;          // [rows][3]: ordered max z, e_out bits, m_out bits
    int8_t *cls;             // [rows] 0 prune, 1 keep, 2 uncertain
    int32_t *ulist;          // [rows] uncertain positions
    int32_t *ccount;         // [rows / kCompactChunk, rounded up] kept rows per chunk of this layer
    long long *alive_count;  // [L] rows kept after layer l
    long long *recheck_count;// [L] rows re-decided in FP64 at layer l
    NetState *st;
    // layer 0 by bit counting (bits_layer.cu): binary inputs as bit planes
    // [(rows+31)/32][N] words, a flag raised when the current input is not
    // binary, and the schedule of layer 0 (l0_k steps per output, 0 = the
    // layer does not qualify: not one weight value per output)
    const uint32_t *y0bits;
    const int *y0nonbin;
    const uint4 *l0_idx;     // [N/32][l0_k/8][32] x 8 input indices (16 bits)
    const float *l0_w;       // [N] the output's weight in the compute type
    int l0_k;
    int l0_small;            // every layer-0 output has |z| <= 16 (max_j |w_j| nnz_j + |bias|)
};

enum { CLS_PRUNE = 0, CLS_KEEP = 1, CLS_UNCERTAIN = 2 };

// Limits of the device-side waits and of the layer loop, in engine memory and
// read by the kernels at every launch (cospdnn_engine_set_test_limits changes
// them between runs so that tests can make a bounded wait or the loop guard
// run out and check the error path).
struct DevLimits {
    long long wait_cycles;  // bounded mbarrier waits of k_layer_tc and k_layer_cs (SM clock cycles)
    int max_iters;          // layer-loop iterations before the guard stops the run
    int withhold_stage;     // 1: CTA 0 of k_layer_tc issues no copy for its first stage, and CTA 0 of
                            // k_layer_cs's first cluster does not send its first partial sums
};
constexpr long long kDefaultWaitCycles = 4000000000LL;  // about 2 s at 1.9 GHz

// Rows per compaction chunk (one CTA of k_compact; a multiple of 32).
constexpr int kCompactChunk = 1024;

// Element index of (row, feature) in an activation buffer of width N.
// layout 0, row-major: row*N + f.
// layout 1, MMA tiles (tcgen05 nets): rows in tiles of 128 and features in
// blocks of 16; each (tile, block) is a contiguous 4 KB operand in the
// canonical K-major core-matrix order of tcgen05 (8 rows x 16 bytes per core
// matrix, the two 8-feature halves 128 bytes apart, 8-row groups 256 bytes
// apart), so one bulk copy brings a whole MMA A operand into shared memory
// and the epilogue writes one output block as one such operand.
// layout TR >= 2 (a power of two), row tiles (CUDA-core tile kernel): rows in
// tiles of TR, feature-major inside a tile: (tile*N + f)*TR + row%TR, so a
// tile is one contiguous block and the TR values of one feature are adjacent.
__host__ __device__ __forceinline__ int64_t act_index(int layout, int N, int64_t row, int f) {
    if (layout == 0) return row * N + f;
    if (layout == 1) {
        const int64_t tile = row >> 7;
        const int m = (int)(row & 127), fb = f >> 4, k = f & 15;
        return (tile * (N >> 4) + fb) * 2048 + (m >> 3) * 128 + (k >> 3) * 64 + (m & 7) * 8 + (k & 7);
    }
    const int64_t tile = row / layout;
    return (tile * N + f) * layout + (row - tile * layout);
}

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
    // CUDA-core kernels: one FMA rounding per term (zero-weight padding is
    // exact) and one for the bias; the feature-split kernel sums each half's
    // terms (at most K - 1 of them when both halves have some) and adds the
    // two sums, so a term still sees at most K + 1 roundings.  tcgen05:
    // accumulation order inside the MMA is not specified, so allow two
    // roundings for every product of every block plus the bias.
    return n.kernel == COSPDNN_KERNEL_TCGEN05 ? 2.0 * (16.0 * lw.max_blocks + 2.0) : (double)(lw.K + 2);
}

// Bound on |stored - clamped| for a value c in [0, 32] stored in the compute
// type: half an ulp, at most 2^-11 c + 2^-25 (FP16; 2^-25 covers the
// subnormal range) or 2^-8 c + 2^-126 (BF16, more than its subnormal half
// spacing); 0 for FP32.
template <typename T>
__device__ __forceinline__ float store_error(float c) {
    if constexpr (sizeof(T) == 4) return 0.0f;
    else if constexpr (std::is_same<T, __half>::value) return __fmaf_ru(c, 4.8828125e-04f, 2.98023224e-08f);
    else return __fmaf_ru(c, 3.90625e-03f, 1.17549435e-38f);
}

// Row statistics from the row's max pre-activation zm, its min |z - 16|
// over the outputs (zd) and its error bound ez:
//   max output  = the stored value of clamp(zm) (rounding is monotone, so
//                 this is the max of the stored outputs);
//   output error: outputs with z <= -ez are 0 in both recurrences and those
//                 with z >= 32 + ez are 32 in both; the others, those with
//                 |z - 16| < 16 + ez (there are some iff zd < 16 + ez), are
//                 within ez of the exact clamp plus their storage rounding,
//                 at most clamp(zm): bound ez + store_error(clamp(zm)), else 0.
template <typename T>
__device__ __forceinline__ void row_stats(float zm, float zd, float ez, float &emax, float &ymax) {
    const float c = clamp32(zm);
    ymax = act_traits<T>::to_f(act_traits<T>::from_f(c));
    emax = zd < 16.0f + ez ? __fadd_ru(ez, store_error<T>(c)) : 0.0f;
}

}  // namespace cospdnn
