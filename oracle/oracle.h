/*
 * CPU oracle for the CoSpDNN sparse-DNN layer path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library calls this code;
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * --impl reference legs load it, and only as the checker or the CPU baseline.
 *
 * What it restates (reference paths are relative to the CoSpDNN repository):
 *   - the greedy BCSC block builder  src/utils/matrix.h:1200-1269 (coo2bcsc),
 *     including its placement of the first value of a new block at offset 0;
 *   - the arithmetic of the reference layer kernel cospdnn_single
 *     src/kernels/kernel.cu:240-379 (two blocks per block column, value
 *     [k*16+r] used as the weight from input row_start+k to output bid*16+r,
 *     bias then clamp to [0,32] as in src/kernels/kernel.cuh:132-136);
 *   - the recurrence Y_{l+1} = clamp(Y_l W_l + b, 0, 32) with the W row =
 *     input, W column = output convention of src/utils/matrix.h:282-289 and
 *     src/utils/cpu_spmm_fuse.h:17-79 (with a float bias, not that file's int);
 *   - the row pruning rule "row alive if any output > 1e-5"
 *     src/kernels/kernel.cu:129-139 and the compaction order of
 *     src/cospdnn.cu:251-262 (surviving rows keep ascending order).
 *
 * FP64 summation order (fixed, replayed bit-for-bit by the GPU recheck):
 * for each output j, acc = +0.0; for each nonzero W[i][j] in ascending input
 * index i with Y[i] != 0: acc = acc + (double(W[i][j]) * Y[i]) (separately
 * rounded multiply and add, no FMA); z = acc + double(bias);
 * y = z < 0 ? 0 : (z > 32 ? 32 : z).
 *
 * Parity pinning: the BCSC restatement is checked against the reference's own
 * builder compiled from its sources (oracle/ref_bcsc_dump.cpp, golden fixtures
 * in tests/golden/); the layer restatement is checked on a B200 against the
 * reference's own kernel compiled from its sources (oracle/ref_kernel_shim.cu).
 */
#ifndef COSPDNN_ORACLE_H
#define COSPDNN_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- seeded synthetic data (SplitMix64 streams) ---- */
uint64_t orc_stream_seed(uint64_t seed, uint64_t a, uint64_t b, uint64_t c);
/* nmask distinct masks drawn uniformly from [0, neuron); neuron a power of two. */
int orc_xor_masks(uint64_t seed, int net, int layer, int neuron, int nmask, int32_t *masks);
/* 32 masks {16*h0+t, 16*h1+t : t<16}, h0 != h1 < neuron/16 (reference-compatible
 * config: every 16-aligned output group has exactly two dense aligned blocks). */
int orc_r1_masks(uint64_t seed, int net, int layer, int neuron, int32_t *masks);
/* Binary input rows: row r density d_r ~ U[dlo, dhi), each entry Bernoulli(d_r).
 * Row r depends only on (seed, net, row0 + r), so samples are prefixes. */
void orc_input_binary(uint64_t seed, int net, int64_t row0, int64_t rows, int neuron,
                      double dlo, double dhi, uint8_t *y0);
/* Uneven multi-network mix: neuron from choices[], layers from lchoices[],
 * batch ~ U[bmin, bmax]. */
void orc_mix_config(uint64_t seed, int nnet, const int *nchoices, int nn, const int *lchoices,
                    int nl, int bmin, int bmax, int *neuron, int *layers, int *batch);

/* XOR-mask weights in CSC form: output j <- inputs j^m_k, ascending input index. */
void orc_masks_to_csc(const int32_t *masks, int nmask, int neuron, float val,
                      int32_t *colptr /*neuron+1*/, int32_t *rowidx /*neuron*nmask*/,
                      float *vals /*neuron*nmask*/);

/* ---- reference BCSC builder (src/utils/matrix.h:1200-1269) ----
 * Input COO (row = input, col = output).  Output arrays are malloc'ed; free
 * with orc_free.  Returns 0 on success. */
int orc_bcsc_greedy(int64_t nnz, const int32_t *row, const int32_t *col, const float *val,
                    int bc, int br, int32_t **col_ptr, int32_t *n_col_ptr,
                    int32_t **row_index, int32_t *n_blocks, int32_t **col_index,
                    float **values);
void orc_free(void *p);

/* ---- one layer in the reference kernel's arithmetic (src/kernels/kernel.cu:240-379) ----
 * a: [2*neuron][batch] (hi rows then lo rows, as float); values: blocks of
 * 256; writes c: [neuron][batch]. Double accumulation (the kernel accumulates
 * in FP32 on mma.sync; comparisons use a tolerance). */
void orc_ref_layer(const float *a, const float *values, float *c, const int32_t *fuse,
                   const int32_t *idx_ptr, const int32_t *index, float bias, int batch,
                   int neuron);

/* ---- one layer of the true BCSC product, any block count per column ----
 * c[o][b] = clamp(bias + sum_blocks sum_{co,ro} V[co*bc+ro] * a[fuse[rs+ro]][b]),
 * o = col_start + co, where col_start = 16-aligned block column bid*bc.
 * a: [neuron][batch] float; double accumulation; rows rs+ro >= neuron skipped. */
void orc_bcsc_layer(const float *a, const float *values, float *c, const int32_t *fuse,
                    const int32_t *idx_ptr, const int32_t *index, int nblockcols, float bias,
                    int batch, int neuron, int bc, int br);

/* ---- FP64 recurrence over a batch (rows independent; OpenMP over rows) ----
 * colptr/rowidx/vals: per-layer CSC (ascending input index within a column).
 * y0_u8 (binary) or y0_f32 (general) row-major [rows][neuron]; exactly one non-null.
 * Outputs:
 *   death[r]  = first layer l whose output row has max <= tau (row pruned after
 *               layer l), or `layers` if the row survives all layers;
 *   maxval    (optional) [rows*layers] max output of each row per layer (0 after death);
 *   final_y   (optional) [rows][neuron] output of the last computed layer
 *               (the layer the row died at, or the final one).
 * Returns 0. */
int orc_infer_fp64(int neuron, int layers, int64_t rows, const int32_t *const *colptr,
                   const int32_t *const *rowidx, const float *const *vals, const uint8_t *y0_u8,
                   const float *y0_f32, float bias, double tau, int threads, int32_t *death,
                   double *maxval, double *final_y);

/* Replays rows through layers [0, upto] and returns their layer-`upto` outputs
 * in FP64 (same order as orc_infer_fp64); used by tests of the GPU recheck. */
int orc_replay_fp64(int neuron, int upto, int64_t nrows, const int64_t *row_ids,
                    const int32_t *const *colptr, const int32_t *const *rowidx,
                    const float *const *vals, const uint8_t *y0_u8, const float *y0_f32,
                    float bias, double *out);

/* ---- CPU baseline: FP32 CSR scatter recurrence, OpenMP over rows, early exit ----
 * rowptr/colidx/vals: per-layer CSR (row = input).  Returns alive-row count
 * after the last layer; death[] as above (optional). */
int64_t orc_infer_fp32_csr(int neuron, int layers, int64_t rows, const int32_t *const *rowptr,
                           const int32_t *const *colidx, const float *const *vals,
                           const uint8_t *y0_u8, float bias, float tau, int threads,
                           int32_t *death);

#ifdef __cplusplus
}
#endif
#endif
