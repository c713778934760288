/*
 * cospdnn_b200 -- C ABI of the B200 (sm_100a) sparse-DNN inference engine.
 *
 * Plain pointers and sizes only.  Every function returns a status code
 * (COSPDNN_OK == 0) instead of exiting the process as the reference's
 * Safe_Call does (src/gpu_lib/gpu_runtime.h:6-17); cospdnn_last_error()
 * gives the message of the calling thread's last failure.  Device pointers
 * are CUDA device memory of the current device; `stream` is a cudaStream_t
 * (NULL = legacy default stream).  Reference paths are relative to the
 * CoSpDNN repository.
 */
#ifndef COSPDNN_B200_H
#define COSPDNN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    COSPDNN_OK = 0,
    COSPDNN_ERR_INVALID = 1,     /* bad argument */
    COSPDNN_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    COSPDNN_ERR_NOMEM = 3,       /* device or host allocation failed */
    COSPDNN_ERR_STATE = 4,       /* call out of order (e.g. run before build) */
    COSPDNN_ERR_DEVICE = 5,      /* a device-side check failed (bounds, loop guard) */
    COSPDNN_ERR_UNSUPPORTED = 6  /* shape or option this build does not handle */
};

/* Message of the calling thread's last failing call ("" if none). */
const char *cospdnn_last_error(void);
/* Library version as major*10000 + minor*100 + patch. */
int cospdnn_version(void);

/* ------------------------------------------------------------------------
 * Layer entry.  Replaces ftxj::cospdnn_single (src/kernels/kernel.cuh:179-189,
 * launched at src/cospdnn.cu:219-229) with the same argument meaning:
 *   A        activations, feature-major, batch contiguous:
 *            default: half [2*neuron][batch], rows 0..neuron-1 the hi parts and
 *            rows neuron..2*neuron-1 the lo parts (src/kernels/kernel.cu:140-152);
 *            COSPDNN_LAYER_A_FLOAT: float [neuron][batch].
 *   B        block values, blocksize_c*blocksize_r per block, value
 *            [col_off*blocksize_c + row_off] (src/utils/matrix.h:1245);
 *            half by default (src/cospdnn.cu:46-56), float with COSPDNN_LAYER_B_FLOAT.
 *   C        float [neuron][batch], every row of every block column written.
 *   fuse     activation row of each weight row (src/cospdnn.cpp:14-44).
 *   idx_ptr  block-column pointer (bcsc_len_), nblockcols+1 entries.
 *   index    start row of each block (bcsc_row_index_).
 *   Output column o = bid*blocksize_c + col_off (block columns are taken as
 *   blocksize_c-aligned, as the reference kernel's output indexing does).
 * Default arithmetic: the true product over every block of the column,
 *   C[o][b] = clamp(bias + sum_blocks sum_ro V[co*bc+ro] * A[fuse[start+ro]][b], 0, 32),
 *   hi+lo summed, FP32 accumulation; weight rows >= neuron are skipped.
 * COSPDNN_LAYER_REFERENCE_ARITH reproduces the reference kernel's arithmetic
 *   instead: only the two blocks starting at idx_ptr[bid], and value
 *   [k*16 + r] applied from input row start+k to output bid*16+r
 *   (src/kernels/kernel.cu:257,306-331,371-375); requires blocksize 16.
 * batch need not be a multiple of 128.  Asynchronous on `stream`.
 */
#define COSPDNN_LAYER_A_FLOAT 0x1u
#define COSPDNN_LAYER_B_FLOAT 0x2u
#define COSPDNN_LAYER_REFERENCE_ARITH 0x4u
int cospdnn_layer(const void *A, const void *B, float *C, const int *fuse, const int *idx_ptr,
                  const int *index, float bias, int batch, int neuron, int blocksize_c,
                  int blocksize_r, int nblockcols, unsigned flags, void *stream);

/* ------------------------------------------------------------------------
 * Pruning entry.  Replaces check_active_f_col (src/kernels/kernel.cu:129-139),
 * the host compaction loop (src/cospdnn.cu:240-270) and matrix_reshape
 * (src/kernels/kernel.cu:156-172) with one device-side pass, no host round trip:
 *   column k of C ([neuron][batch] float) survives if any C[n][k] > threshold
 *   (the reference uses 1e-5);
 *   survivors keep ascending order: category[j] = k of the j-th survivor,
 *   map_out[j] = map_in[k] (map_in NULL = identity), *count_dev = survivors;
 *   A_out [neuron][stride], stride = count rounded up to a multiple of 128,
 *   gets the surviving columns and zero padding; with COSPDNN_PRUNE_OUT_HALF_HILO
 *   A_out is half [2*neuron][stride] hi/lo rows, ready for cospdnn_layer.
 * A_out needs room for batch columns rounded up to a multiple of 128,
 * category and map_out for batch entries.  `workspace` is
 * device memory of cospdnn_prune_workspace_bytes(batch) bytes, owned by the
 * caller.  Asynchronous; read *count_dev after synchronizing.
 */
#define COSPDNN_PRUNE_OUT_HALF_HILO 0x1u
size_t cospdnn_prune_workspace_bytes(int batch);
int cospdnn_prune_compact(const float *C, int neuron, int batch, float threshold, void *A_out,
                          int *category, const int *map_in, int *map_out, int *count_dev,
                          unsigned flags, void *workspace, size_t workspace_bytes, void *stream);

/* Allocation-free variant of cospdnn_prune_compact (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc: code that must not
 * implicitly synchronize the device (cudaMalloc/cudaFree can), code whose
 * device memory is owned by another allocator or fixed budget, or code that
 * simply has no place to keep a workspace between calls.  Same arguments and
 * results as cospdnn_prune_compact minus the workspace: the per-column flags
 * live in a file-scope device array of 1048576 ints (4 MiB), held on every
 * GPU that loads this library until the process exits; batch > 1048576 is
 * rejected with COSPDNN_ERR_INVALID.  The first call on a device looks up
 * that array's device address (cudaGetSymbolAddress, with the device
 * current), so make the first call on each device before any stream capture;
 * that address is kept for the life of the process, so the entry is not for
 * use on a device after cudaDeviceReset (the library's module is then loaded
 * again at a new address).  Every call clears the flags it uses; all calls share the one array, so
 * calls that overlap on the GPU (other streams, other threads) race.  No
 * cudaMalloc, cudaFree or other allocating call is made. */
int cospdnn_prune_compact_noalloc(const float *C, int neuron, int batch, float threshold,
                                  void *A_out, int *category, const int *map_in, int *map_out,
                                  int *count_dev, unsigned flags, void *stream);

/* ------------------------------------------------------------------------
 * Whole-network engine.  Replaces the host layer loop test_graph_challenge_tc
 * (src/cospdnn.cu:3-369) and the two-network path test_graph_challenge_tc_co
 * (src/cospdnn_double.cu:208-1214): any number of networks of any sizes run
 * in one captured CUDA graph whose device-side loop advances every live
 * network by one layer per iteration and stops when all are finished.
 * Each network computes Y_{l+1} = clamp(Y_l W_l + bias, 0, 32); a row is
 * pruned after the first layer whose outputs are all <= threshold; the
 * categories are the original ids of the rows alive after the last layer.
 * Rows whose keep/prune decision is within the proven error bound of the
 * fast precision are re-decided by an exact FP64 replay from Y0, so the
 * categories equal those of the FP64 recurrence.
 */
typedef struct cospdnn_engine cospdnn_engine;

#define COSPDNN_PREC_FP32 0 /* FP32 activations, CUDA-core kernel */
#define COSPDNN_PREC_FP16 1 /* FP16 activations, FP32 accumulation */
#define COSPDNN_PREC_BF16 2 /* BF16 activations, FP32 accumulation */

#define COSPDNN_KERNEL_AUTO 0      /* chosen at build from the weights: tcgen05 for FP16/BF16 when the
                                      16x16 blocks are at least 1/4 full or the row tile does not fit
                                      shared memory, else CUDA cores; FP32 on CUDA cores */
#define COSPDNN_KERNEL_CUDA_CORE 1 /* gather-FMA kernel, any precision */
#define COSPDNN_KERNEL_TCGEN05 2   /* tcgen05 block MMA kernel (FP16/BF16) */

typedef struct {
    int neuron;      /* features per layer */
    int layers;      /* number of layers */
    int rows;        /* input rows (batch) */
    float bias;      /* bias of every neuron (reference table src/cospdnn.cpp:97-102) */
    float threshold; /* prune rule: row alive if any output > threshold (reference 1e-5) */
    int precision;   /* COSPDNN_PREC_* */
    int kernel;      /* COSPDNN_KERNEL_* */
} cospdnn_net_desc;

int cospdnn_engine_create(cospdnn_engine **out, int device);
void cospdnn_engine_destroy(cospdnn_engine *e);
int cospdnn_engine_add_net(cospdnn_engine *e, const cospdnn_net_desc *d, int *net_id);
/* W_l in CSC form (row = input, column = output; src/utils/matrix.h:282-289),
 * host arrays, rows ascending within each column. */
int cospdnn_engine_set_layer_csc(cospdnn_engine *e, int net, int layer, const int32_t *colptr,
                                 const int32_t *rowidx, const float *vals);
/* W_l in the reference's BCSC form (host arrays from BCSRCSCMatrix, values
 * [col_off*bs + row_off]) plus the layer's fuse row (NULL = identity).  Block
 * value [co*bs + ro] of block column bid is the weight from activation row
 * fuse[start + ro] to output bid*bs + co (the true product of cospdnn_layer's
 * default arithmetic); the engine folds the fuse into its own weight layout. */
int cospdnn_engine_set_layer_bcsc(cospdnn_engine *e, int net, int layer, const int32_t *col_ptr,
                                  int n_col_ptr, const int32_t *row_index, int n_blocks,
                                  const float *values, int blocksize, const int32_t *fuse);
/* Uploads weights, allocates every device buffer and captures the CUDA graph. */
int cospdnn_engine_build(cospdnn_engine *e);

#define COSPDNN_INPUT_U8 0   /* [rows][neuron] bytes (binary images) */
#define COSPDNN_INPUT_F32 1  /* [rows][neuron] float */
#define COSPDNN_INPUT_BITS 2 /* [rows][neuron/8] bytes, bit j%8 of byte j/8, LSB first */
/* Copies Y0 of one network (host pointer: pinned memory keeps it async; a
 * device pointer, on_device = 1, must be 16-byte aligned) and converts it to
 * the compute type.  Asynchronous on `stream`.  Inputs are
 * double buffered: this fills the network's back buffers and the next run
 * (cospdnn_engine_run / _run_timed / _profile_layers) makes them current,
 * so the next batch can be set on another stream while a run is in flight.
 * The caller orders set_input before the run that should use it (same
 * stream, or an event), and the second set_input after a run only after
 * the run before it has finished (the buffers alternate). */
int cospdnn_engine_set_input(cospdnn_engine *e, int net, const void *y0, int format,
                             int on_device, void *stream);
/* ------------------------------------------------------------------------
 * One call for the persistent multi-network launch (the whole host loop of
 * test_graph_challenge_tc / _co, src/cospdnn.cuh:14-35, for any number of
 * networks): an engine on `device` is built from each network's CSC layers,
 * the inputs are set, every network runs in one graph launch, and each
 * network's results are copied back; the engine is destroyed before the
 * call returns.  Networks given as BCSC + fuse rows go through
 * cospdnn_engine_set_layer_bcsc instead.  *ms (may be NULL) receives the
 * device time of the run, as cospdnn_engine_run_timed.
 */
typedef struct {
    cospdnn_net_desc desc;          /* sizes, bias, threshold, precision, kernel */
    const int32_t *const *colptr;   /* [layers] CSC column pointers, neuron + 1 each */
    const int32_t *const *rowidx;   /* [layers] row (input) indices */
    const float *const *vals;       /* [layers] weights */
    const void *y0;                 /* host rows in `format` (COSPDNN_INPUT_*) */
    int format;
    int32_t *categories;            /* out: surviving original rows, room for desc.rows */
    int64_t *count;                 /* out: number of categories */
    int64_t *alive_per_layer;       /* out (may be NULL): rows kept after each layer */
} cospdnn_network;
int cospdnn_run_networks(const cospdnn_network *nets, int n, int device, float *ms);

/* Number of CUDA devices visible to this process (0 when none, or on error);
 * replaces cudaGetDeviceCount in the reference's multi-GPU launcher
 * (src/cospdnn.cpp:155-163). */
int cospdnn_device_count(void);
/* Runs every network to completion: one graph launch, asynchronous. */
int cospdnn_engine_run(cospdnn_engine *e, void *stream);
/* cospdnn_engine_run bracketed by CUDA events on `stream`; waits for the run
 * and returns its device time in *ms.  Replaces the event timing around the
 * reference's layer loop that prints "Kernel Exec Time" (src/cospdnn.cu:303-310,
 * src/cospdnn_double.cu:1142). */
int cospdnn_engine_run_timed(cospdnn_engine *e, void *stream, float *ms);
/* Synchronizes `stream`, then copies results of one network to host memory:
 * categories (ascending original row ids, room for `rows`), their count,
 * alive rows after each layer (room for `layers`, may be NULL) and rows
 * re-decided in FP64 at each layer (may be NULL). */
int cospdnn_engine_result(cospdnn_engine *e, int net, int32_t *categories, int64_t *count,
                          int64_t *alive_per_layer, int64_t *rechecked_per_layer, void *stream);
/* Copies the activations of the last computed layer for the surviving rows
 * (in category order) into a host float buffer: min(max_rows, count) rows of
 * `neuron` floats are written (count as returned by cospdnn_engine_result;
 * nothing is written when it is 0), so `out` needs room for
 * min(max_rows, count) * neuron floats.  max_rows < 0 is rejected.  For checks. */
int cospdnn_engine_final_values(cospdnn_engine *e, int net, float *out, int64_t max_rows,
                                void *stream);
/* Runs the layer loop eagerly (as cospdnn_engine_profile_layers) until
 * network `net` has computed layer `layer` (0-based), then copies that
 * layer's outputs for the rows kept after it, in ascending original-row
 * order: min(max_rows, kept) rows of `neuron` floats into `out`, their
 * original row ids into `ids` (may be NULL), each row's proven bound on
 * |value - FP64 recurrence value| over its outputs into `bounds` (may be
 * NULL; the bound behind the exact keep/prune decisions), the row count into
 * *count (0 when every row was pruned at or before `layer`).  Replaces the reference's
 * -DPRINT_RESULT dump of C (src/cospdnn.cu:311-320) for any layer; for checks
 * against an FP64 recurrence.  The eager pass then runs on to the end, so
 * afterwards every network's cospdnn_engine_result and final values are
 * those of a complete run on the current inputs.  Synchronizes `stream`. */
int cospdnn_engine_layer_values(cospdnn_engine *e, int net, int layer, float *out, int32_t *ids,
                                float *bounds, int64_t max_rows, int64_t *count, void *stream);
/* Largest of the surviving rows' proven bounds on |final value - FP64
 * recurrence value| after the last run (0 when no row survived): the
 * maximum error of the result against an FP64 oracle of the same
 * recurrence, as the engine tracks it to decide every row exactly.
 * Synchronizes `stream`. */
int cospdnn_engine_final_bound(cospdnn_engine *e, int net, float *max_bound, void *stream);
/* What the engine resolved for network `net` at build and did in its last
 * run: *kernel the layer kernel (COSPDNN_KERNEL_CUDA_CORE or _TCGEN05, never
 * AUTO), *row_tile the rows per activation tile of the CUDA-core row-tile
 * kernel (0 for the tcgen05 MMA-tile layout and the row-major gather kernel;
 * 2 for an FP16/BF16 net: the feature-split kernel, whose 2-row tiles are
 * split by feature over the two CTAs of a cluster),
 * *layer0_counted 1 when layer 0 of the last run was computed by counting
 * the bits of a binary input.  Synchronizes `stream`. */
int cospdnn_engine_net_info(cospdnn_engine *e, int net, int *kernel, int *row_tile,
                            int *layer0_counted, void *stream);
/* Test hooks for the device-side failure paths (no counterpart in the
 * reference, whose Safe_Call exits the process, src/gpu_lib/gpu_runtime.h:6-17).
 * Every wait in the engine's kernels is bounded and the layer loop has an
 * iteration guard; when one runs out the run stops and
 * cospdnn_engine_result returns COSPDNN_ERR_DEVICE, and the next run starts
 * clean.  These set, for the following runs: wait_cycles, the limit of each
 * bounded wait of the tcgen05 and feature-split layer kernels in SM clock
 * cycles (0 = the default of 4e9, about 2 s; values below 1e6 are rejected);
 * max_iters, the layer-loop iterations after which the guard stops the run
 * (0 = the default of the deepest network's layers + 2); withhold_stage = 1
 * makes the first block of the tcgen05 layer kernel skip the copies of its
 * first stage, and the first block of the feature-split kernel skip its
 * first message to the other block of its cluster, so that the waits for
 * them run out (data that never arrives, made on purpose; no fault, no
 * hang).  (0, 0, 0) restores the defaults.
 * Synchronizes the device. */
int cospdnn_engine_set_test_limits(cospdnn_engine *e, long long wait_cycles, int max_iters,
                                   int withhold_stage);
/* Number of launches of this library's kernels the last run made (device
 * counter, read after synchronizing). */
int cospdnn_engine_launch_count(cospdnn_engine *e, int64_t *launches, void *stream);
/* Asynchronous result copy for end-to-end pipelines: after the run on `stream`,
 * packs one network's result and copies it to host_buf (pinned memory keeps it
 * asynchronous): int64 count, int64 alive_per_layer[layers], int32
 * categories[rows].  Needs 8*(1+layers) + 4*rows bytes. */
int cospdnn_engine_result_async(cospdnn_engine *e, int net, void *host_buf, size_t bytes,
                                void *stream);
/* Runs the same kernels as cospdnn_engine_run layer by layer from the host
 * (synchronizing after each layer) and times the layer kernels of each
 * iteration with CUDA events on `stream`: layer_ms[i] for iteration i (all
 * networks advance one layer per iteration), up to max_iters; *iters gets the
 * number of iterations.  Results equal those of cospdnn_engine_run. */
int cospdnn_engine_profile_layers(cospdnn_engine *e, void *stream, int max_iters,
                                  float *layer_ms, int *iters);

/* ------------------------------------------------------------------------
 * Synthetic Graph-Challenge-style input rows, generated on the GPU: row r
 * (global index row0 + r) of network `net` has density
 * d = dlo + (dhi-dlo)*u and element j = (u_j < d), from SplitMix64 streams
 * keyed by (seed, net, row).  format COSPDNN_INPUT_U8 writes [rows][neuron]
 * bytes, COSPDNN_INPUT_BITS [rows][neuron/8] packed bits.  Asynchronous.
 */
int cospdnn_synth_input(void *out, int64_t rows, int neuron, uint64_t seed, int net, int64_t row0,
                        double dlo, double dhi, int format, void *stream);

#ifdef __cplusplus
}
#endif
#endif
