/*
 * CPU oracle for the CoSpDNN sparse-DNN layer path -- TEST INFRASTRUCTURE.
 * See oracle.h for what each function restates and where in the reference.
 * Built with -ffp-contract=off so the FP64 recurrence has separately rounded
 * multiplies and adds (the GPU recheck replays exactly that order).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* SplitMix64 (Steele, Lea & Flood, "Fast splittable pseudorandom number
 * generators", OOPSLA 2014).                                          */
static inline uint64_t sm64(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static inline double u01(uint64_t *s) { return (double)(sm64(s) >> 11) * (1.0 / 9007199254740992.0); }

uint64_t orc_stream_seed(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) {
    uint64_t s = seed ^ 0x5851F42D4C957F2DULL;
    uint64_t x = sm64(&s);
    s = x ^ (a + 0x632BE59BD9B4E019ULL);
    x = sm64(&s);
    s = x ^ (b + 0x9E3779B97F4A7C15ULL);
    x = sm64(&s);
    s = x ^ (c + 0xD1B54A32D192ED03ULL);
    return sm64(&s);
}

enum { STREAM_MASKS = 1, STREAM_INPUT = 2, STREAM_MIX = 3, STREAM_R1 = 4 };

int orc_xor_masks(uint64_t seed, int net, int layer, int neuron, int nmask, int32_t *masks) {
    if (neuron <= 0 || nmask <= 0 || nmask > neuron) return -1;
    uint64_t s = orc_stream_seed(seed, STREAM_MASKS, (uint64_t)net, (uint64_t)layer);
    int n = 0;
    while (n < nmask) {
        int32_t m = (int32_t)(sm64(&s) % (uint64_t)neuron);
        int dup = 0;
        for (int k = 0; k < n; ++k) dup |= (masks[k] == m);
        if (!dup) masks[n++] = m;
    }
    return 0;
}

int orc_r1_masks(uint64_t seed, int net, int layer, int neuron, int32_t *masks) {
    int nb = neuron / 16;
    if (nb < 2) return -1;
    uint64_t s = orc_stream_seed(seed, STREAM_R1, (uint64_t)net, (uint64_t)layer);
    int h0 = (int)(sm64(&s) % (uint64_t)nb), h1;
    do { h1 = (int)(sm64(&s) % (uint64_t)nb); } while (h1 == h0);
    for (int t = 0; t < 16; ++t) {
        masks[t] = 16 * h0 + t;
        masks[16 + t] = 16 * h1 + t;
    }
    return 0;
}

void orc_input_binary(uint64_t seed, int net, int64_t row0, int64_t rows, int neuron,
                      double dlo, double dhi, uint8_t *y0) {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < rows; ++r) {
        uint64_t s = orc_stream_seed(seed, STREAM_INPUT, (uint64_t)net, (uint64_t)(row0 + r));
        double d = dlo + (dhi - dlo) * u01(&s);
        uint8_t *y = y0 + r * (int64_t)neuron;
        for (int j = 0; j < neuron; ++j) y[j] = (uint8_t)(u01(&s) < d);
    }
}

void orc_mix_config(uint64_t seed, int nnet, const int *nchoices, int nn, const int *lchoices,
                    int nl, int bmin, int bmax, int *neuron, int *layers, int *batch) {
    uint64_t s = orc_stream_seed(seed, STREAM_MIX, 0, 0);
    for (int i = 0; i < nnet; ++i) {
        neuron[i] = nchoices[sm64(&s) % (uint64_t)nn];
        layers[i] = lchoices[sm64(&s) % (uint64_t)nl];
        batch[i] = bmin + (int)(sm64(&s) % (uint64_t)(bmax - bmin + 1));
    }
}

void orc_masks_to_csc(const int32_t *masks, int nmask, int neuron, float val, int32_t *colptr,
                      int32_t *rowidx, float *vals) {
    for (int j = 0; j <= neuron; ++j) colptr[j] = j * nmask;
    for (int j = 0; j < neuron; ++j) {
        int32_t *r = rowidx + (int64_t)j * nmask;
        for (int k = 0; k < nmask; ++k) {
            int32_t v = j ^ masks[k], p = k;
            while (p > 0 && r[p - 1] > v) { r[p] = r[p - 1]; --p; }
            r[p] = v;
        }
        for (int k = 0; k < nmask; ++k) vals[(int64_t)j * nmask + k] = val;
    }
}

void orc_free(void *p) { free(p); }

/* ------------------------------------------------------------------ */
/* Greedy BCSC builder, restating src/utils/matrix.h:1200-1269.
 * Elements are visited in (column, row) order.  A block column starts at the
 * first column that is >= bc away from the current block column's start.
 * Inside a block column, an element joins the most recently created block
 * whose row range [start, start+br) holds its row (searched newest first);
 * otherwise it starts a new block at its own row.  The value lands at
 * [(col - blockcol_start) * bc + (row - block_start)] -- except for the
 * element that creates a block, which the reference stores at offset 0 of the
 * new block (matrix.h:1249-1251 and :1256-1261 push the value first and then
 * 255 zeros), whatever its column offset. */
typedef struct { int32_t r, c; float v; } coo_t;

static int coo_colmajor_cmp(const void *a, const void *b) {
    const coo_t *x = (const coo_t *)a, *y = (const coo_t *)b;
    if (x->c != y->c) return x->c < y->c ? -1 : 1;
    if (x->r != y->r) return x->r < y->r ? -1 : 1;
    return 0;
}

typedef struct { void *p; int64_t n, cap; size_t esz; } vec_t;
static int vec_push(vec_t *v, const void *e, int64_t cnt) {
    if (v->n + cnt > v->cap) {
        int64_t nc = v->cap ? v->cap : 64;
        while (nc < v->n + cnt) nc *= 2;
        void *q = realloc(v->p, (size_t)nc * v->esz);
        if (!q) return -1;
        v->p = q;
        v->cap = nc;
    }
    if (e) memcpy((char *)v->p + (size_t)v->n * v->esz, e, (size_t)cnt * v->esz);
    else memset((char *)v->p + (size_t)v->n * v->esz, 0, (size_t)cnt * v->esz);
    v->n += cnt;
    return 0;
}

int orc_bcsc_greedy(int64_t nnz, const int32_t *row, const int32_t *col, const float *val, int bc,
                    int br, int32_t **col_ptr, int32_t *n_col_ptr, int32_t **row_index,
                    int32_t *n_blocks, int32_t **col_index, float **values) {
    if (nnz <= 0 || bc <= 0 || br <= 0) return -1;
    coo_t *e = (coo_t *)malloc((size_t)nnz * sizeof(coo_t));
    if (!e) return -1;
    for (int64_t i = 0; i < nnz; ++i) { e[i].r = row[i]; e[i].c = col[i]; e[i].v = val[i]; }
    qsort(e, (size_t)nnz, sizeof(coo_t), coo_colmajor_cmp);

    const int64_t bsz = (int64_t)bc * br;
    vec_t len = {0, 0, 0, sizeof(int32_t)}, rix = {0, 0, 0, sizeof(int32_t)};
    vec_t cix = {0, 0, 0, sizeof(int32_t)}, vals = {0, 0, 0, sizeof(float)};
    int32_t zero = 0;
    int rc = 0;
    rc |= vec_push(&len, &zero, 1);
    rc |= vec_push(&cix, &e[0].c, 1);
    rc |= vec_push(&rix, &e[0].r, 1);
    rc |= vec_push(&vals, &e[0].v, 1);
    rc |= vec_push(&vals, NULL, bsz - 1);
    int64_t blk_col_ptr = 0;
    for (int64_t t = 1; t < nnz && !rc; ++t) {
        int32_t blk_col = ((int32_t *)cix.p)[blk_col_ptr];
        int32_t r = e[t].r, c = e[t].c;
        if (c - blk_col < bc) {
            int64_t i, lo = ((int32_t *)len.p)[blk_col_ptr];
            int found = 0;
            for (i = rix.n - 1; i >= lo; --i) {
                int32_t br0 = ((int32_t *)rix.p)[i];
                if (r >= br0 && r - br0 < br) { found = 1; break; }
            }
            if (found) {
                int64_t pos = i * bsz + (int64_t)(c - blk_col) * bc + (r - ((int32_t *)rix.p)[i]);
                ((float *)vals.p)[pos] = e[t].v;
            } else {
                rc |= vec_push(&rix, &r, 1);
                rc |= vec_push(&vals, &e[t].v, 1);
                rc |= vec_push(&vals, NULL, bsz - 1);
            }
        } else {
            rc |= vec_push(&cix, &c, 1);
            blk_col_ptr++;
            rc |= vec_push(&rix, &r, 1);
            int32_t l = (int32_t)(rix.n - 1);
            rc |= vec_push(&len, &l, 1);
            rc |= vec_push(&vals, &e[t].v, 1);
            rc |= vec_push(&vals, NULL, bsz - 1);
        }
    }
    int32_t nb = (int32_t)rix.n;
    rc |= vec_push(&len, &nb, 1);
    free(e);
    if (rc) { free(len.p); free(rix.p); free(cix.p); free(vals.p); return -1; }
    *col_ptr = (int32_t *)len.p;
    *n_col_ptr = (int32_t)len.n;
    *row_index = (int32_t *)rix.p;
    *n_blocks = nb;
    *col_index = (int32_t *)cix.p;
    *values = (float *)vals.p;
    return 0;
}

/* ------------------------------------------------------------------ */
static inline double relu32(double x) { return x < 0.0 ? 0.0 : (x > 32.0 ? 32.0 : x); }

/* src/kernels/kernel.cu:240-379: block column bid reads the two blocks that
 * start at idx_ptr[bid]; for stage k it gathers activation rows
 * fuse[index[p + k/2] + (k%2)*8 + w] (w < 8) and the 128 values
 * [k*128, k*128+128) of that block span; the ldmatrix.trans fragment mapping
 * (:306-307, :331) pairs value [kk*16 + r] with input row start+kk and output
 * bid*16 + r; the hi and lo halves are multiplied by the same weight. */
void orc_ref_layer(const float *a, const float *values, float *c, const int32_t *fuse,
                   const int32_t *idx_ptr, const int32_t *index, float bias, int batch,
                   int neuron) {
    const int nbc = neuron / 16;
#pragma omp parallel for schedule(static)
    for (int bid = 0; bid < nbc; ++bid) {
        const int p = idx_ptr[bid];
        for (int rr = 0; rr < 16; ++rr) {
            float *crow = c + (int64_t)(bid * 16 + rr) * batch;
            for (int b = 0; b < batch; ++b) {
                double acc = 0.0;
                for (int j = 0; j < 2; ++j) {
                    const float *v = values + (int64_t)(p + j) * 256;
                    for (int kk = 0; kk < 16; ++kk) {
                        double w = v[kk * 16 + rr];
                        if (w == 0.0) continue;
                        int f = fuse[index[p + j] + kk];
                        acc += w * a[(int64_t)f * batch + b] + w * a[(int64_t)(f + neuron) * batch + b];
                    }
                }
                crow[b] = (float)relu32(acc + (double)bias);
            }
        }
    }
}

void orc_bcsc_layer(const float *a, const float *values, float *c, const int32_t *fuse,
                    const int32_t *idx_ptr, const int32_t *index, int nblockcols, float bias,
                    int batch, int neuron, int bc, int br) {
    const int64_t bsz = (int64_t)bc * br;
    for (int64_t i = 0; i < (int64_t)neuron * batch; ++i) c[i] = 0.0f;
#pragma omp parallel for schedule(static)
    for (int bid = 0; bid < nblockcols; ++bid) {
        double *acc = (double *)calloc((size_t)bc * batch, sizeof(double));
        for (int blk = idx_ptr[bid]; blk < idx_ptr[bid + 1]; ++blk) {
            const float *v = values + (int64_t)blk * bsz;
            const int rs = index[blk];
            for (int co = 0; co < bc; ++co) {
                for (int ro = 0; ro < br; ++ro) {
                    int r = rs + ro;
                    if (r >= neuron) continue;
                    double w = v[(int64_t)co * bc + ro];
                    if (w == 0.0) continue;
                    int f = fuse ? fuse[r] : r;
                    const float *arow = a + (int64_t)f * batch;
                    for (int b = 0; b < batch; ++b) acc[(int64_t)co * batch + b] += w * arow[b];
                }
            }
        }
        for (int co = 0; co < bc; ++co) {
            int o = bid * bc + co;
            if (o >= neuron) continue;
            for (int b = 0; b < batch; ++b)
                c[(int64_t)o * batch + b] = (float)relu32(acc[(int64_t)co * batch + b] + (double)bias);
        }
        free(acc);
    }
}

/* ------------------------------------------------------------------ */
/* One FP64 layer for one row in the fixed order described in oracle.h. */
static double layer_fp64(int neuron, const int32_t *cp, const int32_t *ri, const float *vv,
                         const double *y, double *out, double bias) {
    double mx = 0.0;
    for (int j = 0; j < neuron; ++j) {
        double acc = 0.0;
        for (int32_t p = cp[j]; p < cp[j + 1]; ++p) {
            double yi = y[ri[p]];
            if (yi != 0.0) {
                double prod = (double)vv[p] * yi;
                acc = acc + prod;
            }
        }
        double z = acc + bias;
        double o = relu32(z);
        out[j] = o;
        if (o > mx) mx = o;
    }
    return mx;
}

int orc_infer_fp64(int neuron, int layers, int64_t rows, const int32_t *const *colptr,
                   const int32_t *const *rowidx, const float *const *vals, const uint8_t *y0_u8,
                   const float *y0_f32, float bias, double tau, int threads, int32_t *death,
                   double *maxval, double *final_y) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
    const double b = (double)bias;
#pragma omp parallel
    {
        double *y = (double *)malloc(sizeof(double) * (size_t)neuron);
        double *z = (double *)malloc(sizeof(double) * (size_t)neuron);
#pragma omp for schedule(dynamic, 16)
        for (int64_t r = 0; r < rows; ++r) {
            for (int j = 0; j < neuron; ++j)
                y[j] = y0_u8 ? (double)y0_u8[r * neuron + j] : (double)y0_f32[r * neuron + j];
            int32_t d = layers;
            int l;
            for (l = 0; l < layers; ++l) {
                double mx = layer_fp64(neuron, colptr[l], rowidx[l], vals[l], y, z, b);
                if (maxval) maxval[r * layers + l] = mx;
                double *t = y; y = z; z = t;
                if (!(mx > tau)) { d = l; ++l; break; }
            }
            if (maxval) for (; l < layers; ++l) maxval[r * layers + l] = 0.0;
            death[r] = d;
            if (final_y) memcpy(final_y + r * neuron, y, sizeof(double) * (size_t)neuron);
        }
        free(y);
        free(z);
    }
    return 0;
}

int orc_replay_fp64(int neuron, int upto, int64_t nrows, const int64_t *row_ids,
                    const int32_t *const *colptr, const int32_t *const *rowidx,
                    const float *const *vals, const uint8_t *y0_u8, const float *y0_f32,
                    float bias, double *out) {
    const double b = (double)bias;
#pragma omp parallel
    {
        double *y = (double *)malloc(sizeof(double) * (size_t)neuron);
        double *z = (double *)malloc(sizeof(double) * (size_t)neuron);
#pragma omp for schedule(dynamic, 4)
        for (int64_t q = 0; q < nrows; ++q) {
            int64_t r = row_ids[q];
            for (int j = 0; j < neuron; ++j)
                y[j] = y0_u8 ? (double)y0_u8[r * neuron + j] : (double)y0_f32[r * neuron + j];
            for (int l = 0; l <= upto; ++l) {
                layer_fp64(neuron, colptr[l], rowidx[l], vals[l], y, z, b);
                double *t = y; y = z; z = t;
            }
            memcpy(out + q * neuron, y, sizeof(double) * (size_t)neuron);
        }
        free(y);
        free(z);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
int64_t orc_infer_fp32_csr(int neuron, int layers, int64_t rows, const int32_t *const *rowptr,
                           const int32_t *const *colidx, const float *const *vals,
                           const uint8_t *y0_u8, float bias, float tau, int threads,
                           int32_t *death) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
    int64_t alive = 0;
#pragma omp parallel reduction(+ : alive)
    {
        float *y = (float *)malloc(sizeof(float) * (size_t)neuron);
        float *acc = (float *)malloc(sizeof(float) * (size_t)neuron);
#pragma omp for schedule(dynamic, 16)
        for (int64_t r = 0; r < rows; ++r) {
            for (int j = 0; j < neuron; ++j) y[j] = (float)y0_u8[r * neuron + j];
            int32_t d = layers;
            for (int l = 0; l < layers; ++l) {
                memset(acc, 0, sizeof(float) * (size_t)neuron);
                const int32_t *rp = rowptr[l], *ci = colidx[l];
                const float *vv = vals[l];
                for (int i = 0; i < neuron; ++i) {
                    float yi = y[i];
                    if (yi == 0.0f) continue;
                    for (int32_t p = rp[i]; p < rp[i + 1]; ++p) acc[ci[p]] += yi * vv[p];
                }
                float mx = 0.0f;
                for (int j = 0; j < neuron; ++j) {
                    float zz = acc[j] + bias;
                    zz = zz < 0.0f ? 0.0f : (zz > 32.0f ? 32.0f : zz);
                    y[j] = zz;
                    mx = zz > mx ? zz : mx;
                }
                if (!(mx > tau)) { d = l; break; }
            }
            if (death) death[r] = d;
            alive += (d == layers);
        }
        free(y);
        free(acc);
    }
    return alive;
}
