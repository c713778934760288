// Layer 0 of binary inputs by bit counting (implementation in bits_layer.cu).
#pragma once

#include <vector>

#include "engine.cuh"

namespace cospdnn {

// Builds the bit-count schedule of layer 0 of a row-tile net (layout >= 4)
// or a 16-row net (layout 1: MMA-tile and feature-split nets) when every output's weights are one value
// (zero entries ignored) and no output has more than 63 of them; sets
// nd.l0_k to the steps per output (a multiple of 8, or of 16 for MMA tiles),
// left 0 when the layer does not qualify (nothing is uploaded then).
int l0_build(const std::vector<int32_t> &colptr, const std::vector<int32_t> &rowidx, const std::vector<float> &vals,
             int N, int prec, int layout, float bias, NetDev &nd, std::vector<void *> &owned);
// Kinds of bit-count launch: row-tile nets (32-row units), MMA-tile nets and
// feature-split nets (16-row units, 16-bit precisions only).
enum { kL0Rows32 = 0, kL0Mma16 = 1, kL0Split16 = 2 };
// Launch of the bit-count kernel of one kind for the qualifying nets of
// precision `prec`, max_n the widest of them.
int l0_spec(KSpec &k, NetDev *nets, int nnets, int prec, int kind, unsigned long long *launches, int sms,
            int max_n);
// Input rows (U8 or packed bits, row-major) as bit planes: word (unit, f)
// holds feature f of rows 32*unit .. 32*unit+31 (bit r = row 32*unit+r is
// non-zero; rows past `rows` are 0); also each row's max value (err0 = 0,
// the row-max kernel's output) and, for bytes, `nonbin` raised when a value
// is above 1 (the caller clears it first).
void l0_convert_bits(const uint8_t *src, int format, int rows, int N, uint32_t *bits, float *err0, float *mx0,
                     int *nonbin, cudaStream_t s);
// Bytes of the bit planes of `rows` rows of width N.
inline size_t l0_bits_bytes(int rows, int N) { return (size_t)((rows + 31) / 32) * N * 4; }

}  // namespace cospdnn
