// Bit-sliced counting of the layer-0 kernels (bits_layer.cu): six counter
// planes hold, at every bit position (a row of a unit), one bit of a count of
// set bits; host and device code, so that the counting is tested on the CPU.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

// loops fully unrolled in device code (the host pass has no such pragma)
#ifdef __CUDA_ARCH__
#define CSP_UNROLL _Pragma("unroll")
#else
#define CSP_UNROLL
#endif

namespace cospdnn {

// carry-save adder: (h, l) = the two bits of a + b + c at every position
__host__ __device__ __forceinline__ void csa(uint32_t &h, uint32_t &l, uint32_t a, uint32_t b, uint32_t c) {
    const uint32_t u = a ^ b;
    h = (a & b) | (u & c);
    l = u ^ c;
}

// count += number of set bits among x[0..7] at every bit position
__host__ __device__ __forceinline__ void add8(uint32_t (&p)[6], const uint32_t (&x)[8]) {
    uint32_t twosA, twosB, foursA, foursB, eightsA;
    csa(twosA, p[0], p[0], x[0], x[1]);
    csa(twosB, p[0], p[0], x[2], x[3]);
    csa(foursA, p[1], p[1], twosA, twosB);
    csa(twosA, p[0], p[0], x[4], x[5]);
    csa(twosB, p[0], p[0], x[6], x[7]);
    csa(foursB, p[1], p[1], twosA, twosB);
    csa(eightsA, p[2], p[2], foursA, foursB);
    const uint32_t c8 = p[3] & eightsA;
    p[3] ^= eightsA;
    const uint32_t c16 = p[4] & c8;
    p[4] ^= c8;
    p[5] ^= c16;  // counts stay below 64
}

// The counters as bytes: byte g of c[k] = the count at bit position 8g + k.
// Planes 0..5 (with 6 and 7 zero) hold, at each bit position, one bit of an
// 8-bit count; transposing the 8x8 bit matrix of each byte column across the
// eight words (three rounds of delta swaps of 4-, 2- and 1-bit blocks) gives
// each position's count as a byte.
__host__ __device__ __forceinline__ void counts8(const uint32_t (&p)[6], uint32_t (&c)[8]) {
CSP_UNROLL
    for (int b = 0; b < 6; ++b) c[b] = p[b];
    c[6] = c[7] = 0u;
CSP_UNROLL
    for (int d = 4; d >= 1; d >>= 1) {
        const uint32_t m = d == 4 ? 0x0F0F0F0Fu : d == 2 ? 0x33333333u : 0x55555555u;
CSP_UNROLL
        for (int i = 0; i < 8; ++i) {
            if (i & d) continue;
            const uint32_t t = ((c[i] >> d) ^ c[i + d]) & m;
            c[i + d] ^= t;
            c[i] ^= t << d;
        }
    }
}

}  // namespace cospdnn
