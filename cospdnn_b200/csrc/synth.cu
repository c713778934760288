// Synthetic Graph-Challenge-style inputs on the GPU: binary image rows with a
// per-row density, from SplitMix64 streams (Steele, Lea & Flood, OOPSLA 2014).
// SplitMix64 draw k of a stream with state s0 is mix(s0 + k*gamma), so every
// element is generated independently.  Stream of row r of network `net`:
// stream_seed(seed, 2, net, r); draw 1 gives the density d = dlo + (dhi-dlo)*u,
// draw j+2 gives element j (1 if u < d), u = (draw >> 11) * 2^-53.
#include "common.cuh"

namespace cospdnn {
namespace {

constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ULL;

__host__ __device__ inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__host__ __device__ inline uint64_t next64(uint64_t &s) {
    s += kGamma;
    return mix64(s);
}

__host__ __device__ inline uint64_t stream_seed(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) {
    uint64_t s = seed ^ 0x5851F42D4C957F2DULL;
    uint64_t x = next64(s);
    s = x ^ (a + 0x632BE59BD9B4E019ULL);
    x = next64(s);
    s = x ^ (b + 0x9E3779B97F4A7C15ULL);
    x = next64(s);
    s = x ^ (c + 0xD1B54A32D192ED03ULL);
    return next64(s);
}

__device__ inline double u01(uint64_t z) { return (double)(z >> 11) * (1.0 / 9007199254740992.0); }

// one CTA row-slab: threads over the row's elements
__global__ void k_synth_rows(uint8_t *__restrict__ out, int64_t rows, int neuron, uint64_t seed, int net,
                             int64_t row0, double dlo, double dhi, int bits) {
    for (int64_t r = blockIdx.x; r < rows; r += gridDim.x) {
        const uint64_t s0 = stream_seed(seed, 2, (uint64_t)net, (uint64_t)(row0 + r));
        const double d = __dadd_rn(dlo, __dmul_rn(dhi - dlo, u01(mix64(s0 + kGamma))));
        if (!bits) {
            uint8_t *o = out + r * neuron;
            for (int j = threadIdx.x; j < neuron; j += blockDim.x)
                o[j] = (uint8_t)(u01(mix64(s0 + (uint64_t)(j + 2) * kGamma)) < d);
        } else {
            uint8_t *o = out + r * (neuron / 8);
            for (int jb = threadIdx.x; jb < neuron / 8; jb += blockDim.x) {
                uint8_t v = 0;
                for (int t = 0; t < 8; ++t) {
                    const int j = jb * 8 + t;
                    v |= (uint8_t)(u01(mix64(s0 + (uint64_t)(j + 2) * kGamma)) < d) << t;
                }
                o[jb] = v;
            }
        }
    }
}

}  // namespace
}  // namespace cospdnn

using namespace cospdnn;

extern "C" int cospdnn_synth_input(void *out, int64_t rows, int neuron, uint64_t seed, int net,
                                   int64_t row0, double dlo, double dhi, int format, void *stream) {
    CSP_CHECK(out && rows >= 0 && neuron > 0, COSPDNN_ERR_INVALID, "synth_input: bad arguments");
    CSP_CHECK(format == COSPDNN_INPUT_U8 || (format == COSPDNN_INPUT_BITS && neuron % 8 == 0),
              COSPDNN_ERR_INVALID, "synth_input: format must be U8 or BITS (neuron % 8 == 0)");
    CSP_CHECK(dlo <= dhi, COSPDNN_ERR_INVALID, "synth_input: dlo > dhi");
    if (rows == 0) return COSPDNN_OK;
    const int blocks = (int)std::min<int64_t>(rows, 148 * 16);
    k_synth_rows<<<blocks, 256, 0, (cudaStream_t)stream>>>((uint8_t *)out, rows, neuron, seed, net, row0,
                                                          dlo, dhi, format == COSPDNN_INPUT_BITS);
    CSP_CUDA(cudaGetLastError());
    return COSPDNN_OK;
}
