// CUDA-core row-tile layer kernel interface (implementation in cc_layer.cu).
#pragma once

#include <vector>

#include "engine.cuh"

namespace cospdnn {

// Row-tile height TR (activation layout TR) for a CUDA-core net of width N in
// precision `prec`, or 0 when a tile of 16-byte feature columns does not fit
// in shared memory (the net then uses the row-major gather kernel).
int cc_tile_rows(int N, int prec);
// Zero feature columns staged after a tile's N inputs (one per bank residue
// of the conflict-free order): the padding entries of compact lists read them.
constexpr int kCcZeroCols = 16;
// Builds the entry list of one layer from its CSC (conflict-free order for
// tile height TR) and uploads it; compact: 16-bit entries (the layer must
// have one weight value, cc_single_weight).
int cc_build_entries(const std::vector<int32_t> &colptr, const std::vector<int32_t> &rowidx,
                     const std::vector<float> &vals, int N, int prec, int TR, bool compact, LayerDev &ld,
                     std::vector<void *> &owned);
// True when every weight of the layer has one value in the compute type and
// that value is not zero (what compact entry lists need).
bool cc_single_weight(const std::vector<int32_t> &colptr, const std::vector<float> &vals, int N, int prec);
// Launch description of the tile kernel for the CUDA-core row-tile nets of
// precision `prec` whose lanes own `lane_bytes` (16 or 8) of a feature
// column; max_tile_bytes = largest N*TR*element size among them.
int cc_layer_spec(KSpec &spec, NetDev *nets, int nnets, int prec, int lane_bytes, bool compact,
                  unsigned long long *launches, int sms, size_t max_tile_bytes);
// Edge colouring of a bipartite multigraph with P vertices on each side
// (edge e joins eu[e] and es[e]): colour[e] in [0, D), D = the max degree, no
// two edges of one colour share a vertex.  Returns D.
int colour_group(int P, const std::vector<int> &eu, const std::vector<int> &es, std::vector<int> &colour);
// Lane bytes of a row-tile net of tile height TR.
inline int cc_lane_bytes(int prec, int TR) { return TR * (prec == COSPDNN_PREC_FP32 ? 4 : 2) >= 16 ? 16 : 8; }
// Shared-memory bytes of one row tile: its N inputs and the zero columns.
inline size_t cc_tile_bytes(int N, int prec, int TR) {
    return (size_t)(N + kCcZeroCols) * TR * (prec == COSPDNN_PREC_FP32 ? 4 : 2);
}

}  // namespace cospdnn
