// CUDA-core feature-split tile kernel interface (implementation in cs_layer.cu).
#pragma once

#include <vector>

#include "engine.cuh"

namespace cospdnn {

// True when a 16-bit net of width N takes the feature-split kernel: no row
// tile of the one-CTA kernel fits shared memory (cc_tile_rows == 0), while
// half of a 2-row tile does (N % 64 == 0, N / 2 + 32 16-bit columns).
bool cs_supported(int N, int prec);
// Builds one layer's split entry lists from its CSC (split bit chosen per
// layer, conflict-free order per half and group of 32 outputs) and uploads
// them; compact: entries without a weight (the layer has one weight value).
int cs_build_entries(const std::vector<int32_t> &colptr, const std::vector<int32_t> &rowidx,
                     const std::vector<float> &vals, int N, int prec, bool compact, LayerDev &ld,
                     std::vector<void *> &owned);
// Launch description of the split kernel for the split nets of precision
// `prec` whose widest has max_n features (grid: the clusters of two CTAs
// that can be resident at once).
int cs_layer_spec(KSpec &spec, NetDev *nets, int nnets, int prec, bool compact, unsigned long long *launches,
                  int *abort_flag, const DevLimits *limits, int sms, int max_n);

}  // namespace cospdnn
