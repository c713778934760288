// tcgen05 layer kernel interface (implementation in tc_layer.cu).
#pragma once

#include <vector>

#include "engine.cuh"

namespace cospdnn {

// true if the tcgen05 path handles this layer width
bool tc_supported(int neuron);
// Builds the 16x16 aligned block view of one layer from its CSC and uploads it.
int tc_build_blocks(const std::vector<int32_t> &colptr, const std::vector<int32_t> &rowidx,
                    const std::vector<float> &vals, int N, int prec, LayerDev &ld,
                    std::vector<void *> &owned);
// Launch description of the layer kernel for the tcgen05 nets of precision `prec`.
int tc_layer_spec(KSpec &spec, NetDev *nets, int nnets, int prec, unsigned long long *launches,
                  int *abort_flag, const DevLimits *limits, int sms);

}  // namespace cospdnn
