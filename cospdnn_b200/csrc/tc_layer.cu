// tcgen05 layer kernel (FP16 / BF16 activations, FP32 accumulation in TMEM).
#include "tc_layer.cuh"

namespace cospdnn {

bool tc_supported(int neuron) { (void)neuron; return false; }

int tc_build_blocks(const std::vector<int32_t> &, const std::vector<int32_t> &, const std::vector<float> &,
                    int, int, LayerDev &, std::vector<void *> &) {
    return fail(COSPDNN_ERR_UNSUPPORTED, "tcgen05 kernel not built");
}

int tc_layer_spec(KSpec &, NetDev *, int, int, unsigned long long *, int) {
    return fail(COSPDNN_ERR_UNSUPPORTED, "tcgen05 kernel not built");
}

}  // namespace cospdnn
