// cospdnn_multi.out: any number of networks in one launch.  The command line
// of cospdnn_double.out (src/cospdnn_double.cpp:81-197) generalised from two
// networks to k >= 1:
//     cospdnn_multi.out neuron1 batch1 layer1 [neuron2 batch2 layer2 ...] gpu_id dataset_dir
// The reference runs at most two networks, and only with equal layer counts
// (src/cospdnn_double.cu:243-248); here every network goes into one engine
// and all run in a single graph launch, whatever their widths, depths and
// batches.  Networks of the same width read the same dataset files.  Prints
// cospdnn_double.out's lines for k networks: "SpDNN i layer l, feature = n"
// (l <= 21), "layer l, batch1 = b1, ..., batchk = bk" (kept rows padded to
// 128), "Layer l exec Time = tms", "[Categoriesi] :n" and "Total Kernel Exec
// Time = X ms".  COSPDNN_PRECISION, COSPDNN_KERNEL, COSPDNN_CACHE,
// COSPDNN_CATEGORIES_i, COSPDNN_TRUTH_i (exit status 2 on a mismatch),
// COSPDNN_LAYER_TIMES and COSPDNN_JSON as in cospdnn_double.out.
#include "reference_io.h"

using namespace cospdnn_cli;

int main(int argc, char *argv[]) {
    if (argc < 6 || (argc - 3) % 3 != 0) {
        std::cout << "Usage: exe neuron1 batch1 layer1 [neuron2 batch2 layer2 ...] gpu_id dataset_dir" << std::endl;
        return 0;
    }
    const int k = (argc - 3) / 3;
    std::vector<int> neuron(k), batch(k), layers(k);
    for (int i = 0; i < k; ++i) {
        neuron[i] = std::atoi(argv[1 + 3 * i]);
        batch[i] = std::atoi(argv[2 + 3 * i]);
        layers[i] = std::atoi(argv[3 + 3 * i]);
        if (neuron[i] <= 0 || batch[i] <= 0 || layers[i] <= 0) die("bad arguments");
    }
    const int dev = std::atoi(argv[argc - 2]);
    const std::string dir(argv[argc - 1]);
    std::cout << "-------------------------------------" << std::endl;
    std::cout << "[BEGIN]..." << std::endl;
    for (int i = 0; i < k; ++i) {
        std::cout << "[Batch" << i + 1 << "] :" << batch[i] << std::endl;
        std::cout << "[Neuron" << i + 1 << "] :" << neuron[i] << std::endl;
        std::cout << "[Layer" << i + 1 << "] :" << layers[i] << std::endl;
        std::cout << "-------------------------------------" << std::endl;
    }
    std::vector<Network> net;
    net.reserve(k);
    for (int i = 0; i < k; ++i) net.push_back(load_network(neuron[i], batch[i], layers[i], dir));
    const int prec = env_precision(), kern = env_kernel();
    cospdnn_engine *e = nullptr;
    check(cospdnn_engine_create(&e, dev), "engine_create");
    std::vector<int> id(k);
    for (int i = 0; i < k; ++i) id[i] = add_network(e, net[i], 0, batch[i], prec, kern);
    check(cospdnn_engine_build(e), "build");
    for (int i = 0; i < k; ++i) set_rows(e, id[i], net[i], 0, batch[i]);
    std::cout << "initial padding batch";
    for (int i = 0; i < k; ++i) std::cout << (i ? " and " : " ") << pad_tile(batch[i]);
    std::cout << std::endl;
    std::cout << "TILE_DIM 128" << std::endl;
    float ms = 0.0f;
    check(cospdnn_engine_run_timed(e, nullptr, &ms), "run");
    int rc = 0;
    std::vector<std::vector<int64_t>> alive(k), rech(k);
    std::vector<std::vector<int32_t>> cats(k);
    std::vector<int64_t> count(k, 0);
    std::vector<float> bound(k, 0.0f);
    int lmax = 0;
    for (int i = 0; i < k; ++i) {
        alive[i].assign(layers[i], 0);
        rech[i].assign(layers[i], 0);
        cats[i].assign((size_t)batch[i], 0);
        check(cospdnn_engine_result(e, id[i], cats[i].data(), &count[i], alive[i].data(), rech[i].data(), nullptr),
              "result");
        check(cospdnn_engine_final_bound(e, id[i], &bound[i], nullptr), "final_bound");
        lmax = std::max(lmax, layers[i]);
    }
    std::vector<float> layer_ms(lmax + 1, 0.0f);
    if (env_layer_times()) {
        int iters = 0;
        check(cospdnn_engine_profile_layers(e, nullptr, lmax + 1, layer_ms.data(), &iters), "profile_layers");
    }
    for (int l = 0; l < lmax; ++l) {
        if (l <= 21)
            for (int i = 0; i < k; ++i)
                if (l < layers[i])
                    std::cout << "SpDNN " << i + 1 << " layer " << l << ", feature = " << alive[i][l] << std::endl;
        std::cout << "layer " << l;
        for (int i = 0; i < k; ++i)
            std::cout << ", batch" << i + 1 << " = " << pad_tile(l < layers[i] ? alive[i][l] : 0);
        std::cout << std::endl;
        std::cout << "Layer " << l << " exec Time = " << layer_ms[l] << "ms" << std::endl;
    }
    for (int i = 0; i < k; ++i) {
        std::cout << "[Categories" << i + 1 << "] :" << count[i] << std::endl;
        const std::vector<int64_t> c64(cats[i].begin(), cats[i].begin() + count[i]);
        const std::string s = std::to_string(i + 1);
        rc = std::max(rc, report_categories(c64, ("COSPDNN_CATEGORIES_" + s).c_str(), ("COSPDNN_TRUTH_" + s).c_str(),
                                            "SpDNN " + s + " "));
        RunReport rep;
        rep.program = "cospdnn_multi";
        rep.network = i + 1;
        rep.neuron = neuron[i];
        rep.batch = batch[i];
        rep.layers = layers[i];
        rep.precision = prec;
        rep.kernel = kern;
        for (const auto &w : net[i].w) rep.weights += (int64_t)w.rowidx.size();
        rep.ms = ms;  // every network runs in the one launch
        rep.dy_bound = bound[i];
        rep.alive = alive[i];
        rep.rechecked = rech[i];
        rep.categories = c64;
        report_json(rep);
    }
    cospdnn_engine_destroy(e);
    std::cout << "Total Kernel Exec Time = " << ms << "ms" << std::endl;
    std::cout << "[END]..." << std::endl;
    return rc;
}
