// cospdnn_double.out: two networks in one launch, the reference's command
// line (src/cospdnn_double.cpp:81-197):
//     cospdnn_double.out neuron1 batch1 layer1 neuron2 batch2 layer2 gpu_id dataset_dir
// Both networks go into one engine and run in a single graph launch (they
// may differ in width, depth and batch).  Prints the reference's lines
// (src/cospdnn_double.cu:249-250,794,841,880-882,1142): "initial padding
// batch B1 and B2", "TILE_DIM 128", per layer "SpDNN 1 layer l, feature = n"
// and "SpDNN 2 layer l, feature = n" (l <= 21), "layer l, batch1 = b1,
// batch2 = b2" (kept rows padded to 128) and "Layer l exec Time = tms" (both
// networks' layer kernels, from a kernel-by-kernel pass unless
// COSPDNN_LAYER_TIMES=0), then "Total Kernel Exec Time = X ms".  COSPDNN_PRECISION / COSPDNN_KERNEL select
// precision and kernel; COSPDNN_CACHE, COSPDNN_CATEGORIES_1/_2,
// COSPDNN_TRUTH_1/_2 (exit status 2 on a mismatch) and COSPDNN_JSON (one
// result line per network, timed over the joint run) as in cospdnn.out.
#include "reference_io.h"

using namespace cospdnn_cli;

int main(int argc, char *argv[]) {
    if (argc != 9) {
        std::cout << "Usage: exe neuron1 batch1 layer1 neuron2 batch2 layer2 gpu_id dataset_dir" << std::endl;
        return 0;
    }
    const int neuron[2] = {std::atoi(argv[1]), std::atoi(argv[4])};
    const int batch[2] = {std::atoi(argv[2]), std::atoi(argv[5])};
    const int layers[2] = {std::atoi(argv[3]), std::atoi(argv[6])};
    const int dev = std::atoi(argv[7]);
    const std::string dir(argv[8]);
    for (int i = 0; i < 2; ++i)
        if (neuron[i] <= 0 || batch[i] <= 0 || layers[i] <= 0) die("bad arguments");
    std::cout << "-------------------------------------" << std::endl;
    std::cout << "[BEGIN]..." << std::endl;
    for (int i = 0; i < 2; ++i) {
        std::cout << "[Batch" << i + 1 << "] :" << batch[i] << std::endl;
        std::cout << "[Neuron" << i + 1 << "] :" << neuron[i] << std::endl;
        std::cout << "[Layer" << i + 1 << "] :" << layers[i] << std::endl;
        std::cout << "-------------------------------------" << std::endl;
    }
    Network net[2] = {load_network(neuron[0], batch[0], layers[0], dir),
                      load_network(neuron[1], batch[1], layers[1], dir)};
    const int prec = env_precision(), kern = env_kernel();
    cospdnn_engine *e = nullptr;
    check(cospdnn_engine_create(&e, dev), "engine_create");
    int id[2];
    for (int i = 0; i < 2; ++i) id[i] = add_network(e, net[i], 0, batch[i], prec, kern);
    check(cospdnn_engine_build(e), "build");
    for (int i = 0; i < 2; ++i) set_rows(e, id[i], net[i], 0, batch[i]);
    std::cout << "initial padding batch " << pad_tile(batch[0]) << " and " << pad_tile(batch[1]) << std::endl;
    std::cout << "TILE_DIM 128" << std::endl;
    float ms = 0.0f;
    check(cospdnn_engine_run_timed(e, nullptr, &ms), "run");
    int rc = 0;
    std::vector<int64_t> alive[2], rech[2], count(2, 0);
    std::vector<int32_t> cats[2];
    float bound[2] = {0.0f, 0.0f};
    for (int i = 0; i < 2; ++i) {
        alive[i].assign(layers[i], 0);
        rech[i].assign(layers[i], 0);
        cats[i].assign((size_t)batch[i], 0);
        check(cospdnn_engine_result(e, id[i], cats[i].data(), &count[i], alive[i].data(), rech[i].data(), nullptr),
              "result");
        check(cospdnn_engine_final_bound(e, id[i], &bound[i], nullptr), "final_bound");
    }
    const int lmax = std::max(layers[0], layers[1]);
    std::vector<float> layer_ms(lmax + 1, 0.0f);
    if (env_layer_times()) {
        int iters = 0;
        check(cospdnn_engine_profile_layers(e, nullptr, lmax + 1, layer_ms.data(), &iters), "profile_layers");
    }
    for (int l = 0; l < lmax; ++l) {
        const int64_t a1 = l < layers[0] ? alive[0][l] : 0, a2 = l < layers[1] ? alive[1][l] : 0;
        if (l <= 21) {
            if (l < layers[0]) std::cout << "SpDNN 1 layer " << l << ", feature = " << a1 << std::endl;
            if (l < layers[1]) std::cout << "SpDNN 2 layer " << l << ", feature = " << a2 << std::endl;
        }
        std::cout << "layer " << l << ", batch1 = " << pad_tile(a1) << ", batch2 = " << pad_tile(a2) << std::endl;
        std::cout << "Layer " << l << " exec Time = " << layer_ms[l] << "ms" << std::endl;
    }
    for (int i = 0; i < 2; ++i) {
        const std::vector<int64_t> &al = alive[i];
        std::cout << "[Categories" << i + 1 << "] :" << count[i] << std::endl;
        const std::vector<int64_t> c64(cats[i].begin(), cats[i].begin() + count[i]);
        const std::string k = std::to_string(i + 1);
        rc = std::max(rc, report_categories(c64, ("COSPDNN_CATEGORIES_" + k).c_str(), ("COSPDNN_TRUTH_" + k).c_str(),
                                            "SpDNN " + k + " "));
        RunReport rep;
        rep.program = "cospdnn_double";
        rep.network = i + 1;
        rep.neuron = neuron[i];
        rep.batch = batch[i];
        rep.layers = layers[i];
        rep.precision = prec;
        rep.kernel = kern;
        for (const auto &w : net[i].w) rep.weights += (int64_t)w.rowidx.size();
        rep.ms = ms;  // both networks run in one launch
        rep.dy_bound = bound[i];
        rep.alive = al;
        rep.rechecked = rech[i];
        rep.categories = c64;
        report_json(rep);
    }
    cospdnn_engine_destroy(e);
    std::cout << "Total Kernel Exec Time = " << ms << "ms" << std::endl;
    std::cout << "[END]..." << std::endl;
    return rc;
}
