// cospdnn_double.out: two networks in one launch, the reference's command
// line (src/cospdnn_double.cpp:81-197):
//     cospdnn_double.out neuron1 batch1 layer1 neuron2 batch2 layer2 gpu_id dataset_dir
// Both networks go into one engine and run in a single graph launch (they
// may differ in width, depth and batch).  Prints the reference's lines
// "SpDNN 1 layer l, feature = n", "SpDNN 2 layer l, feature = n" and
// "Total Kernel Exec Time = X ms".  COSPDNN_PRECISION / COSPDNN_KERNEL select
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
    float ms = 0.0f;
    check(cospdnn_engine_run_timed(e, nullptr, &ms), "run");
    int rc = 0;
    for (int i = 0; i < 2; ++i) {
        std::vector<int64_t> alive(layers[i], 0), rech(layers[i], 0);
        std::vector<int32_t> cats((size_t)batch[i], 0);
        int64_t count = 0;
        check(cospdnn_engine_result(e, id[i], cats.data(), &count, alive.data(), rech.data(), nullptr), "result");
        for (int l = 0; l < layers[i]; ++l)
            std::cout << "SpDNN " << i + 1 << " layer " << l << ", feature = " << alive[l] << std::endl;
        std::cout << "[Categories" << i + 1 << "] :" << count << std::endl;
        const std::vector<int64_t> c64(cats.begin(), cats.begin() + count);
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
        rep.alive = alive;
        rep.rechecked = rech;
        rep.categories = c64;
        report_json(rep);
    }
    cospdnn_engine_destroy(e);
    std::cout << "Total Kernel Exec Time = " << ms << "ms" << std::endl;
    std::cout << "[END]..." << std::endl;
    return rc;
}
