// cospdnn.out: one network, the reference's command line
// (src/cospdnn.cpp:80-189):
//     cospdnn.out neuron batch layer gpu_num gpu_id dataset_dir
// Reads the dataset files (reference_io.h), runs every layer on the engine
// (one graph launch per GPU) and prints the reference's lines
// (src/cospdnn.cu:27,262-264,302-310): "initial padding batch B",
// per layer "layer l, feature = n" (rows alive after layer l, l <= 21),
// "layer l, batch = b" (the kept rows padded to 128) and
// "Layer l exec Time = t" (the layer's kernels, from a second, kernel by
// kernel pass unless COSPDNN_LAYER_TIMES=0), then "Kernel Exec Time = X ms"
// (the graph run).  With gpu_num > 1 the batch is split into
// contiguous row ranges, one engine and host thread per GPU, and the counts
// are summed.  COSPDNN_PRECISION / COSPDNN_KERNEL select precision and kernel;
// COSPDNN_CACHE keeps parsed datasets in binary form; COSPDNN_CATEGORIES /
// COSPDNN_TRUTH write the categories in Graph Challenge format and check them
// against a truth file (exit status 2 on a mismatch); COSPDNN_JSON=1 (or a
// file name) adds one JSON result line (edges/s, rows alive and rechecked
// per layer, category count and hash).  See reference_io.h.
#include <algorithm>
#include <thread>

#include "reference_io.h"

using namespace cospdnn_cli;

int main(int argc, char *argv[]) {
    if (argc != 7) {
        std::cout << "Usage: exe neuron batch layer gpu_num gpu_id dataset_dir" << std::endl;
        return 0;
    }
    const int neuron = std::atoi(argv[1]), batch = std::atoi(argv[2]), layers = std::atoi(argv[3]);
    int gpu_num = std::atoi(argv[4]);
    const int dev = std::atoi(argv[5]);
    const std::string dir(argv[6]);
    if (neuron <= 0 || batch <= 0 || layers <= 0 || gpu_num <= 0) die("bad arguments");
    std::cout << "[BEGIN]..." << std::endl;
    std::cout << "[Batch] :" << batch << std::endl;
    std::cout << "[Neuron] :" << neuron << std::endl;
    std::cout << "[Layer] :" << layers << std::endl;
    const Network net = load_network(neuron, batch, layers, dir);
    const int prec = env_precision(), kern = env_kernel();

    std::vector<int> devices;
    if (gpu_num == 1) {
        devices.push_back(dev);
    } else {
        const int avail = cospdnn_device_count();
        if (avail < 1) die("no CUDA device visible");
        if (gpu_num > avail) {
            std::cout << "Exceeding Maximum GPU Number! Automatically Change to Max GPU Number " << avail << std::endl;
            gpu_num = avail;
        }
        for (int g = 0; g < gpu_num; ++g) devices.push_back(g);
    }
    const int ng = (int)devices.size();
    std::vector<std::vector<int64_t>> alive(ng, std::vector<int64_t>(layers, 0)), rech(alive);
    std::vector<int64_t> count(ng, 0);
    std::vector<std::vector<int32_t>> cats(ng);
    std::vector<float> ms(ng, 0.0f), bound(ng, 0.0f);
    std::vector<std::vector<float>> layer_ms(ng, std::vector<float>(layers + 1, 0.0f));
    const bool times = env_layer_times();
    for (int g = 0; g < ng; ++g) {
        const int64_t r0 = (int64_t)batch * g / ng, r1 = (int64_t)batch * (g + 1) / ng;
        std::cout << "initial padding batch " << pad_tile(r1 - r0) << std::endl;
    }
    // each worker exits the process with the reference's style of message on
    // any error (as Safe_Call does in the reference)
    auto work = [&](int g) {
        const int r0 = (int)((int64_t)batch * g / ng), r1 = (int)((int64_t)batch * (g + 1) / ng);
        cospdnn_engine *e = nullptr;
        check(cospdnn_engine_create(&e, devices[g]), "engine_create");
        const int id = add_network(e, net, r0, r1, prec, kern);
        check(cospdnn_engine_build(e), "build");
        set_rows(e, id, net, r0, r1);
        check(cospdnn_engine_run_timed(e, nullptr, &ms[g]), "run");
        cats[g].assign((size_t)std::max(1, r1 - r0), 0);
        check(cospdnn_engine_result(e, id, cats[g].data(), &count[g], alive[g].data(), rech[g].data(), nullptr),
              "result");
        cats[g].resize((size_t)count[g]);
        for (auto &c : cats[g]) c += r0;  // rows of the whole batch
        check(cospdnn_engine_final_bound(e, id, &bound[g], nullptr), "final_bound");
        if (times) {
            int iters = 0;
            check(cospdnn_engine_profile_layers(e, nullptr, layers + 1, layer_ms[g].data(), &iters), "profile_layers");
        }
        cospdnn_engine_destroy(e);
    };
    if (ng == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (int g = 0; g < ng; ++g) th.emplace_back(work, g);
        for (auto &t : th) t.join();
    }
    int64_t total = 0;
    for (int g = 0; g < ng; ++g) total += count[g];
    for (int l = 0; l < layers; ++l) {
        int64_t f = 0, padded = 0;
        float t = 0.0f;
        for (int g = 0; g < ng; ++g) {
            f += alive[g][l];
            padded += pad_tile(alive[g][l]);
            t = std::max(t, layer_ms[g][l]);
        }
        if (l <= 21) std::cout << "layer " << l << ", feature = " << f << std::endl;
        std::cout << "layer " << l << ", batch = " << padded << std::endl;
        std::cout << "Layer " << l << " exec Time = " << t << std::endl;
    }
    float tmax = 0.0f;
    for (int g = 0; g < ng; ++g) {
        if (ng > 1) std::cout << "GPU[" << devices[g] << "] Kernel Exec Time = " << ms[g] << "ms" << std::endl;
        tmax = std::max(tmax, ms[g]);
    }
    std::cout << "[Categories] :" << total << std::endl;
    std::vector<int64_t> all;
    for (int g = 0; g < ng; ++g) all.insert(all.end(), cats[g].begin(), cats[g].end());
    const int rc = report_categories(all, "COSPDNN_CATEGORIES", "COSPDNN_TRUTH", "");
    RunReport rep;
    rep.program = "cospdnn";
    rep.neuron = neuron;
    rep.batch = batch;
    rep.layers = layers;
    rep.precision = prec;
    rep.kernel = kern;
    rep.gpus = ng;
    for (const auto &w : net.w) rep.weights += (int64_t)w.rowidx.size();
    rep.ms = tmax;
    for (int g = 0; g < ng; ++g) rep.dy_bound = std::max(rep.dy_bound, bound[g]);
    rep.alive.assign(layers, 0);
    rep.rechecked.assign(layers, 0);
    for (int g = 0; g < ng; ++g)
        for (int l = 0; l < layers; ++l) {
            rep.alive[l] += alive[g][l];
            rep.rechecked[l] += rech[g][l];
        }
    rep.categories = all;
    report_json(rep);
    std::cout << "Kernel Exec Time = " << tmax << "ms" << std::endl;
    std::cout << "[END]..." << std::endl;
    return rc;
}
