// Readers for the reference's dataset files and the shared driver of the
// cospdnn.out / cospdnn_double.out command lines.
//
// Files under the dataset directory (src/cospdnn.cpp:13-79):
//   sparse-images-N.tsv                  "b n val", 1-based image row b (rows
//                                        past the batch are skipped) and
//                                        neuron n
//   neuronN/N-l{l+1}.tsv                 "u v val", 1-based input neuron u,
//                                        output neuron v (COOMatrix with
//                                        T = true, src/utils/matrix.h:270-303)
//   fuse_matrix/neuronN/N_L_fuse.tsv     L rows of N numbers: the activation
//                                        row that block row r of layer l reads
//
// The reference multiplies the value of weight (u, v) with activation row
// fuse[l][u] (src/kernels/kernel.cu:257-275); the layer handed to the engine
// is therefore W[fuse[l][u]][v] += val, the true product over every weight.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <utility>
#include <vector>

#include "cospdnn_b200.h"

namespace cospdnn_cli {

inline void die(const std::string &msg) {
    std::cout << msg << std::endl;
    std::exit(-1);
}

inline void check(int rc, const char *what) {
    if (rc != COSPDNN_OK) die(std::string(what) + ": " + cospdnn_last_error());
}

inline float bias_of(int neuron) {
    switch (neuron) {
        case 65536: return -0.45f;
        case 16384: return -0.4f;
        case 4096: return -0.35f;
        case 1024: return -0.3f;
        default: return -0.3f;
    }
}

// Dense rows [batch][neuron]; `integral` stays true while every value is an
// integer in 0..255 (then the rows are handed over as bytes).
struct Input {
    std::vector<float> rows;
    bool integral = true;
    long read = 0;
};

inline Input read_input(int neuron, int batch, const std::string &dir) {
    const std::string name = dir + "/sparse-images-" + std::to_string(neuron) + ".tsv";
    std::ifstream f(name);
    if (!f) die("FILE:" + name + " does not exists.");
    Input in;
    in.rows.assign((size_t)batch * neuron, 0.0f);
    long b, n;
    float val;
    while (f >> b >> n >> val) {
        if (b < 1 || b > batch) continue;
        if (n < 1 || n > neuron) die("input neuron index out of range in " + name);
        in.rows[(size_t)(b - 1) * neuron + (n - 1)] = val;
        if (!(val >= 0.0f && val <= 255.0f && (float)(int)val == val)) in.integral = false;
        ++in.read;
    }
    std::cout << "Read Input success! read_numeber = " << in.read << std::endl;
    return in;
}

inline std::vector<std::vector<int32_t>> read_fuse(int neuron, int layers, const std::string &dir) {
    const std::string name = dir + "/fuse_matrix/neuron" + std::to_string(neuron) + "/" + std::to_string(neuron) +
                             "_" + std::to_string(layers) + "_fuse.tsv";
    std::ifstream f(name);
    if (!f) die("FILE:" + name + " does not exists.");
    std::vector<std::vector<int32_t>> fuse(layers, std::vector<int32_t>(neuron));
    for (int l = 0; l < layers; ++l)
        for (int j = 0; j < neuron; ++j) {
            float t;
            if (!(f >> t)) die(" read error");
            fuse[l][j] = (int32_t)t;
            if (fuse[l][j] < 0 || fuse[l][j] >= neuron) die("fuse entry out of range in " + name);
        }
    std::cout << "Read fuse success!" << std::endl;
    return fuse;
}

// One layer as CSC over (activation row, output), fuse applied, duplicates summed.
struct Csc {
    std::vector<int32_t> colptr, rowidx;
    std::vector<float> vals;
};

inline Csc read_layer(int neuron, int l, const std::vector<int32_t> &fuse, const std::string &dir) {
    const std::string name =
        dir + "/neuron" + std::to_string(neuron) + "/" + std::to_string(neuron) + "-l" + std::to_string(l + 1) + ".tsv";
    std::ifstream f(name);
    if (!f) die("File:" + name + " does not exists.");
    std::vector<std::vector<std::pair<int32_t, float>>> cols(neuron);
    long u, v;
    float val;
    while (f >> u >> v >> val) {
        if (u < 1 || u > neuron || v < 1 || v > neuron) die("weight index out of range in " + name);
        cols[v - 1].push_back({fuse[u - 1], val});
    }
    Csc c;
    c.colptr.assign(neuron + 1, 0);
    for (int j = 0; j < neuron; ++j) {
        auto &e = cols[j];
        std::sort(e.begin(), e.end(),
                  [](const std::pair<int32_t, float> &a, const std::pair<int32_t, float> &b) { return a.first < b.first; });
        for (size_t t = 0; t < e.size(); ++t) {
            if ((int)c.rowidx.size() > c.colptr[j] && c.rowidx.back() == e[t].first) c.vals.back() += e[t].second;
            else {
                c.rowidx.push_back(e[t].first);
                c.vals.push_back(e[t].second);
            }
        }
        c.colptr[j + 1] = (int32_t)c.rowidx.size();
    }
    return c;
}

// One network as the engine sees it.
struct Network {
    int neuron = 0, batch = 0, layers = 0;
    Input input;
    std::vector<Csc> w;
};

inline Network load_network(int neuron, int batch, int layers, const std::string &dir) {
    Network n;
    n.neuron = neuron;
    n.batch = batch;
    n.layers = layers;
    n.input = read_input(neuron, batch, dir);
    const auto fuse = read_fuse(neuron, layers, dir);
    for (int l = 0; l < layers; ++l) n.w.push_back(read_layer(neuron, l, fuse[l], dir));
    return n;
}

// Adds rows [r0, r1) of `net` to engine `e`; returns the net id.
inline int add_network(cospdnn_engine *e, const Network &net, int r0, int r1, int precision, int kernel) {
    cospdnn_net_desc d{};
    d.neuron = net.neuron;
    d.layers = net.layers;
    d.rows = r1 - r0;
    d.bias = bias_of(net.neuron);
    d.threshold = 1e-5f;
    d.precision = precision;
    d.kernel = kernel;
    int id = -1;
    check(cospdnn_engine_add_net(e, &d, &id), "add_net");
    for (int l = 0; l < net.layers; ++l)
        check(cospdnn_engine_set_layer_csc(e, id, l, net.w[l].colptr.data(), net.w[l].rowidx.data(),
                                           net.w[l].vals.data()),
              "set_layer_csc");
    return id;
}

inline void set_rows(cospdnn_engine *e, int id, const Network &net, int r0, int r1) {
    if (r1 <= r0) return;
    const float *src = net.input.rows.data() + (size_t)r0 * net.neuron;
    if (net.input.integral) {
        std::vector<uint8_t> b((size_t)(r1 - r0) * net.neuron);
        for (size_t i = 0; i < b.size(); ++i) b[i] = (uint8_t)src[i];
        // from pageable memory the copy has left `b` when the call returns
        check(cospdnn_engine_set_input(e, id, b.data(), COSPDNN_INPUT_U8, 0, nullptr), "set_input");
    } else {
        check(cospdnn_engine_set_input(e, id, src, COSPDNN_INPUT_F32, 0, nullptr), "set_input");
    }
}

// Precision and kernel from the environment (COSPDNN_PRECISION = fp32 | fp16
// | bf16, default fp16; COSPDNN_KERNEL = auto | cuda-core | tcgen05).
inline int env_precision() {
    const char *p = std::getenv("COSPDNN_PRECISION");
    const std::string s = p ? p : "fp16";
    if (s == "fp32") return COSPDNN_PREC_FP32;
    if (s == "bf16") return COSPDNN_PREC_BF16;
    return COSPDNN_PREC_FP16;
}
inline int env_kernel() {
    const char *p = std::getenv("COSPDNN_KERNEL");
    const std::string s = p ? p : "auto";
    if (s == "cuda-core") return COSPDNN_KERNEL_CUDA_CORE;
    if (s == "tcgen05") return COSPDNN_KERNEL_TCGEN05;
    return COSPDNN_KERNEL_AUTO;
}

}  // namespace cospdnn_cli
