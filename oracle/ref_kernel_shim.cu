// Checker / reference-timing harness (TEST INFRASTRUCTURE).  Compiled together
// with the reference's own, unmodified src/kernels/kernel.cu and src/cospdnn.cu
// (for sm_100a) into oracle/_ref/libref_cospdnn.so.  It only adds plain C entry
// points so that Python tests and bench.py can:
//   * launch the reference layer kernel ftxj::cospdnn_single with the launch
//     shape of src/cospdnn.cu:219-229 (grid (block columns, batch/128), 256 threads);
//   * run the reference's whole host layer loop test_graph_challenge_tc
//     (src/cospdnn.cuh:14-21) on in-memory data, capturing what it prints.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "cospdnn.cuh"

extern "C" int ref_cospdnn_single(const void *A, const void *B, float *C, const int *fuse,
                                  const int *idx_ptr, const int *index, float bias, int batch,
                                  int neuron, int nblockcols, void *stream) {
    dim3 grid(nblockcols, (batch + 127) / 128);
    dim3 block(256);
    ftxj::cospdnn_single<<<grid, block, 0, (cudaStream_t)stream>>>(
        (half *)A, (half *)B, C, (int *)fuse, (int *)idx_ptr, (int *)index, bias, batch, neuron,
        16, 16);
    return (int)cudaGetLastError();
}

// Runs test_graph_challenge_tc on one GPU.  y0: [batch][neuron] bytes (binary
// images); per layer l: values[l] (nval[l] floats), row_index[l] (nrow[l]),
// col_ptr[l] (ncol[l]); fuse_rows[l] (neuron ints: the activation row block
// row r of layer l reads), or the identity when fuse_rows is NULL.  Returns the reference's own printed
// "Kernel Exec Time" in *kernel_ms, the wall time of the call in *wall_ms,
// the last "feature = " count it printed in *last_feature, and every printed
// "layer l, feature = n" count in features[l] (the reference prints these for
// the layers it compacts, l <= 21; src/cospdnn.cu:262-264).
extern "C" int ref_run_network(const uint8_t *y0, int batch, int neuron, int layers,
                               const float *const *values, const int64_t *nval,
                               const int *const *row_index, const int64_t *nrow,
                               const int *const *col_ptr, const int64_t *ncol, float bias,
                               double *kernel_ms, double *wall_ms, int *last_feature,
                               int *features, int max_features, char *log_tail,
                               int log_tail_len, const int *const *fuse_rows) {
    std::vector<std::vector<float>> input(batch, std::vector<float>(neuron));
    for (int b = 0; b < batch; ++b)
        for (int j = 0; j < neuron; ++j) input[b][j] = (float)y0[(int64_t)b * neuron + j];
    std::vector<std::vector<float>> weight(layers);
    std::vector<std::vector<int>> ridx(layers), ptr(layers);
    for (int l = 0; l < layers; ++l) {
        weight[l].assign(values[l], values[l] + nval[l]);
        ridx[l].assign(row_index[l], row_index[l] + nrow[l]);
        ptr[l].assign(col_ptr[l], col_ptr[l] + ncol[l]);
    }
    std::vector<std::vector<int>> fuse(layers + 1, std::vector<int>(neuron));
    for (int l = 0; l <= layers; ++l)
        for (int j = 0; j < neuron; ++j) fuse[l][j] = (fuse_rows && l < layers) ? fuse_rows[l][j] : j;

    std::stringstream captured;
    std::streambuf *old = std::cout.rdbuf(captured.rdbuf());
    cudaDeviceSynchronize();
    auto t0 = std::chrono::steady_clock::now();
    test_graph_challenge_tc(input, weight, ridx, ptr, fuse, batch, neuron, bias, 16, 16, 0, 1);
    cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    std::cout.rdbuf(old);
    *wall_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();

    std::string text = captured.str();
    *kernel_ms = -1.0;
    *last_feature = -1;
    std::istringstream lines(text);
    std::string line;
    while (std::getline(lines, line)) {
        const char *k = "Kernel Exec Time = ";
        size_t p = line.find(k);
        if (p != std::string::npos) *kernel_ms = atof(line.c_str() + p + strlen(k));
        const char *f = ", feature = ";
        p = line.find(f);
        if (p != std::string::npos && line.compare(0, 6, "layer ") == 0) {
            int l = atoi(line.c_str() + 6);
            int n = atoi(line.c_str() + p + strlen(f));
            *last_feature = n;
            if (features && l >= 0 && l < max_features) features[l] = n;
        }
    }
    if (log_tail && log_tail_len > 0) {
        size_t n = text.size() < (size_t)(log_tail_len - 1) ? text.size() : (size_t)(log_tail_len - 1);
        memcpy(log_tail, text.data() + text.size() - n, n);
        log_tail[n] = 0;
    }
    // Once every row is pruned the reference launches its kernels with a zero
    // grid (src/cospdnn.cu:222-229), a non-sticky launch error it never checks;
    // clear it and report only errors that outlive it.
    cudaGetLastError();
    return (int)cudaDeviceSynchronize();
}
