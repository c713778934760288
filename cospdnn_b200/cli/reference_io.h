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
//
// Binary cache (COSPDNN_CACHE=<dir>): a parsed network is kept in
// <dir>/cospdnn-n{N}-b{B}-l{L}.bin -- the input rows (bytes when integral)
// and every layer's CSC with the fuse applied -- behind a header holding the
// size and modification time of every source file; a run whose sources no
// longer match the header parses the TSV files again and rewrites the cache
// (written to a temporary name, then renamed).
//
// Categories (Graph Challenge format): the surviving input rows, 1-based,
// one per line, ascending.  COSPDNN_CATEGORIES=<file> writes them and
// COSPDNN_TRUTH=<file> compares them with a truth file of that format
// (cospdnn_double.out: COSPDNN_CATEGORIES_1/_2, COSPDNN_TRUTH_1/_2).
#pragma once

#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <string>
#include <thread>
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

// Whitespace-separated decimal numbers of a file, read in blocks (the files
// of the 65536-neuron networks hold tens of millions of lines): integers as
// strtol and values as strtof read them, which is what the stream
// extraction of the reference's readers (`f >> u >> v >> val`) yields for
// such tokens.  next() is false at the end of the file and at a token that
// is not a number of its kind; the readers stop there, as the reference's
// `while (f >> ...)` loops do.
class NumReader {
  public:
    // block: bytes read at a time (at least twice the longest token)
    explicit NumReader(const std::string &name, size_t block = 16u << 20)
        : f_(std::fopen(name.c_str(), "rb")), block_(std::max(block, 2 * kToken)), buf_(block_ + 1) {}
    ~NumReader() {
        if (f_) std::fclose(f_);
    }
    NumReader(const NumReader &) = delete;
    NumReader &operator=(const NumReader &) = delete;
    bool ok() const { return f_ != nullptr; }
    // a read failed (a directory, an I/O error): the numbers stopped there
    bool failed() const { return err_; }
    bool next(long &x) {
        if (!token()) return false;
        char *e = nullptr;
        x = std::strtol(p_, &e, 10);
        if (e == p_) return false;
        p_ = e;
        return true;
    }
    bool next(float &x) {
        if (!token()) return false;
        // decimal and exponent forms, as the stream extraction takes them:
        // no inf or nan; "0x..." is the value 0 followed by the token "x..."
        const char *d = p_ + (*p_ == '+' || *p_ == '-');
        if (!((*d >= '0' && *d <= '9') || *d == '.')) return false;
        if (d[0] == '0' && (d[1] == 'x' || d[1] == 'X')) {
            x = *p_ == '-' ? -0.0f : 0.0f;
            p_ = const_cast<char *>(d) + 1;
            return true;
        }
        char *e = nullptr;
        x = std::strtof(p_, &e);
        if (e == p_) return false;
        // an exponent without digits ("1e", "1e+") fails the stream extraction
        if ((*e == 'e' || *e == 'E') && std::find_if(p_, e, [](char ch) { return ch == 'e' || ch == 'E'; }) == e)
            return false;
        p_ = e;
        return true;
    }

  private:
    static constexpr size_t kToken = 4096;  // longest token read whole
    // skips white space; true when a token starts at p_ with at least kToken
    // bytes (or the rest of the file) behind it in the buffer
    bool token() {
        for (;;) {
            while (p_ < end_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r' || *p_ == '\v' ||
                                 *p_ == '\f'))
                ++p_;
            if (eof_ || (size_t)(end_ - p_) >= kToken) return p_ < end_;
            const size_t keep = (size_t)(end_ - p_);
            if (keep) std::memmove(buf_.data(), p_, keep);
            const size_t got = f_ ? std::fread(buf_.data() + keep, 1, block_ - keep, f_) : 0;
            eof_ = got < block_ - keep;
            if (eof_ && f_ && std::ferror(f_)) err_ = true;
            p_ = buf_.data();
            end_ = p_ + keep + got;
            *end_ = '\0';  // strtol/strtof stop here
        }
    }
    std::FILE *f_;
    size_t block_;
    std::vector<char> buf_;
    char *p_ = nullptr, *end_ = nullptr;
    bool eof_ = false, err_ = false;
};

// Dense rows [batch][neuron]; `integral` stays true while every value is an
// integer in 0..255 (then the rows are handed over as bytes).
struct Input {
    std::vector<float> rows;
    bool integral = true;
    long read = 0;
};

// Reads the images into in; returns "" or what is wrong with the file (read
// on its own thread while the layers are parsed, the caller reports it).
inline std::string read_input(int neuron, int batch, const std::string &dir, Input &in) {
    const std::string name = dir + "/sparse-images-" + std::to_string(neuron) + ".tsv";
    NumReader f(name);
    if (!f.ok()) return "FILE:" + name + " does not exists.";
    in = Input();
    in.rows.assign((size_t)batch * neuron, 0.0f);
    long b, n;
    float val;
    while (f.next(b) && f.next(n) && f.next(val)) {
        if (b < 1 || b > batch) continue;
        if (n < 1 || n > neuron) return "input neuron index out of range in " + name;
        in.rows[(size_t)(b - 1) * neuron + (n - 1)] = val;
        if (!(val >= 0.0f && val <= 255.0f && (float)(int)val == val)) in.integral = false;
        ++in.read;
    }
    if (f.failed()) return "FILE:" + name + " cannot be read.";
    return "";
}

// Reads the fuse rows of every layer; returns "" or what is wrong with the file.
inline std::string read_fuse(int neuron, int layers, const std::string &dir, std::vector<std::vector<int32_t>> &fuse) {
    const std::string name = dir + "/fuse_matrix/neuron" + std::to_string(neuron) + "/" + std::to_string(neuron) +
                             "_" + std::to_string(layers) + "_fuse.tsv";
    NumReader f(name);
    if (!f.ok()) return "FILE:" + name + " does not exists.";
    fuse.assign(layers, std::vector<int32_t>(neuron));
    for (int l = 0; l < layers; ++l)
        for (int j = 0; j < neuron; ++j) {
            float t;
            if (!f.next(t)) return f.failed() ? "FILE:" + name + " cannot be read." : " read error";
            fuse[l][j] = (int32_t)t;
            if (fuse[l][j] < 0 || fuse[l][j] >= neuron) return "fuse entry out of range in " + name;
        }
    return "";
}

// One layer as CSC over (activation row, output), fuse applied, duplicates summed.
struct Csc {
    std::vector<int32_t> colptr, rowidx;
    std::vector<float> vals;
};

// Reads layer l into c; returns "" or the message of what is wrong with the
// file (layers are read on several threads, the caller reports it).  The
// message prefix is the one each of the reference's readers prints: "FILE:"
// for the images and the fuse file (src/cospdnn.cpp:21,52), "File:" for a
// layer file (src/utils/matrix.h:277); a file that exists but cannot be read
// takes the same prefix as its missing-file line.
inline std::string read_layer(int neuron, int l, const std::vector<int32_t> &fuse, const std::string &dir, Csc &c) {
    const std::string name =
        dir + "/neuron" + std::to_string(neuron) + "/" + std::to_string(neuron) + "-l" + std::to_string(l + 1) + ".tsv";
    NumReader f(name);
    if (!f.ok()) return "File:" + name + " does not exists.";
    std::vector<std::vector<std::pair<int32_t, float>>> cols(neuron);
    long u, v;
    float val;
    while (f.next(u) && f.next(v) && f.next(val)) {
        if (u < 1 || u > neuron || v < 1 || v > neuron) return "weight index out of range in " + name;
        cols[v - 1].push_back({fuse[u - 1], val});
    }
    if (f.failed()) return "File:" + name + " cannot be read.";
    c = Csc();
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
    return "";
}

// One network as the engine sees it.
struct Network {
    int neuron = 0, batch = 0, layers = 0;
    Input input;
    std::vector<Csc> w;
};

inline std::string input_path(int neuron, const std::string &dir) {
    return dir + "/sparse-images-" + std::to_string(neuron) + ".tsv";
}
inline std::string fuse_path(int neuron, int layers, const std::string &dir) {
    return dir + "/fuse_matrix/neuron" + std::to_string(neuron) + "/" + std::to_string(neuron) + "_" +
           std::to_string(layers) + "_fuse.tsv";
}
inline std::string layer_path(int neuron, int l, const std::string &dir) {
    return dir + "/neuron" + std::to_string(neuron) + "/" + std::to_string(neuron) + "-l" + std::to_string(l + 1) +
           ".tsv";
}

inline Network parse_network(int neuron, int batch, int layers, const std::string &dir) {
    Network n;
    n.neuron = neuron;
    n.batch = batch;
    n.layers = layers;
    // the images on one thread; the fuse, then the layer files (independent)
    // on one thread per core; messages in file order once all are read
    std::string ein, efuse;
    std::thread tin([&] { ein = read_input(neuron, batch, dir, n.input); });
    std::vector<std::vector<int32_t>> fuse;
    efuse = read_fuse(neuron, layers, dir, fuse);
    n.w.resize(layers);
    std::vector<std::string> err(layers);
    if (efuse.empty()) {
        std::atomic<int> next{0};
        auto work = [&] {
            for (int l; (l = next++) < layers;) err[l] = read_layer(neuron, l, fuse[l], dir, n.w[l]);
        };
        const int nt = std::max(1, std::min(layers, (int)std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t) pool.emplace_back(work);
        work();
        for (auto &t : pool) t.join();
    }
    tin.join();
    if (!ein.empty()) die(ein);
    std::cout << "Read Input success! read_numeber = " << n.input.read << std::endl;
    if (!efuse.empty()) die(efuse);
    std::cout << "Read fuse success!" << std::endl;
    for (int l = 0; l < layers; ++l)
        if (!err[l].empty()) die(err[l]);
    return n;
}

// ---- binary cache ---------------------------------------------------------
constexpr char kCacheMagic[8] = {'C', 'S', 'P', 'D', 'N', 'N', 'C', '1'};

// (size, mtime in ns) of every source file, in a fixed order; empty if one is missing
inline std::vector<int64_t> source_signature(int neuron, int layers, const std::string &dir) {
    std::vector<std::string> files = {input_path(neuron, dir), fuse_path(neuron, layers, dir)};
    for (int l = 0; l < layers; ++l) files.push_back(layer_path(neuron, l, dir));
    std::vector<int64_t> sig;
    for (const auto &f : files) {
        struct stat st;
        if (stat(f.c_str(), &st) != 0) return {};
        sig.push_back((int64_t)st.st_size);
        sig.push_back((int64_t)st.st_mtim.tv_sec * 1000000000LL + st.st_mtim.tv_nsec);
    }
    return sig;
}

inline std::string cache_path(const std::string &cache_dir, int neuron, int batch, int layers) {
    return cache_dir + "/cospdnn-n" + std::to_string(neuron) + "-b" + std::to_string(batch) + "-l" +
           std::to_string(layers) + ".bin";
}

template <typename T>
inline bool put(std::FILE *f, const T *p, size_t n) {
    return n == 0 || std::fwrite(p, sizeof(T), n, f) == n;
}
template <typename T>
inline bool get(std::FILE *f, T *p, size_t n) {
    return n == 0 || std::fread(p, sizeof(T), n, f) == n;
}

inline bool write_cache(const std::string &path, const Network &n, const std::vector<int64_t> &sig) {
    const std::string tmp = path + ".tmp" + std::to_string((long)getpid());
    std::FILE *f = std::fopen(tmp.c_str(), "wb");
    if (!f) return false;
    const int32_t hdr[4] = {n.neuron, n.batch, n.layers, n.input.integral ? 1 : 0};
    const int64_t nsig = (int64_t)sig.size(), nread = n.input.read;
    bool ok = put(f, kCacheMagic, 8) && put(f, hdr, 4) && put(f, &nsig, 1) && put(f, sig.data(), sig.size()) &&
              put(f, &nread, 1);
    if (n.input.integral) {
        std::vector<uint8_t> b(n.input.rows.size());
        for (size_t i = 0; i < b.size(); ++i) b[i] = (uint8_t)n.input.rows[i];
        ok = ok && put(f, b.data(), b.size());
    } else {
        ok = ok && put(f, n.input.rows.data(), n.input.rows.size());
    }
    for (const auto &c : n.w) {
        const int64_t nnz = (int64_t)c.rowidx.size();
        ok = ok && put(f, &nnz, 1) && put(f, c.colptr.data(), c.colptr.size()) && put(f, c.rowidx.data(), c.rowidx.size()) &&
             put(f, c.vals.data(), c.vals.size());
    }
    ok = (std::fclose(f) == 0) && ok;
    if (ok) ok = std::rename(tmp.c_str(), path.c_str()) == 0;
    if (!ok) std::remove(tmp.c_str());
    return ok;
}

// true when `path` holds this network and its header matches `sig`
inline bool read_cache(const std::string &path, int neuron, int batch, int layers, const std::vector<int64_t> &sig,
                       Network &n) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    char magic[8];
    int32_t hdr[4];
    int64_t nsig = 0;
    bool ok = get(f, magic, 8) && std::memcmp(magic, kCacheMagic, 8) == 0 && get(f, hdr, 4) && hdr[0] == neuron &&
              hdr[1] == batch && hdr[2] == layers && get(f, &nsig, 1) && nsig == (int64_t)sig.size();
    std::vector<int64_t> old(ok ? (size_t)nsig : 0);
    ok = ok && get(f, old.data(), old.size()) && old == sig;
    int64_t nread = 0;
    ok = ok && get(f, &nread, 1);
    if (ok) {
        n.neuron = neuron;
        n.batch = batch;
        n.layers = layers;
        n.input.integral = hdr[3] != 0;
        n.input.read = (long)nread;
        n.input.rows.assign((size_t)batch * neuron, 0.0f);
        if (n.input.integral) {
            std::vector<uint8_t> b(n.input.rows.size());
            ok = get(f, b.data(), b.size());
            for (size_t i = 0; ok && i < b.size(); ++i) n.input.rows[i] = (float)b[i];
        } else {
            ok = get(f, n.input.rows.data(), n.input.rows.size());
        }
    }
    for (int l = 0; ok && l < layers; ++l) {
        Csc c;
        int64_t nnz = -1;
        ok = get(f, &nnz, 1) && nnz >= 0 && nnz <= (int64_t)neuron * neuron;
        if (!ok) break;
        c.colptr.resize(neuron + 1);
        c.rowidx.resize((size_t)nnz);
        c.vals.resize((size_t)nnz);
        ok = get(f, c.colptr.data(), c.colptr.size()) && get(f, c.rowidx.data(), c.rowidx.size()) &&
             get(f, c.vals.data(), c.vals.size()) && c.colptr[0] == 0 && c.colptr[neuron] == nnz;
        for (int j = 0; ok && j < neuron; ++j) ok = c.colptr[j] <= c.colptr[j + 1];
        for (int64_t t = 0; ok && t < nnz; ++t) ok = c.rowidx[t] >= 0 && c.rowidx[t] < neuron;
        if (ok) n.w.push_back(std::move(c));
    }
    std::fclose(f);
    if (!ok) n = Network();
    return ok;
}

// The network from the TSV files, through the binary cache when COSPDNN_CACHE
// names a directory.
inline Network load_network(int neuron, int batch, int layers, const std::string &dir) {
    const char *cdir = std::getenv("COSPDNN_CACHE");
    if (!cdir || !*cdir) return parse_network(neuron, batch, layers, dir);
    const std::string path = cache_path(cdir, neuron, batch, layers);
    const auto sig = source_signature(neuron, layers, dir);
    Network n;
    if (!sig.empty() && read_cache(path, neuron, batch, layers, sig, n)) {
        std::cout << "Read cache success! file = " << path << std::endl;
        return n;
    }
    n = parse_network(neuron, batch, layers, dir);
    if (!sig.empty() && !write_cache(path, n, sig)) std::cout << "cache not written: " << path << std::endl;
    return n;
}

// ---- categories -------------------------------------------------------------
// 0-based surviving rows -> file of 1-based ids, one per line
inline bool write_categories(const std::string &path, const std::vector<int64_t> &cats0) {
    std::ofstream f(path);
    if (!f) return false;
    for (int64_t c : cats0) f << c + 1 << "\n";
    return (bool)f;
}

// 1-based ids of a categories file; false when it cannot be read or holds
// anything but positive integers
inline bool read_categories(const std::string &path, std::vector<int64_t> &ids) {
    struct stat st;
    if (stat(path.c_str(), &st) != 0 || !S_ISREG(st.st_mode)) return false;  // a directory reads as empty
    std::ifstream f(path);
    if (!f) return false;
    ids.clear();
    std::string tok;
    while (f >> tok) {
        char *end = nullptr;
        const long long v = std::strtoll(tok.c_str(), &end, 10);
        if (end == tok.c_str() || *end != '\0' || v < 1) return false;
        ids.push_back(v);
    }
    return true;
}

struct CategoryCheck {
    size_t ours = 0, truth = 0, missing = 0, extra = 0;
    bool ok() const { return missing == 0 && extra == 0; }
};

// ours0: 0-based rows; truth1: 1-based ids
inline CategoryCheck compare_categories(const std::vector<int64_t> &ours0, std::vector<int64_t> truth1) {
    std::vector<int64_t> ours1(ours0.size());
    for (size_t i = 0; i < ours0.size(); ++i) ours1[i] = ours0[i] + 1;
    std::sort(ours1.begin(), ours1.end());
    ours1.erase(std::unique(ours1.begin(), ours1.end()), ours1.end());
    std::sort(truth1.begin(), truth1.end());
    truth1.erase(std::unique(truth1.begin(), truth1.end()), truth1.end());
    std::vector<int64_t> d;
    CategoryCheck r;
    r.ours = ours1.size();
    r.truth = truth1.size();
    std::set_difference(truth1.begin(), truth1.end(), ours1.begin(), ours1.end(), std::back_inserter(d));
    r.missing = d.size();
    d.clear();
    std::set_difference(ours1.begin(), ours1.end(), truth1.begin(), truth1.end(), std::back_inserter(d));
    r.extra = d.size();
    return r;
}

// Writes and checks the categories as the environment asks; returns 0, or 2
// when a truth file was given and does not match.
inline int report_categories(const std::vector<int64_t> &cats0, const char *out_env, const char *truth_env,
                             const std::string &label) {
    const char *out = std::getenv(out_env);
    if (out && *out) {
        if (!write_categories(out, cats0)) die(std::string("cannot write ") + out);
        std::cout << label << "categories written: " << out << std::endl;
    }
    const char *truth = std::getenv(truth_env);
    if (!truth || !*truth) return 0;
    std::vector<int64_t> t;
    if (!read_categories(truth, t)) die(std::string("cannot read truth file ") + truth);
    const CategoryCheck r = compare_categories(cats0, t);
    std::cout << label << "categories check: " << (r.ok() ? "PASS" : "FAIL") << " (ours " << r.ours << ", truth "
              << r.truth << ", missing " << r.missing << ", extra " << r.extra << ")" << std::endl;
    return r.ok() ? 0 : 2;
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
// FNV-1a (64-bit) of the categories file these rows make (Graph Challenge
// format: 1-based ids, one per line, ascending), so that a run can be compared
// with a truth file by its hash (cospdnn_b200.categories computes the same).
inline uint64_t categories_hash(const std::vector<int64_t> &cats0) {
    std::vector<int64_t> c(cats0);
    std::sort(c.begin(), c.end());
    c.erase(std::unique(c.begin(), c.end()), c.end());
    uint64_t h = 0xcbf29ce484222325ull;  // FNV-1a offset basis; prime 2^40 + 2^8 + 0xb3
    for (int64_t r : c) {
        const std::string line = std::to_string(r + 1) + "\n";
        for (unsigned char ch : line) h = (h ^ ch) * 1099511628211ull;
    }
    return h;
}

// What a run reports in its JSON result line.
struct RunReport {
    std::string program;
    int network = 0;  // 1 or 2 in the two-network program, else 0
    int neuron = 0, batch = 0, layers = 0, precision = COSPDNN_PREC_FP16, kernel = COSPDNN_KERNEL_AUTO, gpus = 1;
    int64_t weights = 0;  // non-zeros over all layers
    float ms = 0.0f;      // device time of the run (max over GPUs)
    float dy_bound = 0.0f;  // max proven |final value - FP64 value| over the categories
    std::vector<int64_t> alive, rechecked, categories;
};

// The result line: sizes, device time, edges = rows x non-zeros of every
// layer and edges/s, the largest proven bound on |final value - FP64 value|
// over the categories (the error against an FP64 recurrence of the same
// network, as the engine tracks it), rows alive and rows re-decided in FP64
// per layer, the number of categories and their hash.
inline std::string json_line(const RunReport &r) {
    static const char *prec[] = {"fp32", "fp16", "bf16"};
    static const char *kern[] = {"auto", "cuda-core", "tcgen05"};
    auto list = [](const std::vector<int64_t> &v) {
        std::string t = "[";
        for (size_t i = 0; i < v.size(); ++i) t += (i ? "," : "") + std::to_string(v[i]);
        return t + "]";
    };
    const double edges = (double)r.batch * (double)r.weights;
    char num[160];
    std::snprintf(num, sizeof num, "\"ms\": %.6g, \"edges\": %.17g, \"edges_per_s\": %.6g, \"max_abs_dy_bound\": %.6g",
                  (double)r.ms, edges, r.ms > 0.0f ? edges / (r.ms * 1e-3) : 0.0, (double)r.dy_bound);
    char hash[40];
    std::snprintf(hash, sizeof hash, "%016llx", (unsigned long long)categories_hash(r.categories));
    std::string j = "{\"program\": \"" + r.program + "\"";
    if (r.network) j += ", \"network\": " + std::to_string(r.network);
    j += ", \"neuron\": " + std::to_string(r.neuron) + ", \"batch\": " + std::to_string(r.batch) +
         ", \"layers\": " + std::to_string(r.layers) + ", \"precision\": \"" +
         prec[std::min(std::max(r.precision, 0), 2)] + "\", \"kernel\": \"" + kern[std::min(std::max(r.kernel, 0), 2)] +
         "\", \"gpus\": " + std::to_string(r.gpus) + ", \"weights\": " + std::to_string(r.weights) + ", " + num +
         ", \"alive\": " + list(r.alive) + ", \"fp64_rechecked\": " + list(r.rechecked) +
         ", \"categories\": " + std::to_string(r.categories.size()) + ", \"category_hash\": \"fnv1a64:" + hash +
         "\"}";
    return j;
}

// COSPDNN_JSON=1 prints the result line; any other value appends it to the
// file it names (unset: nothing, the output stays the reference's).
inline void report_json(const RunReport &r) {
    const char *dst = std::getenv("COSPDNN_JSON");
    if (!dst || !*dst) return;
    const std::string line = json_line(r);
    if (std::string(dst) == "1") {
        std::cout << line << std::endl;
        return;
    }
    std::FILE *f = std::fopen(dst, "a");
    if (!f) die(std::string("cannot write ") + dst);
    std::fprintf(f, "%s\n", line.c_str());
    std::fclose(f);
}

// Per-layer lines of the reference's host loops (printed under its default
// -DPRINT_TEST, src/cospdnn.cu:262-264,302-305 and src/cospdnn_double.cu:
// 794,841,880-882): rows are padded to its 128-column tile.  It compacts
// rows after layers 0..21 only and prints their counts there; this engine
// compacts after every layer, so the batch line carries the padded count of
// the rows it keeps after every layer.
inline int64_t pad_tile(int64_t rows) { return (rows + 127) / 128 * 128; }

// COSPDNN_LAYER_TIMES=0 skips the per-layer timing pass (the layer lines then
// show 0 ms); by default the layer loop is run once more kernel by kernel to
// time each layer's kernels, as the reference's per-layer events do.
inline bool env_layer_times() {
    const char *p = std::getenv("COSPDNN_LAYER_TIMES");
    return !(p && std::string(p) == "0");
}

inline int env_precision() {
    const char *p = std::getenv("COSPDNN_PRECISION");
    const std::string s = p && *p ? p : "fp16";
    if (s == "fp32") return COSPDNN_PREC_FP32;
    if (s == "bf16") return COSPDNN_PREC_BF16;
    if (s != "fp16") die("COSPDNN_PRECISION must be fp32, fp16 or bf16, not " + s);
    return COSPDNN_PREC_FP16;
}
inline int env_kernel() {
    const char *p = std::getenv("COSPDNN_KERNEL");
    const std::string s = p && *p ? p : "auto";
    if (s == "cuda-core") return COSPDNN_KERNEL_CUDA_CORE;
    if (s == "tcgen05") return COSPDNN_KERNEL_TCGEN05;
    if (s != "auto") die("COSPDNN_KERNEL must be auto, cuda-core or tcgen05, not " + s);
    return COSPDNN_KERNEL_AUTO;
}

}  // namespace cospdnn_cli
