"""The edge colouring behind the bank-conflict-free entry schedules of the
row-tile and bit-count kernels (cospdnn::colour_group, host code in the
CUDA library), on the CPU: for bipartite multigraphs of lanes x banks it
uses exactly D colours, D = the largest degree (Koenig's theorem), and no two
edges of one colour share a lane or a bank, so the 32 lanes of one step read
32 distinct banks."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "cospdnn_b200")

HARNESS = r"""
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>
namespace cospdnn {
int colour_group(int P, const std::vector<int> &eu, const std::vector<int> &es, std::vector<int> &colour);
}
static unsigned long long s = 88172645463325252ull;
static unsigned rnd(unsigned n) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (unsigned)(s % n); }
int main() {
    int graphs = 0;
    for (int P : {1, 4, 8, 16, 32})
        for (int rep = 0; rep < 300; ++rep, ++graphs) {
            // lane degrees up to 63 (real entries per output); banks drawn
            // uniformly, or from a few banks (heavy multi-edges) every third graph
            std::vector<int> eu, es;
            const int span = rep % 3 == 0 ? std::min(P, 1 + (int)rnd(3)) : P;
            for (int u = 0; u < P; ++u) {
                const int deg = rep % 5 == 0 ? 0 : (int)rnd(64);
                for (int k = 0; k < deg; ++k) {
                    eu.push_back(u);
                    es.push_back((int)rnd(span));
                }
            }
            std::vector<int> du(P, 0), ds(P, 0);
            int D = 0;
            for (size_t e = 0; e < eu.size(); ++e) {
                D = std::max(D, ++du[eu[e]]);
                D = std::max(D, ++ds[es[e]]);
            }
            std::vector<int> colour;
            const int got = cospdnn::colour_group(P, eu, es, colour);
            if (got != D || colour.size() != eu.size()) {
                printf("P=%d rep=%d: %d colours for max degree %d\n", P, rep, got, D);
                return 1;
            }
            std::vector<char> usedU((size_t)P * (D + 1), 0), usedS((size_t)P * (D + 1), 0);
            for (size_t e = 0; e < eu.size(); ++e) {
                const int c = colour[e];
                if (c < 0 || c >= D || usedU[(size_t)eu[e] * D + c] || usedS[(size_t)es[e] * D + c]) {
                    printf("P=%d rep=%d: edge %zu colour %d clashes\n", P, rep, e, c);
                    return 1;
                }
                usedU[(size_t)eu[e] * D + c] = usedS[(size_t)es[e] * D + c] = 1;
            }
        }
    printf("ok %d\n", graphs);
    return 0;
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    gxx = shutil.which("g++")
    lib = os.path.join(LIBDIR, "libcospdnn_b200.so")
    if gxx is None or not os.path.exists(lib):
        pytest.skip("g++ or the built library missing")
    d = tmp_path_factory.mktemp("colour")
    src = d / "h.cpp"
    src.write_text(HARNESS)
    exe = d / "h"
    subprocess.run([gxx, "-O1", "-std=c++17", str(src), "-o", str(exe), "-L", LIBDIR, "-lcospdnn_b200",
                    f"-Wl,-rpath,{LIBDIR}"], check=True, timeout=300)
    return str(exe)


def test_colouring_uses_max_degree_colours_and_is_proper(harness):
    out = subprocess.run([harness], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "ok 1500"
