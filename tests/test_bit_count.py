"""The integer logic of the layer-0 bit-count kernels on the CPU
(cospdnn_b200/csrc/bit_count.cuh, host and device code): carry-save
counters fed eight words at a time, then the 8x8 bit transpose that gives
every bit position's count as a byte.  Checked against plain popcounts per
position for the 32-row units of row-tile nets (byte b of word k = row 8b + k)
and for the 16-row units of MMA-tile nets (two entries' 16-bit words per
32-bit word; word k plus itself shifted by 16 gives rows k and 8 + k in bytes
0 and 1), over entry counts 0..63 and densities from empty to full.  Also the
exact count-to-float step: 2^23 + count as a float's bits, less 2^23."""
import os
import shutil
import struct
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r"""
#include <cstdio>
#include "bit_count.cuh"
using namespace cospdnn;

static uint64_t s = 0x9E3779B97F4A7C15ull;
static uint32_t rnd() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (uint32_t)s; }
// a word whose bits are set with probability d/8
static uint32_t word(int d) {
    if (d == 0) return 0u;
    if (d == 8) return 0xFFFFFFFFu;
    uint32_t w = 0;
    for (int b = 0; b < 32; ++b) w |= (uint32_t)((rnd() & 7u) < (uint32_t)d) << b;
    return w;
}
static void count(const uint32_t *x, int n, uint32_t (&c)[8]) {
    uint32_t p[6] = {0u, 0u, 0u, 0u, 0u, 0u};
    for (int t = 0; t < n; t += 8) {
        uint32_t y[8];
        for (int i = 0; i < 8; ++i) y[i] = t + i < n ? x[t + i] : 0u;  // zero padding words
        add8(p, y);
    }
    counts8(p, c);
}
int main() {
    int cases = 0;
    for (int K = 0; K <= 63; ++K)
        for (int d = 0; d <= 8; ++d)
            for (int rep = 0; rep < 4; ++rep, ++cases) {
                // 32-row units: K words of 32 rows
                uint32_t x[64], c[8];
                for (int i = 0; i < K; ++i) x[i] = word(d);
                count(x, K, c);
                for (int r = 0; r < 32; ++r) {
                    int want = 0;
                    for (int i = 0; i < K; ++i) want += (x[i] >> r) & 1u;
                    const int got = (c[r % 8] >> (8 * (r / 8))) & 0xFFu;
                    if (got != want) {
                        printf("32-row K=%d d=%d row %d: %d != %d\n", K, d, r, got, want);
                        return 1;
                    }
                }
                // 16-row units: K entries of 16 rows, two per word (even entry low)
                uint16_t h[64];
                for (int i = 0; i < K; ++i) h[i] = (uint16_t)word(d);
                uint32_t pk[32];
                const int n = (K + 1) / 2;
                for (int t = 0; t < n; ++t)
                    pk[t] = (uint32_t)h[2 * t] | (2 * t + 1 < K ? (uint32_t)h[2 * t + 1] << 16 : 0u);
                count(pk, n, c);
                for (int r = 0; r < 16; ++r) {
                    int want = 0;
                    for (int i = 0; i < K; ++i) want += (h[i] >> r) & 1u;
                    const uint32_t s2 = c[r % 8] + (c[r % 8] >> 16);
                    const int got = (s2 >> (8 * (r / 8))) & 0xFFu;
                    if (got != want) {
                        printf("16-row K=%d d=%d row %d: %d != %d\n", K, d, r, got, want);
                        return 1;
                    }
                }
            }
    printf("ok %d\n", cases);
    return 0;
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    d = tmp_path_factory.mktemp("bitcount")
    src = d / "h.cu"
    src.write_text(HARNESS)
    exe = d / "h"
    subprocess.run([nvcc, "-O1", "-std=c++17", "-Wno-deprecated-gpu-targets", "-I",
                    os.path.join(ROOT, "cospdnn_b200", "csrc"), str(src), "-o", str(exe)], check=True, timeout=300)
    return str(exe)


def test_counters_and_transpose(harness):
    out = subprocess.run([harness], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == f"ok {64 * 9 * 4}"


def test_count_as_float_exact():
    for c in range(256):
        f = struct.unpack("<f", struct.pack("<I", 0x4B000000 | c))[0]
        assert f - 8388608.0 == c
