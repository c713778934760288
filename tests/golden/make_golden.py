"""Generates the BCSC golden fixtures in this directory.

Each case writes a COO weight file in the reference's TSV format
(src/cospdnn.cpp:72-79: 'u v val', 1-based, u = input row), runs the
reference's own COO reader + greedy BCSC builder (src/utils/matrix.h,
compiled from the reference sources into oracle/_ref/ref_bcsc_dump by
`make -C oracle ref`), and stores the input triplets together with the
reference's col_ptr / row_index / col_index / values arrays in bcsc_<case>.npz.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import pyoracle as po  # noqa: E402

DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_bcsc_dump")
OUT = os.path.dirname(os.path.abspath(__file__))


def xor_case(seed, n, nmask):
    m = po.xor_masks(seed, 0, 0, n, nmask)
    cp, ri, vv = po.masks_to_csc(m, n)
    return po.csc_to_coo(cp, ri, vv)


def r1_case(seed, n):
    m = po.r1_masks(seed, 0, 0, n)
    cp, ri, vv = po.masks_to_csc(m, n)
    return po.csc_to_coo(cp, ri, vv)


def random_case(seed, n, nnz, empty_cols=()):
    rng = np.random.default_rng(seed)
    cells = set()
    while len(cells) < nnz:
        r, c = int(rng.integers(n)), int(rng.integers(n))
        if c in empty_cols:
            continue
        cells.add((r, c))
    cells = sorted(cells)
    row = np.array([x[0] for x in cells], np.int32)
    col = np.array([x[1] for x in cells], np.int32)
    # values exactly representable in the TSV's %.6g and in float
    val = (rng.integers(-16, 17, len(cells)) / 8.0).astype(np.float32)
    val[val == 0] = 0.125
    return row, col, val


CASES = {
    "xor_n64_m8": (lambda: xor_case(11, 64, 8), 16),
    "xor_n128_m32": (lambda: xor_case(12, 128, 32), 16),
    "xor_n256_m32": (lambda: xor_case(13, 256, 32), 16),
    "r1_n256": (lambda: r1_case(14, 256), 16),
    "rand_n96": (lambda: random_case(15, 96, 400), 16),
    "rand_n80_gaps": (lambda: random_case(16, 80, 250, empty_cols=(17, 18, 40)), 16),
    "xor_n64_bs8": (lambda: xor_case(17, 64, 8), 8),
}


def main():
    if not os.path.exists(DUMP):
        sys.exit("build the reference checker first: make -C oracle ref")
    with tempfile.TemporaryDirectory() as td:
        for name, (gen, bs) in CASES.items():
            row, col, val = gen()
            tsv = os.path.join(td, name + ".tsv")
            po.write_weight_tsv(tsv, row, col, val)
            out = os.path.join(td, name + ".bin")
            subprocess.check_call([DUMP, tsv, str(bs), out])
            cp, ri, ci, vals = po.read_bcsc_dump(out, bs)
            np.savez_compressed(os.path.join(OUT, f"bcsc_{name}.npz"), row=row, col=col, val=val,
                                bs=np.int32(bs), col_ptr=cp, row_index=ri, col_index=ci,
                                values=vals)
            print(f"{name}: nnz={len(row)} blocks={len(ri)} blockcols={len(cp) - 1}")


if __name__ == "__main__":
    main()
