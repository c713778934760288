"""Categories in Graph Challenge format and the check against a truth file.

A categories file lists the input rows (images) that are still alive after
the last layer, as 1-based ids, one per line, ascending -- the format of the
challenge's truth files.  The engine returns 0-based rows.

    python -m cospdnn_b200.categories OURS TRUTH
    python -m cospdnn_b200.categories --hash FILE

compares two such files and exits 0 when they hold the same ids, 2 if not;
--hash prints the FNV-1a (64-bit) hash of the file's ids in that format, the
`category_hash` of the command lines' COSPDNN_JSON result line.
"""
import sys

import numpy as np


def write(path, rows0):
    """Writes 0-based rows as 1-based ids, one per line, ascending."""
    ids = np.unique(np.asarray(rows0, np.int64)) + 1
    with open(path, "w") as f:
        for v in ids.tolist():
            f.write(f"{v}\n")


def read(path):
    """1-based ids of a categories file as sorted unique 0-based rows."""
    with open(path) as f:
        toks = f.read().split()
    ids = []
    for t in toks:
        v = int(t)  # raises ValueError on anything but an integer
        if v < 1:
            raise ValueError(f"{path}: id {v} is not positive")
        ids.append(v - 1)
    return np.unique(np.asarray(ids, np.int64))


def digest(rows0):
    """FNV-1a (64-bit) of the categories file these 0-based rows make (the
    bytes of write()), as 16 hex digits."""
    h = 0xCBF29CE484222325  # FNV-1a offset basis; prime 2^40 + 2^8 + 0xb3
    for v in (np.unique(np.asarray(rows0, np.int64)) + 1).tolist():
        for ch in f"{v}\n".encode():
            h = ((h ^ ch) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return f"{h:016x}"


def check(rows0, truth_path):
    """Compares 0-based rows with a truth file: dict(ok, ours, truth,
    missing, extra) where missing/extra are 0-based rows."""
    ours = np.unique(np.asarray(rows0, np.int64))
    truth = read(truth_path)
    missing = np.setdiff1d(truth, ours)
    extra = np.setdiff1d(ours, truth)
    return {"ok": missing.size == 0 and extra.size == 0, "ours": int(ours.size), "truth": int(truth.size),
            "missing": missing, "extra": extra}


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 2:
        print("usage: python -m cospdnn_b200.categories OURS TRUTH | --hash FILE")
        return 1
    try:
        if argv[0] == "--hash":
            print(f"fnv1a64:{digest(read(argv[1]))}")
            return 0
        r = check(read(argv[0]), argv[1])
    except (OSError, ValueError) as e:  # a missing or malformed file (status 2 is a mismatch)
        print(f"categories: {e}")
        return 1
    print(f"categories check: {'PASS' if r['ok'] else 'FAIL'} (ours {r['ours']}, truth {r['truth']}, "
          f"missing {r['missing'].size}, extra {r['extra'].size})")
    return 0 if r["ok"] else 2


if __name__ == "__main__":
    sys.exit(main())
