"""Store the reference's shipped interior Gauss-Lobatto nodes as a golden fixture.

Reads ``src/workingData/mesh/legendreRoots/roots%05d.txt`` of the reference (the node files that
internal.py:526 loads) for N = 32 .. 1024 and writes ``tests/golden/lobatto_roots.npz``
(``roots02048.txt`` is all NaN in the reference and is skipped).

Usage:  python tests/golden/make_lobatto_fixture.py /root/reference/src/workingData/mesh/legendreRoots
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(src):
    out = {}
    for n in (32, 64, 128, 256, 512, 1024):
        out[f"n{n}"] = np.genfromtxt(os.path.join(src, f"roots{n:05d}.txt"), delimiter=",")
    np.savez_compressed(os.path.join(HERE, "lobatto_roots.npz"), **out)


if __name__ == "__main__":
    main(sys.argv[1])
