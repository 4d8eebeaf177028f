"""Records the reference's own binary-CSR converter output as golden fixtures.

Needs oracle/_ref/greader, built from the reference's
scripts/gbin_reader/greader.cpp by `make -C oracle gbin` where the reference
is mounted.  For each input below (text the converter accepts) it runs

    greader <input.mtx> <outdir>

and stores graph.vertex.bin, graph.edge.bin and graph.meta.txt in
gbin_golden.npz next to this file (the inputs are stored too).

    python tests/golden/make_gbin_golden.py
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
GREADER = os.path.join(ROOT, "oracle", "_ref", "greader")


def inputs():
    out = [
        "5 5 4\n1 2\n2 3\n3 3\n5 1\n",            # self-loop kept, ids from 1
        "4 4 3\n1 2 5\n2 3\n3 4\n",               # a three-token line is skipped
        "4 4 3\n1  2\n2 3\n3 4\n",                # runs of spaces
        "3 3 2\n0 1\n1 2\n",                      # ids from 0
        "3 3 2\n1\t2\n2 3\n",                     # a tab does not separate
        "3 3 2\n1 2\n2 3",                        # last line without a newline
        "3 3 2\r\n1 2\r\n2 3\r\n",                # CRLF
        "6 6 5\n6 1\n2 6\n6 2\n1 6\n4 5\n",       # lists in file order, gaps
    ]
    rng = np.random.default_rng(99)
    e = rng.integers(3, 700, size=(2000, 2))
    out.append("700 700 2000\n" + "".join(f"{a} {b}\n" for a, b in e))
    return out


def main():
    rec = {}
    texts = inputs()
    metas = []
    with tempfile.TemporaryDirectory() as td:
        for i, text in enumerate(texts):
            src = os.path.join(td, f"in{i}.mtx")
            with open(src, "w") as f:
                f.write(text)
            dst = os.path.join(td, f"out{i}")
            subprocess.run([GREADER, src, dst], check=True, capture_output=True)
            rec[f"off{i}"] = np.fromfile(os.path.join(dst, "graph.vertex.bin"), np.int64)
            rec[f"idx{i}"] = np.fromfile(os.path.join(dst, "graph.edge.bin"), np.int32)
            metas.append(open(os.path.join(dst, "graph.meta.txt")).read())
    np.savez_compressed(os.path.join(HERE, "gbin_golden.npz"), inputs=np.array(texts), meta=np.array(metas), **rec)
    print("wrote gbin_golden.npz:", len(texts), "inputs")


if __name__ == "__main__":
    main()
