"""Store the reference's cylindrical Laplacian golden matrix as a fixture.

The reference ships lap.txt: the dense matrix that src/Solvers.py:306-310
writes for Laplacian_cylindrical_csr(10, 10, 1, 1), printed with '%.2f'.
This script keeps its non-zero entries (row, column, value) in
lap_cylindrical_10x10.npz so that the CPU tests can pin the oracle's
restatement of the builder without the reference tree.

    python tests/golden/make_golden_lap.py [--reference DIR]

The reference tree is --reference DIR, else $PIC_REFERENCE_DIR, else the
container's read-only checkout.
"""
from __future__ import annotations

import argparse
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PIC_REFERENCE_DIR", "/root/reference"))
    L = np.loadtxt(os.path.join(ap.parse_args().reference, "lap.txt"))
    rows, cols = np.nonzero(L)
    np.savez_compressed(os.path.join(HERE, "lap_cylindrical_10x10.npz"), shape=np.array(L.shape),
                        rows=rows.astype(np.int32), cols=cols.astype(np.int32), vals=L[rows, cols])
    print(f"{rows.size} non-zeros of a {L.shape} matrix")


if __name__ == "__main__":
    main()
