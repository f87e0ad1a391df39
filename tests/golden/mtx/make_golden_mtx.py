"""Golden CSR arrays of the Matrix-Market fixtures in tests/golden/mtx/, made by the
REFERENCE's own import (mtx_read + mtx_values_convert_to_real + coo_to_csr with sorted
columns, src/bench.cpp:127-238), compiled from its sources into oracle/_ref/libref_mtx.so:

    make -C oracle ref REF=<reference checkout> && python tests/golden/mtx/make_golden_mtx.py

For every fixture <name>.mtx, <name>.npz holds, for expand_symmetry 1 and 0 (prefix e1_ /
e0_): row_ptr, col_ind, values and info = [m, n, nnz, nnz_diag, nnz_non_diag, symmetric,
expanded].
"""
from __future__ import annotations

import glob
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402


def main():
    for path in sorted(glob.glob(os.path.join(HERE, "*.mtx"))):
        out = {}
        for e in (1, 0):
            r = O.ref_read_mtx(path, expand_symmetry=bool(e))
            out[f"e{e}_row_ptr"] = r["row_ptr"]
            out[f"e{e}_col_ind"] = r["col_ind"]
            out[f"e{e}_values"] = r["values"]
            out[f"e{e}_info"] = np.array([r[k] for k in ("m", "n", "nnz", "nnz_diag", "nnz_non_diag", "symmetric",
                                                         "expanded")], np.int64)
        np.savez(os.path.splitext(path)[0] + ".npz", **out)
        print(os.path.basename(path), out["e1_info"].tolist(), out["e0_info"].tolist())


if __name__ == "__main__":
    main()
