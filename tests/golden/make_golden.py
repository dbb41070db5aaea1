"""Generate the golden fixtures from the reference itself.

Runs the reference's serial HODLRMatrix / HSSMatrix (compiled unmodified from
chenxinye/hmat-omp include/*.h into oracle/_ref/ by ``make -C oracle``, with seed
injection) on seeded inputs and stores what the reference computed: tree layout and
ranks, multiply(x), and solve(b).  The reference has no test vectors of its own
(its drivers only print errors), so these files are its known answers.

    python tests/golden/make_golden.py           # rewrites tests/golden/*.npz
    python tests/golden/make_golden.py NAME ...  # only the named cases

Inputs are regenerated from the parameters stored in each file (``cases.py``), so
only outputs are stored.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import ref  # noqa: E402
from cases import CASES, make_matrix, make_vectors  # noqa: E402


def main(names=None):
    for name, c in CASES.items():
        if names and name not in names:
            continue
        A = make_matrix(c)
        N = A.shape[0]
        x, b = make_vectors(c, N)
        gauss = c.get("sketch", "uniform") == "normal"
        if c["kind"] == "hodlr":
            R = ref.RefHODLR(A, c["leaf"], c["tol"], c["rsvd_rank"], seed=c["seed"], gaussian=gauss)
            t = R.tree()
            y = R.multiply(x)
            xs = R.solve(b)
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), start=t.start, end=t.end,
                                is_leaf=t.is_leaf, depth=t.depth, rank12=t.rank12, rank21=t.rank21,
                                y=y, xs=xs)
            R.close()
        else:
            R = ref.RefHSS(A, c["leaf"], c["tol"], c["rsvd_rank"], seed=c["seed"], gaussian=gauss)
            t = R.tree()
            y = R.multiply(x)
            xs = R.solve(b)
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **t, y=y, xs=xs)
            R.close()
        print(f"{name}: N={N} nodes={len(t['start'] if isinstance(t, dict) else t.start)}")


if __name__ == "__main__":
    main(sys.argv[1:])
