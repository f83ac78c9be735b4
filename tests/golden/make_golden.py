"""Generates the golden fixtures in this directory from the oracle.

The reference cannot be built here and ships no golden vectors for this path,
so these fixtures pin the oracle (the CPU restatement of the reference's dd_pcg
path) on small seeded inputs: later changes to the oracle or the generator must
reproduce them.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from hierarchicaldd_b200 import domains  # noqa: E402
from hierarchicaldd_b200.domains import ACTIVE, INTERFACE  # noqa: E402
from oracle_ffi import Oracle  # noqa: E402

CASES = {"small16_sub8": dict(n=16, sub=8, radius=3, seed=1), "small32_sub16": dict(n=32, sub=16, radius=5, seed=2)}


def compute(name):
    c = CASES[name]
    d = domains.small(c["n"], c["sub"], c["radius"], seed=c["seed"])
    m = d.meta
    o = Oracle(d.size, d.sub_size, d.flags, vlevels=m["vlevels"], nVcycles=m["nVcycles"],
               interior_smoothing=m["interior_smoothing"], boundary_smoothing=m["boundary_smoothing"],
               sigma_levels=m["sigma_levels"], sigma_smoothing=m["sigma_smoothing"], sigma_mg=m["sigma_mg"])
    f0 = o.level_flags(0)
    solve_mask = (f0 & (ACTIVE | INTERFACE)) != 0
    rng = np.random.default_rng(100 + c["seed"])
    x = rng.standard_normal(d.size).astype(np.float32)
    x[~solve_mask] = 0
    b = rng.standard_normal(d.size).astype(np.float32)
    b[(f0 & ACTIVE) == 0] = 0
    u, _ = o.vcycle(x, np.zeros_like(x), b)
    arr = o.matrix("Arr", 0)
    _, it, info = o.solve(d.rhs, tol=1e-6)
    return dict(flags=d.flags, rhs=d.rhs, level0_flags=f0, x=x, b=b, laplacian=o.multiply(x), vcycle=u,
                arr_ptr=arr.indptr.astype(np.int32), arr_col=arr.indices.astype(np.int32),
                arr_val=arr.data.astype(np.float32), iterations=np.int32(it), history=info["history"])


if __name__ == "__main__":
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **compute(name))
        print("wrote", name)
