"""Generates tests/golden/two_level_oracle.npz: the oracle's two-level DD
solves (the reference's -multilevel yes, demos/Domain_Decomposition_CPU_Only_Two_Levels)
for the GPU parity tests at the two-level demo's defaults
(tests/test_gpu_two_level.py):

* tl128 (128^3 cells, centred Dirichlet sphere r=24, U[-1, 1] right-hand side,
  64^3 subdomains split into 32^3 boxes, vlevels 3, smoothing 1/3,
  sigma_levels 3): the FP32 oracle's PCG iteration count and max|r| history
  at 1e-6 relative max-norm residual, and the FP64 oracle's discrete solution
  at 1e-10, stored (as float32) at every 4th cell along each axis plus its L2
  norm over all cells;
* c2ml (the 256^3 workload's domain and right-hand side, same two-level
  settings): the FP32 oracle's iteration count and history.

The oracle is the CPU restatement of the reference's dd_pcg path.  This takes
about an hour on 8 cores (the c2ml part most of it; ``--c2ml-only`` redoes just
that part, keeping the tl128 entries).  Run from the repository root:

    python tests/golden/make_two_level_fixture.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from hierarchicaldd_b200 import domains  # noqa: E402
from oracle_ffi import Oracle  # noqa: E402

STRIDE = 4


def oracle(d, dtype):
    m = d.meta
    return Oracle(d.size, d.sub_size, d.flags, vlevels=m["vlevels"], nVcycles=m["nVcycles"],
                  interior_smoothing=m["interior_smoothing"], boundary_smoothing=m["boundary_smoothing"],
                  sigma_levels=m["sigma_levels"], sigma_smoothing=m["sigma_smoothing"], sigma_mg=m["sigma_mg"],
                  dtype=dtype, multilevel=m["multilevel"])


def fp32(d):
    t0 = time.time()
    o = oracle(d, np.float32)
    _, it, info = o.solve(d.rhs, tol=1e-6, max_it=400)
    print(f"{d.name}: FP32 oracle {it} iterations, true residual {info['true_res_inf'] / info['b_inf']:.3e} "
          f"({time.time() - t0:.0f} s)", flush=True)
    return it, info["history"]


def save(out):
    np.savez_compressed(os.path.join(HERE, "two_level_oracle.npz"), stride=np.int32(STRIDE), **out)


def main():
    path = os.path.join(HERE, "two_level_oracle.npz")
    out = {}
    if "--c2ml-only" in sys.argv and os.path.exists(path):  # keep the tl128 entries of an earlier run
        with np.load(path) as g:
            out = {k: g[k] for k in g.files if k.startswith("tl128")}
    else:
        out.update(tl128(domains.CONFIGS["tl128"]()))
        save(out)
    d = domains.CONFIGS["c2ml"]()
    out["c2ml_iterations_fp32"], out["c2ml_history_fp32"] = fp32(d)
    save(out)


def tl128(d):
    out = {}
    out["tl128_iterations_fp32"], out["tl128_history_fp32"] = fp32(d)
    t0 = time.time()
    o64 = oracle(d, np.float64)
    x64, it64, info64 = o64.solve(d.rhs, tol=1e-10, max_it=600)
    del o64
    print(f"{d.name}: FP64 oracle {it64} iterations, true residual {info64['true_res_inf'] / info64['b_inf']:.3e} "
          f"({time.time() - t0:.0f} s)", flush=True)
    out.update(tl128_iterations_fp64=np.int32(it64),
               tl128_x64_sub=x64[::STRIDE, ::STRIDE, ::STRIDE].astype(np.float32),
               tl128_x64_l2=np.float64(np.sqrt(np.sum(x64.astype(np.float64) ** 2))))
    return out


if __name__ == "__main__":
    main()
