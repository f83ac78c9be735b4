"""Generates tests/golden/c2_oracle.npz: the oracle's solve of the 256^3
workload (257^3 flags, Dirichlet sphere of radius 48 at the centre, a delta at
(64, 64, 64) plus U[-1e-3, 1e-3] noise, 32^3 subdomains, vlevels 4,
interior/boundary smoothing 4, sigma_levels 4, sigma_smoothing 3, sigma_mg 1)
for the GPU parity test at that size (tests/test_gpu_c2_parity.py).

* The FP32 oracle (the reference's precision: FP32 vectors, FP64 dot
  accumulation) to 1e-6 relative max-norm residual: its PCG iteration count
  and the max|r| history.
* The FP64 oracle to 1e-10 relative max-norm residual: the discrete solution
  the GPU's is compared with, stored (as float32) at every 4th cell along each axis (65^3
  values) plus its L2 norm over all cells.

The oracle is the CPU restatement of the reference's dd_pcg path.  This takes
about 15 minutes on 8 cores.  Run from the repository root:

    python tests/golden/make_c2_fixture.py
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
                  dtype=dtype)


def main():
    d = domains.CONFIGS["c2"]()
    t0 = time.time()
    o32 = oracle(d, np.float32)
    _, it32, info32 = o32.solve(d.rhs, tol=1e-6, max_it=200)
    del o32
    print(f"FP32 oracle: {it32} iterations, true residual {info32['true_res_inf'] / info32['b_inf']:.3e} "
          f"({time.time() - t0:.0f} s)", flush=True)
    t0 = time.time()
    o64 = oracle(d, np.float64)
    x64, it64, info64 = o64.solve(d.rhs, tol=1e-10, max_it=400)
    print(f"FP64 oracle: {it64} iterations, true residual {info64['true_res_inf'] / info64['b_inf']:.3e} "
          f"({time.time() - t0:.0f} s)", flush=True)
    np.savez_compressed(os.path.join(HERE, "c2_oracle.npz"), iterations_fp32=np.int32(it32),
                        history_fp32=info32["history"], iterations_fp64=np.int32(it64),
                        x64_sub=x64[::STRIDE, ::STRIDE, ::STRIDE].astype(np.float32),
                        x64_l2=np.float64(np.sqrt(np.sum(x64.astype(np.float64) ** 2))), stride=np.int32(STRIDE),
                        true_residual_fp64=np.float64(info64["true_res_inf"] / info64["b_inf"]))
    print("wrote c2_oracle.npz")


if __name__ == "__main__":
    main()
