"""Summarises the reference's shipped 2D SPGrid directory
(demos/SPGrid_Create_Simple_Domain/Create_2D_Domain/output, written by
Create_2D_Domain with -size 256 256) into tests/golden/spgrid2d_fixture.json:
its size, block count, and SHA-256 digests of the dense flags and data it
decodes to.  The reference tree is only read by this script; the tests compare
the restated generator against these digests everywhere, and against the
directory itself where it exists.

Usage: python tests/golden/make_spgrid2d_golden.py <reference_root>  (or HDD_REFERENCE_ROOT)
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from spgrid_format import read_spgrid_dir_any  # noqa: E402

REL = os.path.join("demos", "SPGrid_Create_Simple_Domain", "Create_2D_Domain", "output")


def main():
    if len(sys.argv) < 2 and not os.environ.get("HDD_REFERENCE_ROOT"):
        sys.exit("usage: make_spgrid2d_golden.py <reference checkout> (or set HDD_REFERENCE_ROOT)")
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ["HDD_REFERENCE_ROOT"]
    size, flags, data, count = read_spgrid_dir_any(os.path.join(root, REL))
    delta = [int(v) for v in np.argwhere(data != 0)[0]]
    out = {
        "source": REL,
        "size": list(size),
        "blocks": count,
        "flags_sha256": hashlib.sha256(np.ascontiguousarray(flags, "<u4").tobytes()).hexdigest(),
        "data_sha256": hashlib.sha256(np.ascontiguousarray(data, "<f4").tobytes()).hexdigest(),
        "cells": {"active": int(np.sum((flags & 0x10000) != 0)), "dirichlet": int(np.sum((flags & 0x20000) != 0)),
                  "exterior": int(np.sum(flags == 0))},
        "delta": delta,
        "delta_value": float(data[tuple(delta)]),
    }
    with open(os.path.join(HERE, "spgrid2d_fixture.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
