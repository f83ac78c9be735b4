"""hdd_test_bench on the GPU: the reference's Test_Bench_3D command line
(-mode no_convertion on a Write_SPGrid directory) gives the same PCG iterations
and the same solution, bit for bit, as the Python mirror of the solver class;
-iomode output and then -iomode input (the interface matrices dumped and read
back) give them again."""
import os
import re
import subprocess

import numpy as np
import pytest

from hierarchicaldd_b200 import build as hdd_build
from hierarchicaldd_b200 import domains
from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
from spgrid_format import write_spgrid_dir

pytestmark = pytest.mark.gpu


def test_command_line_matches_the_library(tmp_path, hdd_lib):
    if not os.path.exists(hdd_build.CLI):
        hdd_build.build()
    d = domains.small(32, 8, 6, seed=1)
    src = tmp_path / "domain"
    src.mkdir()
    write_spgrid_dir(str(src), d.flags, d.rhs)
    m = d.meta
    cmd = [hdd_build.CLI, "-mode", "no_convertion", "-d", str(src), "-size", *map(str, d.size),
           "-sub_size", *map(str, d.sub_size), "-vlevels", str(m["vlevels"]), "-sigma_levels",
           str(m["sigma_levels"]), "-sigma_smoothing", str(m["sigma_smoothing"]), "-sigma_mg", str(m["sigma_mg"]),
           "-interior_smoothing", str(m["interior_smoothing"]), "-boundary_smoothing",
           str(m["boundary_smoothing"]), "-nVcycles", str(m["nVcycles"]), "-o", str(tmp_path / "dump")]
    runs = {}
    for io in ("output", "input"):
        xf = tmp_path / f"x_{io}.bin"
        p = subprocess.run(cmd + ["-iomode", io, "-solution", str(xf)], capture_output=True, text=True,
                           timeout=600)
        assert p.returncode == 0, (io, p.stdout, p.stderr)
        it = int(re.search(r"cg iterations\s*:\s*(\d+)", p.stdout).group(1))
        runs[io] = (it, np.fromfile(xf, np.float32).reshape(d.size))
    a = SPGrid_Domain_Decomposition_Solver()
    try:
        a.Read_SPGrid(str(src))
        a.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"])
        r, x = a.Solve(), a.Solution()
    finally:
        a.close()
    for io, (it, xc) in runs.items():
        assert it == r["iterations"] and np.array_equal(xc, x), io


def test_command_line_two_level_matches_the_library(tmp_path, hdd_lib):
    """-multilevel yes (the two-level demo's flag): the same iterations and
    solution as the library's two-level solve; no interface dump by default."""
    if not os.path.exists(hdd_build.CLI):
        hdd_build.build()
    d = domains.small(32, 16, 6, seed=3)
    src = tmp_path / "domain"
    src.mkdir()
    write_spgrid_dir(str(src), d.flags, d.rhs)
    m = dict(d.meta, sigma_levels=2)
    xf = tmp_path / "x.bin"
    cmd = [hdd_build.CLI, "-mode", "no_convertion", "-d", str(src), "-size", *map(str, d.size),
           "-sub_size", *map(str, d.sub_size), "-vlevels", str(m["vlevels"]), "-sigma_levels",
           str(m["sigma_levels"]), "-interior_smoothing", str(m["interior_smoothing"]), "-boundary_smoothing",
           str(m["boundary_smoothing"]), "-o", str(tmp_path / "dump"), "-multilevel", "yes", "-solution", str(xf)]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, (p.stdout, p.stderr)
    assert not (tmp_path / "dump").exists()
    it = int(re.search(r"cg iterations\s*:\s*(\d+)", p.stdout).group(1))
    a = SPGrid_Domain_Decomposition_Solver()
    try:
        a.Read_SPGrid(str(src))
        a.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"], multilevel=True)
        r, x = a.Solve(), a.Solution()
    finally:
        a.close()
    assert it == r["iterations"] and np.array_equal(np.fromfile(xf, np.float32).reshape(d.size), x)
