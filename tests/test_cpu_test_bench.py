"""The hdd_test_bench command line (the reference's Test_Bench_3D flags,
demos/Domain_Decomposition_CPU_Only/Test_Bench_3D/main.cpp:236-301) without a GPU:
help and usage errors, the unsupported fluids-format modes, and no CPU fallback."""
import os
import subprocess

import pytest

from conftest import gpu_available
from hierarchicaldd_b200 import build as hdd_build

CLI = hdd_build.CLI


@pytest.fixture(scope="module")
def cli(hdd_lib):
    if not os.path.exists(CLI):
        hdd_build.build()
    return CLI


def run(cli, *args):
    return subprocess.run([cli, *args], capture_output=True, text=True, timeout=120)


def test_help_lists_the_reference_flags(cli):
    p = run(cli, "-help")
    assert p.returncode == 0
    for flag in ("-size", "-sub_size", "-vlevels", "-sigma_levels", "-sigma_smoothing", "-sigma_mg",
                 "-interior_smoothing", "-boundary_smoothing", "-nVcycles", "-threads", "-d", "-o", "-mode",
                 "-iomode", "-multilevel"):
        assert flag in p.stdout, flag


@pytest.mark.parametrize("args", [("-bogus",), ("-size", "33", "33"), ("-vlevels", "x"), ("-iomode", "both"),
                                  ("-precision", "half"), ("-mode", "no_convertion"), ("-multilevel", "maybe")])
def test_usage_errors_exit_2(cli, args):
    p = run(cli, *args)
    assert p.returncode == 2 and "usage" in p.stderr, (args, p.stderr)


@pytest.mark.parametrize("mode", ["velocity", "rhs"])
def test_fluids_modes_are_unsupported(cli, mode, tmp_path):
    p = run(cli, "-mode", mode, "-d", str(tmp_path))
    assert p.returncode == 3 and "unsupported input" in p.stderr and "no_convertion" in p.stderr


@pytest.mark.skipif(gpu_available(), reason="checks the GPU-less failure path")
def test_no_cpu_fallback(cli, tmp_path):
    p = run(cli, "-mode", "no_convertion", "-d", str(tmp_path), "-size", "33", "33", "33", "-sub_size", "8", "8",
            "8", "-iomode", "neither")
    assert p.returncode == 3 and "CUDA error" in p.stderr and "cg iterations" not in p.stdout
