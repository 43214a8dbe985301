"""A compiled C99 program calls the library the way the Fortran DNS calls
the reference (tests/c/legacy_abi.c): mc_gpu_ / get_results_ with every
argument by reference, configured from the reference-format param.h,
NarrowBand.h and table files, and the same solve through the explicit
context API must give identical arrays."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _build(tmp_path):
    exe = str(tmp_path / "legacy_abi")
    cmd = ["gcc", "-std=c99", "-O2", "-D_POSIX_C_SOURCE=200112L", os.path.join(HERE, "c", "legacy_abi.c"),
           "-I" + os.path.join(ROOT, "include"), "-L" + os.path.join(ROOT, "radchan_b200"), "-lradchan",
           "-Wl,-rpath," + os.path.join(ROOT, "radchan_b200"), "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_caller_compiles_and_links_against_the_library(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_c_caller_legacy_entry_points_equal_context_api(tmp_path):
    exe = _build(tmp_path)
    props = tmp_path / "properties"
    props.mkdir()
    gold = os.path.join(HERE, "golden")
    r = subprocess.run([exe, os.path.join(gold, "param_channel64.h"), os.path.join(gold, "narrowband_channel64.h"),
                        str(props)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "identical 1 finite 1 nonzero 1" in r.stdout
