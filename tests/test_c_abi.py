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


def _build(tmp_path, name="legacy_abi"):
    exe = str(tmp_path / name)
    cmd = ["gcc", "-std=c99", "-O2", "-D_POSIX_C_SOURCE=200112L", os.path.join(HERE, "c", name + ".c"),
           "-I" + os.path.join(ROOT, "include"), "-L" + os.path.join(ROOT, "radchan_b200"), "-lradchan",
           "-Wl,-rpath," + os.path.join(ROOT, "radchan_b200"), "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_caller_compiles_and_links_against_the_library(tmp_path):
    assert os.path.exists(_build(tmp_path))
    assert os.path.exists(_build(tmp_path, "slab_abi"))
    assert os.path.exists(_build(tmp_path, "slab_group"))


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


@pytest.mark.gpu
def test_c_caller_slabs_over_ranks_equal_the_one_gpu_solve(tmp_path):
    """The reference's decomposition over several GPUs through the legacy
    entry points (tests/c/slab_abi.c): with p_col = 2 in param.h each rank's
    mc_gpu_ / get_results_ returns its z slab, equal bit for bit to the same
    planes of the one-GPU solve."""
    exe = _build(tmp_path, "slab_abi")
    gold = os.path.join(HERE, "golden")
    src = open(os.path.join(gold, "param_channel64.h")).read()
    assert "#define  p_col      1" in src
    ph = tmp_path / "param_pcol2.h"
    ph.write_text(src.replace("#define  p_col      1", "#define  p_col      2"))
    props = tmp_path / "properties"
    props.mkdir()
    r = subprocess.run([exe, str(ph), os.path.join(gold, "narrowband_channel64.h"), str(props)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "in 2 slabs: identical 1 nonzero 1" in r.stdout


@pytest.mark.gpu
def test_c_caller_slab_group_equals_the_plain_solve(tmp_path):
    """One solve over a group of GPUs from C (tests/c/slab_group.c): the
    group id, joining, rc_slab_solve on host arrays (the library's own
    NCCL, field broadcast, in-place gathers) on a one-rank group equal the
    plain solve of the same field bit for bit."""
    exe = _build(tmp_path, "slab_group")
    gold = os.path.join(HERE, "golden")
    props = tmp_path / "properties"
    props.mkdir()
    r = subprocess.run([exe, os.path.join(gold, "param_channel64.h"), os.path.join(gold, "narrowband_channel64.h"),
                        str(props)], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, NCCL_NVLS_ENABLE="0"))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "identical 1 nonzero 1" in r.stdout

