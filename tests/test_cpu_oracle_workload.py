"""The oracle builds the benchmark's inputs on its own (oracle/workload.py:
parameters, synthetic tables, field) so that bench.py's CPU reference arm
never loads the product library.  Those inputs must equal the product's
(radchan_b200/workloads.py through libradchan.so) byte for byte, or the two
arms would not time the same workload."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from oracle import workload as OW
from radchan_b200 import workloads as W


def test_params_equal_byte_for_byte():
    for a, b in ((OW.params_nb64(), W.config_nb_64()),
                 (OW.params_nb64(photmax=64), W.config_nb_64(photmax=64)),
                 (OW.channel_params(32, 32, 32, grey=True), W.config_grey_32())):
        assert C.sizeof(a) == C.sizeof(b)
        assert bytes(a) == bytes(b)


@pytest.mark.parametrize("spec", [dict(), dict(nB=24, nQ=4, nT=32), dict(logk_lo=-1.0, logk_hi=2.0, seed=5)])
def test_synthetic_tables_equal_the_library_tables(spec):
    o = OW.tables_nb(**spec).arrays()
    t = W.tables_nb(**spec).arrays()
    for k in ("Tnb", "kP", "wvl", "wvr", "wvc", "kavg", "kq", "prob", "probg", "wq"):
        assert np.array_equal(o[k].reshape(-1), np.asarray(t[k]).reshape(-1)), k


def test_field_equals_the_library_field():
    p = OW.params_nb64()
    assert np.array_equal(OW.channel_field(p), W.channel_field(W.config_nb_64()))


def test_oracle_solve_on_its_own_inputs_equals_the_library_inputs():
    p, tabs, T = OW.nb64(photmax=4)
    a = O.solve(p, tabs, T, rpt=4, cell_begin=0, cell_end=256, walls=False)
    q = W.config_nb_64(photmax=4)
    b = O.solve(q, W.tables_nb(), W.channel_field(q), rpt=4, cell_begin=0, cell_end=256, walls=False)
    assert np.array_equal(a["q64"], b["q64"], equal_nan=True) and a["steps"] == b["steps"]


def test_reference_format_files_read_back_as_the_library_files(tmp_path):
    """The oracle's writer (used to feed the reference's own readT when its
    CUDA build is timed) and the library's rc_tables_write_dir produce files
    that read back to the same tables."""
    from oracle.workload import write_reference_dir
    from radchan_b200 import api
    write_reference_dir(OW.tables_nb(nB=24, nQ=4, nT=32), str(tmp_path / "o"))
    (tmp_path / "l").mkdir()
    W.tables_nb(nB=24, nQ=4, nT=32).write_dir(str(tmp_path / "l"))
    a = api.TableSet.read_dir(str(tmp_path / "o"), 32, 24, 4).arrays()
    b = api.TableSet.read_dir(str(tmp_path / "l"), 32, 24, 4).arrays()
    for k in ("Tnb", "kP", "wvl", "wvr", "wvc", "kavg", "kq", "prob", "probg"):
        assert np.array_equal(a[k], b[k]), k


def test_both_bench_arms_report_the_same_config():
    import bench
    for name in ("nb64", "grey32"):
        po = bench.workload_oracle(name)[0]
        pl = bench.workload(name)[0]
        assert bytes(po) == bytes(pl)
        for ws in (1, 4):
            assert bench.bench_config(bench.workload_desc(name, po), ws) == \
                bench.bench_config(bench.workload_desc(name, pl), ws)
