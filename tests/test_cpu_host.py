"""Host-side logic: parameter headers, multigrid geometry, spectral tables
(reference file formats), and the work decomposition -- no GPU needed."""
import os

import numpy as np
import pytest

from oracle.ref_build import REF
from radchan_b200 import api
from radchan_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
# the reference checkout's parameter headers, where the reference build
# recipe finds the checkout (skipped when it is absent)
REF_PARAM = os.path.join(REF, "src", "param")


def test_parse_channel_headers():
    p = api.params_from_headers(os.path.join(GOLD, "param_channel64.h"), os.path.join(GOLD, "narrowband_channel64.h"))
    assert (p.imax, p.jmax, p.kmax) == (64, 64, 64)
    assert abs(p.Ly - 6.283185307179586) < 1e-6 and abs(p.Lz - np.pi) < 1e-6
    assert p.grid_num == 3
    assert list(p.maxi)[:3] == [64, 32, 16] and list(p.maxk)[:3] == [64, 32, 16]
    assert list(p.maxs)[:3] == [5, 5, 100000]
    assert (p.nVar, p.photmax, p.srt, p.grey, p.calcwalls) == (4, 256, 1, 0, 1)
    assert (p.adiabw, p.adiabe) == (1, 0)
    assert list(p.Tw)[:2] == [955.0, 573.0]
    assert list(p.bd) == [2, 2, 1, 1, 1, 1]
    assert (p.nT, p.nQ, p.nB) == (64, 8, 100)
    assert api.validate(p) == ""


@pytest.mark.skipif(not os.path.isdir(REF_PARAM), reason="reference headers not mounted")
def test_parse_reference_headers_as_shipped():
    p = api.params_from_headers(os.path.join(REF_PARAM, "param.h"), os.path.join(REF_PARAM, "NarrowBand.h"))
    d = api.default_params()
    for f in ("imax", "jmax", "kmax", "nVar", "photmax", "grid_num", "srt", "grey", "calcwalls", "nT", "nQ", "nB"):
        assert getattr(p, f) == getattr(d, f), f
    assert list(p.maxi)[:9] == list(d.maxi)[:9] and list(p.maxs)[:9] == list(d.maxs)[:9]
    assert list(p.bd) == list(d.bd)
    assert p.p_col == 48  # multi-node slab count of the production run


@pytest.mark.parametrize("dims,levels", [((32, 32, 32), [(32, 32, 32)]),
                                         ((64, 48, 40), [(64, 48, 40), (32, 24, 20), (16, 12, 10)]),
                                         ((406, 8, 8), [(406, 8, 8), (14, 4, 4)]),
                                         ((17, 9, 5), [(17, 9, 5)])])
def test_grid_levels_equal_oracle_bit_for_bit(dims, levels):
    from oracle import oracle as O
    p = W.channel_params(*dims, levels=levels, maxs=[5] * (len(levels) - 1) + [100000], fact_mesh=1.6)
    for l in range(len(levels)):
        a = api.grid_level(p, l)
        b = O.grid_level(p, l)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])
        xu = a["xu"]
        assert xu[0] == 0 and abs(xu[-1] - p.Lx) < 1e-6
        if p.maxi[0] % 2 == 0:
            assert np.all(np.diff(xu) > 0)
        else:
            # the reference's law (definitions.h:108-123) leaves a zero-width
            # centre cell when imax is odd
            assert np.all(np.diff(xu) >= 0) and (np.diff(xu) == 0).sum() == 1
        # parabolic spacing: finest at the walls, symmetric about the centre
        np.testing.assert_allclose(xu, p.Lx - xu[::-1], atol=1e-5)


def test_synthetic_tables_are_consistent():
    t = W.tables_nb(nB=50, nQ=8, nT=32).arrays()
    assert np.all(np.diff(t["wvc"]) > 0) and t["wvl"][0] == 500.0 and t["wvr"][-1] == 10000.0
    np.testing.assert_allclose(t["wq"].sum(), 1.0, rtol=1e-6)
    assert np.all(np.diff(t["prob"], axis=1) >= 0) and np.all(t["prob"][:, -1] == 1.0)
    assert np.all(np.diff(t["probg"], axis=2) >= 0) and np.all(t["probg"][:, :, -1] == 1.0)
    # k increases with g (xi ascending, exp(1.5 xi))
    assert np.all(np.diff(t["kq"], axis=2) > 0)
    assert np.all(t["kP"] > 0)


def _i_black(T, nu):
    """Spectral blackbody intensity, nu in cm^-1 (nbcorrk/ckdist_hitran_part.cpp:229-233)."""
    c1, c2 = 3.741771790075259e-16, 0.014387741858429
    return c1 * (nu * 100.0) ** 3 / (np.pi * np.expm1(c2 * nu * 100.0 / T))


@pytest.mark.parametrize("nB,nQ,nT", [(50, 8, 32), (7, 4, 3), (1, 1, 2)])
def test_synthetic_tables_follow_reference_cdf_law(nB, nQ, nT):
    """The band and g cumulative probabilities and the Planck-mean
    coefficient restated from nbcorrk/calc_prob.cpp:54-116 on the table's own
    k, weights and band edges: band CDF ~ sum_g w_g k_bg I_b(T, nu_b) dnu_b,
    g CDF within a band ~ w_g k_bg, kP = pi sum k I_b dnu / (sigma T^4)."""
    t = W.tables_nb(nB=nB, nQ=nQ, nT=nT).arrays()
    kq = t["kq"].astype(np.float64).reshape(nB, nT, nQ)
    wq = t["wq"].astype(np.float64)
    nu = t["wvc"].astype(np.float64)
    dnu = (t["wvr"].astype(np.float64) - t["wvl"].astype(np.float64)) * 100.0
    sigma = 5.670373e-08
    for i, T in enumerate(t["Tnb"].astype(np.float64)):
        k = kq[:, i, :]                                           # [nB, nQ]
        pb = (k * wq).sum(axis=1) * _i_black(T, nu) * dnu         # calc_prob.cpp:73-76
        np.testing.assert_allclose(t["prob"][i], np.cumsum(pb) / pb.sum(), rtol=2e-5, atol=1e-9)
        cg = np.cumsum(k * wq, axis=1)                            # calc_prob.cpp:97-116
        np.testing.assert_allclose(t["probg"][i], cg / cg[:, -1:], rtol=2e-6, atol=1e-9)
        kP = np.pi * pb.sum() / (sigma * T ** 4)                  # calc_prob.cpp:54-56
        np.testing.assert_allclose(t["kP"][i], kP, rtol=2e-5)


def test_reference_table_files_round_trip(tmp_path):
    ts = W.tables_nb(nB=12, nQ=8, nT=16)
    ts.write_dir(tmp_path)
    names = sorted(os.listdir(tmp_path))
    assert "planck-mean.txt" in names and "prob_new2.txt" in names and "NarrBand11.txt" in names
    back = api.TableSet.read_dir(tmp_path, 16, 12, 8)
    a, b = ts.arrays(), back.arrays()
    for k in ("Tnb", "wvl", "wvr", "wvc"):
        np.testing.assert_allclose(b[k], a[k], rtol=2e-6)
    np.testing.assert_allclose(b["kq"], a["kq"], rtol=1e-5)       # %le: 6 significant digits
    np.testing.assert_allclose(b["prob"], a["prob"], rtol=1e-7)   # %30.20le
    np.testing.assert_allclose(b["probg"], a["probg"], rtol=1e-7)
    # prob_new2.txt: "T j cuprob cuprob_new2[nQ]" per line (nbcorrk/write_tables.cpp:40-53)
    lines = open(os.path.join(tmp_path, "prob_new2.txt")).read().split("\n")
    assert len(lines[0].split()) == 3 + 8


def _edit_token(path, line, col, value):
    lines = open(path).read().split("\n")
    tok = lines[line].split()
    tok[col] = value
    lines[line] = " ".join(tok)
    open(path, "w").write("\n".join(lines))


@pytest.mark.parametrize("fname,line,col,value,msg", [
    ("prob_new2.txt", 3, 2, "1.0e-3", "band cumulative"),      # band CDF decreases
    ("prob_new2.txt", 2, 4, "nan", "g cumulative"),             # NaN in a g CDF
    ("prob_new2.txt", 1, 6, "1.5", "g cumulative"),             # g CDF above 1
    ("NarrBand3.txt", 2, 4, "-2.0e-03", "absorption"),          # negative k
    ("NarrBand1.txt", 4, 3, "inf", "absorption"),               # infinite k
    ("planck-mean.txt", 2, 0, "1200.0", "uniformly"),           # uneven temperature step
    ("planck-mean.txt", 3, 1, "nan", "Planck-mean"),            # NaN kP
])
def test_malformed_table_files_are_rejected(tmp_path, fname, line, col, value, msg):
    """Table files that read but break what the device searches assume
    (monotone CDFs in [0, 1], finite k >= 0, uniform temperature steps)
    are rejected before any upload, with the first violation named."""
    ts = W.tables_nb(nB=6, nQ=4, nT=5)
    assert ts.validate() == ""
    ts.write_dir(tmp_path)
    assert api.TableSet.read_dir(tmp_path, 5, 6, 4).validate() == ""
    _edit_token(os.path.join(tmp_path, fname), line, col, value)
    bad = api.TableSet.read_dir(tmp_path, 5, 6, 4)
    assert msg in bad.validate()


def test_truncated_table_file_is_reported(tmp_path):
    ts = W.tables_nb(nB=6, nQ=4, nT=5)
    ts.write_dir(tmp_path)
    path = os.path.join(tmp_path, "prob_new2.txt")
    text = open(path).read()
    open(path, "w").write(text[: len(text) // 2])
    with pytest.raises(Exception) as e:
        api.TableSet.read_dir(tmp_path, 5, 6, 4)
    assert "prob_new2" in str(e.value)


def test_missing_table_file_is_reported(tmp_path):
    with pytest.raises(Exception) as e:
        api.TableSet.read_dir(tmp_path, 16, 12, 8)
    assert "planck-mean" in str(e.value)


def test_field_recipe_walls_and_periodicity():
    p = W.config_nb_64(photmax=4)
    T = W.channel_field(p)
    # face averages equal the wall temperatures; y/z ghosts are periodic images
    np.testing.assert_allclose((T[:, :, 0] + T[:, :, 1]) / 2, 955.0, rtol=1e-6)
    np.testing.assert_allclose((T[:, :, -1] + T[:, :, -2]) / 2, 573.0, rtol=1e-6)
    np.testing.assert_array_equal(T[:, 0, :], T[:, -2, :])
    np.testing.assert_array_equal(T[0], T[-2])
    assert 500 < T[1:-1, 1:-1, 1:-1].min() and T[1:-1, 1:-1, 1:-1].max() < 1050
