"""CPU checks of the seeded scenario builder (restated EFDC+ set-up)."""
import numpy as np

import scenario as S


def test_config1_size_and_maps():
    scn = S.config1()
    assert 5400 <= scn.ncell <= 5800  # "about 5,600 wet cells"
    g = scn.grid
    la, lc = scn.la, scn.lc
    L = np.arange(2, la + 1)
    lec, lwc, lnc, lsc = (g[k][L - 1] for k in ("lec", "lwc", "lnc", "lsc"))
    # neighbour maps are mutually consistent (cellmap.f90:80-134)
    e = lec != lc
    assert np.all(g["lwc"][lec[e] - 1] == L[e])
    n = lnc != lc
    assert np.all(g["lsc"][lnc[n] - 1] == L[n])
    # row-major L order: J outer, I inner
    key = g["jl"][L - 1].astype(np.int64) * 10**6 + g["il"][L - 1]
    assert np.all(np.diff(key) > 0)


def test_open_boundary_switches_follow_setbcs():
    scn = S.config1()
    g = scn.grid
    for L in g["obc"]["W"]["l"]:
        assert scn.state["sub"][L - 1] == 0.0 and scn.state["svb"][L - 1] == 0.0
        LE = g["lec"][L - 1]
        assert scn.state["sub"][LE - 1] == 1.0  # the connection to the interior stays open
        assert scn.state["svb"][LE - 1] == 0.0  # ISPBW<=1 (setbcs.f90:188-192)
    np.testing.assert_array_equal(g["subo"], scn.state["sub"])


def test_metrics():
    scn = S.config2(n=128)
    g = scn.grid
    i0 = np.arange(1, scn.la)
    assert np.allclose(g["dxyip"][i0] * g["dxyp"][i0], 1.0)
    assert np.all((g["dxyu"][i0] > 2400) & (g["dxyu"][i0] < 40001))
    assert np.all(g["hruo"][i0][g["subo"][i0] == 0] == 0)
    assert g["dxyp"][scn.lc - 1] > 0  # ghost DXYP(LC)=DX*DY (ainit.f90:44)


def test_config3_sizes():
    n = S.config3_sizes()
    assert n.size == 256 and n.min() >= 10_000 and n.max() <= 400_000
    assert 15e6 < n.sum() < 40e6


def test_three_levels_start_at_level_n():
    scn = S.add_three_levels(S.config1(seed=4))
    st = scn.state
    for dst, src in (("p1", "p"), ("h2p", "hp"), ("h1p", "hp"), ("uhdy1e", "uhdye"),
                     ("uhdy2e", "uhdye"), ("vhdx2e", "vhdxe"), ("h1u", "hu"), ("h1v", "hv"),
                     ("tbx1", "tbx"), ("tsy1", "tsy")):
        assert np.array_equal(st[dst], st[src]) and st[dst] is not st[src], dst
    assert "fpgxe" not in st  # no baroclinic terms: no gradient state


def test_bed_and_drag_inputs():
    scn = S.config1(seed=5)
    bed = S.make_bed(scn, seed=2, kc=4, smooth_frac=0.2)
    n = scn.lc + 1
    for k in ("zbr", "stbxo", "stbyo", "dxp", "dyp", "dzc1", "sgzu1", "sgzv1"):
        assert bed[k].shape == (n,) and bed[k].dtype == np.float64, k
    z = bed["zbr"]
    assert 0.1 < np.mean(z == 0.0) < 0.3 and z.max() <= 0.05
    assert np.allclose(bed["dzc1"], 0.25)
    st = scn.copy_state()
    d = S.drag_inputs(scn, st, st["hu"], st["hv"], seed=1)
    for k in ("ub", "vb", "vu", "uv", "h1u", "h1v"):
        assert d[k].shape == (n,) and np.all(np.isfinite(d[k])), k
    assert d["h1u"] is not st["hu"]
