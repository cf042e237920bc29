"""CALPUV9C, the three-time-level external mode (calpuv9c.f90), through the
same C-ABI as CALPUV2C with params.tl3_istl = 3 (leapfrog over DT2 = 2*DT) or
2 (the trapezoidal correction), driven in HDMT's order
(scenario.three_level_schedule: a correction after every NTSTBC-th step).

Bars:
* (CPU) CALPUV9C(2) from a state whose level n-1 equals level n is CALPUV2C:
  the same system, so P and the face discharges bit for bit, HP within
  1e-13 relative (the continuity is written DELT*(Q - S/2) there and
  DELT/2*(2Q - S) in CALPUV2C);
* (CPU) a closed basin keeps its volume from level n-1 (ISTL = 3) or n
  (ISTL = 2) to level n+1; the leapfrog runs stay finite and bounded;
* FP64 GPU: the same CG iteration counts as the oracle on every call,
  elevation within 1e-9 m, every time level returned alike, for the plain,
  wet/dry (ISDRY = 99 and the legacy drying), radiation-boundary, channel and
  baroclinic cases;
* MIXED: elevation within 1e-6 m of the FP64 oracle from the same input;
* batched: each member bit-identical to its own single-basin run.
"""
import numpy as np
import pytest

import cases
import efdc_xm as X
import oracle as O
import scenario as S

LEVELS = ("p", "hp", "h1p", "h2p", "p1", "uhdye", "vhdxe", "uhdy1e", "vhdx1e", "uhdy2e",
          "vhdx2e", "hu", "hv", "h1u", "h1v")


def prm3(scn, call, tm, precision=X.PREC_FP64):
    n, istl, nctbc, rold, rnew = call
    return X.make_params(S.three_level_params(scn.params, istl, nctbc, rold, rnew), n=n,
                         tn=scn.tn(n) * tm, precision=precision)


def case(name):
    if name == "channels":
        scn, steps, tm = cases.channels(1, qcherr=0.5), 12, 10.0
        scn.params["qcherr"] = 0.5
    elif name == "channels_as_written":
        scn, steps, tm = cases.channels(0, qcherr=0.25), 12, 10.0
    elif name == "baroclinic":
        scn, steps, tm = cases.baroclinic(), 12, 10.0
    elif name == "baroclinic_wetdry":
        scn, steps, tm = cases.baroclinic(wetdry=True), 20, 60.0
    else:
        scn, steps, tm = cases.build(name)
    return S.add_three_levels(scn), steps, tm


def volume(scn, h):
    return float(np.sum(scn.grid["dxyp"][1:scn.la] * h[1:scn.la]))


@pytest.mark.parametrize("name", ["basin_fp64", "noise_forcing", "baroclinic"])
def test_oracle_istl2_at_level_n_is_calpuv2c(name):
    scn, _, tm = case(name)
    a = scn.copy_state()
    b = scn.copy_state()
    o = O.Oracle(scn.grid)
    if scn.layers:
        o.set_layers(scn.layers)
    r2 = o.step(X.make_params(scn.params, n=1, tn=scn.tn(1) * tm), a)
    o.close()
    o = O.Oracle(scn.grid)
    if scn.layers:
        o.set_layers(scn.layers)
    r9 = o.step(prm3(scn, (1, 2, 0, 0.0, 1.0), tm), b)
    o.close()
    assert r2.status == r9.status == X.OK
    assert r2.iters_total == r9.iters_total
    la = scn.la
    for k in ("p", "uhdye", "vhdxe"):
        assert np.array_equal(a[k][1:la], b[k][1:la]), k
    assert float(np.abs(a["hp"] - b["hp"])[1:la].max() / np.abs(a["hp"][1:la]).max()) < 1e-13


def test_oracle_three_level_volume_closed_basin():
    scn = S.make_scenario(50, 40, seed=41, obc_sides=(), amp=0.3, dt=10.0, explicit_noise=3e-4)
    S.add_three_levels(scn)
    o = O.Oracle(scn.grid)
    st = scn.copy_state()
    for call in S.three_level_schedule(16, 4):
        base = volume(scn, st["h2p"] if call[1] == 3 else st["h1p"])
        assert o.step(prm3(scn, call, 10.0), st).status == X.OK
        assert abs(volume(scn, st["hp"]) - base) / base < 1e-10, call
    o.close()


@pytest.mark.parametrize("name", ["basin_fp64", "tidal_flat_99", "legacy_dry_1", "noise_forcing",
                                  "channels", "baroclinic_wetdry"])
def test_oracle_three_level_runs_bounded(name):
    scn, steps, tm = case(name)
    o = O.Oracle(scn.grid)
    if scn.channels:
        o.set_channels(scn.channels)
    if scn.layers:
        o.set_layers(scn.layers)
    st = scn.copy_state()
    h0 = float(np.abs(st["hp"][1:scn.la]).max())
    for call in S.three_level_schedule(steps, 4):
        r = o.step(prm3(scn, call, tm), st)
        assert r.status in (X.OK, X.NEG_DEPTH), (call, r.as_dict())
    assert np.all(np.isfinite(st["p"]))
    assert float(np.abs(st["hp"][1:scn.la]).max()) < 2 * h0 + 5.0
    o.close()


def test_oracle_rejects_missing_levels():
    scn, _, tm = case("basin_fp64")
    st = scn.copy_state()
    del st["h2p"]
    o = O.Oracle(scn.grid)
    assert o.step(prm3(scn, (1, 3, 1, 0.0, 1.0), tm), st).status == X.BAD_ARGUMENT
    o.close()


def run_oracle(scn, steps, tm):
    o = O.Oracle(scn.grid)
    if scn.channels:
        o.set_channels(scn.channels)
    if scn.layers:
        o.set_layers(scn.layers)
    st = scn.copy_state()
    out = []
    for call in S.three_level_schedule(steps, 4):
        r = o.step(prm3(scn, call, tm), st)
        out.append((r.as_dict(), {k: v.copy() for k, v in st.items() if isinstance(v, np.ndarray)}))
    o.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["basin_fp64", "tidal_flat_99", "legacy_dry_1", "noise_forcing",
                                  "radiation_all_sides", "channels", "channels_as_written",
                                  "baroclinic", "baroclinic_wetdry"])
def test_gpu_three_level_fp64_matches_oracle(name):
    X.load()
    scn, steps, tm = case(name)
    ref = run_oracle(scn, steps, tm)
    sol = X.Solver(scn.grid)
    if scn.channels:
        sol.set_channels(scn.channels)
    if scn.layers:
        sol.set_layers(scn.layers)
    st = scn.copy_state()
    la = scn.la
    for i, call in enumerate(S.three_level_schedule(steps, 4)):
        a = sol.step(prm3(scn, call, tm), st)
        r, so = ref[i]
        assert a.status == r["status"], (call, a.as_dict(), r)
        assert a.iters_total == r["iters_total"], (call, a.iters_total, r["iters_total"])
        assert a.solves == r["solves"], call
        for k in LEVELS:
            scale = 1.0 / S.G if k in ("p", "p1") else 1.0
            err = float(np.abs(st[k][1:la] - so[k][1:la]).max()) * scale
            tol = 1e-9 if k in ("p", "p1", "hp", "h1p", "h2p", "hu", "hv", "h1u", "h1v") else \
                1e-9 * max(1.0, float(np.abs(so[k][1:la]).max()))
            assert err <= tol, (call, k, err)
    for k in ("sub", "svb", "lmaskdry", "iscdry", "natdry", "qdwaste", "fpgxe", "fpgye",
              "qchanu", "qchanv", "qchanun", "qchanvn"):
        if k in so:
            scale = max(1.0, float(np.abs(so[k]).max()))
            assert float(np.abs(st[k] - so[k]).max()) <= 1e-9 * scale, k
    sol.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["basin_fp64", "tidal_flat_99", "channels", "baroclinic"])
def test_gpu_three_level_mixed_within_1e6_m(name):
    X.load()
    scn, steps, tm = case(name)
    o = O.Oracle(scn.grid)
    sol = X.Solver(scn.grid)
    if scn.channels:
        o.set_channels(scn.channels)
        sol.set_channels(scn.channels)
    if scn.layers:
        o.set_layers(scn.layers)
        sol.set_layers(scn.layers)
    so = scn.copy_state()
    worst = 0.0
    for call in S.three_level_schedule(steps, 4):
        sg = {k: (v.copy() if isinstance(v, np.ndarray) else
                  {s: a.copy() for s, a in v.items()} if isinstance(v, dict) else v)
              for k, v in so.items()}
        a = sol.step(prm3(scn, call, tm, X.PREC_MIXED), sg)
        b = o.step(prm3(scn, call, tm), so)
        assert a.status == b.status, (call, a.as_dict())
        if a.solves == b.solves:  # same wet/dry sweeps: compare the surfaces
            worst = max(worst, float(np.abs(sg["p"][1:scn.la] - so["p"][1:scn.la]).max()) / S.G)
    assert worst <= 1e-6, worst
    sol.close()
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [X.PREC_FP64, X.PREC_MIXED])
def test_gpu_three_level_batch_equals_single(precision):
    X.load()
    ms = [case("basin_fp64")[0], case("tidal_flat_99")[0], case("noise_forcing")[0]]
    tm = 10.0
    bs = X.BatchSolver([m.grid for m in ms])
    singles = [X.Solver(m.grid) for m in ms]
    sb = [m.copy_state() for m in ms]
    ss = [m.copy_state() for m in ms]
    for call in S.three_level_schedule(10, 3):
        prm = [prm3(m, call, tm, precision) for m in ms]
        stb = bs.step(prm, sb)
        for k, m in enumerate(ms):
            st1 = singles[k].step(prm[k], ss[k])
            assert stb[k].status == st1.status, (k, call)
            assert stb[k].iters_total == st1.iters_total, (k, call)
            for f in ("p", "hp", "h1p", "h2p", "uhdy1e", "uhdy2e"):
                assert np.array_equal(sb[k][f][1:m.la], ss[k][f][1:m.la]), (k, call, f)
    bs.close()
    for s in singles:
        s.close()


@pytest.mark.gpu
def test_gpu_three_level_argument_errors():
    X.load()
    scn, _, tm = case("basin_fp64")
    sol = X.Solver(scn.grid)
    st = scn.copy_state()
    del st["uhdy2e"]
    with pytest.raises(RuntimeError, match="UHDY2E"):
        sol.step(prm3(scn, (1, 3, 1, 0.0, 1.0), tm), st)
    st = scn.copy_state()
    p = prm3(scn, (1, 3, 1, 0.0, 1.0), tm)
    p.tl3_istl = 4
    with pytest.raises(RuntimeError, match="tl3_istl"):
        sol.step(p, st)
    bs = X.BatchSolver([scn.grid, scn.grid])
    with pytest.raises(RuntimeError, match="same"):
        bs.step([prm3(scn, (1, 3, 1, 0.0, 1.0), tm), prm3(scn, (1, 2, 0, 0.5, 0.5), tm)],
                [scn.copy_state(), scn.copy_state()])
    bs.close()
    sol.close()


def test_schedule_follows_hdmt():
    """HDMT's order (hdmt.f90:299-305, 1009-1029): NCTBC starts at 1; after the
    leapfrog step on which NCTBC reaches NTSTBC comes the trapezoidal
    correction of the same step with NCTBC = 0 and ROLD = RNEW = 0.5."""
    sch = S.three_level_schedule(9, 4)
    assert [c[:3] for c in sch[:6]] == [(1, 3, 1), (2, 3, 2), (3, 3, 3), (4, 3, 4), (4, 2, 0),
                                        (5, 3, 1)]
    assert all(c[3:] == ((0.0, 1.0) if c[1] == 3 else (0.5, 0.5)) for c in sch)
    assert [c[0] for c in sch if c[1] == 2] == [4, 8]
    assert sch[-1][0] == 9
    p = X.make_params(S.three_level_params(dict(cases.build("basin_fp64")[0].params), 3, 1, 0.0,
                                           1.0), n=1, tn=0.0)
    assert p.tl3_istl == 3 and p.delt == 2.0 * cases.build("basin_fp64")[0].params["dt"]


def test_oracle_fpgxe_blend():
    """CALPUV9C's baroclinic gradients are blended with the last ones
    (calpuv9c.f90:164-190): with ROLD = RNEW = 0.5 the result is the mean of
    the FPGXE passed in and the gradient of the current state (ROLD = 0,
    RNEW = 1 on a copy)."""
    scn, _, tm = case("baroclinic")
    o = O.Oracle(scn.grid)
    o.set_layers(scn.layers)
    st = scn.copy_state()
    assert o.step(prm3(scn, (1, 3, 1, 0.0, 1.0), tm), st).status == X.OK
    old = st["fpgxe"].copy()
    fresh = {k: (v.copy() if isinstance(v, np.ndarray) else
                 {q: a.copy() for q, a in v.items()} if isinstance(v, dict) else v)
             for k, v in st.items()}
    assert o.step(prm3(scn, (1, 2, 0, 0.0, 1.0), tm), fresh).status == X.OK
    assert o.step(prm3(scn, (1, 2, 0, 0.5, 0.5), tm), st).status == X.OK
    la = scn.la
    want = 0.5 * old[1:la] + 0.5 * fresh["fpgxe"][1:la]
    assert np.abs(old[1:la]).max() > 0
    assert np.allclose(st["fpgxe"][1:la], want, rtol=1e-13, atol=1e-20)
    o.close()
