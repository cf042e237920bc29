"""GPU parity tests: the CUDA library (through its C-ABI) against the oracle.

Bars:
* FP64 drop-in: the same CG iteration count as the oracle on every solve,
  surface elevation within 1e-9 m (FP64 roundoff of a different dot-product
  order), wet/dry mask and face switches bit-exact.
* MIXED: surface elevation within 1e-6 m of the FP64 oracle (the bar of the
  FP32-inner/FP64-refinement form), same masks.
* volume budget closed to 1e-10 relative.
"""
import numpy as np
import pytest

import cases
import efdc_xm as X
import oracle as O
import scenario as S

pytestmark = pytest.mark.gpu

STATE_F = ("p", "hp", "h1p", "hu", "hv", "uhdye", "vhdxe", "uhe", "vhe")
MASK_F = ("sub", "svb", "sbx", "sby", "lmaskdry", "iscdry", "lopenbcdry", "natdry")


@pytest.fixture(scope="module", autouse=True)
def _lib():
    X.load()  # fails loudly when libefdc_xm.so is missing: no CPU fallback


def run_both(scn, steps, tm=1.0, precision=X.PREC_FP64, same_input=False, lists=False):
    """Run the GPU library and the oracle side by side; yields per-step data."""
    sol = X.Solver(scn.grid)
    orc = O.Oracle(scn.grid)
    sg, so = scn.copy_state(), scn.copy_state()
    out = []
    for n in range(1, steps + 1):
        if same_input:
            sg = {k: (v.copy() if isinstance(v, np.ndarray) else
                      {s: a.copy() for s, a in v.items()} if isinstance(v, dict) else v)
                  for k, v in so.items()}
        prm = X.make_params(scn.params, n=n, tn=scn.tn(n) * tm, precision=precision)
        a = sol.step(prm, sg, lists=lists)
        b = orc.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * tm), so, lists=lists)
        snap = lambda d: {k: (v.copy() if isinstance(v, np.ndarray) else v)  # noqa: E731
                          for k, v in d.items()}
        out.append((a.as_dict(), b.as_dict(), snap(sg), snap(so)))
    sol.close()
    orc.close()
    return out


def eta_err(a, b, la):
    return float(np.abs(a["p"][1:la] - b["p"][1:la]).max() / S.G)


@pytest.mark.parametrize("name", cases.GOLDEN)
def test_fp64_matches_oracle(name):
    scn, steps, tm = cases.build(name)
    res = run_both(scn, steps, tm, lists=True)
    for n, (a, b, sg, so) in enumerate(res, 1):
        assert a["status"] == b["status"], (n, a, b)
        assert a["solves"] == b["solves"], (n, a, b)
        assert abs(a["iters_total"] - b["iters_total"]) <= 0, (n, a["iters_total"], b["iters_total"])
        assert a["n_wasted"] == b["n_wasted"] and a["n_negdep"] == b["n_negdep"]
    a, b, sg, so = res[-1]
    la = scn.la
    assert eta_err(sg, so, la) < 1e-9
    for k in STATE_F:
        scale = max(1.0, float(np.abs(so[k][1:la]).max()))
        assert np.abs(sg[k][1:la] - so[k][1:la]).max() <= 1e-9 * scale, k
    for k in MASK_F:
        np.testing.assert_array_equal(sg[k][1:la], so[k][1:la], err_msg=k)
    np.testing.assert_array_equal(sg["lwet"][: a["lawet"]], so["lwet"][: b["lawet"]])
    assert a["lawet"] == b["lawet"] and a["ladry"] == b["ladry"]


@pytest.mark.parametrize("name", cases.GOLDEN)
def test_fp64_matches_golden_fixture(name):
    """Against the committed fixture (what the oracle produced when committed)."""
    from pathlib import Path
    scn, steps, tm = cases.build(name)
    g = np.load(Path(__file__).resolve().parent / "golden" / f"{name}.npz")
    sol = X.Solver(scn.grid)
    st = scn.copy_state()
    its = []
    for n in range(1, steps + 1):
        s = sol.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * tm), st)
        its.append(s.iters_total)
    sol.close()
    np.testing.assert_array_equal(its, g["stat_iters_total"])
    assert float(np.abs(st["p"] - g["state_p"]).max()) / S.G < 1e-9
    np.testing.assert_array_equal(st["lmaskdry"], g["state_lmaskdry"])
    np.testing.assert_array_equal(st["sub"], g["state_sub"])


def test_fp64_config1_long_run():
    """200 steps of the 100x60 basin: identical iteration counts throughout."""
    scn = S.config1()
    res = run_both(scn, 200)
    assert all(a["iters_total"] == b["iters_total"] for a, b, _, _ in res)
    assert eta_err(res[-1][2], res[-1][3], scn.la) < 1e-9


def test_mixed_config1_within_1e6_m():
    """Solver error of the MIXED form: from the same inputs, every step's
    surface is within 1e-6 m of the FP64 oracle's."""
    scn = S.config1()
    res = run_both(scn, 300, precision=X.PREC_MIXED, same_input=True)
    worst = max(eta_err(sg, so, scn.la) for _, _, sg, so in res)
    assert worst <= 1e-6, worst
    assert all(a["status"] == X.OK for a, _, _, _ in res)


def test_mixed_free_run_drift_matches_fp64_tolerance():
    """Run freely for 300 steps, the MIXED trajectory departs from the FP64
    oracle's by no more than the oracle's own trajectory departs when RSQM is
    tightened 100x: the drift comes from RSQM, not from FP32."""
    scn = S.config1()
    res = run_both(scn, 300, precision=X.PREC_MIXED)
    drift_mixed = max(eta_err(sg, so, scn.la) for _, _, sg, so in res)
    tight = S.config1()
    tight.params["rsqm"] = scn.params["rsqm"] * 1e-2
    a, _ = O.run(scn, 300)
    b, _ = O.run(tight, 300)
    drift_fp64 = eta_err(a, b, scn.la)
    assert drift_mixed <= 2.0 * drift_fp64 + 1e-7, (drift_mixed, drift_fp64)


def test_mixed_wetdry_masks_bit_exact_stepwise():
    """Mixed precision on the wetting/drying flat, same inputs every step:
    masks and face switches equal the FP64 oracle's."""
    scn, steps, tm = cases.build("tidal_flat_99")
    res = run_both(scn, steps, tm, precision=X.PREC_MIXED, same_input=True)
    for n, (a, b, sg, so) in enumerate(res, 1):
        for k in ("lmaskdry", "sub", "svb", "iscdry"):
            np.testing.assert_array_equal(sg[k][1:scn.la], so[k][1:scn.la], err_msg=f"{n}:{k}")
        assert eta_err(sg, so, scn.la) <= 1e-6


def test_congrad_standalone():
    scn, _, tm = cases.build("noise_forcing")
    st = scn.copy_state()
    orc = O.Oracle(scn.grid)
    p_in = st["p"].copy()
    orc.step(X.make_params(scn.params, n=1, tn=scn.tn(1) * tm), st, diag=True)
    ccci = np.zeros_like(st["ccc"])
    ccci[1:scn.la] = 1.0 / st["ccc"][1:scn.la]
    po = p_in.copy()
    r1 = orc.congrad(st["ccc"], st["ccs"], st["ccn"], st["ccw"], st["cce"], ccci, st["fptmp"], po,
                     1e-10, 200)
    sol = X.Solver(scn.grid)
    for prec, tol in ((X.PREC_FP64, 1e-9), (X.PREC_MIXED, 1e-6)):
        pg = p_in.copy()
        r2 = sol.congrad(st["ccc"], st["ccs"], st["ccn"], st["ccw"], st["cce"], ccci, st["fptmp"],
                         pg, 1e-10, 200, precision=prec)
        assert r2[0] == 0, sol.last_error()
        if prec == X.PREC_FP64:
            assert r2[1] == r1[1]
        assert np.abs(pg - po)[1:scn.la].max() / S.G < tol
        assert pg[0] == p_in[0] and pg[scn.lc - 1] == p_in[scn.lc - 1]  # ghosts untouched
    sol.close()


def test_volume_budget_gpu():
    scn = S.make_scenario(60, 40, seed=24, obc_sides=(), manning=0.02, dt=10.0,
                          explicit_noise=1e-4)
    for prec in (X.PREC_FP64, X.PREC_MIXED):
        sol = X.Solver(scn.grid)
        st = scn.copy_state()
        dxyp = scn.grid["dxyp"][1:scn.la]
        v0 = float(np.sum(dxyp * st["hp"][1:scn.la]))
        src = 0.0
        for n in range(1, 21):
            sol.step(X.make_params(scn.params, n=n, tn=scn.tn(n), precision=prec), st)
            src += scn.params["dt"] * float(np.sum(st["qsume"][1:scn.la]))
        v1 = float(np.sum(dxyp * st["hp"][1:scn.la]))
        assert abs((v1 - v0) - src) / v0 < 1e-10
        sol.close()


def test_device_resident_equals_host_path():
    scn, steps, tm = cases.build("tidal_flat_99")
    sol = X.Solver(scn.grid)
    a = scn.copy_state()
    for n in range(1, steps + 1):
        sol.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * tm), a)
    sol.close()
    sol = X.Solver(scn.grid)
    b = scn.copy_state()
    sol.upload(b)
    for n in range(1, steps + 1):
        sol.step_device(X.make_params(scn.params, n=n, tn=scn.tn(n) * tm))
    sol.download(b)
    sol.close()
    for k in STATE_F + MASK_F:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_failure_statuses_keep_context_usable():
    """ITERM=1 -> CG_MAXITER (the reference STOPs); NaN forcing -> NONFINITE;
    an unknown precision -> BAD_ARGUMENT.  The context keeps working."""
    scn = S.config1()
    sol = X.Solver(scn.grid)
    st = scn.copy_state()
    prm = X.make_params(dict(scn.params, iterm=1), n=1, tn=scn.tn(1))
    s = sol.step(prm, st)
    assert s.status == X.CG_MAXITER and "maximum iterations" in sol.last_error()
    st = scn.copy_state()
    st["tbx"] = st["tbx"].copy()
    st["tbx"][100] = np.nan
    s = sol.step(X.make_params(scn.params, n=1, tn=scn.tn(1)), st)
    assert s.status == X.NONFINITE
    prm = X.make_params(scn.params, n=1, tn=scn.tn(1))
    prm.precision = 7
    with pytest.raises(RuntimeError, match="BAD_ARGUMENT"):
        sol.step(prm, scn.copy_state())
    st = scn.copy_state()
    s = sol.step(X.make_params(scn.params, n=1, tn=scn.tn(1)), st)
    assert s.status == X.OK
    sol.close()


def test_periodic_maps_rejected():
    scn = S.make_scenario(20, 12, seed=3)
    g = dict(scn.grid)
    g["lwc"] = g["lwc"].copy()
    L = 2 + 5
    g["lwc"][L - 1] = scn.la  # an east-west periodic link
    with pytest.raises(RuntimeError, match="structured grid"):
        X.Solver(g)


def test_large_basin_mixed_vs_fp64():
    """1024x1024 curvilinear basin: mixed within 1e-6 m of the FP64 GPU solve
    after 10 steps, and both meet RSQ <= RSQM."""
    scn = S.config2(n=1024)
    out = {}
    for prec in (X.PREC_FP64, X.PREC_MIXED):
        sol = X.Solver(scn.grid)
        st = scn.copy_state()
        sol.upload(st)
        for n in range(1, 11):
            s = sol.step_device(X.make_params(scn.params, n=n, tn=scn.tn(n), precision=prec))
            assert s.status == X.OK
            assert s.rsq_last <= scn.params["rsqm"]
        sol.download(st)
        out[prec] = st
        sol.close()
    assert eta_err(out[X.PREC_MIXED], out[X.PREC_FP64], scn.la) <= 1e-6


def test_wetdry_fields_left_on_host_by_dry_free_step():
    """efdc_xm_step without wetting and drying neither uploads nor returns the
    fields only wetting and drying reads; a device-resident ISDRY > 0 step is
    then refused until they are uploaded, and gives the oracle's result after."""
    scn, steps, tm = cases.build("tidal_flat_99")
    st = scn.copy_state()
    sol = X.Solver(scn.grid)
    dry_free = X.make_params(dict(scn.params, isdry=0), n=1, tn=scn.tn(1) * tm)
    before = {k: st[k].copy() for k in ("sbx", "sby", "lmaskdry", "iscdry", "natdry")}
    assert sol.step(dry_free, st).status in (X.OK, X.NEG_DEPTH)
    for k, v in before.items():  # untouched on the host
        assert np.array_equal(st[k], v), k
    prm = X.make_params(scn.params, n=2, tn=scn.tn(2) * tm)
    with pytest.raises(RuntimeError, match="upload them first"):
        sol.step_device(prm)
    sol.upload(st)
    a = sol.step_device(prm)
    so = {k: (v.copy() if isinstance(v, np.ndarray) else
              {s: x.copy() for s, x in v.items()} if isinstance(v, dict) else v)
          for k, v in st.items()}
    b = O.Oracle(scn.grid).step(X.make_params(scn.params, n=2, tn=scn.tn(2) * tm), so)
    assert a.iters_total == b.iters_total
    out = {k: np.zeros_like(st[k]) for k in ("p", "lmaskdry")}
    sol.download(out)
    assert float(np.abs(out["p"][1:scn.la] - so["p"][1:scn.la]).max()) / S.G < 1e-9
    assert np.array_equal(out["lmaskdry"][1:scn.la], so["lmaskdry"][1:scn.la])
    sol.close()
