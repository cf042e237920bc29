"""Steps whose loops run on the device (EFDC_XM_OPT_DEVICE_LOOPS, the default).

A step is one CUDA graph whose three data-dependent loops -- the CG
iterations (congrad.f90:91-169), the MIXED refinement passes with their inner
iterations, and the wet/dry re-solves (GOTO 1000, calpuv2c.f90:597-601,
726-749) -- are conditional nodes decided on the device.  The host-driven
form (option 0) runs the same kernels in the same order and polls between
groups of iterations.  Checked here:

* both forms give the same result bit for bit (FP64 in every scenario family,
  MIXED where a step has one sweep), for single basins, a batch, the
  three-time-level schedule and other iterations per loop body;
* a device-driven step waits for the device once;
* the failure statuses the reference STOPs on or reports (ITERM exceeded,
  the NCORDRY sweep cap, negative depths, non-finite values) come back as the
  oracle's, and the context keeps working after them.
"""
import numpy as np
import pytest

import cases
import efdc_xm as X
import oracle as O
import scenario as S

pytestmark = pytest.mark.gpu

FIELDS = ("p", "hp", "h1p", "hu", "hv", "uhdye", "vhdxe", "uhe", "vhe", "sub", "svb", "sbx",
          "sby", "lmaskdry", "iscdry", "natdry", "qdwaste", "vdwaste")
STATS = ("status", "iters_total", "iters_last", "solves", "lawet", "ladry", "n_negdep",
         "n_wasted", "outer_refinements")


@pytest.fixture(scope="module", autouse=True)
def _lib():
    X.load()


def scenario(name):
    if name == "channels":
        return cases.channels(1, qcherr=0.5), 12, 10.0
    if name == "baroclinic_wetdry":
        return cases.baroclinic(wetdry=True), 20, 60.0
    return cases.build(name)


def solver(scn):
    sol = X.Solver(scn.grid)
    if scn.channels is not None:
        sol.set_channels(scn.channels)
    if scn.layers is not None:
        sol.set_layers(scn.layers)
    return sol


def run(scn, steps, tm, device_loops, precision=X.PREC_FP64, iters=None, params=None):
    sol = solver(scn)
    sol.set_option(X.OPT_DEVICE_LOOPS, device_loops)
    if iters is not None:
        sol.set_option(X.OPT_GRAPH_ITERS, iters)
    st = scn.copy_state()
    stats = []
    for n in range(1, steps + 1):
        prm = params(n) if params else X.make_params(scn.params, n=n, tn=scn.tn(n) * tm,
                                                     precision=precision)
        stats.append(sol.step(prm, st, lists=True).as_dict())
    sol.close()
    return st, stats


def same(a, b, la):
    (sa, ta), (sb, tb) = a, b
    for n, (x, y) in enumerate(zip(ta, tb), 1):
        for k in STATS:
            assert x[k] == y[k], (n, k, x[k], y[k])
    for k in FIELDS:
        np.testing.assert_array_equal(sa[k][1:la], sb[k][1:la], err_msg=k)
    np.testing.assert_array_equal(sa["lwet"], sb["lwet"])


@pytest.mark.parametrize("name", ["basin_fp64", "tidal_flat_99", "legacy_dry_1",
                                  "radiation_all_sides", "noise_forcing", "radiation_closed_face",
                                  "channels", "baroclinic_wetdry"])
def test_device_and_host_loops_equal_fp64(name):
    scn, steps, tm = scenario(name)
    same(run(scn, steps, tm, 1), run(scn, steps, tm, 0), scn.la)


@pytest.mark.parametrize("name", ["basin_fp64", "noise_forcing", "radiation_all_sides"])
def test_device_and_host_loops_equal_mixed_one_sweep(name):
    scn, steps, tm = scenario(name)
    same(run(scn, steps, tm, 1, X.PREC_MIXED), run(scn, steps, tm, 0, X.PREC_MIXED), scn.la)


@pytest.mark.parametrize("iters", [1, 3, 8])
def test_iterations_per_loop_body_do_not_change_results(iters):
    scn, steps, tm = cases.build("tidal_flat_99")
    same(run(scn, steps, tm, 1, iters=iters), run(scn, steps, tm, 1), scn.la)


def test_three_level_schedule_equal():
    scn, steps, tm = cases.build("tidal_flat_99")
    scn = S.add_three_levels(scn)
    sched = S.three_level_schedule(steps, 4)

    def prm(k):
        n, istl, nctbc, rold, rnew = sched[k - 1]
        return X.make_params(S.three_level_params(scn.params, istl, nctbc, rold, rnew), n=n,
                             tn=scn.tn(n) * tm)

    a = run(scn, len(sched), tm, 1, params=prm)
    b = run(scn, len(sched), tm, 0, params=prm)
    same(a, b, scn.la)
    for k in ("p1", "h2p", "uhdy2e", "vhdx2e", "h1u", "h1v"):
        np.testing.assert_array_equal(a[0][k], b[0][k], err_msg=k)


def test_batch_equal():
    mem = [cases.build(n)[0] for n in ("tidal_flat_99", "basin_fp64", "noise_forcing")]
    out = []
    for mode in (1, 0):
        bs = X.BatchSolver([m.grid for m in mem])
        bs.set_option(X.OPT_DEVICE_LOOPS, mode)
        sts = [m.copy_state() for m in mem]
        stats = []
        for n in range(1, 16):
            r = bs.step([X.make_params(m.params, n=n, tn=m.tn(n) * 20.0) for m in mem], sts)
            stats.append([x.as_dict() for x in r])
        bs.close()
        out.append((sts, stats))
    for m, scn in enumerate(mem):
        for n in range(15):
            for k in STATS:
                assert out[0][1][n][m][k] == out[1][1][n][m][k], (m, n, k)
        for k in FIELDS:
            np.testing.assert_array_equal(out[0][0][m][k], out[1][0][m][k], err_msg=f"{m}:{k}")


def test_one_host_wait_per_device_driven_step():
    scn = S.config1()
    for mode, check in ((1, lambda w, n: w == n), (0, lambda w, n: w > n)):
        sol = X.Solver(scn.grid)
        sol.set_option(X.OPT_DEVICE_LOOPS, mode)
        sol.upload(scn.copy_state())
        sol.step_device(X.make_params(scn.params, n=1, tn=scn.tn(1)))  # builds the graphs
        w0 = X.host_waits()
        for n in range(2, 12):
            assert sol.step_device(X.make_params(scn.params, n=n, tn=scn.tn(n))).status == X.OK
        waits = X.host_waits() - w0
        sol.close()
        assert check(waits, 10), (mode, waits)


def test_cg_maxiter_and_nonfinite():
    scn = S.config1()
    sol = X.Solver(scn.grid)
    st = scn.copy_state()
    s = sol.step(X.make_params(dict(scn.params, iterm=1), n=1, tn=scn.tn(1)), st)
    assert s.status == X.CG_MAXITER and "maximum iterations" in sol.last_error()
    st = scn.copy_state()
    st["tbx"] = st["tbx"].copy()
    st["tbx"][100] = np.nan
    assert sol.step(X.make_params(scn.params, n=1, tn=scn.tn(1)), st).status == X.NONFINITE
    st = scn.copy_state()
    assert sol.step(X.make_params(scn.params, n=1, tn=scn.tn(1)), st).status == X.OK
    sol.close()


def test_wetdry_sweep_cap():
    """NCORDRY reaching its cap (calpuv2c.f90:597-601; 500 in the reference, 2
    here) gives WETDRY_MAXSWEEP after the same solves as the oracle; the next
    step with the normal cap succeeds."""
    scn, _, tm = cases.build("tidal_flat_99")
    capped = dict(scn.params, max_sweeps=2)
    sol = X.Solver(scn.grid)
    sg, so = scn.copy_state(), scn.copy_state()
    a = sol.step(X.make_params(capped, n=1, tn=scn.tn(1) * tm), sg)
    o = O.Oracle(scn.grid)
    b = o.step(X.make_params(capped, n=1, tn=scn.tn(1) * tm), so)
    assert a.status == b.status == X.WETDRY_MAXSWEEP, (a.as_dict(), b.as_dict())
    assert a.solves == b.solves == 2 and a.iters_total == b.iters_total
    assert "NCORDRY" in sol.last_error()
    st = scn.copy_state()
    assert sol.step(X.make_params(scn.params, n=1, tn=scn.tn(1) * tm), st).status == X.OK
    sol.close()
    o.close()


def test_negative_depth_status_like_oracle():
    """A shallow basin under a 1 m tide without wetting/drying: from step 53
    some HP <= 0 (negdep.f90:34-45, reported and not fatal).  Every step's
    status and count of negative depths equal the oracle's."""
    scn = S.make_scenario(40, 30, seed=51, depth=(0.3, 1.5), amp=1.0, obc_sides=("W",), dt=10.0,
                          isdry=0, land_frac=0.03)
    res = cases.run_both(scn, 62, tm=20.0, keep=lambda n: False)
    neg = 0
    for n, (a, b, _, _) in enumerate(res, 1):
        assert a["status"] == b["status"], (n, a, b)
        assert a["n_negdep"] == b["n_negdep"], (n, a["n_negdep"], b["n_negdep"])
        assert a["iters_total"] == b["iters_total"], n
        neg += a["status"] == X.NEG_DEPTH
    assert neg >= 5
