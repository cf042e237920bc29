"""The implicit bottom and vegetation drag (ISITB >= 1, ISVEG > 0;
calpuv2c.f90:222-243, calpuv9c.f90:220-240) and the separate RCX (u faces)
and RCY (v faces) it produces.

CPU: the oracle's RCX, RCY and their effect are checked against an
independent numpy statement of the reference's formulas: the coefficients
on a cell's faces, FUHDYE*RCX entering the assembly, and CS built with RCY
(a mix-up of RCX and RCY would show, since the two differ here).
GPU: FP64 steps with ISITB = 1, ISITB = 2 with vegetation, and ISVEG alone
match the oracle (same CG iterations, surface within 1e-9 m), on their own,
in a batch with members without drag, and in the three-time-level schedule;
MIXED is within 1e-6 m.
"""
import numpy as np
import pytest

import cases
import efdc_xm as X
import oracle as O
import scenario as S


def bottom_velocity(scn, st):
    """U(L,KSZU(L)), V(L,KSZV(L)) from the current transports, as the internal
    mode provides them: 0.8 of the depth-averaged velocity UHE/HU (a host
    update before each step; then TMPX = 0.8 wherever UHE /= 0)."""
    la = scn.la
    for b, q, h in (("ubot", "uhe", "hu"), ("vbot", "vhe", "hv")):
        a = np.zeros_like(st[q])
        a[1:la] = 0.8 * st[q][1:la] / st[h][1:la]
        st[b] = a


def run_both_drag(scn, steps, precision=X.PREC_FP64, same_input=False):
    """cases.run_both with the bottom velocities updated before each step."""
    sol, orc = X.Solver(scn.grid), O.Oracle(scn.grid)
    sg, so = scn.copy_state(), scn.copy_state()
    out = []
    for n in range(1, steps + 1):
        if same_input:
            sg = cases.copy_state(so)
        bottom_velocity(scn, sg)
        bottom_velocity(scn, so)
        a = sol.step(X.make_params(scn.params, n=n, tn=scn.tn(n), precision=precision), sg)
        b = orc.step(X.make_params(scn.params, n=n, tn=scn.tn(n)), so)
        out.append((a.as_dict(), b.as_dict(), cases.copy_state(sg), cases.copy_state(so)))
    sol.close()
    orc.close()
    return out


def drag_case(isitb=1, isveg=0, veg=0.0, seed=0):
    scn = S.make_scenario(50, 36, seed=61 + seed, obc_sides=("W",), amp=0.4, dt=10.0,
                          explicit_noise=1e-4)
    return S.add_implicit_drag(scn, isitb, isveg=isveg, veg=veg, seed=seed)


def expected_rc(scn, st):
    """RCX, RCY of the first step restated in numpy (UHE = VHE = 0 at the
    start: TMPX = TMPY = 1)."""
    p, la = scn.params, scn.la
    i = np.arange(1, la)
    dt = p["dt"]
    if p["isitb"] >= 1:
        hui, hvi = 1.0 / st["hu"][i], 1.0 / st["hv"][i]
        rx = 1.0 / (1.0 + p["ritb"] * dt * hui * st["stbx"][i] *
                    np.sqrt(st["vu"][i] ** 2 + st["ubot"][i] ** 2) + dt * st["fxvege"][i])
        ry = 1.0 / (1.0 + p["ritb"] * dt * hvi * st["stby"][i] *
                    np.sqrt(st["uv"][i] ** 2 + st["vbot"][i] ** 2) + dt * st["fyvege"][i])
    else:
        rx = 1.0 / (1.0 + dt * st["fxvege"][i])
        ry = 1.0 / (1.0 + dt * st["fyvege"][i])
    return rx, ry


@pytest.mark.parametrize("isitb,isveg,veg", [(1, 0, 0.0), (2, 1, 2e-3), (0, 1, 2e-3)])
def test_oracle_drag_coefficients_and_assembly(isitb, isveg, veg):
    scn = drag_case(isitb, isveg, veg)
    st = scn.copy_state()
    st0 = scn.copy_state()
    o = O.Oracle(scn.grid)
    o.step(X.make_params(scn.params, n=1, tn=scn.tn(1)), st, diag=True)
    o.close()
    rx, ry = expected_rc(scn, st0)
    assert np.all(rx < 1.0) and np.all(ry < 1.0)
    assert np.abs(rx - ry).max() > 1e-3  # RCX and RCY differ, so a mix-up would show
    # CS of the scaled system is C1*SVB*HRVO*RCY*HV / CCMNM (calpuv2c.f90:306-344)
    g, la = scn.grid, scn.la
    i = np.arange(1, la)
    c1 = -0.5 * 0.5 * scn.params["dt"] * scn.params["g"]
    cs = c1 * st0["svb"][i] * g["hrvo"][i] * ry * st0["hv"][i]
    cw = c1 * st0["sub"][i] * g["hruo"][i] * rx * st0["hu"][i]
    inner = (g["subo"][i] > 0) & (g["svbo"][i] > 0)
    ratio_s = st["ccs"][i][inner] / cs[inner]
    ratio_w = st["ccw"][i][inner] / cw[inner]
    nz = (np.abs(cs[inner]) > 0) & (np.abs(cw[inner]) > 0)
    # one common scale (1/CCMNM) for both couplings of every cell
    assert ratio_s[nz].std() / ratio_s[nz].mean() < 1e-12
    assert abs(ratio_w[nz].mean() - ratio_s[nz].mean()) / ratio_s[nz].mean() < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("isitb,isveg,veg", [(1, 0, 0.0), (2, 1, 2e-3), (0, 1, 2e-3)])
def test_gpu_drag_matches_oracle(isitb, isveg, veg):
    X.load()
    scn = drag_case(isitb, isveg, veg)
    res = run_both_drag(scn, 30)
    for n, (a, b, sg, so) in enumerate(res, 1):
        assert a["status"] == b["status"] == X.OK, (n, a, b)
        assert a["iters_total"] == b["iters_total"], (n, a["iters_total"], b["iters_total"])
        assert cases.state_err(sg, so, scn.la) < 1e-9, n
    a, b, sg, so = res[-1]
    for k in ("uhdye", "vhdxe", "uhe", "vhe", "hu", "hv"):
        scale = max(1.0, float(np.abs(so[k][1:scn.la]).max()))
        assert np.abs(sg[k][1:scn.la] - so[k][1:scn.la]).max() <= 1e-9 * scale, k
    resm = run_both_drag(scn, 15, precision=X.PREC_MIXED, same_input=True)
    assert max(cases.state_err(sg, so, scn.la) for _, _, sg, so in resm) <= 1e-6


@pytest.mark.gpu
def test_gpu_drag_in_batch_with_plain_members():
    X.load()
    mem = [drag_case(1), cases.build("basin_fp64")[0], drag_case(0, 1, 2e-3, seed=3)]
    # the plain member gives the drag arrays too (all or none), with ISITB = ISVEG = 0
    S.add_implicit_drag(mem[1], 0, isveg=0)
    single = []
    for m in mem:
        sol = X.Solver(m.grid)
        st = m.copy_state()
        for n in range(1, 11):
            bottom_velocity(m, st)
            sol.step(X.make_params(m.params, n=n, tn=m.tn(n)), st)
        sol.close()
        single.append(st)
    bs = X.BatchSolver([m.grid for m in mem])
    sts = [m.copy_state() for m in mem]
    for n in range(1, 11):
        for m, st in zip(mem, sts):
            bottom_velocity(m, st)
        out = bs.step([X.make_params(m.params, n=n, tn=m.tn(n)) for m in mem], sts)
        assert all(r.status == X.OK for r in out)
    bs.close()
    for m in range(len(mem)):
        for k in ("p", "hp", "uhdye", "vhdxe"):
            np.testing.assert_array_equal(sts[m][k], single[m][k], err_msg=f"{m}:{k}")


@pytest.mark.gpu
def test_gpu_drag_three_levels():
    X.load()
    scn = S.add_three_levels(drag_case(1))
    sched = S.three_level_schedule(16, 4)
    sol = X.Solver(scn.grid)
    o = O.Oracle(scn.grid)
    sg, so = scn.copy_state(), scn.copy_state()
    for (n, istl, nctbc, rold, rnew) in sched:
        prm = X.make_params(S.three_level_params(scn.params, istl, nctbc, rold, rnew), n=n,
                            tn=scn.tn(n))
        bottom_velocity(scn, sg)
        bottom_velocity(scn, so)
        a = sol.step(prm, sg)
        b = o.step(prm, so)
        assert a.status == b.status == X.OK and a.iters_total == b.iters_total
    sol.close()
    o.close()
    assert cases.state_err(sg, so, scn.la) < 1e-9
