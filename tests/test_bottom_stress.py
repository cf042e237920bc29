"""The bottom-stress producer: CALTBXY's drag coefficients STBX, STBY (the
rough log-law form of caltbxy.f90:504-537 and the smooth viscous form of
:480-502) and the bottom stresses TBX, TBY of hdmt2t.f90:670-684, on the
device from the state the last step left there (efdc_xm_set_bed,
efdc_xm_bottom_stress_batch).

Bars:
* (CPU) the oracle's restatement against an independent numpy evaluation of
  the same formulas, for one layer and several, on every wet cell;
* (CPU) the faces of the cells of LDRY get TBX = TBY = 0 and the other dry
  cells keep theirs;
* GPU: from the same state and inputs, STBX, STBY, TBX, TBY within 1e-14
  relative of the oracle (the device's and the host's log may differ in the
  last bit), the dry-face zeros at the same faces;
* GPU: a step given TBX, TBY = NULL after the producer uses the stresses the
  producer left on the device: the same CG iteration counts as the oracle
  fed the oracle's stresses, elevation within 1e-9 m;
* GPU: a batch gives each member's single-basin result bit for bit.
"""
import numpy as np
import pytest

import cases
import efdc_xm as X
import oracle as O
import scenario as S

TM = 60.0


def setup(name, kc=1, seed=5):
    scn, steps, tm = cases.build(name)
    return scn, S.make_bed(scn, seed=seed, kc=kc), min(steps, 8), tm


def numpy_stress(scn, bed, st, drag, delt, avcon1, tbx, tby):
    """caltbxy.f90:476-539 and hdmt2t.f90:670-684 in numpy, over the wet cells."""
    g = scn.grid
    la = scn.la
    L = np.arange(2, la + 1)
    i = L - 1
    lw = np.asarray(g["lwc"])[i] - 1
    ls = np.asarray(g["lsc"])[i] - 1
    wet = np.ones(L.size, bool) if scn.params["isdry"] == 0 else st["lmaskdry"][i] != 0
    zbr, dxp, dyp = bed["zbr"], bed["dxp"], bed["dyp"]
    zu = 0.5 * (dxp[lw] * zbr[lw] + dxp[i] * zbr[i]) * g["dxiu"][i]
    zv = 0.5 * (dyp[ls] * zbr[ls] + dyp[i] * zbr[i]) * g["dyiv"][i]
    U, V, VU, UV = drag["ub"][i], drag["vb"][i], drag["vu"][i], drag["uv"][i]
    hu, hv = st["hu"][i], st["hv"][i]
    so, to = bed["stbxo"][i], bed["stbyo"][i]
    rough = zbr[i] > 1e-6
    um_r = np.sqrt(VU * VU + U * U + 1e-12)
    vm_r = np.sqrt(UV * UV + V * V + 1e-12)
    um_s = np.sqrt(U * U + VU * VU + 1e-12)
    vm_s = np.sqrt(UV * UV + V * V + 1e-12)
    um = np.where(rough, um_r, um_s)
    vm = np.where(rough, vm_r, vm_s)
    cdu = 0.5 * so * hu / (delt * um)
    cdv = 0.5 * to * hv / (delt * vm)
    with np.errstate(all="ignore"):
        hur = np.maximum(zu, drag["h1u"][i])
        hvr = np.maximum(zv, drag["h1v"][i])
        if bed["kc"] == 1:
            lu = np.log(np.maximum(0.5 * hur / zu, 7.5)) - 1.0
            lv = np.log(np.maximum(0.5 * hvr / zv, 7.5)) - 1.0
            sx_r = so * 0.16 / (lu * lu)
            sy_r = to * 0.16 / (lv * lv)
        else:
            sg = 0.5 * np.maximum(bed["dzc1"][i], bed["sgzu1"][i])
            sh = 0.5 * np.maximum(bed["dzc1"][i], bed["sgzv1"][i])
            lu = np.log(np.maximum(1.0 + sg * hur / zu, 7.5))
            lv = np.log(np.maximum(1.0 + sh * hvr / zv, 7.5))
            sx_r = bed["avcon"] * so * 0.16 / (lu * lu)
            sy_r = bed["avcon"] * to * 0.16 / (lv * lv)
    visfac = 0.0258 * bed["coeftsbl"] ** (2.0 / 7.0)
    sx_s = visfac * bed["avcon"] * so * ((bed["vismud"] * (1.0 / hu) / um) * (2.0 / 7.0))
    sy_s = visfac * bed["avcon"] * to * ((bed["vismud"] * (1.0 / hv) / vm) * (2.0 / 7.0))
    sx = np.minimum(cdu, np.where(rough, sx_r, sx_s))
    sy = np.minimum(cdv, np.where(rough, sy_r, sy_s))
    tx = (avcon1 * (1.0 / hu) + sx * np.sqrt(VU * VU + U * U)) * U
    ty = (avcon1 * (1.0 / hv) + sy * np.sqrt(UV * UV + V * V)) * V
    return wet, i, sx, sy, tx, ty


def rel(a, b):
    s = np.maximum(np.abs(b), 1e-300)
    return float(np.max(np.abs(a - b) / s)) if a.size else 0.0


def oracle_run(scn, bed, steps, tm, avcon1=0.0, device_like=False):
    """Steps with the producer after each; yields per step the state and the drag."""
    o = O.Oracle(scn.grid)
    o.set_bed(bed)
    st = scn.copy_state()
    out = []
    for n in range(1, steps + 1):
        h1u, h1v = st["hu"].copy(), st["hv"].copy()
        r = o.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * tm), st)
        drag = S.drag_inputs(scn, st, h1u, h1v, seed=n)
        drag["stbx"] = np.zeros(scn.lc)
        drag["stby"] = np.zeros(scn.lc)
        drag["tbx"], drag["tby"] = st["tbx"], st["tby"]
        dp = X.make_drag_params(dict(scn.params, avcon1=avcon1), n=n)
        assert o.bottom_stress(dp, st, drag) == X.OK
        out.append((r.as_dict(), {k: v.copy() for k, v in st.items() if isinstance(v, np.ndarray)},
                    {k: v.copy() for k, v in drag.items()}))
    o.close()
    return out


@pytest.mark.parametrize("name,kc", [("basin_fp64", 1), ("basin_fp64", 4), ("tidal_flat_99", 1)])
def test_oracle_matches_numpy(name, kc):
    scn, bed, steps, tm = setup(name, kc)
    o = O.Oracle(scn.grid)
    o.set_bed(bed)
    st = scn.copy_state()
    for n in range(1, 4):
        h1u, h1v = st["hu"].copy(), st["hv"].copy()
        o.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * tm), st)
        drag = S.drag_inputs(scn, st, h1u, h1v, seed=n)
        drag.update(stbx=np.zeros(scn.lc), stby=np.zeros(scn.lc), tbx=st["tbx"].copy(),
                    tby=st["tby"].copy())
        tbx0 = drag["tbx"].copy()
        dp = X.make_drag_params(dict(scn.params, avcon1=1e-3), n=n)
        assert o.bottom_stress(dp, st, drag) == X.OK
        wet, i, sx, sy, tx, ty = numpy_stress(scn, bed, st, drag, dp.delt, 1e-3, None, None)
        assert wet.sum() > 0
        for got, want in ((drag["stbx"][i][wet], sx[wet]), (drag["stby"][i][wet], sy[wet]),
                          (drag["tbx"][i][wet], tx[wet]), (drag["tby"][i][wet], ty[wet])):
            assert rel(got, want) < 1e-13
        if scn.params["isdry"] > 0:  # dry cells: zero or kept, never anything else
            d = ~wet
            assert np.all((drag["tbx"][i][d] == 0.0) | (drag["tbx"][i][d] == tbx0[i][d]))
    o.close()


def test_oracle_dry_faces_zeroed():
    scn, bed, _, tm = setup("tidal_flat_99")
    o = O.Oracle(scn.grid)
    o.set_bed(bed)
    st = scn.copy_state()
    for n in range(1, 6):
        h1u, h1v = st["hu"].copy(), st["hv"].copy()
        o.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * tm), st)
    drag = S.drag_inputs(scn, st, h1u, h1v, seed=9)
    drag.update(tbx=np.full(scn.lc + 1, 7.0), tby=np.full(scn.lc + 1, 7.0))
    dp = X.make_drag_params(dict(scn.params, ntstbc=3), n=1)  # N < NTSTBC+1: all dry in LDRY
    assert o.bottom_stress(dp, st, drag) == X.OK
    la = scn.la
    L = np.arange(2, la + 1)
    dry = st["lmaskdry"][L - 1] == 0
    assert dry.sum() > 10
    lec = np.asarray(scn.grid["lec"])[L - 1]
    assert np.all(drag["tbx"][L[dry] - 1] == 0.0)
    east = lec[dry]
    east = east[east <= la]
    wet_e = st["lmaskdry"][east - 1] != 0
    assert np.all(drag["tbx"][east[~wet_e] - 1] == 0.0)
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,kc", [("basin_fp64", 1), ("noise_forcing", 4), ("tidal_flat_99", 1),
                                     ("legacy_dry_1", 1)])
def test_gpu_bottom_stress_matches_oracle(name, kc):
    """From the oracle's state after each step (uploaded; the device's entry
    mask from a step of the same entry state) and the same internal-mode
    inputs, the device's stresses equal the oracle's but for the last bits of
    log."""
    X.load()
    scn, bed, steps, tm = setup(name, kc)
    o = O.Oracle(scn.grid)
    o.set_bed(bed)
    sol = X.Solver(scn.grid)
    sol.set_bed(bed)
    st = scn.copy_state()
    i = np.arange(1, scn.la)
    for n in range(1, steps + 1):
        prm = X.make_params(scn.params, n=n, tn=scn.tn(n) * tm)
        entry = {k: (v.copy() if isinstance(v, np.ndarray) else
                     {q: a.copy() for q, a in v.items()} if isinstance(v, dict) else v)
                 for k, v in st.items()}
        h1u, h1v = st["hu"].copy(), st["hv"].copy()
        assert o.step(prm, st).status in (X.OK, X.NEG_DEPTH)
        sol.step(prm, entry)
        sol.upload(st)
        drag = S.drag_inputs(scn, st, h1u, h1v, seed=n)
        d_o = dict(drag, stbx=np.zeros(scn.lc), stby=np.zeros(scn.lc), tbx=st["tbx"].copy(),
                   tby=st["tby"].copy())
        d_g = dict(drag, stbx=np.zeros(scn.lc), stby=np.zeros(scn.lc), tbx=st["tbx"].copy(),
                   tby=st["tby"].copy())
        dp = X.make_drag_params(dict(scn.params, avcon1=1e-3), n=n)
        assert o.bottom_stress(dp, st, d_o) == X.OK
        sol.bottom_stress(dp, d_g)
        for k in ("stbx", "stby", "tbx", "tby"):
            assert rel(d_g[k][i], d_o[k][i]) < 1e-14, (n, k)
            assert np.array_equal(d_g[k][i] == 0.0, d_o[k][i] == 0.0), (n, k)
        st["tbx"], st["tby"] = d_o["tbx"], d_o["tby"]
    sol.close()
    o.close()


@pytest.mark.gpu
def test_gpu_stresses_stay_on_device():
    """A step given TBX, TBY = NULL uses the producer's stresses."""
    X.load()
    scn, bed, steps, tm = setup("noise_forcing", 1)
    ref = oracle_run(scn, bed, steps, tm, avcon1=1e-3)
    sol = X.Solver(scn.grid)
    sol.set_bed(bed)
    st = scn.copy_state()
    for n in range(1, steps + 1):
        h1u, h1v = st["hu"].copy(), st["hv"].copy()
        a = sol.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * tm), st)
        r, so, _ = ref[n - 1]
        assert a.iters_total == r["iters_total"], n
        assert float(np.abs(st["p"][1:scn.la] - so["p"][1:scn.la]).max()) / S.G < 1e-9, n
        drag = S.drag_inputs(scn, st, h1u, h1v, seed=n)
        sol.bottom_stress(X.make_drag_params(dict(scn.params, avcon1=1e-3), n=n), drag)
        st.pop("tbx", None)  # the next step reads them on the device
        st.pop("tby", None)
    sol.close()


@pytest.mark.gpu
def test_gpu_bottom_stress_batch_equals_single():
    X.load()
    items = [setup("basin_fp64", 1, seed=1), setup("tidal_flat_99", 1, seed=2)]
    bs = X.BatchSolver([scn.grid for scn, _, _, _ in items])
    singles = [X.Solver(scn.grid) for scn, _, _, _ in items]
    for m, (scn, bed, _, _) in enumerate(items):
        bs.set_bed(bed, m)
        singles[m].set_bed(bed)
    sb = [scn.copy_state() for scn, _, _, _ in items]
    ss = [scn.copy_state() for scn, _, _, _ in items]
    for n in range(1, 5):
        prm = [X.make_params(scn.params, n=n, tn=scn.tn(n) * tm) for scn, _, _, tm in items]
        h1 = [(s["hu"].copy(), s["hv"].copy()) for s in sb]
        bs.step(prm, sb)
        for m in range(len(items)):
            singles[m].step(prm[m], ss[m])
        db = [S.drag_inputs(scn, sb[m], *h1[m], seed=n) for m, (scn, _, _, _) in enumerate(items)]
        ds = [dict((k, v.copy()) for k, v in d.items()) for d in db]
        for d, s_ in zip(db, sb):
            d.update(tbx=s_["tbx"], tby=s_["tby"], stbx=np.zeros(s_["p"].size - 1))
        for d, s_ in zip(ds, ss):
            d.update(tbx=s_["tbx"], tby=s_["tby"], stbx=np.zeros(s_["p"].size - 1))
        dps = [X.make_drag_params(scn.params, n=n) for scn, _, _, _ in items]
        bs.bottom_stress(dps, db)
        for m in range(len(items)):
            singles[m].bottom_stress(dps[m], ds[m])
            la = items[m][0].la
            for k in ("tbx", "tby", "stbx"):
                assert np.array_equal(db[m][k][1:la], ds[m][k][1:la]), (m, n, k)
    bs.close()
    for s in singles:
        s.close()
