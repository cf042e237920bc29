"""An unsymmetric external-mode operator: a radiation boundary whose
interior faces are closed in the state (cases.unsymmetric).

Every other seeded case assembles a symmetric operator (CE(L) = CW(LE),
CN(L) = CS(LN) bit for bit), so this case is the one that drives the
library's four-array CG path from a CALPUV2C step.

Bars:
* (CPU) the oracle's assembled system is unsymmetric at the closed faces;
* FP64: the same CG iteration counts as the oracle, elevation within 1e-9 m;
* MIXED: elevation within 1e-6 m of the FP64 oracle from the same input;
* batched with a symmetric basin: each member bit-identical to its own
  single-basin run.
"""
import numpy as np
import pytest

import cases
import efdc_xm as X
import oracle as O
import scenario as S

STEPS = 6
TM = 20.0


def unsymmetric_faces(scn, st):
    g = scn.grid
    L = np.arange(2, scn.la + 1)
    n = 0
    for a, b, key in (("cce", "ccw", "lec"), ("ccn", "ccs", "lnc")):
        nb = np.asarray(g[key])[L - 1]
        ok = nb != scn.lc
        n += int((st[a][L - 1][ok] != st[b][nb[ok] - 1]).sum())
    return n


def params(scn, n, precision=X.PREC_FP64):
    return X.make_params(scn.params, n=n, tn=scn.tn(n) * TM, precision=precision)


def test_case_is_unsymmetric():
    scn = cases.unsymmetric()
    orc = O.Oracle(scn.grid)
    st = scn.copy_state()
    counts = []
    for n in range(1, STEPS + 1):
        assert orc.step(params(scn, n), st, diag=True).status == X.OK
        counts.append(unsymmetric_faces(scn, st))
    orc.close()
    assert min(counts) == 3, counts


@pytest.mark.gpu
def test_gpu_unsymmetric_fp64_matches_oracle():
    X.load()
    scn = cases.unsymmetric()
    sol, orc = X.Solver(scn.grid), O.Oracle(scn.grid)
    sg, so = scn.copy_state(), scn.copy_state()
    for n in range(1, STEPS + 1):
        a = sol.step(params(scn, n), sg)
        b = orc.step(params(scn, n), so)
        assert a.status == b.status == X.OK, (n, a.as_dict())
        assert a.iters_total == b.iters_total, (n, a.iters_total, b.iters_total)
    err = float(np.abs(sg["p"][1:scn.la] - so["p"][1:scn.la]).max()) / S.G
    assert err < 1e-9, err
    sol.close()
    orc.close()


@pytest.mark.gpu
def test_gpu_unsymmetric_mixed_within_1e6_m():
    X.load()
    scn = cases.unsymmetric()
    sol, orc = X.Solver(scn.grid), O.Oracle(scn.grid)
    so = scn.copy_state()
    worst = 0.0
    for n in range(1, STEPS + 1):
        sg = {k: (v.copy() if isinstance(v, np.ndarray) else
                  {s: a.copy() for s, a in v.items()} if isinstance(v, dict) else v)
              for k, v in so.items()}
        a = sol.step(params(scn, n, X.PREC_MIXED), sg)
        orc.step(params(scn, n), so)
        assert a.status == X.OK, (n, a.as_dict())
        worst = max(worst, float(np.abs(sg["p"][1:scn.la] - so["p"][1:scn.la]).max()) / S.G)
    assert worst <= 1e-6, worst
    sol.close()
    orc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [X.PREC_FP64, X.PREC_MIXED])
def test_gpu_unsymmetric_in_batch_equals_single(precision):
    X.load()
    ms = [cases.unsymmetric(), cases.build("basin_fp64")[0]]
    bs = X.BatchSolver([m.grid for m in ms])
    singles = [X.Solver(m.grid) for m in ms]
    sb = [m.copy_state() for m in ms]
    ss = [m.copy_state() for m in ms]
    for n in range(1, STEPS + 1):
        prm = [params(m, n, precision) for m in ms]
        stb = bs.step(prm, sb)
        for k, m in enumerate(ms):
            st1 = singles[k].step(prm[k], ss[k])
            assert stb[k].status == st1.status == X.OK
            assert stb[k].iters_total == st1.iters_total, (k, n)
            assert np.array_equal(sb[k]["p"][1:m.la], ss[k]["p"][1:m.la]), (k, n)
    bs.close()
    for s in singles:
        s.close()


@pytest.mark.gpu
def test_gpu_unsymmetric_congrad_standalone():
    """CONGRAD on the unsymmetric scaled system the oracle assembled, through
    efdc_xm_congrad in both precisions."""
    X.load()
    scn = cases.unsymmetric()
    st = scn.copy_state()
    orc = O.Oracle(scn.grid)
    p_in = st["p"].copy()
    orc.step(params(scn, 1), st, diag=True)
    assert unsymmetric_faces(scn, st) == 3
    ccci = np.zeros_like(st["ccc"])
    ccci[1:scn.la] = 1.0 / st["ccc"][1:scn.la]
    po = p_in.copy()
    r1 = orc.congrad(st["ccc"], st["ccs"], st["ccn"], st["ccw"], st["cce"], ccci, st["fptmp"], po,
                     1e-10, 200)
    orc.close()
    sol = X.Solver(scn.grid)
    for prec, tol in ((X.PREC_FP64, 1e-9), (X.PREC_MIXED, 1e-6)):
        pg = p_in.copy()
        r2 = sol.congrad(st["ccc"], st["ccs"], st["ccn"], st["ccw"], st["cce"], ccci, st["fptmp"],
                         pg, 1e-10, 200, precision=prec)
        assert r2[0] == 0, sol.last_error()
        if prec == X.PREC_FP64:
            assert r2[1] == r1[1]
        assert np.abs(pg - po)[1:scn.la].max() / S.G < tol, prec
    sol.close()
