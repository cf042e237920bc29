"""Baroclinic terms: CALEBI's external buoyancy integrals (standard sigma
grid) and the density gradients FPGXE, FPGYE of CALPUV2C's explicit
transports (calpuv2c.f90:161, 192-220; calebi.f90:73-120).

Bars:
* (CPU) with BSC = 0 the layers and B change nothing; with BSC = 1 the
  oracle's transports change, and a closed basin keeps its volume;
* FP64: the same CG iteration counts as the oracle, elevation within 1e-9 m
  (a basin with an open boundary, and a wetting/drying flat whose dry cells
  keep their integrals);
* MIXED: elevation within 1e-6 m of the FP64 oracle from the same input;
* batched with a basin without them: each member bit-identical to its own
  single-basin run;
* BSC > 0 without layers or without B is an argument error.
"""
import numpy as np
import pytest

import cases
import efdc_xm as X
import oracle as O
import scenario as S


def run_oracle(scn, steps, tm):
    o = O.Oracle(scn.grid)
    o.set_layers(scn.layers)
    st = scn.copy_state()
    out = []
    for n in range(1, steps + 1):
        r = o.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * tm), st)
        out.append((r.as_dict(), {k: v.copy() for k, v in st.items() if isinstance(v, np.ndarray)}))
    o.close()
    return out


def test_oracle_bsc_zero_changes_nothing_and_volume_kept():
    scn = cases.baroclinic(closed=True)
    on = run_oracle(scn, 10, 10.0)
    scn.params["bsc"] = 0.0
    off = run_oracle(scn, 10, 10.0)
    plain = cases.baroclinic(closed=True)
    del plain.state["b"]
    plain.params["bsc"] = 0.0
    o = O.Oracle(plain.grid)
    st = plain.copy_state()
    for n in range(1, 11):
        o.step(X.make_params(plain.params, n=n, tn=plain.tn(n) * 10.0), st)
    o.close()
    assert np.array_equal(off[-1][1]["p"], st["p"])  # BSC = 0: no trace of B
    assert float(np.abs(on[-1][1]["uhdye"] - off[-1][1]["uhdye"]).max()) > 1e-3
    dxyp = scn.grid["dxyp"][1:scn.la]
    v0 = float(np.sum(dxyp * scn.state["hp"][1:scn.la]))
    v1 = float(np.sum(dxyp * on[-1][1]["hp"][1:scn.la]))
    assert abs(v1 - v0) / v0 < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("wetdry,steps,tm", [(False, 12, 10.0), (True, 30, 60.0)])
def test_gpu_baroclinic_fp64_matches_oracle(wetdry, steps, tm):
    X.load()
    scn = cases.baroclinic(wetdry)
    ref = run_oracle(scn, steps, tm)
    sol = X.Solver(scn.grid)
    sol.set_layers(scn.layers)
    st = scn.copy_state()
    for n in range(1, steps + 1):
        a = sol.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * tm), st)
        r, so = ref[n - 1]
        assert a.status == r["status"], (n, a.as_dict(), r)
        assert a.iters_total == r["iters_total"], (n, a.iters_total, r["iters_total"])
        assert a.solves == r["solves"], n
    la = scn.la
    assert float(np.abs(st["p"][1:la] - so["p"][1:la]).max()) / S.G < 1e-9
    for k in ("lmaskdry", "sub", "svb"):
        assert np.array_equal(st[k][1:la], so[k][1:la]), k
    sol.close()


@pytest.mark.gpu
def test_gpu_baroclinic_mixed_within_1e6_m():
    X.load()
    scn = cases.baroclinic()
    o = O.Oracle(scn.grid)
    o.set_layers(scn.layers)
    sol = X.Solver(scn.grid)
    sol.set_layers(scn.layers)
    so = scn.copy_state()
    worst = 0.0
    for n in range(1, 13):
        sg = {k: (v.copy() if isinstance(v, np.ndarray) else
                  {s: a.copy() for s, a in v.items()} if isinstance(v, dict) else v)
              for k, v in so.items()}
        a = sol.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * 10.0,
                                   precision=X.PREC_MIXED), sg)
        o.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * 10.0), so)
        assert a.status == X.OK, (n, a.as_dict())
        worst = max(worst, float(np.abs(sg["p"][1:scn.la] - so["p"][1:scn.la]).max()) / S.G)
    assert worst <= 1e-6, worst
    sol.close()
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [X.PREC_FP64, X.PREC_MIXED])
def test_gpu_baroclinic_in_batch_equals_single(precision):
    X.load()
    ms = [cases.baroclinic(), cases.build("basin_fp64")[0]]
    bs = X.BatchSolver([m.grid for m in ms])
    bs.set_layers(ms[0].layers, 0)
    singles = [X.Solver(m.grid) for m in ms]
    singles[0].set_layers(ms[0].layers)
    sb = [m.copy_state() for m in ms]
    ss = [m.copy_state() for m in ms]
    for n in range(1, 7):
        prm = [X.make_params(m.params, n=n, tn=m.tn(n) * 10.0, precision=precision) for m in ms]
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
def test_gpu_baroclinic_argument_errors():
    X.load()
    scn = cases.baroclinic()
    sol = X.Solver(scn.grid)
    with pytest.raises(RuntimeError, match="layers"):
        sol.step(X.make_params(scn.params, n=1, tn=scn.tn(1)), scn.copy_state())
    sol.set_layers(scn.layers)
    st = scn.copy_state()
    del st["b"]
    with pytest.raises(RuntimeError, match="needs B"):
        sol.step(X.make_params(scn.params, n=1, tn=scn.tn(1)), st)
    bad = dict(dzc=scn.layers["dzc"][:2], zz=scn.layers["zz"][:2])
    with pytest.raises(RuntimeError, match="KC"):
        sol.set_layers(bad)
    sol.close()
