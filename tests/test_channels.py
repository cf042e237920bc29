"""Sub-grid channels: SUBCHAN, CONGRADC and the channel exchange of CALPUV2C.

The reference's CONGRADC adds the host-guest coupling CCCCHH with the same
sign to its initial residual and to A*p (congradc.f90:59-77, 99-116), so its
CG solves (A+C)P = b + 2C*P0; the library reproduces that by default, and
with chan_consistent = 1 solves the conductance system (A-C)P = b instead.

Bars:
* (CPU) the oracle's channels activate, a closed basin keeps its volume
  (the exchange moves water between host and guest only), and the two
  operators give different P;
* FP64: the same CG iteration counts as the oracle on every step, elevation
  within 1e-9 m, the channel flows within 1e-9 relative, for both operators;
* MIXED: elevation within 1e-6 m of the FP64 oracle from the same input;
* batched with a basin without channels: each member bit-identical to its
  own single-basin run;
* argument errors: open-boundary or out-of-range cells, unsupported types,
  missing flow arrays.
"""
import numpy as np
import pytest

import cases
import efdc_xm as X
import oracle as O
import scenario as S

TM = 10.0
FLOWS = ("qchanu", "qchanv", "qchanun", "qchanvn")


def params(scn, n, precision=X.PREC_FP64):
    return X.make_params(scn.params, n=n, tn=scn.tn(n) * TM, precision=precision)


def run_oracle(scn, steps):
    o = O.Oracle(scn.grid)
    o.set_channels(scn.channels)
    st = scn.copy_state()
    out = []
    for n in range(1, steps + 1):
        r = o.step(params(scn, n), st)
        out.append((r.as_dict(), {k: v.copy() for k, v in st.items() if isinstance(v, np.ndarray)}))
    o.close()
    return out


@pytest.mark.parametrize("consistent", [0, 1])
def test_oracle_channels_active_and_volume_kept(consistent):
    scn = cases.channels(consistent, closed=True, qcherr=0.25)
    res = run_oracle(scn, 20)
    assert all(r["status"] == X.OK for r, _ in res)
    active = max(int(np.count_nonzero(s["qchanu"]) + np.count_nonzero(s["qchanv"]))
                 for _, s in res)
    assert active >= 6, active
    dxyp = scn.grid["dxyp"][1:scn.la]
    v0 = float(np.sum(dxyp * scn.state["hp"][1:scn.la]))
    v1 = float(np.sum(dxyp * res[-1][1]["hp"][1:scn.la]))
    assert abs(v1 - v0) / v0 < 1e-10


def test_oracle_channel_operators_differ():
    a = run_oracle(cases.channels(0, qcherr=0.25), 6)[-1][1]["p"]
    b = run_oracle(cases.channels(1, qcherr=0.25), 6)[-1][1]["p"]
    assert float(np.abs(a - b).max()) / S.G > 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("consistent,qcherr,steps", [(0, 0.25, 12), (0, 1.0, 4), (1, 1.0, 12)])
def test_gpu_channels_fp64_matches_oracle(consistent, qcherr, steps):
    X.load()
    scn = cases.channels(consistent, qcherr=qcherr)
    ref = run_oracle(scn, steps)
    sol = X.Solver(scn.grid)
    sol.set_channels(scn.channels)
    st = scn.copy_state()
    for n in range(1, steps + 1):
        a = sol.step(params(scn, n), st)
        r, so = ref[n - 1]
        assert a.status == r["status"], (n, a.as_dict(), r)
        assert a.iters_total == r["iters_total"], (n, a.iters_total, r["iters_total"])
    la = scn.la
    assert float(np.abs(st["p"][1:la] - so["p"][1:la]).max()) / S.G < 1e-9
    for k in FLOWS:
        scale = max(1.0, float(np.abs(so[k]).max()))
        assert float(np.abs(st[k] - so[k]).max()) <= 1e-9 * scale, k
    sol.close()


@pytest.mark.gpu
@pytest.mark.parametrize("consistent,qcherr", [(0, 0.25), (1, 1.0)])
def test_gpu_channels_mixed_within_1e6_m(consistent, qcherr):
    """From the same input every step, the MIXED step's surface is within
    1e-6 m of the FP64 oracle's."""
    X.load()
    scn = cases.channels(consistent, qcherr=qcherr)
    o = O.Oracle(scn.grid)
    o.set_channels(scn.channels)
    sol = X.Solver(scn.grid)
    sol.set_channels(scn.channels)
    so = scn.copy_state()
    worst = 0.0
    for n in range(1, 13):
        sg = {k: (v.copy() if isinstance(v, np.ndarray) else
                  {s: a.copy() for s, a in v.items()} if isinstance(v, dict) else v)
              for k, v in so.items()}
        a = sol.step(params(scn, n, X.PREC_MIXED), sg)
        o.step(params(scn, n), so)
        assert a.status == X.OK, (n, a.as_dict())
        worst = max(worst, float(np.abs(sg["p"][1:scn.la] - so["p"][1:scn.la]).max()) / S.G)
    assert worst <= 1e-6, worst
    sol.close()
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [X.PREC_FP64, X.PREC_MIXED])
def test_gpu_channels_in_batch_equal_single(precision):
    X.load()
    ms = [cases.channels(1, qcherr=1.0), cases.build("basin_fp64")[0]]
    for m in ms[1:]:
        m.params["qcherr"] = 1.0
        m.params["chan_consistent"] = 1
    bs = X.BatchSolver([m.grid for m in ms])
    bs.set_channels(ms[0].channels, 0)
    singles = [X.Solver(m.grid) for m in ms]
    singles[0].set_channels(ms[0].channels)
    sb = [m.copy_state() for m in ms]
    ss = [m.copy_state() for m in ms]
    for n in range(1, 9):
        prm = [params(m, n, precision) for m in ms]
        stb = bs.step(prm, sb)
        for k, m in enumerate(ms):
            st1 = singles[k].step(prm[k], ss[k])
            assert stb[k].status == st1.status == X.OK
            assert stb[k].iters_total == st1.iters_total, (k, n)
            assert np.array_equal(sb[k]["p"][1:m.la], ss[k]["p"][1:m.la]), (k, n)
    assert np.array_equal(sb[0]["qchanu"], ss[0]["qchanu"])
    bs.close()
    for s in singles:
        s.close()


@pytest.mark.gpu
def test_gpu_channel_argument_errors():
    X.load()
    scn = cases.channels(1)
    sol = X.Solver(scn.grid)
    ch = dict(scn.channels)
    obc = int(scn.grid["obc"]["W"]["l"][3])
    bad = dict(ch, lhost=np.r_[obc, ch["lhost"][1:]].astype(np.int32))
    with pytest.raises(RuntimeError, match="open-boundary"):
        sol.set_channels(bad)
    bad = dict(ch, type=np.r_[3, ch["type"][1:]].astype(np.int32))
    with pytest.raises(RuntimeError, match="MDCHTYP"):
        sol.set_channels(bad)
    sol.set_channels(ch)
    st = scn.copy_state()
    del st["qchanv"]
    with pytest.raises(RuntimeError, match="QCHANU"):
        sol.step(params(scn, 1), st)
    sol.set_channels(None)  # removed: the basin steps as a plain one
    st = scn.copy_state()
    assert sol.step(params(scn, 1), st).status == X.OK
    sol.close()
