"""Batched contexts: several basins (ensemble members) in one context.

Bars:
* each member of a batch gives bit-identical results to the same basin run
  alone in its own context (FP64 and MIXED): every reduction is per member
  and taken in the same fixed order, so batching changes nothing;
* each member matches the oracle as the single-basin drop-in does (same CG
  iteration counts, elevation within 1e-9 m, masks bit-exact);
* a member that fails (CG_MAXITER) is reported in its own stats and does not
  disturb the others;
* the single-basin entry points refuse a batch context, and a field given
  for some members only is an argument error.
"""
import ctypes as C

import numpy as np
import pytest

import cases
import efdc_xm as X
import oracle as O
import scenario as S

pytestmark = pytest.mark.gpu

STATE_F = ("p", "hp", "h1p", "hu", "hv", "uhdye", "vhdxe", "uhe", "vhe")
MASK_F = ("sub", "svb", "sbx", "sby", "lmaskdry", "iscdry", "lopenbcdry", "natdry")
STEPS = 8


@pytest.fixture(scope="module", autouse=True)
def _lib():
    X.load()  # fails loudly when libefdc_xm.so is missing: no CPU fallback


def members():
    """The golden cases plus three uneven ensemble-style basins."""
    out = [cases.build(n) for n in cases.GOLDEN]
    for k, ncell in enumerate((900, 4_000, 15_000)):
        out.append((S.config3_member(k, ncell, seed=31), STEPS, 1.0))
    return out


def params_at(ms, n, precision=X.PREC_FP64):
    return [X.make_params(scn.params, n=n, tn=scn.tn(n) * tm, precision=precision)
            for scn, _, tm in ms]


def assert_same(a, b, la, what):
    for k in STATE_F + MASK_F:
        if k in a:
            assert np.array_equal(a[k][1:la], b[k][1:la]), f"{what}: {k} differs"


@pytest.mark.parametrize("precision", [X.PREC_FP64, X.PREC_MIXED])
def test_batch_equals_single(precision):
    ms = members()
    bs = X.BatchSolver([scn.grid for scn, _, _ in ms])
    assert bs.lib.efdc_xm_nmembers(bs.ctx) == len(ms)
    sb = [scn.copy_state() for scn, _, _ in ms]
    singles = [X.Solver(scn.grid) for scn, _, _ in ms]
    ss = [scn.copy_state() for scn, _, _ in ms]
    for n in range(1, STEPS + 1):
        prm = params_at(ms, n, precision)
        stb = bs.step(prm, sb, lists=True)
        for m, (scn, _, _) in enumerate(ms):
            st1 = singles[m].step(prm[m], ss[m], lists=True)
            assert stb[m].status == st1.status, (m, n)
            assert stb[m].iters_total == st1.iters_total, (m, n)
            assert stb[m].solves == st1.solves, (m, n)
            assert stb[m].lawet == st1.lawet and stb[m].ladry == st1.ladry, (m, n)
            assert_same(sb[m], ss[m], scn.la, f"member {m} step {n}")
            nw = st1.lawet
            assert np.array_equal(sb[m]["lwet"][:nw], ss[m]["lwet"][:nw])
    bs.close()
    for s in singles:
        s.close()


def test_batch_matches_oracle_fp64():
    ms = members()
    bs = X.BatchSolver([scn.grid for scn, _, _ in ms])
    orcs = [O.Oracle(scn.grid) for scn, _, _ in ms]
    sb = [scn.copy_state() for scn, _, _ in ms]
    so = [scn.copy_state() for scn, _, _ in ms]
    for n in range(1, STEPS + 1):
        prm = params_at(ms, n)
        stb = bs.step(prm, sb)
        for m, (scn, _, _) in enumerate(ms):
            sto = orcs[m].step(prm[m], so[m])
            assert stb[m].status == sto.status, (m, n)
            assert stb[m].iters_total == sto.iters_total, (m, n)
            err = float(np.abs(sb[m]["p"][1:scn.la] - so[m]["p"][1:scn.la]).max() / S.G)
            assert err < 1e-9, (m, n, err)
            for k in MASK_F:
                assert np.array_equal(sb[m][k][1:scn.la], so[m][k][1:scn.la]), (m, n, k)
    bs.close()
    for o in orcs:
        o.close()


def test_failing_member_is_isolated():
    ms = members()[:4]
    bs = X.BatchSolver([scn.grid for scn, _, _ in ms])
    singles = [X.Solver(scn.grid) for scn, _, _ in ms]
    sb = [scn.copy_state() for scn, _, _ in ms]
    ss = [scn.copy_state() for scn, _, _ in ms]
    prm = params_at(ms, 1)
    prm[1].iterm = 2  # member 1 cannot converge in two iterations
    stb = bs.step(prm, sb)
    assert stb[1].status == X.CG_MAXITER
    assert stb[1].iters_last == 2
    for m in (0, 2, 3):
        st1 = singles[m].step(prm[m], ss[m])
        assert stb[m].status == st1.status == X.OK
        assert stb[m].iters_total == st1.iters_total
        assert_same(sb[m], ss[m], ms[m][0].la, f"member {m}")
    bs.close()
    for s in singles:
        s.close()


def test_batch_argument_errors():
    ms = members()[:2]
    bs = X.BatchSolver([scn.grid for scn, _, _ in ms])
    states = [scn.copy_state() for scn, _, _ in ms]
    prm = params_at(ms, 1)
    # the single-basin entry points refuse a context of two members
    f, _k = X.make_fields(states[0])
    st = X.Stats()
    rc = bs.lib.efdc_xm_step(bs.ctx, C.byref(prm[0]), C.byref(f), C.byref(st))
    assert rc == X.BAD_ARGUMENT and "members" in bs.last_error()
    # a field given for one member only
    del states[1]["qsume"]
    with pytest.raises(RuntimeError, match="qsume"):
        bs.step(prm, states)
    # members must share the precision
    states = [scn.copy_state() for scn, _, _ in ms]
    prm[1].precision = X.PREC_MIXED
    with pytest.raises(RuntimeError, match="precision"):
        bs.step(prm, states)
    bs.close()


def field_major(states):
    """The same states with each field's member arrays back to back in one
    buffer (an ensemble held as one (LCM, members) array per field)."""
    out = [dict() for _ in states]
    for k, v in states[0].items():
        if isinstance(v, np.ndarray):
            buf = np.concatenate([st[k] for st in states])
            off = 0
            for i, st in enumerate(states):
                n = st[k].size
                out[i][k] = buf[off:off + n]
                off += n
        else:
            for i, st in enumerate(states):
                out[i][k] = {s: a.copy() for s, a in st[k].items()} if isinstance(st[k], dict) \
                    else st[k]
    return out


@pytest.mark.parametrize("precision", [X.PREC_FP64, X.PREC_MIXED])
def test_field_major_host_layout(precision):
    """Member arrays that lie back to back go up in one copy per field: the
    results equal those of separately allocated arrays."""
    ms = members()
    # one solver per layout: a MIXED solver carries per-member history (the
    # iteration estimate that picks each member's inner preconditioner)
    ba = X.BatchSolver([scn.grid for scn, _, _ in ms])
    bf = X.BatchSolver([scn.grid for scn, _, _ in ms])
    sa = [scn.copy_state() for scn, _, _ in ms]
    sf = field_major([scn.copy_state() for scn, _, _ in ms])
    def edges(st, scn):  # L = 1, L = LC and the element after LC
        return {k: (st[k][0], st[k][scn.lc - 1], st[k][-1]) for k in STATE_F + MASK_F
                if k in st and isinstance(st[k], np.ndarray)}
    for n in range(1, 4):
        prm = params_at(ms, n, precision)
        before = [edges(sf[m], scn) for m, (scn, _, _) in enumerate(ms)]
        sta = ba.step(prm, sa)
        stf = bf.step(prm, sf)
        for m, (scn, _, _) in enumerate(ms):
            assert sta[m].iters_total == stf[m].iters_total, (m, n)
            assert_same(sa[m], sf[m], scn.la, f"member {m} step {n}")
            # whole-run copies leave the caller's ghost and padding elements alone
            after = edges(sf[m], scn)
            for k, v in before[m].items():
                assert np.array_equal(np.array(v), np.array(after[k])), (m, n, k)
    ba.close()
    bf.close()


def test_chunked_step_equals_device_resident():
    """efdc_xm_step_batch runs a batch in member chunks whose transfers and
    steps overlap: with several members per chunk, back to back in host
    memory, it gives what the unchunked upload / step_device / download gives,
    bit for bit, and leaves the caller's ghost and padding elements alone."""
    ms = members() + [(S.config3_member(k, 600 + 700 * k, seed=41), STEPS, 1.0)
                      for k in range(16)]
    ba = X.BatchSolver([scn.grid for scn, _, _ in ms])
    bd = X.BatchSolver([scn.grid for scn, _, _ in ms])
    sa = field_major([scn.copy_state() for scn, _, _ in ms])
    sd = [scn.copy_state() for scn, _, _ in ms]
    def edges(st, scn):
        return {k: (st[k][0], st[k][scn.lc - 1], st[k][-1]) for k in STATE_F + MASK_F
                if k in st and isinstance(st[k], np.ndarray)}
    for n in range(1, 4):
        prm = params_at(ms, n, X.PREC_MIXED)
        before = [edges(sa[m], scn) for m, (scn, _, _) in enumerate(ms)]
        sta = ba.step(prm, sa, lists=True)
        bd.upload(sd)
        std = bd.step_device(prm)
        bd.download(sd, lists=True)
        for m, (scn, _, _) in enumerate(ms):
            assert sta[m].status == std[m].status, (m, n)
            assert sta[m].iters_total == std[m].iters_total, (m, n)
            assert_same(sa[m], sd[m], scn.la, f"member {m} step {n}")
            after = edges(sa[m], scn)
            for k, v in before[m].items():
                assert np.array_equal(np.array(v), np.array(after[k])), (m, n, k)
    ba.close()
    bd.close()
