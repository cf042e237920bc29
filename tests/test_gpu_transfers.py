"""efdc_xm_fields.unchanged: arrays the caller did not touch since this
context's last transfer of them are not sent again.

* Steps on host arrays with the state arrays declared unchanged give the
  results of steps that send everything, bit for bit, in the chunked batch
  path (two or more members) and the single-basin path, and upload fewer bytes:
  exactly the bytes of the arrays left out.
* The library sends a declared-unchanged array anyway when its device copy is
  no longer that transfer's (here: after a device-resident step, whose
  results the caller has not downloaded).
"""
import numpy as np
import pytest

import cases
import efdc_xm as X

pytestmark = pytest.mark.gpu

KEPT = ("p", "hp", "hu", "hv", "uhdye", "vhdxe", "sub", "svb", "lopenbcdry")
FIELDS = ("p", "hp", "h1p", "hu", "hv", "uhdye", "vhdxe", "uhe", "vhe", "sub", "svb")


@pytest.fixture(scope="module", autouse=True)
def _lib():
    X.load()


def members():
    return [cases.build(n)[0] for n in ("basin_fp64", "noise_forcing", "radiation_all_sides")]


def run_batch(mem, steps, unchanged, precision=X.PREC_FP64):
    bs = X.BatchSolver([m.grid for m in mem])
    sts = [m.copy_state() for m in mem]
    prep = bs.prepare(sts, unchanged=unchanged)
    up = []
    for n in range(1, steps + 1):
        b0 = X.transfer_bytes()[0]
        out = bs.step_prepared([X.make_params(m.params, n=n, tn=m.tn(n) * 10.0,
                                              precision=precision) for m in mem], prep)
        assert all(r.status == X.OK for r in out)
        up.append(X.transfer_bytes()[0] - b0)
    bs.close()
    return sts, up


@pytest.mark.parametrize("precision", [X.PREC_FP64, X.PREC_MIXED])
def test_batch_unchanged_same_results_fewer_bytes(precision):
    mem = members()
    a, up_a = run_batch(mem, 8, 0, precision)
    b, up_b = run_batch(mem, 8, X.same_bits(KEPT), precision)
    for m, scn in enumerate(mem):
        for k in FIELDS:
            np.testing.assert_array_equal(a[m][k], b[m][k], err_msg=f"{m}:{k}")
    # the first step sends everything; later ones leave out the kept arrays
    assert up_b[0] == up_a[0]
    lcs = sum(m.lc for m in mem)
    saved = 8 * 8 * lcs + 4 * lcs  # eight double arrays and LOPENBCDRY, every member
    # (member arrays that happen to lie back to back move in one copy that
    # includes the element between them)
    slack = 9 * 8 * (len(mem) - 1)
    for n in range(1, 8):
        assert saved <= up_a[n] - up_b[n] <= saved + slack, (n, up_a[n], up_b[n], saved)


def test_single_basin_unchanged():
    scn = cases.build("basin_fp64")[0]
    res = []
    for bits in (0, X.same_bits(KEPT)):
        sol = X.Solver(scn.grid)
        st = scn.copy_state()
        f, _k = X.make_fields(st, unchanged=bits)
        for n in range(1, 6):
            s = X.Stats()
            rc = sol.lib.efdc_xm_step(sol.ctx, X.make_params(scn.params, n=n, tn=scn.tn(n)),
                                      f, s)
            assert rc == X.OK, sol.last_error()
        sol.close()
        res.append(st)
    for k in FIELDS:
        np.testing.assert_array_equal(res[0][k], res[1][k], err_msg=k)


def test_stale_device_copy_is_sent_anyway():
    """A device-resident step between two host-array steps leaves the device
    copies newer than the caller's arrays: the next step must upload them
    although they are declared unchanged."""
    mem = members()

    def run(bits):
        bs = X.BatchSolver([m.grid for m in mem])
        sts = [m.copy_state() for m in mem]
        prep = bs.prepare(sts, unchanged=bits)
        prm = lambda n: [X.make_params(m.params, n=n, tn=m.tn(n) * 10.0) for m in mem]  # noqa
        bs.step_prepared(prm(1), prep)
        bs.step_device(prm(2))  # not downloaded: the host keeps step 1's state
        bs.step_prepared(prm(3), prep)
        bs.close()
        return sts

    a, b = run(0), run(X.same_bits(KEPT))
    for m in range(len(mem)):
        for k in FIELDS:
            np.testing.assert_array_equal(a[m][k], b[m][k], err_msg=f"{m}:{k}")
