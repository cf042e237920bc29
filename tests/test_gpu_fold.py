"""Member reductions folded into the CG kernels (EFDC_XM_OPT_FOLD_REDUCE).

With folding on, each CG kernel counts its stored per-unit partial sums
towards their member, and the CTA that stores a member's last one sums the
member's partials and runs its epilogue (ALPHA, BETA, the stop tests); off, a
member-reduce kernel follows each CG kernel.  The sums run in the same fixed
order either way, so a batch steps to the same state bit for bit with the same
iterations: FP64 and MIXED, every MIXED kernel variant, Jacobi and polynomial
members, an unsymmetric (radiation) member, wetting and drying, host- and
device-driven loops, and a 2048 x 2048 basin whose members span thousands of
units (many CTAs arrive per member).
"""
import numpy as np
import pytest

import cases
import efdc_xm as X
import scenario as S

pytestmark = pytest.mark.gpu

FIELDS = ("p", "hp", "hu", "hv", "uhdye", "vhdxe", "sub", "svb", "lmaskdry")


@pytest.fixture(scope="module", autouse=True)
def _lib():
    X.load()


def run(mem, steps, tm, prec, fold, variant=0, device_loops=1):
    bs = X.BatchSolver([m.grid for m in mem])
    bs.set_option(X.OPT_FOLD_REDUCE, 2 * fold)
    bs.set_option(X.OPT_KERNEL_VARIANT, variant)
    bs.set_option(X.OPT_DEVICE_LOOPS, device_loops)
    sts = [m.copy_state() for m in mem]
    stats = []
    for n in range(1, steps + 1):
        r = bs.step([X.make_params(m.params, n=n, tn=m.tn(n) * tm, precision=prec)
                     for m in mem], sts)
        stats.append([(x.status, x.iters_total, x.solves, x.outer_refinements) for x in r])
    bs.close()
    return sts, stats


def same(a, b, n):
    assert a[1] == b[1]
    for m in range(n):
        for k in FIELDS:
            np.testing.assert_array_equal(a[0][m][k], b[0][m][k], err_msg=f"{m}:{k}")


MEMBERS = ("basin_fp64", "noise_forcing", "radiation_all_sides", "tidal_flat_99")


@pytest.mark.parametrize("prec,variant,loops", [(X.PREC_FP64, 0, 1), (X.PREC_FP64, 0, 0),
                                                (X.PREC_MIXED, 0, 1), (X.PREC_MIXED, 1, 1),
                                                (X.PREC_MIXED, 2, 1), (X.PREC_MIXED, 3, 1),
                                                (X.PREC_MIXED, 3, 0)])
def test_fold_equals_reduce_kernels(prec, variant, loops):
    mem = [cases.build(n)[0] for n in MEMBERS]
    a = run(mem, 12, 20.0, prec, 0, variant, loops)
    b = run(mem, 12, 20.0, prec, 1, variant, loops)
    same(a, b, len(mem))


@pytest.mark.parametrize("prec", [X.PREC_FP64, X.PREC_MIXED])
def test_fold_large_member(prec):
    mem = [S.config2(n=2048)]
    a = run(mem, 3, 1.0, prec, 0, 3)
    b = run(mem, 3, 1.0, prec, 1, 3)
    same(a, b, 1)


def test_fold_matches_oracle():
    """The folded FP64 form against the oracle: the same CG iterations and
    the surface within 1e-9 m at every step."""
    scn = cases.build("noise_forcing")[0]
    res = cases.run_both(scn, 20)
    for n, (a, b, sg, so) in enumerate(res, 1):
        assert a["status"] == b["status"] == X.OK
        assert a["iters_total"] == b["iters_total"], n
        assert cases.state_err(sg, so, scn.la) < 1e-9, n
