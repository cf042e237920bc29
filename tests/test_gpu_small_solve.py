"""CONGRAD of small members in one CTA each (EFDC_XM_OPT_SMALL_SOLVE).

A context whose members all fit one CTA's shared memory runs each member's
whole FP64 CG as one launch (k_cg_small): its vectors stay in shared memory,
its rows, per-unit partial sums, member sums and epilogues are the multi-kernel
CG's.  The two forms must step to the same state bit for bit, with the same
CG iterations: the reference's sample-model grids and the 100 x 60 basin,
alone and as one batch, with device-driven and host-driven loops, and with a
wetting-and-drying lake whose re-solves restart the CG.
"""
from pathlib import Path

import numpy as np
import pytest

import cases
import efdc_xm as X
import scenario as S

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
FIELDS = ("p", "hp", "hu", "hv", "uhdye", "vhdxe", "lmaskdry", "sub", "svb")


@pytest.fixture(scope="module", autouse=True)
def _lib():
    X.load()


def models():
    out = []
    for name, kw in (("Lake_T_HYD_WQ", dict(wind=(2e-4, 1e-4), drawdown=0.6)),
                     ("Lake_Washington", dict(wind=(1e-4, 2e-4))), ("Ohio_River_4", {})):
        out.append(S.sample_model(dict(np.load(GOLD / f"sample_{name}.npz")), **kw))
    return out


def run(mem, steps, small, device_loops=1):
    bs = X.BatchSolver([m.grid for m in mem])
    bs.set_option(X.OPT_SMALL_SOLVE, small)
    bs.set_option(X.OPT_DEVICE_LOOPS, device_loops)
    sts = [m.copy_state() for m in mem]
    its = []
    for n in range(1, steps + 1):
        out = bs.step([X.make_params(m.params, n=n, tn=m.tn(n)) for m in mem], sts)
        assert all(r.status == X.OK for r in out), [r.as_dict() for r in out]
        its.append([(r.iters_total, r.solves) for r in out])
    bs.close()
    return sts, its


@pytest.mark.parametrize("device_loops", [1, 0])
def test_small_solve_equals_multi_kernel_cg(device_loops):
    mem = models()
    a = run(mem, 25, 1, device_loops)
    b = run(mem, 25, 0, device_loops)
    assert a[1] == b[1]
    for m in range(len(mem)):
        for k in FIELDS:
            np.testing.assert_array_equal(a[0][m][k], b[0][m][k], err_msg=f"{m}:{k}")


def test_small_solve_single_basin_matches_oracle():
    """Lake Washington alone (its window of 15 tiles takes the small solve)
    against the oracle: the same CG iterations every step."""
    for scn in (models()[1],):
        res = cases.run_both(scn, 40)
        for n, (a, b, sg, so) in enumerate(res, 1):
            assert a["status"] == b["status"] == X.OK
            assert a["iters_total"] == b["iters_total"], n
            assert cases.state_err(sg, so, scn.la) < 1e-9, n
