"""GPU parity at the workload configurations' own sizes.

The other parity tests use basins of a few thousand cells.  These run the
full-size cases against the oracle (its OpenMP form, whose results do not
depend on the thread count; test_oracle_properties.py checks that):

* the 100 x 60 basin (~5,600 cells) for its full 1,000 steps;
* the 2048 x 2048 curvilinear basin (3.4 M cells, 13,890 tiles), 20 steps;
* the largest member of the 256-basin ensemble (~400 k cells), 50 steps;
* one 1024 x 1024 wetting/drying tidal flat (1.05 M cells, ISDRY = 99), 30
  steps of the tidal phase in which its flats dry and flood.

Bars as in test_gpu_parity.py: FP64 has the oracle's CG iteration count and
sweep count on every step, surface within 1e-9 m and bit-exact masks, face
switches and wet lists; MIXED, from the oracle's state each step, is within
1e-6 m with bit-exact masks.  Multi-tile Morton order, quads that span
thousands of tiles and members near the ensemble's upper size are covered
here and nowhere else.
"""
import os

import numpy as np
import pytest

import cases
import efdc_xm as X
import scenario as S

pytestmark = pytest.mark.gpu

NT = os.cpu_count() or 1
MASKS = ("sub", "svb", "sbx", "sby", "lmaskdry", "iscdry", "natdry")


@pytest.fixture(scope="module", autouse=True)
def _lib():
    X.load()


def check_fp64(scn, steps, tm=1.0, every_state=False):
    last = steps  # states kept: the last step's (and every step's if asked)
    res = cases.run_both(scn, steps, tm, lists=True, nthreads=NT,
                         keep=None if every_state else (lambda n: n == last))
    la = scn.la
    for n, (a, b, sg, so) in enumerate(res, 1):
        assert a["status"] == b["status"], (n, a, b)
        assert a["solves"] == b["solves"], (n, a["solves"], b["solves"])
        assert a["iters_total"] == b["iters_total"], (n, a["iters_total"], b["iters_total"])
        if sg is not None:
            assert cases.state_err(sg, so, la) < 1e-9, n
            for k in MASKS:
                np.testing.assert_array_equal(sg[k][1:la], so[k][1:la], err_msg=f"{n}:{k}")
            assert a["lawet"] == b["lawet"] and a["ladry"] == b["ladry"]
            np.testing.assert_array_equal(sg["lwet"][:a["lawet"]], so["lwet"][:b["lawet"]])
    return res


def check_mixed(scn, steps, tm=1.0):
    res = cases.run_both(scn, steps, tm, precision=X.PREC_MIXED, same_input=True, nthreads=NT)
    worst = 0.0
    for n, (a, b, sg, so) in enumerate(res, 1):
        assert a["status"] == b["status"], (n, a, b)
        worst = max(worst, cases.state_err(sg, so, scn.la))
        for k in ("lmaskdry", "sub", "svb", "iscdry"):
            np.testing.assert_array_equal(sg[k][1:scn.la], so[k][1:scn.la], err_msg=f"{n}:{k}")
    assert worst <= 1e-6, worst
    return worst


def test_config1_full_1000_steps():
    scn = S.config1()
    res = check_fp64(scn, 1000)
    assert sum(a["iters_total"] for a, _, _, _ in res) > 1000


def test_config2_2048_fp64():
    scn = S.config2(n=2048)
    assert scn.ncell > 3_300_000
    check_fp64(scn, 20)


def test_config2_2048_mixed():
    check_mixed(S.config2(n=2048), 5)


def test_config3_largest_member():
    sizes = S.config3_sizes()
    k = int(np.argmax(sizes))
    scn = S.config3_member(k, int(sizes[k]))
    assert scn.ncell > 390_000
    check_fp64(scn, 50)
    check_mixed(scn, 10)


def test_config5_tidal_flat_1024():
    scn = S.tidal_flat(n=1024, seed=5)
    assert scn.ncell == 1024 * 1024
    res = check_fp64(scn, 30, tm=60.0)
    assert sum(a["solves"] for a, _, _, _ in res) > 30  # wet/dry re-solves happened
    check_mixed(scn, 5, tm=60.0)
