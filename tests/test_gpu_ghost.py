"""Each member of a batch reads its own ghost cell LC.

EFDC+ points every missing neighbour of a cell at one ghost element, LC, and
some reads of it are not multiplied by a closed face's zero switch: FP1 and
the continuity read UHDYE(LEC(L)) and VHDXE(LNC(L)) as they are
(calpuv2c.f90:282-290, 466-486), so a nonzero ghost transport enters the
step.  In a batch each member has a ghost tile of its own, and its land slots
hold its own LC values.  Here two members carry different nonzero ghost
transports: each member of the batch must step exactly as its single-basin
run (EFDC+ itself keeps them 0: it zeroes them at allocation and writes only
zeros there).
"""
import numpy as np
import pytest

import cases
import efdc_xm as X

pytestmark = pytest.mark.gpu

FIELDS = ("p", "hp", "hu", "hv", "uhdye", "vhdxe", "uhe", "vhe")
GHOST = {0: (0.02, -0.01), 1: (-0.03, 0.015)}


@pytest.fixture(scope="module", autouse=True)
def _lib():
    X.load()


def members():
    out = []
    for m, name in enumerate(("basin_fp64", "noise_forcing")):
        scn = cases.build(name)[0]
        g = scn.grid["lc"] - 1
        u, v = GHOST[m]
        scn.state["uhdye"][g] = u
        scn.state["vhdxe"][g] = v
        out.append(scn)
    return out


def test_batch_members_read_their_own_ghost():
    mem = members()
    steps = 8
    single = []
    for scn in mem:
        sol = X.Solver(scn.grid)
        st = scn.copy_state()
        its = [sol.step(X.make_params(scn.params, n=n, tn=scn.tn(n)), st).iters_total
               for n in range(1, steps + 1)]
        sol.close()
        single.append((st, its))
    bs = X.BatchSolver([m.grid for m in mem])
    sts = [m.copy_state() for m in mem]
    its = [[] for _ in mem]
    for n in range(1, steps + 1):
        out = bs.step([X.make_params(m.params, n=n, tn=m.tn(n)) for m in mem], sts)
        for m, r in enumerate(out):
            assert r.status == X.OK
            its[m].append(r.iters_total)
    bs.close()
    for m, scn in enumerate(mem):
        assert its[m] == single[m][1], m
        for k in FIELDS:
            np.testing.assert_array_equal(sts[m][k], single[m][0][k], err_msg=f"{m}:{k}")


def test_ghost_transports_enter_the_step():
    """The control: the same basin with zero ghosts steps to another surface."""
    import scenario as S
    scn = members()[1]
    base = cases.build("noise_forcing")[0]
    out = []
    for sc in (scn, base):
        sol = X.Solver(sc.grid)
        st = sc.copy_state()
        sol.step(X.make_params(sc.params, n=1, tn=sc.tn(1)), st)
        sol.close()
        out.append(st["p"][1:sc.la])
    assert np.abs(out[0] - out[1]).max() / S.G > 1e-9
