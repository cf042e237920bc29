"""efdc_xm_autotune on the GPU: it measures a schedule for the context's
workload, applies it, appends it to the table; a second call with the same
workload replays the table line without measuring; the tuned context still
steps within the MIXED bar of the FP64 oracle (and FP64 bit for bit: the
schedule does not touch FP64 results)."""
import numpy as np
import pytest

import cases
import efdc_xm as X

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    X.load()


def test_autotune_measure_replay_and_results(tmp_path):
    mem = [cases.build(n)[0] for n in ("basin_fp64", "noise_forcing", "radiation_all_sides")]
    table = tmp_path / "tune.txt"
    bs = X.BatchSolver([m.grid for m in mem])
    sts = [m.copy_state() for m in mem]
    prm = lambda n, p: [X.make_params(m.params, n=n, tn=m.tn(n) * 10.0, precision=p)  # noqa
                        for m in mem]
    bs.step(prm(1, X.PREC_MIXED), sts)
    sch, ms = bs.autotune(X.PREC_MIXED, table, measure=False)  # key absent: measures
    assert ms > 0
    key = bs.tune_key(X.PREC_MIXED)
    assert key.startswith("prec=mixed members=2^1 ")
    assert X.tune_lookup(table, key) == sch
    assert table.read_text().count("\n") == 1
    # the tuned context's next steps: MIXED within 1e-6 m of the oracle's FP64
    import oracle as O
    orcs = [O.Oracle(m.grid) for m in mem]
    for n in range(2, 8):
        ref = [cases.copy_state(st) for st in sts]
        out = bs.step(prm(n, X.PREC_MIXED), sts)
        for m, (o, r) in enumerate(zip(orcs, ref)):
            o.step(X.make_params(mem[m].params, n=n, tn=mem[m].tn(n) * 10.0), r)
            assert out[m].status == X.OK
            assert cases.state_err(sts[m], r, mem[m].la) <= 1e-6
    bs.close()
    # the same workload in a new context: replayed, not measured
    bs2 = X.BatchSolver([m.grid for m in mem])
    sch2, ms2 = bs2.autotune(X.PREC_MIXED, table)
    assert sch2 == sch and ms2 == 0.0
    assert table.read_text().count("\n") == 1
    bs2.close()


def test_fp64_results_do_not_depend_on_the_schedule(tmp_path):
    scn = cases.build("tidal_flat_99")[0]
    out = []
    for tune in (False, True):
        sol = X.Solver(scn.grid)
        st = scn.copy_state()
        for n in range(1, 13):
            sol.step(X.make_params(scn.params, n=n, tn=scn.tn(n) * 60.0), st)
            if tune and n == 1:
                sol.autotune(X.PREC_FP64, tmp_path / "t.txt", measure=True)
        sol.close()
        out.append(st)
    for k in ("p", "hp", "uhdye", "lmaskdry"):
        np.testing.assert_array_equal(out[0][k], out[1][k], err_msg=k)
