"""The sample-model fixtures (tests/golden/sample_*.npz) on the CPU.

* Where the reference tree is present, make_sample_models.py regenerates
  each fixture from the model's input files identically.
* Each fixture's water-cell count is the model's own LC - 2 (card C9), and
  its flow sources sit on water cells.
* The oracle steps every variant without a failure, and the closed lakes
  keep their volume budget: the change of volume equals the source volume.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

import efdc_xm as X
import oracle as O
import scenario as S

GOLD = Path(__file__).resolve().parent / "golden"
REF = Path("/root/reference")
MODELS = ("Lake_T_HYD_WQ", "Lake_Washington", "Ohio_River_4")


@pytest.mark.skipif(not (REF / "SampleModels").exists(), reason="reference tree not present")
def test_fixtures_regenerate_identically():
    sys.path.insert(0, str(GOLD))
    import make_sample_models as M
    for m in MODELS:
        new = M.make(REF, m)
        old = np.load(GOLD / f"sample_{m}.npz")
        assert sorted(new) == sorted(old.files)
        for k, v in new.items():
            np.testing.assert_array_equal(np.asarray(v), old[k], err_msg=f"{m}:{k}")


@pytest.mark.parametrize("m", MODELS)
def test_fixture_matches_model_cell_count(m):
    f = dict(np.load(GOLD / f"sample_{m}.npz"))
    water = (f["ijct"] == 5)
    assert int(water.sum()) + 2 == int(f["lc_reference"])
    for i, j, _q in f["sources"]:
        assert water[int(j) - 1, int(i) - 1]
    scn = S.sample_model(f)
    assert scn.la - 1 == int(water.sum())
    assert scn.params["rsqm"] == 1e-9 and scn.params["iterm"] == 200


@pytest.mark.parametrize("m,kw", [("Lake_T_HYD_WQ", dict(wind=(2e-4, 1e-4), drawdown=0.6)),
                                  ("Lake_Washington", dict(wind=(1e-4, 2e-4))),
                                  ("Ohio_River_4", dict())])
def test_oracle_steps_sample_models(m, kw):
    scn = S.sample_model(dict(np.load(GOLD / f"sample_{m}.npz")), **kw)
    st = scn.copy_state()
    o = O.Oracle(scn.grid)
    for n in range(1, 101):
        r = o.step(X.make_params(scn.params, n=n, tn=scn.tn(n)), st)
        assert r.status == X.OK, (n, r.as_dict())
        assert r.iters_last <= scn.params["iterm"]
    o.close()
    assert np.isfinite(st["p"][1:scn.la]).all()


def test_closed_lake_volume_budget():
    """Lake_T has no open boundary: after 50 steps its volume has changed by
    DT times the sum of its sources, to 1e-10 relative."""
    scn = S.sample_model(dict(np.load(GOLD / "sample_Lake_T_HYD_WQ.npz")), wind=(2e-4, 1e-4))
    st = scn.copy_state()
    o = O.Oracle(scn.grid)
    la = scn.la
    dxyp = scn.grid["dxyp"][1:la]
    v0 = float(np.sum(dxyp * st["hp"][1:la]))
    src = 0.0
    for n in range(1, 51):
        o.step(X.make_params(scn.params, n=n, tn=scn.tn(n)), st)
        src += scn.params["dt"] * float(np.sum(st["qsume"][1:la]))
    o.close()
    v1 = float(np.sum(dxyp * st["hp"][1:la]))
    assert abs((v1 - v0) - src) / v0 < 1e-10
