"""efdc_xm_congrad_noalloc: the CONGRAD entry point that allocates nothing.

It exists for callers that cannot let the library allocate GPU memory (a host
code that budgets all device memory through its own pool, a time-critical loop
where an allocation could stall or fail, or a caller that already keeps its
data in device arrays it manages).  The caller passes device arrays; the
solver's vectors live in a fixed array of device memory inside the library.
This test hands it device arrays it allocated itself (with torch) and checks
two calls in a row against the context-based efdc_xm_congrad, with the
tolerances of the other FP64 tests (same iteration count to within one, and
surface elevation within 1e-9 m).  The file is named so that pytest collects
it last.
"""
import ctypes as C

import numpy as np
import pytest

import cases
import efdc_xm as X
import oracle as O
import scenario as S

pytestmark = pytest.mark.gpu


# LA-1 of the two large cases: exactly the fixed scratch's limit (a 1024 x 512
# all-water basin, the last padded element of the scratch in use), and a basin
# above 296 CTAs x 256 threads = 75,776 cells, so that every thread of the
# fixed grid loops over several cells
LIMIT = 524288


def _build(name):
    if name == "at_limit_1024x512":
        return S.make_scenario(1024, 512, seed=41, land_frac=0.0, obc_sides=("W",), amp=0.5,
                               dt=10.0), 1.0
    if name == "multi_cell_320x300":
        return S.make_scenario(320, 300, seed=41, land_frac=0.05, obc_sides=("W",), amp=0.5,
                               dt=10.0), 1.0
    scn, _, tm = cases.build(name)
    return scn, tm


def _system(name):
    scn, tm = _build(name)
    st = scn.copy_state()
    p_in = st["p"].copy()
    orc = O.Oracle(scn.grid)
    orc.step(X.make_params(scn.params, n=1, tn=scn.tn(1) * tm), st, diag=True)
    orc.close()
    ccci = np.zeros_like(st["ccc"])
    ccci[1:scn.la] = 1.0 / st["ccc"][1:scn.la]
    return scn, st, ccci, p_in


@pytest.mark.parametrize("name", ["noise_forcing", "basin_fp64", "multi_cell_320x300",
                                  "at_limit_1024x512"])
def test_noalloc_matches_context_congrad_twice(name):
    import torch
    lib = X.load()
    scn, st, ccci, p_in = _system(name)
    if name == "at_limit_1024x512":
        assert scn.la - 1 == LIMIT
    if name == "multi_cell_320x300":
        assert scn.la - 1 > 296 * 256
    # the existing entry point
    sol = X.Solver(scn.grid)
    p_ref = p_in.copy()
    rc, it_ref, _ = sol.congrad(st["ccc"], st["ccs"], st["ccn"], st["ccw"], st["cce"], ccci,
                                st["fptmp"], p_ref, scn.params["rsqm"], scn.params["iterm"])
    sol.close()
    assert rc == X.OK
    dev = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.ascontiguousarray(scn.grid[k], dtype=np.int32)).to(dev)
         for k in ("lnc", "lsc", "lec", "lwc")}
    for k in ("ccc", "ccs", "ccn", "ccw", "cce", "fptmp"):
        t[k] = torch.from_numpy(st[k]).to(dev)
    for call in range(2):
        p = torch.from_numpy(p_in.copy()).to(dev)
        its = C.c_int32(-1)
        rsq = C.c_double(-1.0)
        torch.cuda.synchronize()
        rc = lib.efdc_xm_congrad_noalloc(
            scn.la, *(t[k].data_ptr() for k in ("lnc", "lsc", "lec", "lwc")),
            *(t[k].data_ptr() for k in ("ccc", "ccs", "ccn", "ccw", "cce", "fptmp")),
            p.data_ptr(), scn.params["rsqm"], scn.params["iterm"], None, C.byref(its), C.byref(rsq))
        assert rc == X.OK, lib.efdc_xm_last_error().decode()
        out = p.cpu().numpy()
        assert abs(its.value - it_ref) <= 1, (call, its.value, it_ref)
        assert rsq.value <= scn.params["rsqm"]
        assert np.abs(out - p_ref)[1:scn.la].max() / S.G < 1e-9, call
        assert out[0] == p_in[0] and out[scn.lc - 1] == p_in[scn.lc - 1]


def test_noalloc_rejects_oversize():
    lib = X.load()
    big = LIMIT + 2  # LA-1 one past the fixed scratch
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.efdc_xm_congrad_noalloc(big, *([dummy] * 11), 1e-10, 10, None, None, None)
    assert rc == X.BAD_ARGUMENT
    assert "exceeds the fixed scratch" in lib.efdc_xm_last_error().decode()
