"""Kernel variants of the MIXED inner iteration (EFDC_XM_OPT_KERNEL_VARIANT).

Variant 0 fetches each 4-tile unit's descriptors one unit ahead, variant 1 in
batches of 32 units into shared memory, variant 2 also stages the units' rows
in shared memory with bulk copies issued one unit ahead, variant 3 fetches them
as 1 does and issues all of a row's loads before its first dependent operation.  They run the same
arithmetic on the same values, so a batch steps to the same state bit for
bit: Jacobi and polynomial members, an unsymmetric (radiation) member, and
wetting and drying.  The staged variant's kernels also time through
efdc_xm_time_kernels.
"""
import numpy as np
import pytest

import cases
import efdc_xm as X

pytestmark = pytest.mark.gpu

FIELDS = ("p", "hp", "hu", "hv", "uhdye", "vhdxe", "sub", "svb", "lmaskdry")


@pytest.fixture(scope="module", autouse=True)
def _lib():
    X.load()


def run(mem, steps, tm, variant, caps=(0, 0), timed=False):
    bs = X.BatchSolver([m.grid for m in mem])
    bs.set_option(X.OPT_KERNEL_VARIANT, variant)
    bs.set_option(X.OPT_CTAS_MATVEC, caps[0])
    bs.set_option(X.OPT_CTAS_UPDATE, caps[1])
    sts = [m.copy_state() for m in mem]
    stats = []
    for n in range(1, steps + 1):
        r = bs.step([X.make_params(m.params, n=n, tn=m.tn(n) * tm, precision=X.PREC_MIXED)
                     for m in mem], sts)
        stats.append([(x.status, x.iters_total, x.solves, x.outer_refinements) for x in r])
    # (kernel timing iterates past convergence: only on a system far from it)
    kt = bs.time_kernels(X.PREC_MIXED, reps=3) if timed else None
    bs.close()
    return sts, stats, kt


@pytest.mark.parametrize("variant,caps", [(1, (0, 0)), (2, (0, 0)), (2, (2, 2)), (3, (0, 0)),
                                           (3, (2, 2))])
def test_variants_equal_variant0(variant, caps):
    mem = [cases.build(n)[0] for n in ("basin_fp64", "noise_forcing", "radiation_all_sides",
                                       "tidal_flat_99")]
    a = run(mem, 12, 20.0, 0)
    b = run(mem, 12, 20.0, variant, caps)
    assert a[1] == b[1]
    for m in range(len(mem)):
        for k in FIELDS:
            np.testing.assert_array_equal(a[0][m][k], b[0][m][k], err_msg=f"{m}:{k}")


def test_variant2_several_batches_per_cta():
    """Two 2048 x 2048 basins (6.8 M cells, ~6,900 units) with the kernels
    capped at one CTA per SM: each CTA runs about 47 units, i.e. two
    descriptor batches and many refills of each stage."""
    import scenario as S
    mem = [S.config2(seed=2), S.config2(seed=3)]
    a = run(mem, 3, 1.0, 0)
    b = run(mem, 3, 1.0, 2, caps=(1, 1), timed=True)
    assert a[1] == b[1]
    assert b[2].ms_matvec > 0 and b[2].ms_update > 0
    for m in range(len(mem)):
        np.testing.assert_array_equal(a[0][m]["p"], b[0][m]["p"])
