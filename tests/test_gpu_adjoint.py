"""Hand-written adjoint of the external mode (efdc_xm_calib_*) on the GPU.

Bars:
* the calibration forward run matches the FP64 torch reference (exact
  solves) to 1e-9 m at the gauges;
* the adjoint gradients w.r.t. log n, the boundary amplitudes and BELV match
  the reference gradient (torch.autograd through exact solves) to 1e-6
  relative (max norm);
* directional derivatives match central finite differences of the GPU model
  (h = 1e-4) to 1e-5 relative;
* checkpointing changes nothing (bit-identical gradients).
"""
import math

import numpy as np
import pytest
import torch

import adjoint_ref as R
import efdc_xm as X
import scenario as S
from calib import CalibLoss, CalibProblem

pytestmark = pytest.mark.gpu

STEPS = 12


@pytest.fixture(scope="module", autouse=True)
def _lib():
    X.load()


def case(seed=31, nx=40, ny=30):
    scn = S.make_scenario(nx, ny, seed=seed, land_frac=0.05, depth=(2.0, 20.0), obc_sides=("W",),
                          amp=0.5, manning=0.0, dt=10.0, isdry=0, rsqm=1e-22, iterm=800,
                          fill_dead_ends=True)
    rng = np.random.default_rng(seed)
    log_true = np.full(scn.lc + 1, math.log(0.025))
    log_true[1:scn.la] = rng.normal(math.log(0.025), 0.2, scn.la - 1)
    il = scn.grid["il"]
    cand = [L for L in range(2, scn.la + 1) if il[L - 1] > 4]
    gauges = np.sort(rng.choice(cand, size=6, replace=False)).astype(np.int32)
    return scn, gauges, log_true, np.array([0.45, 0.55, 0.5, 0.6])


def make_problem(every=5):
    scn, gauges, log_true, a_true = case()
    pb = CalibProblem(scn, gauges, STEPS, every=every, adj_rel_tol=1e-13)
    pb.obs = pb.forward(log_true, a_true, keep=False)
    log0 = np.full(scn.lc + 1, math.log(0.025))
    a0 = np.full(4, 0.5)
    return pb, scn, gauges, log0, a0


def reference(scn, gauges, log0, a0, obs, pb):
    m = R.RefModel(scn.grid, scn.params, scn.state)
    pcb, psb = pb.harmonics(a0)
    k = torch.tensor(log0, requires_grad=True)
    pc = torch.tensor(pcb, requires_grad=True)
    ps = torch.tensor(psb, requires_grad=True)
    belv = torch.tensor(np.asarray(scn.grid["belv"], dtype=np.float64), requires_grad=True)
    loss, eta = m.loss(k, pc, ps, STEPS, gauges, obs, belv=belv)
    loss.backward()
    da = np.zeros(4)
    np.add.at(da, pb.groups, (pc.grad.numpy() * pb.ucos + ps.grad.numpy() * pb.usin).sum(axis=1))
    return float(loss.detach()), eta, k.grad.numpy(), da, belv.grad.numpy()


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_forward_matches_reference():
    pb, scn, gauges, log0, a0 = make_problem()
    eta = pb.forward(log0, a0)
    _, eta_ref, _, _, _ = reference(scn, gauges, log0, a0, pb.obs, pb)
    assert np.abs(eta - eta_ref).max() < 1e-9
    pb.close()


def test_adjoint_matches_reference_gradient():
    pb, scn, gauges, log0, a0 = make_problem()
    loss = pb.loss(log0, a0)
    dk, da, db, iters = pb.backward()
    lref, _, dk_ref, da_ref, db_ref = reference(scn, gauges, log0, a0, pb.obs, pb)
    assert abs(loss - lref) <= 1e-9 * lref
    la = scn.la
    assert rel(dk[1:la], dk_ref[1:la]) < 1e-6
    assert rel(da, da_ref) < 1e-6
    assert rel(db[1:la], db_ref[1:la]) < 1e-6
    assert iters > 0
    pb.close()


def test_adjoint_matches_central_differences():
    pb, scn, gauges, log0, a0 = make_problem()
    pb.loss(log0, a0)
    dk, da, _, _ = pb.backward()
    rng = np.random.default_rng(9)
    h = 1e-4
    v = np.zeros_like(log0)
    v[1:scn.la] = rng.standard_normal(scn.la - 1)
    fd = (pb.loss(log0 + h * v, a0) - pb.loss(log0 - h * v, a0)) / (2 * h)
    an = float((dk * v).sum())
    assert abs(fd - an) <= 1e-5 * abs(an), (fd, an)
    for j in range(4):
        e = np.zeros(4)
        e[j] = 1.0
        fd = (pb.loss(log0, a0 + h * e) - pb.loss(log0, a0 - h * e)) / (2 * h)
        assert abs(fd - da[j]) <= 1e-5 * abs(da[j]), (j, fd, da[j])
    pb.close()


def test_checkpointing_is_exact():
    grads = []
    for every in (5, STEPS):
        pb, scn, gauges, log0, a0 = make_problem(every=every)
        pb.loss(log0, a0)
        dk, da, db, _ = pb.backward()
        grads.append((dk, da, db))
        pb.close()
    for a, b in zip(grads[0], grads[1]):
        assert np.array_equal(a, b)


def test_autograd_function():
    pb, scn, gauges, log0, a0 = make_problem()
    k = torch.tensor(log0, requires_grad=True)
    a = torch.tensor(a0, requires_grad=True)
    loss = CalibLoss.apply(k, a, pb)
    loss.backward()
    pb.loss(log0, a0)
    dk, da, _, _ = pb.backward()
    assert np.allclose(k.grad.numpy(), dk, rtol=0, atol=0)
    assert np.allclose(a.grad.numpy(), da, rtol=0, atol=0)
    pb.close()


def test_calib_rejects_wet_dry_and_mixed():
    scn, gauges, log_true, a_true = case()
    sol = X.Solver(scn.grid)
    sol.calib_enable(2)
    sol.upload(scn.state)
    prm = X.make_params(scn.params, n=1, tn=scn.tn(1), precision=X.PREC_MIXED)
    with pytest.raises(RuntimeError):
        sol.calib_step(prm)
    sol.close()
