#!/usr/bin/env python
"""External-mode throughput on one B200: cell-iterations per second.

Headline workload (default, ``--workload ensemble``): a batched ensemble of
256 independent basins with wet-cell counts drawn log-uniformly from 10k to
400k (26.3M cells in total), each with its own seeded bathymetry (1-40 m),
Manning n (0.015-0.04) and M2 amplitude (0.1-1.0 m), dt=10 s, RSQM=1e-10.
Synthetic and seeded.  A "step" is one CALPUV2C call for every member
(assembly, open boundaries, scaling, PCG, back-substitution, continuity,
finalisation), all members in one launch sequence.

* value: the batched MIXED solver (FP32 inner PCG, FP64 refinement and dot
  products), state resident in HBM.  cell-iterations = wet cells x CG
  iterations of the FP64 solve of the same step and member (the batched FP64
  run over the same steps gives the credit; it is bit-identical to the
  single-basin drop-in), so extra inner iterations of the mixed solver earn
  nothing.
* fp64_dropin_value: the plain FP64 drop-in, efdc_xm_step_device once per
  member per step (one context per basin, as a host that calls CALPUV2C per
  basin would run it).
* fp64_batched_value: FP64, all members in one context.
* e2e: the same metric through efdc_xm_step_batch with pinned host arrays:
  every step uploads every member's fields and downloads the outputs.
* roofline: the dominant kernel (FP32 CG matrix-vector kernel over all
  members) timed live with CUDA events on the library's stream, against
  MEASURED_PEAKS.json.
* cpu_baseline: the FP64 C++ restatement of the reference (OpenMP, NOPTIMAL
  range split, serial dot products) on a bounded sample of members.
* single_domain: the same three figures on the 2048x2048 curvilinear basin
  (3.4M cells, dt=5 s); ``--workload basin`` makes it the headline.

--impl reference times that CPU restatement alone (the reference itself is
Intel Fortran and cannot be built here).  With --gpus N>1 the ensemble has
N x 256 members, partitioned over the ranks by wet cells (ensemble.partition;
the members shard with no exchange), and value is the sum over ranks divided
by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "efdcplus8.5_b200"))

import efdc_xm as X  # noqa: E402
import ensemble as E  # noqa: E402
import scenario as S  # noqa: E402

METRIC = "external-mode cell-iter/s on 1 B200: mixed/batched vs plain FP64 at 1e-6 m err"
UNIT = "cell-iter/s"
# Algorithmic bytes per water cell of the MIXED inner iteration's two kernels
# (FP32, 4 B per value): the matvec reads z (r for Jacobi members), p_old, AS,
# AW and x and writes p_new, Ap and x (the previous iteration's x += alpha*p
# rides on it); the update reads r, Ap and writes r (Jacobi), plus AS, AW in
# and z out for a polynomial member.
MV_B, UP_B, UP_POLY_B = 32.0, 12.0, 12.0
# and of the FP64 drop-in's matrix-vector kernel: reads z, CCC, p_old, CCS, CCW
# and P, writes p_new, Ap and P (the previous iteration's P += alpha*p)
FP64_MV_B = 72.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=("ensemble", "basin"), default="ensemble")
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--size", type=int, default=2048, help="basin workload: grid size")
    ap.add_argument("--dropin-steps", type=int, default=10)
    ap.add_argument("--basin-steps", type=int, default=50,
                    help="single-domain side measurement (0: skip)")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--wetdry-members", type=int, default=64)
    ap.add_argument("--wetdry-steps", type=int, default=20,
                    help="wetting/drying batch side measurement, 1024x1024 flats (0: skip)")
    ap.add_argument("--tl3-calls", type=int, default=40,
                    help="three-time-level (CALPUV9C) side measurement on the ensemble: timed "
                         "calls of the leapfrog/correction schedule (0: skip)")
    ap.add_argument("--small-steps", type=int, default=200,
                    help="small-basin latency side measurement: steps per model (0: skip)")
    ap.add_argument("--calib-steps", type=int, default=200,
                    help="adjoint calibration side measurement, 512x512 basin (0: skip)")
    ap.add_argument("--explicit-calls", type=int, default=20,
                    help="explicit momentum producer side measurement on the ensemble: timed "
                         "calls (0: skip)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="CPU baseline: seconds per thread setting (two settings)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--host-loops", action="store_true",
                    help="drive the CG, refinement and wet/dry loops from the host "
                         "(EFDC_XM_OPT_DEVICE_LOOPS 0): the same kernels, each launch visible to "
                         "a kernel profiler (kernels inside graphs with conditional nodes are not)")
    ap.add_argument("--profile-prec", choices=("mixed", "fp64", "both"), default="mixed",
                    help="which timed steps of the headline workload are the profiler range "
                         "(ncu --profile-from-start off)")
    ap.add_argument("--variant", type=int, default=-1,
                    help="MIXED inner-iteration kernel variant (EFDC_XM_OPT_KERNEL_VARIANT); "
                         "-1: the schedule efdc_xm_autotune measures for the workload")
    ap.add_argument("--ref-seconds", type=float, default=240.0,
                    help="--impl reference: stop the timed steps after this many seconds")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ensemble(members, seed, pick=None):
    """The seeded ensemble, or the members `pick` of it (threaded: numpy
    releases the GIL)."""
    sizes = S.config3_sizes(seed=seed, members=members)
    ks = range(members) if pick is None else pick
    with ThreadPoolExecutor(os.cpu_count() or 4) as ex:
        return list(ex.map(lambda k: S.config3_member(k, int(sizes[k]), seed=seed), ks))


def ensemble_config(scns, seed):
    cells = [s.ncell for s in scns]
    return {"workload": f"batched ensemble of {len(scns)} basins, wet cells log-uniform "
                        f"10k-400k, depth 1-40 m, Manning 0.015-0.04, M2 0.1-1.0 m, dt=10 s, "
                        f"RSQM=1e-10, FP64-iteration credit",
            "members": len(scns), "cells": int(sum(cells)), "min_cells": int(min(cells)),
            "max_cells": int(max(cells)), "seed": seed,
            "l2": "inputs larger than L2 (all members resident, >10 GB)"}


def basin_config(scn, size):
    return {"workload": f"single-domain basin {size}x{size} curvilinear, west M2 boundary "
                        f"0.2-1.5 m, dt=5 s, RSQM=1e-10, FP64-iteration credit",
            "cells": int(scn.ncell), "grid": f"{size}x{size}",
            "l2": "flushed between timed steps (256 MiB write); working set > L2"}


# ------------------------------------------------------------------ clocks
class Clocks:
    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------- CPU runs
def cpu_run(scns, seconds, max_steps, warmup=0, threads=None, cap=None):
    """The oracle port (FP64, OpenMP): steps of the given basins, all basins
    per step, until `seconds` or `max_steps`.  threads defaults to all host
    threads; cap is the NOPTIMAL thread cap (the reference's is 8)."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    cores = threads or os.cpu_count() or 1
    orcs = [O.Oracle(s.grid, nthreads=cores, noptimal_cap=cap or cores) for s in scns]
    sts = [s.copy_state() for s in scns]
    n = 0
    for _ in range(warmup):
        n += 1
        for s, o, st in zip(scns, orcs, sts):
            o.step(X.make_params(s.params, n=n, tn=s.tn(n)), st)
    cell_iters = 0
    t0 = time.perf_counter()
    k = 0
    while k < max_steps:
        n += 1
        for s, o, st in zip(scns, orcs, sts):
            r = o.step(X.make_params(s.params, n=n, tn=s.tn(n)), st)
            cell_iters += s.ncell * r.iters_total
        k += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    nopt = orcs[0].noptimal
    for o in orcs:
        o.close()
    return cell_iters / dt, k, dt, nopt


def cpu_sample(scns):
    """A bounded, size-spread sample of the ensemble for the CPU port: every
    32nd member in size order (8 of 256)."""
    order = sorted(range(len(scns)), key=lambda k: scns[k].ncell)
    pick = order[::max(1, len(order) // 8)][:8]
    return [scns[k] for k in pick]


def volume_residual(scn, before, after):
    """|dV - (boundary inflow + sources - wasted volume)| / V over the
    non-boundary cells for one step (calpuv2c.f90:466-486 summed: interior
    faces cancel; the faces next to open-boundary cells carry the inflow)."""
    g = scn.grid
    la = scn.la
    bc = np.zeros(scn.lc + 1, bool)
    for s_ in ("W", "E", "S", "N"):
        bc[np.asarray(g["obc"][s_]["l"], dtype=np.int64) - 1] = True
    ii = np.arange(1, la)
    ii = ii[~bc[ii]]
    dxyp = g["dxyp"]
    v0 = float(np.sum(dxyp[ii] * before["hp"][ii]))
    v1 = float(np.sum(dxyp[ii] * after["hp"][ii]))
    d2 = 0.5 * float(scn.params["dt"])
    flow = 0.0
    for s_, key, nbk, sign in (("W", "uhdye", "lec", 1.0), ("E", "uhdye", None, -1.0),
                               ("S", "vhdxe", "lnc", 1.0), ("N", "vhdxe", None, -1.0)):
        for L in np.asarray(g["obc"][s_]["l"], dtype=np.int64):
            f = (g[nbk][L - 1] - 1) if nbk else (L - 1)  # the face between the cell and its target
            flow += sign * d2 * (after[key][f] + before[key][f])
    src = 2.0 * d2 * float(np.sum(after["qsume"][ii]))
    waste = float(np.sum(after["vdwaste"][ii]) - np.sum(before["vdwaste"][ii]))
    return abs((v1 - v0) - (flow + src - waste)) / v0


def wetdry(args, torch, dev, rank):
    """Config-5 style batch: tidal flats (1024x1024, bed ramp -2..15 m +
    N(0, 0.3 m), 2 m M2, ISDRY=99, NDRYSTP=-10), FP64 and MIXED batched
    runs, the MIXED masks checked against FP64 from the same inputs and the
    volume budget, on the first two members."""
    from concurrent.futures import ThreadPoolExecutor as TPE
    K = args.wetdry_steps
    with TPE(os.cpu_count() or 4) as ex:
        scns = list(ex.map(lambda k: S.tidal_flat(n=1024, seed=5 + 97 * k + 1000 * rank),
                           range(args.wetdry_members)))
    cells = np.array([sc.ncell for sc in scns], dtype=np.int64)
    bs = X.BatchSolver([sc.grid for sc in scns], device=dev.index)
    stream = torch.cuda.ExternalStream(bs.stream(), device=dev)
    tmul = 60.0  # a tidal phase in which the flat wets and dries within the run

    def prm(n, prec):
        return [X.make_params(sc.params, n=n, tn=sc.tn(n) * tmul, precision=prec) for sc in scns]

    def run(prec):
        bs.upload([sc.state for sc in scns])
        bs.step_device(prm(1, prec))
        its = np.zeros(len(scns), np.int64)
        sweeps = 0
        t = 0.0
        for n in range(2, K + 2):
            with Timer(torch, stream) as tm:
                sts = bs.step_device(prm(n, prec))
            t += tm.ms / 1e3
            for m, st in enumerate(sts):
                assert st.status in (X.OK, X.NEG_DEPTH), (m, st.as_dict())
            its += np.array([st.iters_total for st in sts])
            sweeps += sum(st.solves for st in sts)
        out = [{"lmaskdry": np.zeros(sc.lc + 1, np.int32), "sub": np.zeros(sc.lc + 1),
                "svb": np.zeros(sc.lc + 1)} for sc in scns]
        bs.download(out)
        return t, its, sweeps, out

    t64, it64, sw64, m64 = run(X.PREC_FP64)
    if args.variant < 0:  # the MIXED schedule for this batch, as for the ensemble
        bs.upload([sc.state for sc in scns])
        bs.step_device(prm(1, X.PREC_MIXED))
        with tempfile.TemporaryDirectory() as td:
            bs.autotune(X.PREC_MIXED, Path(td) / "schedules.txt", measure=True)
    else:
        bs.set_option(X.OPT_KERNEL_VARIANT, args.variant)
    tmx, _itmx, swmx, mmx = run(X.PREC_MIXED)
    credit = float((cells * it64).sum())
    free_diff = sum(int(np.sum(a[k][1:sc.la] != b[k][1:sc.la])) for a, b, sc in
                    zip(m64, mmx, scns) for k in ("lmaskdry", "sub", "svb"))
    bs.close()
    # same-input check, member by member, and the volume budget
    step_diff, vres, toggled = 0, 0.0, 0
    for sc in scns[:2]:
        s64, smx = X.Solver(sc.grid, device=dev.index), X.Solver(sc.grid, device=dev.index)
        st = sc.copy_state()
        wet0 = st["lmaskdry"][1:sc.la].copy()
        for n in range(1, K + 2):
            a, b = {k: (v.copy() if isinstance(v, np.ndarray) else
                        {q: w.copy() for q, w in v.items()} if isinstance(v, dict) else v)
                    for k, v in st.items()}, None
            b = {k: (v.copy() if isinstance(v, np.ndarray) else
                     {q: w.copy() for q, w in v.items()} if isinstance(v, dict) else v)
                 for k, v in st.items()}
            p = X.make_params(sc.params, n=n, tn=sc.tn(n) * tmul)
            s64.step(p, a)
            pm = X.make_params(sc.params, n=n, tn=sc.tn(n) * tmul, precision=X.PREC_MIXED)
            smx.step(pm, b)
            for k in ("lmaskdry", "sub", "svb", "iscdry"):
                step_diff += int(np.sum(a[k][1:sc.la] != b[k][1:sc.la]))
            vres = max(vres, volume_residual(sc, st, b))
            st = a
        toggled += int(np.sum(st["lmaskdry"][1:sc.la] != wet0))
        s64.close()
        smx.close()
    return {"config": {"workload": f"{len(scns)} wetting/drying tidal flats 1024x1024 (bed ramp "
                                   f"-2..15 m + N(0, 0.3 m), 2 m M2, ISDRY=99, NDRYSTP=-10), "
                                   f"{K} timed steps after 1, batched",
                       "members": len(scns), "cells": int(cells.sum())},
            "value": credit / tmx, "fp64_value": credit / t64, "speedup_vs_fp64": t64 / tmx,
            "ms_per_step": 1000 * tmx / K, "fp64_ms_per_step": 1000 * t64 / K,
            "solves_per_member_step": sw64 / (K * len(scns)),
            "mask_diff_cells_free_run": free_diff,
            "mask_diff_cells_same_input_2_members": step_diff,
            "cells_toggled_2_members": toggled,
            "volume_residual_max_2_members": vres}


def small_basins(args, torch, dev):
    """Per-step latency of the FP64 drop-in on small real-size models: the
    100x60 basin of the CPU-runnable configuration (~5,600 cells) and the
    reference's three sample-model grids (tests/golden/sample_*.npz: 355 to
    1,183 cells, their own RSQM and ISDRY), as a host that calls CALPUV2C once
    per time step sees it -- device-resident (efdc_xm_step_device) and on host
    arrays (efdc_xm_step) -- beside the CPU restatement on 1 thread and at
    the reference's thread cap NOPTIMAL = MIN(NTHREADS, 8, MAX(LA/100, 1))."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    gold = REPO / "tests" / "golden"
    models = [("config1_100x60", S.config1(), 1.0)]
    for name, kw in (("Lake_T_HYD_WQ", dict(wind=(2e-4, 1e-4))),
                     ("Lake_Washington", dict(wind=(1e-4, 2e-4))), ("Ohio_River_4", {})):
        f = gold / f"sample_{name}.npz"
        if f.exists():
            models.append((name, S.sample_model(dict(np.load(f)), **kw), 1.0))
    K = args.small_steps
    out = {}
    for name, scn, tm in models:
        prm = [X.make_params(scn.params, n=n, tn=scn.tn(n) * tm) for n in range(1, K + 4)]
        sol = X.Solver(scn.grid, device=dev.index)
        sol.upload(scn.copy_state())
        for k in range(3):
            sol.step_device(prm[k])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        its = 0
        for k in range(3, K + 3):
            its += sol.step_device(prm[k]).iters_total
        t_dev = (time.perf_counter() - t0) / K
        st = scn.copy_state()
        for k in range(3):
            sol.step(prm[k], st)
        t0 = time.perf_counter()
        for k in range(3, K + 3):
            sol.step(prm[k], st)
        t_host = (time.perf_counter() - t0) / K
        sol.close()
        cpu = {}
        for label, nt in (("1_thread", 1), ("noptimal", min(os.cpu_count() or 1, 8))):
            o = O.Oracle(scn.grid, nthreads=nt, noptimal_cap=8)
            so = scn.copy_state()
            for k in range(3):
                o.step(prm[k], so)
            t0 = time.perf_counter()
            for k in range(3, K + 3):
                o.step(prm[k], so)
            cpu[label] = {"ms_per_step": 1000 * (time.perf_counter() - t0) / K,
                          "threads": o.noptimal}
            o.close()
        out[name] = {"cells": int(scn.ncell), "steps": K, "cg_iters_per_step": its / K,
                     "gpu_device_resident_ms_per_step": 1000 * t_dev,
                     "gpu_host_arrays_ms_per_step": 1000 * t_host, "cpu": cpu,
                     "how": "wall clock per step over the timed steps after 3 warm-up "
                            "steps; one host wait per GPU step"}
    return out


def explicit_producer(args, torch, dev, bs, scns, peak):
    """CALEXP2T's external-mode terms (efdc_xm_explicit_batch) on the headline
    ensemble with one layer: a first call takes the layer velocities and
    transports from host arrays; the timed calls reuse them on the device
    (inputs NULL) and keep the sums there, timed with CUDA events on the
    library's stream.  Algorithmic bytes per cell: every input read once (U, V,
    UHDY, VHDX, HP; FCORC, DYDI, DXDJ, DXYP, SCAX, SCAY, SGZU, SGZV, FSGZU,
    FSGZV as FP64, the NW and SE slots as int32) and every output written once
    (FCAXE, FCAYE, FXE, FYE; FCAX, FCAY, FX, FY, CAC): 120 + 8 + 72 = 200 B."""
    M = len(scns)
    for m, s in enumerate(scns):
        bs.set_momentum(S.add_momentum(s, kc=1, seed=m), m)
    prm = [X.make_explicit_params(1.0, 1, 0) for _ in scns]
    first = []
    for m, s in enumerate(scns):
        f = S.momentum_fields(s, seed=m)
        first.append({k: f[k] for k in ("u", "v", "uhdy", "vhdx", "hp")})
    t0 = time.perf_counter()
    bs.explicit(prm, first)
    t_first = time.perf_counter() - t0
    del first
    stream = torch.cuda.ExternalStream(bs.stream(), device=dev)
    none = [{} for _ in scns]
    for _ in range(3):
        bs.explicit(prm, none)
    torch.cuda.synchronize()
    K = args.explicit_calls
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.profiler.start()  # the timed calls are a profiler range too
    e0.record(stream)
    for _ in range(K):
        bs.explicit(prm, none)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.profiler.stop()
    ms = e0.elapsed_time(e1) / K
    cells = float(sum(s.ncell for s in scns))
    gbs = 200.0 * cells / (ms * 1e-3) / 1e9
    return {"calls": K, "members": M, "cells": int(cells), "layers": 1,
            "ms_per_call": ms, "algorithmic_bytes_per_cell": 200,
            "achieved_gbs": gbs, "frac_of_measured_hbm": gbs / peak,
            "first_call_host_arrays_s": t_first,
            "kernels": "k_mom_flux, k_mom_accel, k_mom_edges, k_mom_sum",
            "how": "device-resident calls (inputs reused, sums kept on the device), CUDA events "
                   "on the library stream around the timed calls; inputs larger than L2"}


def calibration(args, torch):
    """Config-4 adjoint: gradient of a 20-gauge elevation misfit over
    `calib_steps` steps w.r.t. per-cell log Manning n and four boundary
    amplitudes on the 512x512 basin, checked by central differences."""
    from calib import CalibProblem
    import math
    scn, gauges, log_true, a_true = S.config4()
    pb = CalibProblem(scn, gauges, args.calib_steps, every=20, adj_rel_tol=1e-12, rsqm=1e-18)
    pb.obs = pb.forward(log_true, a_true, keep=False)
    log0 = np.full(scn.lc + 1, math.log(0.025))
    a0 = np.full(4, 0.5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss = pb.loss(log0, a0)
    t1 = time.perf_counter()
    dk, da, db, iters = pb.backward()
    t2 = time.perf_counter()
    rng = np.random.default_rng(44)
    h = 1e-4
    v = np.zeros_like(log0)
    v[1:scn.la] = rng.standard_normal(scn.la - 1)
    fd = (pb.loss(log0 + h * v, a0) - pb.loss(log0 - h * v, a0)) / (2 * h)
    an = float((dk * v).sum())
    errs = {"log_n_direction": abs(fd - an) / abs(an)}
    for j in range(4):
        e = np.zeros(4)
        e[j] = 1.0
        fdj = (pb.loss(log0, a0 + h * e) - pb.loss(log0, a0 - h * e)) / (2 * h)
        errs[f"amplitude_{j}"] = abs(fdj - da[j]) / abs(da[j])
    pb.close()
    return {"config": {"workload": "adjoint calibration, 512x512 basin, 20 gauges, per-cell log "
                                   "Manning n ~ N(log 0.025, 0.2) and 4 boundary amplitudes, "
                                   "checkpoints every 20 steps, FP64",
                       "cells": int(scn.ncell), "steps": args.calib_steps},
            "loss": loss, "forward_s": t1 - t0, "gradient_s": t2 - t1,
            "gradient_over_forward": (t2 - t1) / (t1 - t0), "adjoint_cg_iterations": int(iters),
            "fd_h": h, "fd_rel_err": errs, "fd_rel_err_max": max(errs.values()),
            "grad_norm_log_n": float(np.linalg.norm(dk)), "grad_amplitudes": da.tolist()}


def reference_arm(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    # the same workload as the GPU arm: every member (all ranks' members for
    # N > 1, since rank 0 alone stands for the whole job here), the same
    # warm-up and timed steps; the wall-time cap only bounds a long default run
    if args.workload == "ensemble":
        seed = 3
        total = args.members * world
        scns = ensemble(total, seed)
        cfg = ensemble_config(scns, seed)
        cfg["members_all_ranks"] = total
        samp = scns
        what = f"all {len(samp)} members ({sum(s.ncell for s in samp)} cells)"
    else:
        scn = S.config2(n=args.size)
        cfg = basin_config(scn, args.size)
        samp = [scn]
        what = f"the {args.size}x{args.size} basin ({scn.ncell} cells)"
    v, k, dt, nopt = cpu_run(samp, seconds=args.ref_seconds, max_steps=args.steps,
                             warmup=args.warmup)
    sample = (f"{k} CALPUV2C steps of {what} after {args.warmup} warm-up steps, FP64 C++ "
              f"restatement, {nopt} OpenMP threads")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": k, "warmup": args.warmup, "ms_per_step": 1000 * dt / max(k, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": cfg,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nopt, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference is Intel Fortran (IFPORT, Windows NetCDF libs); its CPU path "
                    "is timed through the project's FP64 C++ restatement"}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU runs
def pinned_states(torch, scns):
    """Copies of the members' states in one pinned host allocation, field by
    field: each field's member arrays back to back, as an ensemble driver
    holds one (LCM, members) array per field."""
    keys = [k for k, v in scns[0].state.items() if isinstance(v, np.ndarray)]
    total = sum(s.state[k].nbytes for s in scns for k in keys)
    buf = torch.empty(total, dtype=torch.uint8, pin_memory=True).numpy()
    out = [dict() for _ in scns]
    off = 0
    for k in keys:
        for st, s in zip(out, scns):
            v = s.state[k]
            a = buf[off:off + v.nbytes].view(v.dtype).reshape(v.shape)
            a[...] = v
            st[k] = a
            off += v.nbytes
    for st, s in zip(out, scns):
        st["pser"] = {q: a.copy() for q, a in s.state["pser"].items()}
    return out, buf


class Timer:
    """CUDA events on the solver's stream around one region."""

    def __init__(self, torch, stream):
        self.torch, self.stream = torch, stream

    def __enter__(self):
        self.e0 = self.torch.cuda.Event(enable_timing=True)
        self.e1 = self.torch.cuda.Event(enable_timing=True)
        self.e0.record(self.stream)
        return self

    def __exit__(self, *a):
        self.e1.record(self.stream)
        self.e1.synchronize()
        self.ms = self.e0.elapsed_time(self.e1)


def ours(args):
    import torch
    import torch.distributed as dist
    rank, local, world = dist_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=900))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(*vals):
        return E.max_over_ranks(vals, device=dev)

    def sum_over_ranks(*vals):
        return E.sum_over_ranks(vals, device=dev)

    lib = X.load()
    peak, peak_kind = measured_peaks()
    ck = Clocks(local)

    # ---------------- the headline ensemble (or the basin) ----------------
    if args.workload == "ensemble":
        # N GPUs: an ensemble of N x members, partitioned by wet cells
        seed = 3
        total = args.members * world
        mine = E.partition(S.config3_sizes(seed=seed, members=total), world)[rank]
        scns = ensemble(total, seed, pick=mine)
        cfg = ensemble_config(scns, seed)
        cfg["members_all_ranks"] = total
    else:
        scns = [S.config2(n=args.size)]
        cfg = basin_config(scns[0], args.size)
    cells = np.array([s.ncell for s in scns], dtype=np.int64)
    M = len(scns)
    bs = X.BatchSolver([s.grid for s in scns], device=local)
    if args.variant >= 0:
        bs.set_option(X.OPT_KERNEL_VARIANT, args.variant)
    if args.host_loops:
        bs.set_option(X.OPT_DEVICE_LOOPS, 0)
        cfg["loops"] = "host-driven (EFDC_XM_OPT_DEVICE_LOOPS 0)"
    stream = torch.cuda.ExternalStream(bs.stream(), device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev) if M == 1 else None

    def params(n, prec):
        return [X.make_params(s.params, n=n, tn=s.tn(n), precision=prec) for s in scns]

    def run_batch(prec, steps, warmup):
        bs.upload([s.state for s in scns])
        n = 0
        for _ in range(warmup):
            n += 1
            for st in bs.step_device(params(n, prec)):
                assert st.status in (X.OK, X.NEG_DEPTH), st.as_dict()
        barrier()
        torch.cuda.synchronize()
        l0 = lib.efdc_xm_kernel_launches()
        w0 = X.host_waits()
        times, iters, outer = [], np.zeros(M, np.int64), 0
        per_step_iters = []
        # the timed steps are the profiler range (ncu --profile-from-start off): the
        # MIXED ones by default, see --profile-prec
        prof = args.profile_prec == "both" or \
            (args.profile_prec == "mixed") == (prec == X.PREC_MIXED)
        if prof:
            torch.cuda.profiler.start()
        for _ in range(steps):
            n += 1
            if flush is not None:
                with torch.cuda.stream(stream):
                    flush.zero_()
            prm = params(n, prec)
            with Timer(torch, stream) as tm:
                sts = bs.step_device(prm)
            for m, st in enumerate(sts):
                assert st.status in (X.OK, X.NEG_DEPTH), (m, st.as_dict())
            it = np.array([st.iters_total for st in sts], dtype=np.int64)
            iters += it
            per_step_iters.append(it)
            outer += sum(st.outer_refinements for st in sts)
            times.append(tm.ms)
        torch.cuda.synchronize()
        if prof:
            torch.cuda.profiler.stop()
        barrier()
        launches = lib.efdc_xm_kernel_launches() - l0
        waits = X.host_waits() - w0
        out = [{"p": np.zeros(s.lc)} for s in scns]
        bs.download(out)
        return dict(times=times, iters=iters, per_step=per_step_iters, outer=outer,
                    launches=launches, waits=waits, p=[o["p"] for o in out])

    r64 = run_batch(X.PREC_FP64, args.steps, args.warmup)
    # the MIXED schedule for this workload: measured by efdc_xm_autotune on the
    # system of a first MIXED step (the table is this run's own, not reused)
    tune = None
    if args.variant < 0:
        bs.upload([s.state for s in scns])
        bs.step_device(params(1, X.PREC_MIXED))
        t0 = time.perf_counter()
        with tempfile.TemporaryDirectory() as td:
            sch, sms = bs.autotune(X.PREC_MIXED, Path(td) / "schedules.txt", measure=True)
        tune = {"schedule": sch, "solve_ms": sms, "seconds": time.perf_counter() - t0,
                "key": bs.tune_key(X.PREC_MIXED), "how": "efdc_xm_autotune (coordinate descent "
                "over the options, each candidate the median of 5 timed solves, kept when 2 % "
                "faster than the incumbent)"}
    rmx = run_batch(X.PREC_MIXED, args.steps, args.warmup)

    # elevation error of the MIXED solver against the FP64 solve of the same
    # input: one step from the FP64 run's final state in each precision
    def one_step(prec, state_src, n, rsqm_scale=1.0):
        bs.upload(state_src)
        prm = params(n, prec)
        for pp in prm:
            pp.rsqm *= rsqm_scale
        bs.step_device(prm)
        out = [{"p": np.zeros(s.lc)} for s in scns]
        bs.download(out)
        return [o["p"] for o in out]

    full = [s.copy_state() for s in scns]
    bs.upload([s.state for s in scns])
    n_end = args.warmup + args.steps
    for k in range(n_end):  # FP64 trajectory to the end of the timed run
        bs.step_device(params(k + 1, X.PREC_FP64))
    bs.download(full)
    p64 = one_step(X.PREC_FP64, full, n_end + 1)
    pmx = one_step(X.PREC_MIXED, full, n_end + 1)
    step_err = max(float(np.abs(a[1:s.la] - b[1:s.la]).max()) for a, b, s in
                   zip(pmx, p64, scns)) / S.G
    # the FP64 solver's own sensitivity to its stop: RSQM/10 over the timed run
    bs.upload([s.state for s in scns])
    for k in range(n_end):
        prm = params(k + 1, X.PREC_FP64)
        for pp in prm:
            pp.rsqm *= 0.1
        bs.step_device(prm)
    tight = [{"p": np.zeros(s.lc)} for s in scns]
    bs.download(tight)
    drift64 = max(float(np.abs(a["p"][1:s.la] - b[1:s.la]).max()) for a, b, s in
                  zip(tight, r64["p"], scns)) / S.G
    credit = float((cells * r64["iters"]).sum())
    t_mx, t_64 = max_over_ranks(sum(rmx["times"]) / 1e3, sum(r64["times"]) / 1e3)
    credit_all, = sum_over_ranks(credit)
    value = credit_all / t_mx
    fp64_batched = credit_all / t_64
    eta_err = max(float(np.abs(a[1:s.la] - b[1:s.la]).max()) for a, b, s in
                  zip(rmx["p"], r64["p"], scns)) / S.G
    # dominant kernel, live: on the last (mixed) system of every member, with
    # the variant the timed run used, and every variant for comparison
    variants = {}
    run_variant = tune["schedule"]["kernel_variant"] if tune else args.variant
    for v in (0, 1, 2, 3):
        bs.set_option(X.OPT_KERNEL_VARIANT, v)
        kv = bs.time_kernels(X.PREC_MIXED, reps=20)
        variants[v] = {"ms_matvec": kv.ms_matvec, "ms_update": kv.ms_update,
                       "frac_matvec": MV_B * kv.ncells / (kv.ms_matvec * 1e-3) / 1e9 / peak,
                       "frac_update": (UP_B * kv.ncells + UP_POLY_B * kv.ncells_poly) /
                                      (kv.ms_update * 1e-3) / 1e9 / peak}
    bs.set_option(X.OPT_KERNEL_VARIANT, run_variant)
    kt = bs.time_kernels(X.PREC_MIXED, reps=20)
    kt64 = bs.time_kernels(X.PREC_FP64, reps=20)

    # ---------------- plain FP64 drop-in: one context per basin ----------------
    dropin = None
    if args.dropin_steps > 0 and M > 1:
        sols = [X.Solver(s.grid, device=local) for s in scns]
        for sol, s in zip(sols, scns):
            sol.upload(s.state)
        n = 0
        for _ in range(args.warmup):
            n += 1
            for sol, s in zip(sols, scns):
                sol.step_device(X.make_params(s.params, n=n, tn=s.tn(n)))
        torch.cuda.synchronize()
        barrier()
        s_first = torch.cuda.ExternalStream(sols[0].stream(), device=dev)
        s_last = torch.cuda.ExternalStream(sols[-1].stream(), device=dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        d_credit = 0.0
        mismatch = 0
        e0.record(s_first)
        for k in range(args.dropin_steps):
            n += 1
            for m, (sol, s) in enumerate(zip(sols, scns)):
                st = sol.step_device(X.make_params(s.params, n=n, tn=s.tn(n)))
                d_credit += s.ncell * st.iters_total
                if k < len(r64["per_step"]):
                    mismatch += int(st.iters_total != r64["per_step"][k][m])
        e1.record(s_last)
        e1.synchronize()
        t_d, = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        d_credit_all, = sum_over_ranks(d_credit)
        dropin = {"value": d_credit_all / t_d, "steps": args.dropin_steps,
                  "ms_per_step": 1000 * t_d / args.dropin_steps,
                  "iteration_count_mismatches_vs_batched_fp64": mismatch,
                  "how": "efdc_xm_step_device per member per step, one context per basin, "
                         "state resident, the same steps as the first timed batched steps"}
        for sol in sols:
            sol.close()
        del sols

    # ---------------- e2e through efdc_xm_step_batch with pinned host arrays ----------------
    e2e = None
    if args.e2e_steps > 0:
        pst, _buf = pinned_states(torch, scns)
        # the Fields structs over the pinned arrays, built once as a driver
        # whose arrays stay in place does.  The driver runs the external mode
        # only: between two steps it rewrites its forcing arrays (FCAXE ...
        # QSUME, sent every step) and leaves the state arrays the library
        # returned untouched, which it declares in efdc_xm_fields.unchanged
        kept = ("p", "hp", "hu", "hv", "uhdye", "vhdxe", "sub", "svb", "lopenbcdry")
        prep = bs.prepare(pst, unchanged=X.same_bits(kept))
        # the same warm-up as the device-resident runs, so that timed e2e step
        # k is timed FP64 step k (whose iteration counts are the credit)
        n = 0
        for _ in range(max(1, args.warmup)):
            n += 1
            bs.step_prepared(params(n, X.PREC_MIXED), prep)
        torch.cuda.synchronize()
        barrier()
        tms, cred = [], 0.0
        b0 = X.transfer_bytes()  # the library's count of the arrays it copies
        for k in range(args.e2e_steps):
            n += 1
            prm = params(n, X.PREC_MIXED)
            with Timer(torch, stream) as tm:
                bs.step_prepared(prm, prep)
            tms.append(tm.ms)
            cred += float((cells * r64["per_step"][min(k, len(r64["per_step"]) - 1)]).sum())
        b1 = X.transfer_bytes()
        h2d = (b1[0] - b0[0]) // len(tms)
        d2h = (b1[1] - b0[1]) // len(tms)
        t_e, = max_over_ranks(sum(tms) / 1e3)
        cred_all, = sum_over_ranks(cred)
        e2e = {"value": cred_all / t_e, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": 1000 * t_e / len(tms),
               "steps": len(tms), "host_buffers": "pinned, one (LCM, members) block per field",
               "api": "efdc_xm_step_batch (BatchSolver.step_prepared)",
               "host_model": "external mode only: the forcing arrays (FCAXE, FCAYE, FXE, FYE, "
                             "TSX, TSY, TBX, TBY, QSUME) and the boundary series are sent every "
                             "step; the state arrays (" + ", ".join(k.upper() for k in kept) +
                             ") are declared unchanged since the library's last download",
               "h2d_bytes_per_cell": h2d / float(cells.sum()),
               "d2h_bytes_per_cell": d2h / float(cells.sum())}
        del prep, pst, _buf

    # ---------------- roofline of the dominant kernel ----------------
    # The two FP32 kernels of the inner iteration launch once each per
    # iteration, so the one with the longer launch has the larger share of the
    # step (profiles/launch_list_ensemble256.md has the shares of every kernel).
    # Algorithmic bytes per water cell: MV_B, UP_B, UP_POLY_B, FP64_MV_B at the
    # top of the file.
    tj = {}
    tf = REPO / "profiles" / "traffic.json"
    if tf.exists():
        tj = json.loads(tf.read_text())

    def traffic_of(name):
        t = tj.get(name)
        if t and name not in tj.get("stale_for", []):
            return float(t["dram_bytes_per_cell"]) * kt.ncells
        return None

    def kentry(name, what, ms, nbytes):
        a = nbytes / (ms * 1e-3) / 1e9
        return {"bound": "hbm", "kernel": f"{name} ({what})", "achieved": a, "peak": peak,
                "unit": "GB/s", "frac": a / peak, "peak_kind": peak_kind,
                "traffic": traffic_of(name), "ms_per_launch": ms, "bytes_per_launch": nbytes,
                "cells_per_launch": kt.ncells, "slots_per_launch": kt.nslots}

    up_name = "k_mx_update_poly" if kt.ncells_poly > 0 else "k_mx_update_jac"
    e_mv = kentry("k_mx_matvec", "FP32 p-update + Ahat*p + p.Ap + the previous x += alpha*p, "
                  "all members, + member reduce", kt.ms_matvec, MV_B * kt.ncells)
    e_up = kentry(up_name, "FP32 r update, z = (2I - Ahat) r, r.z, r.r, all members, "
                  "+ member reduce", kt.ms_update, UP_B * kt.ncells + UP_POLY_B * kt.ncells_poly)
    e_up["cells_polynomial"] = kt.ncells_poly
    first, second = (e_up, e_mv) if kt.ms_update >= kt.ms_matvec else (e_mv, e_up)
    roof = dict(first)
    roof["dominant_by"] = ("the larger device time per inner iteration of the two kernels "
                           "that launch once per iteration")
    roof["second_kernel"] = second
    roof["variant"] = run_variant
    roof["variants_measured"] = variants
    roof["fp64_matvec"] = {"ms_per_launch": kt64.ms_matvec,
                           "bytes_per_launch": FP64_MV_B * kt.ncells,
                           "achieved": FP64_MV_B * kt.ncells / (kt64.ms_matvec * 1e-3) / 1e9,
                           "frac": FP64_MV_B * kt.ncells / (kt64.ms_matvec * 1e-3) / 1e9 / peak}
    # ---------------- three time levels (CALPUV9C) on the same ensemble ----------------
    tl3_res = None
    if args.tl3_calls > 0 and args.workload == "ensemble":
        warm3 = 3
        sched = S.three_level_schedule(10 * (args.tl3_calls + warm3), 4)[:warm3 + args.tl3_calls]
        lv = (("p1", "p"), ("h2p", "hp"), ("h1p", "hp"), ("uhdy1e", "uhdye"), ("uhdy2e", "uhdye"),
              ("vhdx1e", "vhdxe"), ("vhdx2e", "vhdxe"), ("h1u", "hu"), ("h1v", "hv"),
              ("tsx1", "tsx"), ("tsy1", "tsy"), ("tbx1", "tbx"), ("tby1", "tby"))

        def run3(prec):
            st3 = []
            for s in scns:  # level n-1 = level n at the start (scenario.add_three_levels)
                d = dict(s.state)
                for dst, src in lv:
                    d[dst] = s.state[src].copy()
                st3.append(d)
            bs.upload(st3)
            del st3
            ms, it = [], np.zeros(M, np.int64)
            for i, (n, istl, nctbc, rold, rnew) in enumerate(sched):
                prm = [X.make_params(S.three_level_params(s.params, istl, nctbc, rold, rnew),
                                     n=n, tn=s.tn(n), precision=prec) for s in scns]
                with Timer(torch, stream) as tm:
                    sts = bs.step_device(prm)
                for st in sts:
                    assert st.status in (X.OK, X.NEG_DEPTH), st.as_dict()
                if i >= warm3:
                    ms.append(tm.ms)
                    it += np.array([st.iters_total for st in sts], dtype=np.int64)
            return ms, it

        ms64, it64_3 = run3(X.PREC_FP64)
        msmx, _ = run3(X.PREC_MIXED)
        t64_3, tmx_3 = max_over_ranks(sum(ms64) / 1e3, sum(msmx) / 1e3)
        c3, = sum_over_ranks(float(np.dot(cells, it64_3)))
        tl3_res = {"calls": args.tl3_calls,
                   "schedule": "HDMT order: ISTL=3 leapfrog over 2*DT, ISTL=2 correction after "
                               "every 4th, NCTBC/ROLD/RNEW as HDMT sets them",
                   "value": c3 / tmx_3, "fp64_value": c3 / t64_3,
                   "ms_per_call": 1000 * tmx_3 / args.tl3_calls,
                   "fp64_ms_per_call": 1000 * t64_3 / args.tl3_calls,
                   "speedup_vs_fp64": t64_3 / tmx_3}
    explicit = None
    if rank == 0 and world == 1 and args.explicit_calls > 0 and args.workload == "ensemble":
        explicit = explicit_producer(args, torch, dev, bs, scns, peak)
    bs.close()
    del bs

    # ---------------- single-domain side measurement ----------------
    single = None
    if args.workload == "ensemble" and args.basin_steps > 0:
        scn = S.config2(n=2048)
        sol = X.Solver(scn.grid, device=local)
        sstream = torch.cuda.ExternalStream(sol.stream(), device=dev)
        fl = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

        def run1(prec):
            sol.upload(scn.state)
            n = 0
            for _ in range(args.warmup):
                n += 1
                sol.step_device(X.make_params(scn.params, n=n, tn=scn.tn(n), precision=prec))
            torch.cuda.synchronize()
            ts, its = [], []
            for _ in range(args.basin_steps):
                n += 1
                with torch.cuda.stream(sstream):
                    fl.zero_()
                with Timer(torch, sstream) as tm:
                    st = sol.step_device(X.make_params(scn.params, n=n, tn=scn.tn(n),
                                                       precision=prec))
                ts.append(tm.ms)
                its.append(st.iters_total)
            return sum(ts) / 1e3, its

        t64b, it64 = run1(X.PREC_FP64)
        # the MIXED schedule for this basin, as for the ensemble
        sched_b = None
        if args.variant < 0:
            sol.upload(scn.state)
            sol.step_device(X.make_params(scn.params, n=1, tn=scn.tn(1), precision=X.PREC_MIXED))
            with tempfile.TemporaryDirectory() as td:
                sched_b, _ms = sol.autotune(X.PREC_MIXED, Path(td) / "schedules.txt",
                                            measure=True)
        elif args.variant >= 0:
            sol.set_option(X.OPT_KERNEL_VARIANT, args.variant)
        tmxb, _ = run1(X.PREC_MIXED)
        kb = sol.time_kernels(X.PREC_MIXED, reps=20)
        t64b, tmxb = max_over_ranks(t64b, tmxb)
        cb, = sum_over_ranks(float(scn.ncell * sum(it64)))
        # the MIXED step's elevation error against the FP64 step from the same
        # state: the FP64 trajectory's state after the timed steps, one more
        # step in each precision
        nb_end = args.warmup + args.basin_steps
        sol.upload(scn.state)
        for n in range(1, nb_end + 1):
            sol.step_device(X.make_params(scn.params, n=n, tn=scn.tn(n)))
        st_end = scn.copy_state()
        sol.download(st_end)
        one = {}
        for prec in (X.PREC_FP64, X.PREC_MIXED):
            sol.upload(st_end)
            sol.step_device(X.make_params(scn.params, n=nb_end + 1, tn=scn.tn(nb_end + 1),
                                          precision=prec))
            o = {"p": np.zeros(scn.lc + 1)}
            sol.download(o)
            one[prec] = o["p"]
        eta_b = float(np.abs(one[X.PREC_MIXED][1:scn.la] - one[X.PREC_FP64][1:scn.la]).max()) / S.G
        single = {"config": basin_config(scn, 2048), "steps": args.basin_steps,
                  "value": cb / tmxb, "fp64_value": cb / t64b, "speedup_vs_fp64": t64b / tmxb,
                  "ms_per_step": 1000 * tmxb / args.basin_steps,
                  "fp64_ms_per_step": 1000 * t64b / args.basin_steps,
                  "eta_err_per_step_mixed_vs_fp64_m": eta_b,
                  "k_mx_matvec_ms": kb.ms_matvec,
                  "k_mx_matvec_frac": MV_B * kb.ncells / (kb.ms_matvec * 1e-3) / 1e9 / peak,
                  "update_ms": kb.ms_update,
                  "update_frac": (UP_B * kb.ncells + UP_POLY_B * kb.ncells_poly) /
                                 (kb.ms_update * 1e-3) / 1e9 / peak,
                  "schedule": sched_b}
        sol.close()
        del fl
    wd_res = None
    if args.wetdry_steps > 0 and args.workload == "ensemble":
        wd_res = wetdry(args, torch, dev, rank)
    calib_res = None
    if rank == 0 and world == 1 and args.calib_steps > 0:
        calib_res = calibration(args, torch)
    small = None
    if rank == 0 and world == 1 and args.small_steps > 0:
        small = small_basins(args, torch, dev)
    clocks = ck.stop()

    # ---------------- CPU baseline (rank 0, N=1) ----------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        samp = cpu_sample(scns) if M > 1 else scns
        v, k, dt, nopt = cpu_run(samp, seconds=args.cpu_seconds, max_steps=2000)
        cpu = {"value": v, "unit": UNIT, "cores": nopt, "kind": "port",
               "sample": f"{k} CALPUV2C steps of {len(samp)} basins "
                         f"({sum(s.ncell for s in samp)} cells), FP64 C++ restatement of "
                         f"CALPUV2C/CONGRAD, {nopt} OpenMP threads, {dt:.1f} s"}
        # the reference's own thread cap, NOPTIMAL = MIN(NTHREADS, 8, LA/100)
        t8 = min(os.cpu_count() or 1, 8)
        v8, k8, dt8, nopt8 = cpu_run(samp, seconds=args.cpu_seconds, max_steps=2000, threads=t8,
                                     cap=8)
        cpu["noptimal_cap_8"] = {"value": v8, "cores": nopt8, "steps": k8,
                                 "seconds": round(dt8, 2)}

    if rank == 0:
        cfg["parallelism"] = (f"{world} GPUs, members partitioned by wet cells (no exchange)"
                              if world > 1 else "single GPU")
        cfg["tiles_32x8"] = kt.nslots // 256
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * t_mx / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner / f64 refinement",
            "data": "synthetic (seeded)", "config": cfg,
            "fp64_batched_value": fp64_batched,
            "fp64_dropin_value": dropin["value"] if dropin else None,
            "speedup_vs_fp64_dropin": value / dropin["value"] if dropin else None,
            "speedup_vs_fp64_batched": value / fp64_batched,
            "fp64_batched_ms_per_step": 1000 * t_64 / args.steps,
            "fp64_dropin": dropin,
            "iters_fp64_total": int(r64["iters"].sum()),
            "iters_mixed_inner_total": int(rmx["iters"].sum()),
            "outer_refinements_per_member_step": rmx["outer"] / (args.steps * M),
            "eta_err_per_step_mixed_vs_fp64_m": step_err,
            "eta_drift_after_run_mixed_vs_fp64_m": eta_err,
            "eta_drift_after_run_fp64_rsqm_div10_vs_fp64_m": drift64,
            "eta_note": "per step: one step from the same FP64 state in each precision "
                        "(the 1e-6 m bar); after run: free-running trajectories, MIXED stops "
                        "at 0.1*RSQM and FP64 at RSQM, so the drift is FP64's own truncation, "
                        "of the size FP64 drifts from itself when RSQM is divided by 10",
            "solves_per_s": world * M * args.steps / t_mx,
            "cell_steps_per_s": world * float(cells.sum()) * args.steps / t_mx,
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(rmx["launches"]), "clocks": clocks,
            "host_waits_per_step": rmx["waits"] / args.steps,
            "schedule": tune,
            "single_domain": single,
            "three_level": tl3_res,
            "wetdry": wd_res,
            "calibration": calib_res,
            "small_basins": small,
            "explicit_producer": explicit,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
