#!/usr/bin/env python
"""External-mode throughput on one B200: cell-iterations per second.

Workload: the single-domain 2048x2048 curvilinear basin (~3.4M wet cells,
DXP/DYP 50-200 m, depth 1-60 m, west tidal boundary 0.2-1.5 m, dt=5 s),
seeded and synthetic.  A "step" is one CALPUV2C call (assembly, open
boundaries, scaling, PCG, back-substitution, continuity, finalisation).

* value: the MIXED solver (FP32 inner PCG, FP64 refinement and dot products),
  state resident in HBM.  cell-iterations = wet cells x CG iterations of the
  FP64 solve of the same step (the FP64 drop-in is run first over the same
  steps; its iteration counts are the credit), so extra inner iterations of
  the mixed solver earn nothing.
* fp64_value: the plain FP64 drop-in on the same steps.
* e2e: the same metric through efdc_xm_step with pinned host arrays: every
  step uploads the caller's fields and downloads the outputs.
* roofline: the dominant kernel (FP32 CG matrix-vector kernel) timed live with
  CUDA events on the library's stream, against MEASURED_PEAKS.json.
* cpu_baseline: the FP64 C++ restatement of the reference (OpenMP, NOPTIMAL
  range split, serial dot products) on a bounded sample of the same workload.

--impl reference times that CPU restatement alone (the reference itself is
Intel Fortran and cannot be built here).  With --gpus N>1 every rank solves its
own replica of the basin (the external mode of one domain does not shard;
members of an ensemble would), and value is the sum over ranks divided by the
slowest rank's time.
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
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "efdcplus8.5_b200"))

import efdc_xm as X  # noqa: E402
import scenario as S  # noqa: E402

METRIC = "external-mode cell-iter/s on 1 B200: mixed/batched vs plain FP64 at 1e-6 m err"
UNIT = "cell-iter/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--size", type=int, default=2048)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def workload_config(scn, size):
    return {"workload": f"single-domain basin {size}x{size} curvilinear, west M2 boundary 0.2-1.5 m, "
                        f"dt=5 s, RSQM=1e-10, FP64-iteration credit",
            "cells": int(scn.ncell), "grid": f"{size}x{size}", "tiles_32x8": None,
            "l2": "flushed between timed steps (256 MiB write); working set > L2",
            "parallelism": "replicas"}


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


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
def cpu_run(scn, seconds, max_steps, warmup=0):
    """The oracle port (FP64, OpenMP over all host threads) on the workload."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    orc = O.Oracle(scn.grid, nthreads=cores, noptimal_cap=cores)
    st = scn.copy_state()
    n = 0
    for _ in range(warmup):
        n += 1
        orc.step(X.make_params(scn.params, n=n, tn=scn.tn(n)), st)
    cell_iters = 0
    t0 = time.perf_counter()
    k = 0
    while k < max_steps:
        n += 1
        s = orc.step(X.make_params(scn.params, n=n, tn=scn.tn(n)), st)
        cell_iters += scn.ncell * s.iters_total
        k += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return cell_iters / dt, k, dt, orc.noptimal


def reference_arm(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    scn = S.config2(n=args.size)
    v, k, dt, nopt = cpu_run(scn, seconds=max(5.0, 6.0 * args.steps), max_steps=args.steps,
                             warmup=min(args.warmup, 1))
    sample = (f"{k} CALPUV2C steps of the {args.size}x{args.size} basin ({scn.ncell} cells) "
              f"after {min(args.warmup, 1)} warm-up, FP64 C++ restatement, {nopt} OpenMP threads")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": k, "warmup": min(args.warmup, 1), "ms_per_step": 1000 * dt / max(k, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": workload_config(scn, args.size),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nopt, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference is Intel Fortran (IFPORT, Windows NetCDF libs); its CPU path "
                    "is timed through the project's FP64 C++ restatement"}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU runs
def transfer_bytes(state, lc, la, isdry):
    """Bytes efdc_xm_step moves per call for a Fortran-shim-like field set:
    uploads LC elements of every input/in-out array, downloads LA-1 elements of
    every output/in-out array (mirrors efdc_xm_upload/efdc_xm_download)."""
    dbl_in = ["p", "hp", "hu", "hv", "uhdye", "vhdxe", "sub", "svb", "sbx", "sby",
              "fcaxe", "fcaye", "fxe", "fye", "tsx", "tsy", "tbx", "tby", "qsume", "qdwaste",
              "vdwaste"]
    int_in = ["lmaskdry", "iscdry", "lopenbcdry", "natdry"]
    dbl_out = ["p", "hp", "h1p", "hu", "hv", "uhdye", "vhdxe", "sub", "svb", "sbx", "sby",
               "uhe", "vhe", "hpi", "hui", "hvi", "qdwaste", "vdwaste"]
    nb = sum(len(v) for v in state["pser"].values())
    h2d = lc * (8 * len(dbl_in) + 4 * len(int_in)) + 8 * nb
    d2h = (la - 1) * (8 * len(dbl_out) + 4 * len(int_in))
    return h2d, d2h


def ours(args):
    import torch
    import torch.distributed as dist
    rank, local, world = dist_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier()

    scn = S.config2(n=args.size)
    sol = X.Solver(scn.grid, device=local)
    stream = torch.cuda.ExternalStream(sol.stream(), device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    lib = sol.lib

    def params(n, prec):
        return X.make_params(scn.params, n=n, tn=scn.tn(n), precision=prec)

    def run(prec, steps, warmup):
        st = scn.copy_state()
        sol.upload(st)
        n = 0
        for _ in range(warmup):
            n += 1
            s = sol.step_device(params(n, prec))
            assert s.status in (X.OK, X.NEG_DEPTH), s.as_dict()
        barrier()
        torch.cuda.synchronize()
        l0 = lib.efdc_xm_kernel_launches()
        times, iters, outer = [], [], []
        for _ in range(steps):
            n += 1
            with torch.cuda.stream(stream):
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s = sol.step_device(params(n, prec))
            e1.record(stream)
            e1.synchronize()
            assert s.status in (X.OK, X.NEG_DEPTH), s.as_dict()
            times.append(e0.elapsed_time(e1))
            iters.append(s.iters_total)
            outer.append(s.outer_refinements)
        torch.cuda.synchronize()
        barrier()
        launches = lib.efdc_xm_kernel_launches() - l0
        out = scn.copy_state()
        sol.download(out)
        return dict(times=times, iters=iters, outer=outer, launches=launches, state=out)

    ck = Clocks(local)
    r64 = run(X.PREC_FP64, args.steps, args.warmup)
    rmx = run(X.PREC_MIXED, args.steps, args.warmup)
    clocks = ck.stop()
    cells = scn.ncell
    credit = cells * sum(r64["iters"])  # FP64 iterations of the same steps
    t_mx = sum(rmx["times"]) / 1000.0
    t_64 = sum(r64["times"]) / 1000.0
    if world > 1:
        tt = torch.tensor([t_mx, t_64], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_mx, t_64 = float(tt[0]), float(tt[1])
    value = world * credit / t_mx
    fp64_value = world * credit / t_64
    eta_err = float(np.abs(rmx["state"]["p"][1:scn.la] - r64["state"]["p"][1:scn.la]).max() / S.G)

    # roofline of the dominant kernel on the last assembled (mixed) system
    kt = sol.time_kernels(X.PREC_MIXED, reps=20)
    kt64 = sol.time_kernels(X.PREC_FP64, reps=20)
    peak, peak_kind = measured_peaks()
    # algorithmic bytes per water cell: the FP32 matvec of the Jacobi-scaled
    # system reads r, p_old, AS, AW and writes p_new, Ap (6 x 4 B); the FP64
    # drop-in's reads r, CCC, p_old, CCS, CCW and writes p_new, Ap (7 x 8 B)
    bytes_mv = 24.0 * kt.ncells
    achieved = bytes_mv / (kt.ms_matvec * 1e-3) / 1e9
    traffic = None
    tf = REPO / "profiles" / "traffic.json"
    if tf.exists():
        tj = json.loads(tf.read_text())
        t = tj.get("k_mx_matvec")
        if t and "k_mx_matvec" not in tj.get("stale_for", []):
            traffic = float(t["dram_bytes_per_cell"]) * kt.ncells
    roof = {"bound": "hbm", "kernel": "k_mx_matvec (FP32 p-update + Ahat*p + p.Ap)",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": peak_kind, "traffic": traffic,
            "ms_per_launch": kt.ms_matvec, "bytes_per_launch": bytes_mv,
            "update_kernel": {"ms_per_launch": kt.ms_update, "bytes_per_launch": 24.0 * kt.ncells,
                              "achieved": 24.0 * kt.ncells / (kt.ms_update * 1e-3) / 1e9},
            "fp64_matvec": {"ms_per_launch": kt64.ms_matvec, "bytes_per_launch": 56.0 * kt.ncells,
                            "achieved": 56.0 * kt.ncells / (kt64.ms_matvec * 1e-3) / 1e9}}

    # e2e: efdc_xm_step with pinned host arrays, mixed precision
    e2e = None
    if args.e2e_steps > 0:
        st = scn.copy_state()
        pinned = {}
        for k, v in st.items():
            if isinstance(v, np.ndarray):
                t = torch.empty(v.shape, dtype=torch.float64 if v.dtype == np.float64 else torch.int32,
                                pin_memory=True)
                a = t.numpy()
                a[...] = v
                pinned[k] = (t, a)
        pst = {k: a for k, (t, a) in pinned.items()}
        pst["pser"] = st["pser"]
        h2d, d2h = transfer_bytes(pst, scn.lc, scn.la, scn.params["isdry"])
        n = 0
        for _ in range(1):
            n += 1
            sol.step(params(n, X.PREC_MIXED), pst)
        torch.cuda.synchronize()
        barrier()
        tms = []
        its = []
        for k in range(args.e2e_steps):
            n += 1
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s = sol.step(params(n, X.PREC_MIXED), pst)
            e1.record(stream)
            e1.synchronize()
            tms.append(e0.elapsed_time(e1))
            its.append(r64["iters"][min(k, len(r64["iters"]) - 1)])
        t_e = sum(tms) / 1000.0
        if world > 1:
            tt = torch.tensor([t_e], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t_e = float(tt[0])
        e2e = {"value": world * cells * sum(its) / t_e, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": 1000 * t_e / len(tms),
               "steps": len(tms), "host_buffers": "pinned (torch pin_memory)"}

    cpu = None
    if rank == 0 and not args.no_cpu:
        v, k, dt, nopt = cpu_run(scn, seconds=args.cpu_seconds, max_steps=50)
        cpu = {"value": v, "unit": UNIT, "cores": nopt, "kind": "port",
               "sample": f"{k} CALPUV2C steps of the same basin ({cells} cells), FP64 C++ "
                         f"restatement of CALPUV2C/CONGRAD, {nopt} OpenMP threads, {dt:.1f} s"}

    if rank == 0:
        cfg = workload_config(scn, args.size)
        cfg["tiles_32x8"] = kt.nslots // 256
        cfg["parallelism"] = f"replicas x{world}" if world > 1 else "single GPU"
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * t_mx / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner / f64 refinement",
            "data": "synthetic (seeded)", "config": cfg,
            "fp64_value": fp64_value, "speedup_vs_fp64": value / fp64_value,
            "fp64_ms_per_step": 1000 * t_64 / args.steps,
            "iters_fp64_total": int(sum(r64["iters"])), "iters_mixed_inner_total": int(sum(rmx["iters"])),
            "outer_refinements_per_step": float(np.mean(rmx["outer"])),
            "max_eta_diff_mixed_vs_fp64_m": eta_err,
            "solves_per_s": world * args.steps / t_mx, "cell_steps_per_s": world * cells * args.steps / t_mx,
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(rmx["launches"]), "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    sol.close()
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
