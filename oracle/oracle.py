"""TEST INFRASTRUCTURE ONLY: ctypes loader for the CPU oracle (liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker.  The oracle is an FP64 C++ restatement of EFDC+'s
CALPUV2C/CONGRAD; parity with the reference is unpinned (see efdc_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import subprocess
import sys
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
REPO = ORACLE_DIR.parent
sys.path.insert(0, str(REPO / "efdcplus8.5_b200"))
import efdc_xm as X  # noqa: E402

LIB = ORACLE_DIR / "liboracle.so"
_lib = None


def build(force: bool = False):
    if force or not LIB.exists() or LIB.stat().st_mtime < max(
            (ORACLE_DIR / f).stat().st_mtime for f in ("efdc_oracle.cpp", "efdc_oracle.h")):
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        lib.oracle_create.restype = C.c_void_p
        lib.oracle_create.argtypes = [C.POINTER(X.Grid), C.c_int, C.c_int]
        lib.oracle_destroy.argtypes = [C.c_void_p]
        lib.oracle_noptimal.restype = C.c_int
        lib.oracle_noptimal.argtypes = [C.c_void_p]
        lib.oracle_step.restype = C.c_int
        lib.oracle_step.argtypes = [C.c_void_p, C.POINTER(X.Params), C.POINTER(X.Fields),
                                    C.POINTER(X.Stats)]
        pd = C.POINTER(C.c_double)
        lib.oracle_set_layers.restype = C.c_int
        lib.oracle_set_layers.argtypes = [C.c_void_p, C.POINTER(X.Layers)]
        lib.oracle_set_channels.restype = C.c_int
        lib.oracle_set_channels.argtypes = [C.c_void_p, C.POINTER(X.Channels)]
        lib.oracle_set_bed.restype = C.c_int
        lib.oracle_set_bed.argtypes = [C.c_void_p, C.POINTER(X.Bed)]
        lib.oracle_bottom_stress.restype = C.c_int
        lib.oracle_bottom_stress.argtypes = [C.c_void_p, C.POINTER(X.DragParams),
                                             C.POINTER(X.Fields), C.POINTER(X.DragFields)]
        lib.oracle_set_momentum.restype = C.c_int
        lib.oracle_set_momentum.argtypes = [C.c_void_p, C.POINTER(X.Momentum)]
        lib.oracle_explicit.restype = C.c_int
        lib.oracle_explicit.argtypes = [C.c_void_p, C.POINTER(X.ExplicitParams),
                                        C.POINTER(X.ExplicitFields)]
        lib.oracle_congrad.restype = C.c_int
        lib.oracle_congrad.argtypes = [C.c_void_p] + [pd] * 8 + [
            C.c_double, C.c_int, C.POINTER(C.c_int), pd]
        _lib = lib
    return _lib


class Oracle:
    """CPU FP64 restatement of CALPUV2C for one basin."""

    def __init__(self, grid: dict, nthreads: int = 1, noptimal_cap: int = 8):
        self.lib = load()
        self._grid, self._keep = X.make_grid(grid)
        self.ctx = self.lib.oracle_create(C.byref(self._grid), nthreads, noptimal_cap)
        if not self.ctx:
            raise RuntimeError("oracle_create failed")
        self.noptimal = self.lib.oracle_noptimal(self.ctx)

    def close(self):
        if self.ctx:
            self.lib.oracle_destroy(self.ctx)
            self.ctx = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def step(self, params: X.Params, state: dict, *, diag=False, lists=False) -> X.Stats:
        f, _k = X.make_fields(state, diag=diag, lists=lists)
        st = X.Stats()
        self.lib.oracle_step(self.ctx, C.byref(params), C.byref(f), C.byref(st))
        return st

    def set_layers(self, ly: dict):
        s, _keep = X.make_layers(ly)
        if self.lib.oracle_set_layers(self.ctx, C.byref(s)) != 0:
            raise RuntimeError("oracle_set_layers: bad layer arrays")

    def set_channels(self, ch: dict | None):
        s, _keep = X.make_channels(ch)
        rc = self.lib.oracle_set_channels(self.ctx, C.byref(s))
        if rc != 0:
            raise RuntimeError("oracle_set_channels: bad channel arrays")

    def set_bed(self, bed: dict):
        s, _keep = X.make_bed(bed)
        if self.lib.oracle_set_bed(self.ctx, C.byref(s)) != 0:
            raise RuntimeError("oracle_set_bed: bad bed arrays")

    def bottom_stress(self, params: X.DragParams, state: dict, drag: dict) -> int:
        """CALTBXY + TBX/TBY on the state the last step left; TBX, TBY of `drag`
        in/out."""
        f, _k = X.make_fields(state)
        d = X.make_drag_fields(drag)
        return self.lib.oracle_bottom_stress(self.ctx, C.byref(params), C.byref(f), C.byref(d))

    def set_momentum(self, mo: dict):
        s, _keep = X.make_momentum(mo)
        if self.lib.oracle_set_momentum(self.ctx, C.byref(s)) != 0:
            raise RuntimeError("oracle_set_momentum: bad momentum arrays")

    def explicit(self, params: X.ExplicitParams, fields: dict) -> int:
        """CALEXP2T's external-mode terms; FCAXE, FCAYE, FXE, FYE of `fields`
        in/out, the layer outputs present written."""
        f, _k = X.make_explicit_fields(fields)
        return self.lib.oracle_explicit(self.ctx, C.byref(params), C.byref(f))

    def congrad(self, ccc, ccs, ccn, ccw, cce, ccci, fptmp, p, rsqm, iterm):
        it = C.c_int(0)
        rsq = C.c_double(0.0)
        dp = X._dp
        rc = self.lib.oracle_congrad(self.ctx, dp(ccc), dp(ccs), dp(ccn), dp(ccw), dp(cce),
                                     dp(ccci), dp(fptmp), dp(p), float(rsqm), int(iterm),
                                     C.byref(it), C.byref(rsq))
        return rc, it.value, rsq.value


def run(scn, steps: int, *, nthreads: int = 1, state=None, precision=X.PREC_FP64,
        n0: int = 1, diag=False, lists=False, record=None, tn_mul: float = 1.0):
    """Run `steps` CALPUV2C calls of a scenario on the oracle.  Returns
    (state, list of stats dicts)."""
    o = Oracle(scn.grid, nthreads=nthreads)
    st = state if state is not None else scn.copy_state()
    out = []
    for k in range(steps):
        n = n0 + k
        prm = X.make_params(scn.params, n=n, tn=scn.tn(n) * tn_mul, precision=precision)
        s = o.step(prm, st, diag=diag, lists=lists)
        out.append(s.as_dict())
        if record is not None:
            record(k, st, s)
    o.close()
    return st, out
