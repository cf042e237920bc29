"""ctypes mirror of include/efdc_xm.h and a thin host-side wrapper.

This is how Python callers (the tests, bench.py, a calibration harness) reach
the CUDA library ``libefdc_xm.so``; Fortran callers bind the same symbols
through ISO_C_BINDING (see the Fortran shim sources in ``fortran/``).

Array convention: every per-cell array is a contiguous numpy array laid out
like EFDC+'s 1-based Fortran array, element L at index L-1.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libefdc_xm.so"

OK, CG_MAXITER, WETDRY_MAXSWEEP, NEG_DEPTH, NONFINITE, CUDA_ERROR, DEVICE_TIMEOUT, \
    BAD_ARGUMENT, UNSUPPORTED = range(9)
STATUS_NAMES = {0: "OK", 1: "CG_MAXITER", 2: "WETDRY_MAXSWEEP", 3: "NEG_DEPTH",
                4: "NONFINITE", 5: "CUDA_ERROR", 6: "DEVICE_TIMEOUT",
                7: "BAD_ARGUMENT", 8: "UNSUPPORTED"}
PREC_FP64, PREC_MIXED = 0, 1
SIDES = ("W", "E", "S", "N")

_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)


class Obc(C.Structure):
    _fields_ = [("n", C.c_int32), ("l", _pi), ("ispb", _pi), ("pcb", _pd),
                ("psb", _pd), ("ld", C.c_int32)]


class Grid(C.Structure):
    _fields_ = [("la", C.c_int32), ("lc", C.c_int32), ("il", _pi), ("jl", _pi),
                ("lnc", _pi), ("lsc", _pi), ("lec", _pi), ("lwc", _pi),
                ("dxyp", _pd), ("dxyip", _pd), ("dxiu", _pd), ("dyiu", _pd),
                ("dxiv", _pd), ("dyiv", _pd), ("dxyu", _pd), ("dxyv", _pd),
                ("hruo", _pd), ("hrvo", _pd), ("subo", _pd), ("svbo", _pd),
                ("sbxo", _pd), ("sbyo", _pd), ("belv", _pd), ("mtide", C.c_int32),
                ("tcp", _pd), ("obc", Obc * 4)]


class Params(C.Structure):
    _fields_ = [("delt", C.c_double), ("g", C.c_double), ("hdry", C.c_double),
                ("rsqm", C.c_double), ("tn", C.c_double), ("pi2", C.c_double),
                ("snlt", C.c_double), ("ritb1", C.c_double), ("iterm", C.c_int32),
                ("isdry", C.c_int32), ("ndrystp", C.c_int32), ("isbal", C.c_int32),
                ("n", C.c_int32), ("ntstbc", C.c_int32), ("max_sweeps", C.c_int32),
                ("precision", C.c_int32), ("mixed_rsq_factor", C.c_double),
                ("qcherr", C.c_double), ("chan_consistent", C.c_int32), ("pad_", C.c_int32),
                ("bsc", C.c_double), ("gp", C.c_double), ("tl3_istl", C.c_int32),
                ("nctbc", C.c_int32), ("rold", C.c_double), ("rnew", C.c_double),
                ("isitb", C.c_int32), ("isveg", C.c_int32), ("ritb", C.c_double)]


class Fields(C.Structure):
    _fields_ = [("p", _pd), ("hp", _pd), ("h1p", _pd), ("hu", _pd), ("hv", _pd),
                ("uhdye", _pd), ("vhdxe", _pd), ("sub", _pd), ("svb", _pd),
                ("sbx", _pd), ("sby", _pd), ("lmaskdry", _pi), ("iscdry", _pi),
                ("lopenbcdry", _pi), ("natdry", _pi), ("fcaxe", _pd), ("fcaye", _pd),
                ("fxe", _pd), ("fye", _pd), ("tsx", _pd), ("tsy", _pd), ("tbx", _pd),
                ("tby", _pd), ("qsume", _pd), ("pser", _pd * 4), ("uhe", _pd),
                ("vhe", _pd), ("hpi", _pd), ("hui", _pd), ("hvi", _pd),
                ("qdwaste", _pd), ("vdwaste", _pd), ("lwet", _pi), ("ldry", _pi),
                ("ccc", _pd), ("ccs", _pd), ("ccw", _pd), ("cce", _pd), ("ccn", _pd),
                ("fptmp", _pd), ("qchanu", _pd), ("qchanv", _pd), ("qchanun", _pd),
                ("qchanvn", _pd), ("b", _pd), ("b_ld", C.c_int32), ("pad_b_", C.c_int32),
                ("p1", _pd), ("h2p", _pd), ("uhdy1e", _pd), ("vhdx1e", _pd), ("uhdy2e", _pd),
                ("vhdx2e", _pd), ("h1u", _pd), ("h1v", _pd), ("tsx1", _pd), ("tsy1", _pd),
                ("tbx1", _pd), ("tby1", _pd), ("fpgxe", _pd), ("fpgye", _pd),
                ("ubot", _pd), ("vbot", _pd), ("vu", _pd), ("uv", _pd), ("stbx", _pd),
                ("stby", _pd), ("fxvege", _pd), ("fyvege", _pd),
                ("unchanged", C.c_int32), ("pad_u_", C.c_int32)]


class Schedule(C.Structure):
    _fields_ = [("kernel_variant", C.c_int32), ("ctas_matvec", C.c_int32),
                ("ctas_update", C.c_int32), ("graph_iters", C.c_int32),
                ("poly_threshold", C.c_int32), ("inner_margin", C.c_int32),
                ("inner_tol", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Layers(C.Structure):
    _fields_ = [("kc", C.c_int32), ("ld", C.c_int32), ("dzc", _pd), ("zz", _pd)]


class Bed(C.Structure):
    _fields_ = [("zbr", _pd), ("stbxo", _pd), ("stbyo", _pd), ("dxp", _pd), ("dyp", _pd),
                ("dzc1", _pd), ("sgzu1", _pd), ("sgzv1", _pd), ("kc", C.c_int32),
                ("pad_", C.c_int32), ("avcon", C.c_double), ("vismud", C.c_double),
                ("coeftsbl", C.c_double)]


class DragParams(C.Structure):
    _fields_ = [("delt", C.c_double), ("avcon1", C.c_double), ("isdry", C.c_int32),
                ("n", C.c_int32), ("ntstbc", C.c_int32), ("pad_", C.c_int32)]


class DragFields(C.Structure):
    _fields_ = [("ub", _pd), ("vb", _pd), ("vu", _pd), ("uv", _pd), ("h1u", _pd), ("h1v", _pd),
                ("stbx", _pd), ("stby", _pd), ("tbx", _pd), ("tby", _pd)]


DRAG_IN = ("ub", "vb", "vu", "uv", "h1u", "h1v")
DRAG_OUT = ("stbx", "stby", "tbx", "tby")


class Momentum(C.Structure):
    _fields_ = [("kc", C.c_int32), ("ld", C.c_int32), ("fcorc", _pd), ("dydi", _pd),
                ("dxdj", _pd), ("scax", _pd), ("scay", _pd), ("saax", _pd), ("saay", _pd),
                ("sgzu", _pd), ("sgzv", _pd), ("fsgzu", _pd), ("fsgzv", _pd), ("stcuv", _pd),
                ("sdx", _pd), ("sdy", _pd), ("lhdmf", _pi), ("lnwc", _pi), ("lsec", _pi),
                ("nbcs", C.c_int32), ("pad_", C.c_int32), ("lbcs", _pi), ("lberc", _pi),
                ("lbnrc", _pi)]


class ExplicitParams(C.Structure):
    _fields_ = [("snlt", C.c_double), ("iscurvature", C.c_int32), ("ishdmf", C.c_int32)]


class ExplicitFields(C.Structure):
    _fields_ = [("u", _pd), ("v", _pd), ("uhdy", _pd), ("vhdx", _pd), ("hp", _pd),
                ("wet", _pi), ("fuhj", _pd), ("fvhj", _pd), ("fmdux", _pd), ("fmduy", _pd),
                ("fmdvx", _pd), ("fmdvy", _pd), ("fcaxe", _pd), ("fcaye", _pd), ("fxe", _pd),
                ("fye", _pd), ("fcax", _pd), ("fcay", _pd), ("fx", _pd), ("fy", _pd),
                ("cac", _pd)]


MOM_D = ("fcorc", "dydi", "dxdj", "scax", "scay", "saax", "saay", "sgzu", "sgzv", "fsgzu",
         "fsgzv", "stcuv", "sdx", "sdy")
MOM_I = ("lhdmf", "lnwc", "lsec", "lbcs", "lberc", "lbnrc")
EXP_IN = ("u", "v", "uhdy", "vhdx", "hp", "fuhj", "fvhj", "fmdux", "fmduy", "fmdvx", "fmdvy")
EXP_OUT = ("fcaxe", "fcaye", "fxe", "fye", "fcax", "fcay", "fx", "fy", "cac")


class Channels(C.Structure):
    _fields_ = [("n", C.c_int32), ("type", _pi), ("lhost", _pi), ("lu", _pi), ("lv", _pi),
                ("chanlen", _pd), ("chanfric", _pd), ("dxp", _pd), ("dyp", _pd)]


class Stats(C.Structure):
    _fields_ = [("status", C.c_int32), ("iters_last", C.c_int32),
                ("iters_total", C.c_int32), ("solves", C.c_int32),
                ("lawet", C.c_int32), ("ladry", C.c_int32), ("n_negdep", C.c_int32),
                ("n_wasted", C.c_int32), ("outer_refinements", C.c_int32),
                ("rsq_last", C.c_double), ("ccmnm_last", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class KTime(C.Structure):
    _fields_ = [("ms_matvec", C.c_double), ("ms_update", C.c_double), ("reps", C.c_int32),
                ("ncells", C.c_int32), ("nslots", C.c_int32), ("ncells_poly", C.c_int32)]


FIELD_DOUBLE_INOUT = ("p", "hp", "h1p", "hu", "hv", "uhdye", "vhdxe", "sub", "svb",
                      "sbx", "sby")
FIELD_INT_INOUT = ("lmaskdry", "iscdry", "lopenbcdry", "natdry")
FIELD_IN = ("fcaxe", "fcaye", "fxe", "fye", "tsx", "tsy", "tbx", "tby", "qsume")
FIELD_OUT = ("uhe", "vhe", "hpi", "hui", "hvi", "qdwaste", "vdwaste")
FIELD_CHAN = ("qchanu", "qchanv", "qchanun", "qchanvn")  # per channel, in/out
FIELD_DIAG = ("ccc", "ccs", "ccw", "cce", "ccn", "fptmp")
# three time levels (CALPUV9C): in/out, and the in-only wind and bed stresses
FIELD_TL3 = ("p1", "h2p", "uhdy1e", "vhdx1e", "uhdy2e", "vhdx2e", "h1u", "h1v", "tsx1",
             "tsy1", "tbx1", "tby1", "fpgxe", "fpgye")
# implicit bottom / vegetation drag (ISITB >= 1, ISVEG > 0): in
FIELD_DRAG = ("ubot", "vbot", "vu", "uv", "stbx", "stby", "fxvege", "fyvege")


def _dp(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_pd)


def _ip(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_pi)


def make_grid(g: dict):
    """Build a Grid struct from a scenario grid dict.  Returns (struct, keepalive)."""
    keep = []

    def d(name):
        a = np.ascontiguousarray(g[name], dtype=np.float64)
        keep.append(a)
        return _dp(a)

    def i(name):
        a = np.ascontiguousarray(g[name], dtype=np.int32)
        keep.append(a)
        return _ip(a)

    s = Grid()
    s.la = int(g["la"])
    s.lc = int(g["lc"])
    for k in ("il", "jl", "lnc", "lsc", "lec", "lwc"):
        setattr(s, k, i(k))
    for k in ("dxyp", "dxyip", "dxiu", "dyiu", "dxiv", "dyiv", "dxyu", "dxyv",
              "hruo", "hrvo", "subo", "svbo", "sbxo", "sbyo", "belv"):
        setattr(s, k, d(k))
    s.mtide = int(g["mtide"])
    tcp = np.ascontiguousarray(g["tcp"], dtype=np.float64)
    keep.append(tcp)
    s.tcp = _dp(tcp)
    for k, side in enumerate(SIDES):
        o = g["obc"][side]
        n = len(o["l"])
        l = np.ascontiguousarray(o["l"], dtype=np.int32)
        isp = np.ascontiguousarray(o["ispb"], dtype=np.int32)
        # column-major PCB(LL,M) with leading dimension n == row-major [m, ll]
        pcb = np.ascontiguousarray(o["pcb"], dtype=np.float64).reshape(-1)
        psb = np.ascontiguousarray(o["psb"], dtype=np.float64).reshape(-1)
        keep += [l, isp, pcb, psb]
        s.obc[k] = Obc(n, _ip(l), _ip(isp), _dp(pcb), _dp(psb), max(n, 1))
    return s, keep


def make_params(p: dict, *, n: int, tn: float, precision: int = PREC_FP64):
    s = Params()
    # CALPUV9C(3), the leapfrog step, advances over DT2 = 2*DT (calpuv9c.f90:105-106)
    s.delt = p["dt"] * (2.0 if int(p.get("tl3_istl", 0)) == 3 else 1.0)
    s.g = p["g"]
    s.hdry = p["hdry"]
    s.rsqm = p["rsqm"]
    s.tn = tn
    s.pi2 = p["pi2"]
    s.snlt = p["snlt"]
    s.ritb1 = p["ritb1"]
    s.iterm = p["iterm"]
    s.isdry = p["isdry"]
    s.ndrystp = p["ndrystp"]
    s.isbal = p["isbal"]
    s.n = n
    s.ntstbc = p.get("ntstbc", 0)
    s.max_sweeps = p.get("max_sweeps", 500)
    s.precision = precision
    s.mixed_rsq_factor = p.get("mixed_rsq_factor", 0.0)
    s.qcherr = p.get("qcherr", 1.0)
    s.chan_consistent = int(p.get("chan_consistent", 0))
    s.bsc = p.get("bsc", 0.0)
    s.gp = p.get("gp", p["g"])
    s.tl3_istl = int(p.get("tl3_istl", 0))
    s.nctbc = int(p.get("nctbc", 0))
    s.rold = p.get("rold", 0.0)
    s.rnew = p.get("rnew", 1.0)
    s.isitb = int(p.get("isitb", 0))
    s.isveg = int(p.get("isveg", 0))
    s.ritb = p.get("ritb", 0.0)
    return s


def make_layers(ly: dict | None):
    """A Layers struct over {"dzc", "zz"}: (KC, LCM) float64 arrays, layer K
    at row K-1.  Returns (struct, kept arrays)."""
    s = Layers()
    if not ly:
        return s, []
    keep = [np.ascontiguousarray(ly[k], dtype=np.float64) for k in ("dzc", "zz")]
    s.kc, s.ld = int(keep[0].shape[0]), int(keep[0].shape[1])
    s.dzc, s.zz = _dp(keep[0]), _dp(keep[1])
    return s, keep


def make_bed(bed: dict):
    """A Bed struct over {"zbr", "stbxo", "stbyo", "dxp", "dyp", "dzc1", "sgzu1",
    "sgzv1"} (float64 over 1..LC) and the scalars kc, avcon, vismud, coeftsbl.
    Returns (struct, kept arrays)."""
    keys = ("zbr", "stbxo", "stbyo", "dxp", "dyp", "dzc1", "sgzu1", "sgzv1")
    keep = [np.ascontiguousarray(bed[k], dtype=np.float64) for k in keys]
    s = Bed()
    for k, a in zip(keys, keep):
        setattr(s, k, _dp(a))
    s.kc = int(bed.get("kc", 1))
    s.avcon = float(bed.get("avcon", 1.0))
    s.vismud = float(bed.get("vismud", 1e-6))
    s.coeftsbl = float(bed.get("coeftsbl", 4.0))
    return s, keep


def make_drag_params(p: dict, *, n: int):
    s = DragParams()
    s.delt = float(p["dt"])
    s.avcon1 = float(p.get("avcon1", 0.0))
    s.isdry = int(p["isdry"])
    s.n = n
    s.ntstbc = int(p.get("ntstbc", 0))
    return s


def make_drag_fields(d: dict):
    """A DragFields struct over the arrays of d (DRAG_IN in, DRAG_OUT out)."""
    s = DragFields()
    for k in DRAG_IN + DRAG_OUT:
        a = d.get(k)
        if a is not None:
            setattr(s, k, _dp(a))
    return s


def make_momentum(mo: dict):
    """A Momentum struct over a dict: kc, ld and the arrays of MOM_D (float64;
    the layer ones sgzu, sgzv, fsgzu, fsgzv as [kc, ld] C-order = Fortran
    (ld, kc)) and MOM_I (int32); stcuv, sdx, sdy, lhdmf may be absent.
    Returns (struct, kept arrays)."""
    s = Momentum()
    keep = []
    s.kc = int(mo["kc"])
    s.ld = int(mo["ld"])
    for k in MOM_D:
        if mo.get(k) is not None:
            a = np.ascontiguousarray(mo[k], dtype=np.float64)
            keep.append(a)
            setattr(s, k, _dp(a))
    for k in MOM_I:
        if mo.get(k) is not None:
            a = np.ascontiguousarray(mo[k], dtype=np.int32)
            keep.append(a)
            setattr(s, k, _ip(a))
    s.nbcs = int(len(mo["lbcs"])) if mo.get("lbcs") is not None else 0
    return s, keep


def make_explicit_params(snlt=1.0, iscurvature=1, ishdmf=0):
    return ExplicitParams(snlt=float(snlt), iscurvature=int(iscurvature), ishdmf=int(ishdmf))


def make_explicit_fields(d: dict):
    """An ExplicitFields struct over the arrays of d (EXP_IN in, EXP_OUT out,
    "wet" int32); absent keys are NULL.  Returns (struct, kept arrays)."""
    s = ExplicitFields()
    keep = []
    for k in EXP_IN + EXP_OUT:
        a = d.get(k)
        if a is not None:
            assert a.dtype == np.float64 and a.flags.c_contiguous, k
            setattr(s, k, _dp(a))
    if d.get("wet") is not None:
        w = np.ascontiguousarray(d["wet"], dtype=np.int32)
        keep.append(w)
        s.wet = _ip(w)
    return s, keep


def make_channels(ch: dict | None):
    """A Channels struct over a dict of numpy arrays (type, lhost, lu, lv:
    int32; chanlen, chanfric: float64 per channel; dxp, dyp: float64 over
    1..LC), or an empty one for None.  Returns (struct, kept arrays)."""
    s = Channels()
    if not ch:
        s.n = 0
        return s, []
    keep = [np.ascontiguousarray(ch[k], dtype=np.int32) for k in ("type", "lhost", "lu", "lv")]
    keep += [np.ascontiguousarray(ch[k], dtype=np.float64)
             for k in ("chanlen", "chanfric", "dxp", "dyp")]
    s.n = int(keep[0].size)
    s.type, s.lhost, s.lu, s.lv = (_ip(a) for a in keep[:4])
    s.chanlen, s.chanfric, s.dxp, s.dyp = (_dp(a) for a in keep[4:])
    return s, keep


# bits of efdc_xm_fields.unchanged (enum efdc_xm_same), one per array
SAME = {k: 1 << i for i, k in enumerate((
    "p", "hp", "hu", "hv", "uhdye", "vhdxe", "sub", "svb", "sbx", "sby", "lmaskdry", "iscdry",
    "lopenbcdry", "natdry", "fcaxe", "fcaye", "fxe", "fye", "tsx", "tsy", "tbx", "tby", "qsume",
    "qdwaste", "vdwaste"))}


def same_bits(names) -> int:
    """The efdc_xm_fields.unchanged bits of the named arrays."""
    b = 0
    for k in names:
        b |= SAME[k]
    return b


def make_fields(st: dict, *, diag: bool = False, lists: bool = False, unchanged: int = 0):
    """Build a Fields struct over the numpy arrays of a state dict (in place).
    unchanged: efdc_xm_fields.unchanged (see same_bits)."""
    s = Fields()
    s.unchanged = unchanged
    keep = []
    for k in FIELD_DOUBLE_INOUT + FIELD_IN + FIELD_OUT + FIELD_CHAN + FIELD_TL3 + FIELD_DRAG:
        a = st.get(k)
        if a is not None:
            setattr(s, k, _dp(a))
    for k in FIELD_INT_INOUT:
        a = st.get(k)
        if a is not None:
            setattr(s, k, _ip(a))
    for k, side in enumerate(SIDES):
        a = st["pser"].get(side) if "pser" in st else None
        if a is not None and a.size:
            s.pser[k] = _dp(a)
    if lists:
        n = st["p"].size
        for k in ("lwet", "ldry"):
            if k not in st:
                st[k] = np.zeros(n, np.int32)
            setattr(s, k, _ip(st[k]))
    if diag:
        n = st["p"].size
        for k in FIELD_DIAG:
            if k not in st:
                st[k] = np.zeros(n)
            setattr(s, k, _dp(st[k]))
    b = st.get("b")
    if b is not None:  # B(L,K) as a (KC, LCM) array: layer K at row K-1
        s.b = _dp(b)
        s.b_ld = int(b.shape[-1])
    return s, keep


OPT_DEVICE_LOOPS = 1
OPT_GRAPH_ITERS = 2
OPT_KERNEL_VARIANT = 3
OPT_CTAS_MATVEC = 4
OPT_CTAS_UPDATE = 5
OPT_POLY_THRESHOLD = 6
OPT_INNER_MARGIN = 7
OPT_INNER_TOL = 8
OPT_SMALL_SOLVE = 9
OPT_FOLD_REDUCE = 10
OPT_CHUNKS = 11


TUNE_MEASURE = 1


def tune_lookup(table, key: str):
    """The schedule (a dict) the tuning table holds for `key`, or None."""
    sch = Schedule()
    rc = load().efdc_xm_tune_lookup(str(table).encode(), key.encode(), C.byref(sch))
    return sch.as_dict() if rc == OK else None


def _autotune(lib, ctx, precision, table, measure):
    sch = Schedule()
    ms = C.c_double(0.0)
    rc = lib.efdc_xm_autotune(ctx, precision, str(table).encode() if table else None,
                              TUNE_MEASURE if measure else 0, C.byref(sch), C.byref(ms))
    if rc != OK:
        raise RuntimeError(f"efdc_xm_autotune: {lib.efdc_xm_last_error().decode()}")
    return sch.as_dict(), ms.value


def _tune_key(lib, ctx, precision):
    buf = C.create_string_buffer(256)
    if lib.efdc_xm_tune_key(ctx, precision, buf, 256) != OK:
        raise RuntimeError("efdc_xm_tune_key failed")
    return buf.value.decode()


def host_waits() -> int:
    """Host synchronisations made by step and solve calls so far."""
    return int(load().efdc_xm_host_waits())


class CudaLibraryMissing(RuntimeError):
    pass


_lib = None


def transfer_bytes() -> tuple[int, int]:
    """Bytes of callers' arrays copied (host->device, device->host) by the
    library in this process so far."""
    lib = load()
    h, d = C.c_int64(0), C.c_int64(0)
    lib.efdc_xm_transfer_bytes(C.byref(h), C.byref(d))
    return h.value, d.value


def load(path: str | os.PathLike | None = None):
    """Load libefdc_xm.so (built in-tree by build.py).  Fails loudly when it is
    missing: there is no CPU fallback."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise CudaLibraryMissing(
            f"{p} not found: build it with `python {PKG_DIR / 'build.py'}` "
            "(the solver has no CPU fallback)")
    lib = C.CDLL(str(p))
    lib.efdc_xm_abi_version.restype = C.c_int32
    lib.efdc_xm_last_error.restype = C.c_char_p
    lib.efdc_xm_create.restype = C.c_void_p
    lib.efdc_xm_create.argtypes = [C.POINTER(Grid), C.c_int32]
    lib.efdc_xm_destroy.argtypes = [C.c_void_p]
    for name in ("efdc_xm_step",):
        fn = getattr(lib, name)
        fn.restype = C.c_int32
        fn.argtypes = [C.c_void_p, C.POINTER(Params), C.POINTER(Fields), C.POINTER(Stats)]
    lib.efdc_xm_upload.restype = C.c_int32
    lib.efdc_xm_upload.argtypes = [C.c_void_p, C.POINTER(Fields)]
    lib.efdc_xm_download.restype = C.c_int32
    lib.efdc_xm_download.argtypes = [C.c_void_p, C.POINTER(Fields)]
    lib.efdc_xm_step_device.restype = C.c_int32
    lib.efdc_xm_step_device.argtypes = [C.c_void_p, C.POINTER(Params), C.POINTER(Stats)]
    lib.efdc_xm_stream.restype = C.c_void_p
    lib.efdc_xm_stream.argtypes = [C.c_void_p]
    lib.efdc_xm_kernel_launches.restype = C.c_int64
    lib.efdc_xm_host_waits.restype = C.c_int64
    lib.efdc_xm_autotune.restype = C.c_int32
    lib.efdc_xm_autotune.argtypes = [C.c_void_p, C.c_int32, C.c_char_p, C.c_int32,
                                     C.POINTER(Schedule), C.POINTER(C.c_double)]
    lib.efdc_xm_tune_key.restype = C.c_int32
    lib.efdc_xm_tune_key.argtypes = [C.c_void_p, C.c_int32, C.c_char_p, C.c_int32]
    lib.efdc_xm_tune_lookup.restype = C.c_int32
    lib.efdc_xm_tune_lookup.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(Schedule)]
    lib.efdc_xm_set_option.restype = C.c_int32
    lib.efdc_xm_set_option.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
    lib.efdc_xm_set_layers.restype = C.c_int32
    lib.efdc_xm_set_layers.argtypes = [C.c_void_p, C.c_int32, C.POINTER(Layers)]
    lib.efdc_xm_set_channels.restype = C.c_int32
    lib.efdc_xm_set_channels.argtypes = [C.c_void_p, C.c_int32, C.POINTER(Channels)]
    lib.efdc_xm_transfer_bytes.restype = None
    lib.efdc_xm_transfer_bytes.argtypes = [C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.efdc_xm_time_kernels.restype = C.c_int32
    lib.efdc_xm_time_kernels.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(KTime)]
    lib.efdc_xm_congrad_noalloc.restype = C.c_int32
    lib.efdc_xm_congrad_noalloc.argtypes = [C.c_int32] + [C.c_void_p] * 11 + [
        C.c_double, C.c_int32, C.c_void_p, _pi, _pd]
    lib.efdc_xm_congrad.restype = C.c_int32
    lib.efdc_xm_congrad.argtypes = [C.c_void_p] + [_pd] * 8 + [C.c_double, C.c_int32,
                                                                C.c_int32, _pi, _pd]
    for name, args in (
            ("efdc_xm_calib_enable", [C.c_void_p, C.c_int32]),
            ("efdc_xm_calib_set_roughness", [C.c_void_p, _pd]),
            ("efdc_xm_calib_set_harmonics", [C.c_void_p, _pd, _pd]),
            ("efdc_xm_calib_snapshot", [C.c_void_p, C.c_int32]),
            ("efdc_xm_calib_restore", [C.c_void_p, C.c_int32]),
            ("efdc_xm_calib_step", [C.c_void_p, C.POINTER(Params), C.POINTER(Stats)]),
            ("efdc_xm_calib_gauges", [C.c_void_p, C.c_int32, _pi, _pd]),
            ("efdc_xm_calib_adjoint_reset", [C.c_void_p]),
            ("efdc_xm_calib_add_p_adjoint", [C.c_void_p, C.c_int32, _pi, _pd]),
            ("efdc_xm_calib_adjoint_step", [C.c_void_p, C.POINTER(Params), C.c_int32, C.c_double,
                                            _pi]),
            ("efdc_xm_calib_gradients", [C.c_void_p, _pd, _pd, _pd, _pd, C.POINTER(_pd), _pi])):
        fn = getattr(lib, name)
        fn.restype = C.c_int32
        fn.argtypes = args
    lib.efdc_xm_create_batch.restype = C.c_void_p
    lib.efdc_xm_create_batch.argtypes = [C.POINTER(Grid), C.c_int32, C.c_int32]
    lib.efdc_xm_nmembers.restype = C.c_int32
    lib.efdc_xm_nmembers.argtypes = [C.c_void_p]
    lib.efdc_xm_step_batch.restype = C.c_int32
    lib.efdc_xm_step_batch.argtypes = [C.c_void_p, C.POINTER(Params), C.POINTER(Fields),
                                       C.POINTER(Stats)]
    lib.efdc_xm_upload_batch.restype = C.c_int32
    lib.efdc_xm_upload_batch.argtypes = [C.c_void_p, C.POINTER(Fields)]
    lib.efdc_xm_download_batch.restype = C.c_int32
    lib.efdc_xm_download_batch.argtypes = [C.c_void_p, C.POINTER(Fields)]
    lib.efdc_xm_step_device_batch.restype = C.c_int32
    lib.efdc_xm_step_device_batch.argtypes = [C.c_void_p, C.POINTER(Params), C.POINTER(Stats)]
    lib.efdc_xm_set_bed.restype = C.c_int32
    lib.efdc_xm_set_bed.argtypes = [C.c_void_p, C.c_int32, C.POINTER(Bed)]
    lib.efdc_xm_bottom_stress_batch.restype = C.c_int32
    lib.efdc_xm_bottom_stress_batch.argtypes = [C.c_void_p, C.POINTER(DragParams),
                                                C.POINTER(DragFields)]
    lib.efdc_xm_set_momentum.restype = C.c_int32
    lib.efdc_xm_set_momentum.argtypes = [C.c_void_p, C.c_int32, C.POINTER(Momentum)]
    lib.efdc_xm_explicit_batch.restype = C.c_int32
    lib.efdc_xm_explicit_batch.argtypes = [C.c_void_p, C.POINTER(ExplicitParams),
                                           C.POINTER(ExplicitFields)]
    if path is None:
        _lib = lib
    return lib


class Solver:
    """Host-side handle over one efdc_xm context (one basin on one GPU)."""

    def __init__(self, grid: dict, device: int = 0, lib=None):
        """Create a context for the static model ``grid`` on CUDA device ``device``."""
        self.lib = lib or load()
        self._grid, self._keep = make_grid(grid)
        self.ctx = self.lib.efdc_xm_create(C.byref(self._grid), device)
        if not self.ctx:
            raise RuntimeError("efdc_xm_create failed: " + self.last_error())
        self.la = int(grid["la"])
        self.lc = int(grid["lc"])

    def last_error(self) -> str:
        return self.lib.efdc_xm_last_error().decode()

    def close(self):
        if self.ctx:
            self.lib.efdc_xm_destroy(self.ctx)
            self.ctx = None

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    def step(self, params: Params, state: dict, *, diag=False, lists=False) -> Stats:
        f, _k = make_fields(state, diag=diag, lists=lists)
        st = Stats()
        rc = self.lib.efdc_xm_step(self.ctx, C.byref(params), C.byref(f), C.byref(st))
        if rc in (CUDA_ERROR, BAD_ARGUMENT, UNSUPPORTED, DEVICE_TIMEOUT):
            raise RuntimeError(f"efdc_xm_step: {STATUS_NAMES.get(rc, rc)}: {self.last_error()}")
        return st

    def upload(self, state: dict):
        f, _k = make_fields(state)
        rc = self.lib.efdc_xm_upload(self.ctx, C.byref(f))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_upload: {self.last_error()}")

    def download(self, state: dict, *, diag=False, lists=False):
        f, _k = make_fields(state, diag=diag, lists=lists)
        rc = self.lib.efdc_xm_download(self.ctx, C.byref(f))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_download: {self.last_error()}")

    def step_device(self, params: Params) -> Stats:
        st = Stats()
        rc = self.lib.efdc_xm_step_device(self.ctx, C.byref(params), C.byref(st))
        if rc in (CUDA_ERROR, BAD_ARGUMENT, UNSUPPORTED, DEVICE_TIMEOUT):
            raise RuntimeError(f"efdc_xm_step_device: {STATUS_NAMES.get(rc, rc)}: "
                               f"{self.last_error()}")
        return st

    def stream(self) -> int:
        return int(self.lib.efdc_xm_stream(self.ctx) or 0)

    def set_option(self, option: int, value: int):
        rc = self.lib.efdc_xm_set_option(self.ctx, option, value)
        if rc != OK:
            raise RuntimeError(f"efdc_xm_set_option: {self.last_error()}")

    def autotune(self, precision: int, table=None, measure: bool = False):
        """efdc_xm_autotune: (schedule dict, measured solve ms or 0 if replayed)."""
        return _autotune(self.lib, self.ctx, precision, table, measure)

    def tune_key(self, precision: int) -> str:
        return _tune_key(self.lib, self.ctx, precision)

    def set_layers(self, ly: dict, member: int = 0):
        s, _keep = make_layers(ly)
        rc = self.lib.efdc_xm_set_layers(self.ctx, member, C.byref(s))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_set_layers: {STATUS_NAMES.get(rc, rc)}: "
                               f"{self.last_error()}")

    def set_bed(self, bed: dict, member: int = 0):
        s, _keep = make_bed(bed)
        rc = self.lib.efdc_xm_set_bed(self.ctx, member, C.byref(s))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_set_bed: {STATUS_NAMES.get(rc, rc)}: {self.last_error()}")

    def bottom_stress(self, params: DragParams, drag: dict):
        """CALTBXY + TBX/TBY on the device (efdc_xm_bottom_stress_batch); the
        outputs present in `drag` are written."""
        f = make_drag_fields(drag)
        rc = self.lib.efdc_xm_bottom_stress_batch(self.ctx, C.byref(params), C.byref(f))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_bottom_stress_batch: {STATUS_NAMES.get(rc, rc)}: "
                               f"{self.last_error()}")

    def set_momentum(self, mo: dict, member: int = 0):
        s, _keep = make_momentum(mo)
        rc = self.lib.efdc_xm_set_momentum(self.ctx, member, C.byref(s))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_set_momentum: {STATUS_NAMES.get(rc, rc)}: "
                               f"{self.last_error()}")

    def explicit(self, params: ExplicitParams, fields: dict):
        """CALEXP2T's external-mode terms on the device (efdc_xm_explicit_batch);
        the outputs present in `fields` are written."""
        f, _keep = make_explicit_fields(fields)
        rc = self.lib.efdc_xm_explicit_batch(self.ctx, C.byref(params), C.byref(f))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_explicit_batch: {STATUS_NAMES.get(rc, rc)}: "
                               f"{self.last_error()}")

    def set_channels(self, ch: dict | None, member: int = 0):
        s, _keep = make_channels(ch)
        rc = self.lib.efdc_xm_set_channels(self.ctx, member, C.byref(s))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_set_channels: {STATUS_NAMES.get(rc, rc)}: "
                               f"{self.last_error()}")

    def time_kernels(self, precision: int, reps: int = 20) -> KTime:
        kt = KTime()
        rc = self.lib.efdc_xm_time_kernels(self.ctx, precision, reps, C.byref(kt))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_time_kernels: {self.last_error()}")
        return kt

    # ---- calibration (adjoint) ----
    def _ok(self, name, rc):
        if rc != OK:
            raise RuntimeError(f"{name}: {STATUS_NAMES.get(rc, rc)}: {self.last_error()}")

    def calib_enable(self, nsnap: int):
        self._ok("efdc_xm_calib_enable", self.lib.efdc_xm_calib_enable(self.ctx, int(nsnap)))

    def calib_set_roughness(self, log_n):
        a = np.ascontiguousarray(log_n, dtype=np.float64)
        self._ok("efdc_xm_calib_set_roughness", self.lib.efdc_xm_calib_set_roughness(self.ctx, _dp(a)))

    def calib_set_harmonics(self, pcb, psb):
        a = np.ascontiguousarray(pcb, dtype=np.float64)
        b = np.ascontiguousarray(psb, dtype=np.float64)
        self._ok("efdc_xm_calib_set_harmonics",
                 self.lib.efdc_xm_calib_set_harmonics(self.ctx, _dp(a), _dp(b)))

    def calib_snapshot(self, slot: int):
        self._ok("efdc_xm_calib_snapshot", self.lib.efdc_xm_calib_snapshot(self.ctx, int(slot)))

    def calib_restore(self, slot: int):
        self._ok("efdc_xm_calib_restore", self.lib.efdc_xm_calib_restore(self.ctx, int(slot)))

    def calib_step(self, params: Params) -> Stats:
        st = Stats()
        rc = self.lib.efdc_xm_calib_step(self.ctx, C.byref(params), C.byref(st))
        if rc not in (OK, NEG_DEPTH):
            raise RuntimeError(f"efdc_xm_calib_step: {STATUS_NAMES.get(rc, rc)}: {self.last_error()}")
        return st

    def calib_gauges(self, cells) -> np.ndarray:
        L = np.ascontiguousarray(cells, dtype=np.int32)
        out = np.zeros(L.size)
        self._ok("efdc_xm_calib_gauges",
                 self.lib.efdc_xm_calib_gauges(self.ctx, L.size, _ip(L), _dp(out)))
        return out

    def calib_adjoint_reset(self):
        self._ok("efdc_xm_calib_adjoint_reset", self.lib.efdc_xm_calib_adjoint_reset(self.ctx))

    def calib_add_p_adjoint(self, cells, w):
        L = np.ascontiguousarray(cells, dtype=np.int32)
        a = np.ascontiguousarray(w, dtype=np.float64)
        self._ok("efdc_xm_calib_add_p_adjoint",
                 self.lib.efdc_xm_calib_add_p_adjoint(self.ctx, L.size, _ip(L), _dp(a)))

    def calib_adjoint_step(self, params: Params, slot: int, rel_tol: float = 1e-12) -> int:
        it = C.c_int32(0)
        self._ok("efdc_xm_calib_adjoint_step",
                 self.lib.efdc_xm_calib_adjoint_step(self.ctx, C.byref(params), int(slot),
                                                     float(rel_tol), C.byref(it)))
        return it.value

    def calib_gradients(self, nobc_mt: int):
        """(d/dlog n, d/dBELV, d/dPCB, d/dPSB, state adjoints dict, n_clamped);
        per-cell arrays have the LCM = LC+1 length of the model's arrays."""
        lc = self.lc + 1
        dk, db = np.zeros(lc), np.zeros(lc)
        dpc, dps = np.zeros(max(nobc_mt, 1)), np.zeros(max(nobc_mt, 1))
        names = ("p", "hp", "hu", "hv", "uhdye", "vhdxe")
        st = {k: np.zeros(lc) for k in names}
        arr = (_pd * 6)(*[_dp(st[k]) for k in names])
        ncl = C.c_int32(0)
        self._ok("efdc_xm_calib_gradients",
                 self.lib.efdc_xm_calib_gradients(self.ctx, _dp(dk), _dp(db), _dp(dpc), _dp(dps),
                                                  arr, C.byref(ncl)))
        return dk, db, dpc[:nobc_mt], dps[:nobc_mt], st, ncl.value

    def congrad(self, ccc, ccs, ccn, ccw, cce, ccci, fptmp, p, rsqm, iterm,
                precision=PREC_FP64):
        it = C.c_int32(0)
        rsq = C.c_double(0.0)
        rc = self.lib.efdc_xm_congrad(self.ctx, _dp(ccc), _dp(ccs), _dp(ccn), _dp(ccw),
                                      _dp(cce), _dp(ccci), _dp(fptmp), _dp(p),
                                      float(rsqm), int(iterm), int(precision),
                                      C.byref(it), C.byref(rsq))
        return rc, it.value, rsq.value


class BatchSolver:
    """Host-side handle over one efdc_xm batch context: M independent basins
    (ensemble members) advanced together, one launch sequence per step."""

    def __init__(self, grids: list, device: int = 0, lib=None):
        self.lib = lib or load()
        self.m = len(grids)
        if self.m < 1:
            raise ValueError("BatchSolver needs at least one grid")
        built = [make_grid(g) for g in grids]
        self._keep = [k for _, k in built]
        self._grids = (Grid * self.m)(*[s for s, _ in built])
        self.ctx = self.lib.efdc_xm_create_batch(self._grids, self.m, device)
        if not self.ctx:
            raise RuntimeError("efdc_xm_create_batch failed: " + self.last_error())
        self.la = [int(g["la"]) for g in grids]

    def last_error(self) -> str:
        return self.lib.efdc_xm_last_error().decode()

    def close(self):
        if self.ctx:
            self.lib.efdc_xm_destroy(self.ctx)
            self.ctx = None

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    def set_layers(self, ly: dict, member: int):
        s, _keep = make_layers(ly)
        rc = self.lib.efdc_xm_set_layers(self.ctx, member, C.byref(s))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_set_layers: {STATUS_NAMES.get(rc, rc)}: "
                               f"{self.last_error()}")

    def set_bed(self, bed: dict, member: int):
        s, _keep = make_bed(bed)
        rc = self.lib.efdc_xm_set_bed(self.ctx, member, C.byref(s))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_set_bed: {STATUS_NAMES.get(rc, rc)}: {self.last_error()}")

    def bottom_stress(self, params: list, drags: list):
        fa = (DragFields * self.m)(*[make_drag_fields(d) for d in drags])
        pa = (DragParams * self.m)(*params)
        rc = self.lib.efdc_xm_bottom_stress_batch(self.ctx, pa, fa)
        if rc != OK:
            raise RuntimeError(f"efdc_xm_bottom_stress_batch: {STATUS_NAMES.get(rc, rc)}: "
                               f"{self.last_error()}")

    def set_momentum(self, mo: dict, member: int):
        s, _keep = make_momentum(mo)
        rc = self.lib.efdc_xm_set_momentum(self.ctx, member, C.byref(s))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_set_momentum: {STATUS_NAMES.get(rc, rc)}: "
                               f"{self.last_error()}")

    def explicit(self, params: list, fields: list):
        made = [make_explicit_fields(d) for d in fields]
        fa = (ExplicitFields * self.m)(*[x[0] for x in made])
        pa = (ExplicitParams * self.m)(*params)
        rc = self.lib.efdc_xm_explicit_batch(self.ctx, pa, fa)
        if rc != OK:
            raise RuntimeError(f"efdc_xm_explicit_batch: {STATUS_NAMES.get(rc, rc)}: "
                               f"{self.last_error()}")

    def set_channels(self, ch: dict | None, member: int):
        s, _keep = make_channels(ch)
        rc = self.lib.efdc_xm_set_channels(self.ctx, member, C.byref(s))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_set_channels: {STATUS_NAMES.get(rc, rc)}: "
                               f"{self.last_error()}")

    def _fields(self, states, **kw):
        if len(states) != self.m:
            raise ValueError(f"need {self.m} member states, got {len(states)}")
        fs = [make_fields(st, **kw) for st in states]
        return (Fields * self.m)(*[f for f, _ in fs]), fs

    def _params(self, params):
        if len(params) != self.m:
            raise ValueError(f"need {self.m} member parameter sets, got {len(params)}")
        return (Params * self.m)(*params)

    def _check(self, name, rc):
        if rc in (CUDA_ERROR, BAD_ARGUMENT, UNSUPPORTED, DEVICE_TIMEOUT):
            raise RuntimeError(f"{name}: {STATUS_NAMES.get(rc, rc)}: {self.last_error()}")

    def step(self, params: list, states: list, *, diag=False, lists=False) -> list:
        return self.step_prepared(params, self.prepare(states, diag=diag, lists=lists))

    def prepare(self, states: list, *, diag=False, lists=False, unchanged: int = 0):
        """The members' Fields structs over `states`, for step_prepared: a driver
        whose arrays stay in place builds them once (256 members: ~30 ms of
        Python per build).  unchanged: the arrays (same_bits) the driver does
        not touch between steps."""
        return self._fields(states, diag=diag, lists=lists, unchanged=unchanged)

    def step_prepared(self, params: list, prepared) -> list:
        """efdc_xm_step_batch on the arrays of prepare(states)."""
        fa, _k = prepared
        pa = self._params(params)
        sa = (Stats * self.m)()
        rc = self.lib.efdc_xm_step_batch(self.ctx, pa, fa, sa)
        self._check("efdc_xm_step_batch", rc)
        return list(sa)

    def upload(self, states: list):
        fa, _k = self._fields(states)
        rc = self.lib.efdc_xm_upload_batch(self.ctx, fa)
        if rc != OK:
            raise RuntimeError(f"efdc_xm_upload_batch: {self.last_error()}")

    def download(self, states: list, *, diag=False, lists=False):
        fa, _k = self._fields(states, diag=diag, lists=lists)
        rc = self.lib.efdc_xm_download_batch(self.ctx, fa)
        if rc != OK:
            raise RuntimeError(f"efdc_xm_download_batch: {self.last_error()}")

    def step_device(self, params: list) -> list:
        pa = self._params(params)
        sa = (Stats * self.m)()
        rc = self.lib.efdc_xm_step_device_batch(self.ctx, pa, sa)
        self._check("efdc_xm_step_device_batch", rc)
        return list(sa)

    def stream(self) -> int:
        return int(self.lib.efdc_xm_stream(self.ctx) or 0)

    def set_option(self, option: int, value: int):
        rc = self.lib.efdc_xm_set_option(self.ctx, option, value)
        if rc != OK:
            raise RuntimeError(f"efdc_xm_set_option: {self.last_error()}")

    def autotune(self, precision: int, table=None, measure: bool = False):
        """efdc_xm_autotune: (schedule dict, measured solve ms or 0 if replayed)."""
        return _autotune(self.lib, self.ctx, precision, table, measure)

    def tune_key(self, precision: int) -> str:
        return _tune_key(self.lib, self.ctx, precision)

    def time_kernels(self, precision: int, reps: int = 20) -> KTime:
        kt = KTime()
        rc = self.lib.efdc_xm_time_kernels(self.ctx, precision, reps, C.byref(kt))
        if rc != OK:
            raise RuntimeError(f"efdc_xm_time_kernels: {self.last_error()}")
        return kt
