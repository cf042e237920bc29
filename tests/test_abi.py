"""CPU checks of the C-ABI library: it loads, exports every function declared
in include/efdc_xm.h, and the ctypes mirror matches the C struct layout.
No compute call is made without a GPU."""
import ctypes as C
import json
import re
import subprocess
from pathlib import Path

import pytest

import efdc_xm as X

REPO = Path(__file__).resolve().parents[1]
HEADER = REPO / "include" / "efdc_xm.h"


def declared_functions():
    txt = HEADER.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(efdc_xm_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = X.load()
    out = subprocess.run(["nm", "-D", "--defined-only", str(X.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (efdc_xm_\w+)", out))
    for fn in declared_functions():
        assert fn in exported, fn
        assert getattr(lib, fn) is not None


def test_abi_version():
    lib = X.load()
    m = re.search(r"#define EFDC_XM_ABI_VERSION (\d+)", HEADER.read_text())
    assert lib.efdc_xm_abi_version() == int(m.group(1))


STRUCTS = {
    "efdc_xm_obc": X.Obc, "efdc_xm_grid": X.Grid, "efdc_xm_params": X.Params,
    "efdc_xm_fields": X.Fields, "efdc_xm_stats": X.Stats, "efdc_xm_channels": X.Channels,
    "efdc_xm_layers": X.Layers, "efdc_xm_bed": X.Bed, "efdc_xm_drag_params": X.DragParams,
    "efdc_xm_drag_fields": X.DragFields, "efdc_xm_ktime": X.KTime,
    "efdc_xm_momentum": X.Momentum, "efdc_xm_explicit_params": X.ExplicitParams,
    "efdc_xm_explicit_fields": X.ExplicitFields,
}


def test_ctypes_layout_matches_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){",
             'printf("{");']
    first = True
    for cname, cls in STRUCTS.items():
        for fname, _ in cls._fields_:
            sep = "" if first else ","
            first = False
            lines.append(f'printf("{sep}\\"{cname}.{fname}\\": %zu", offsetof({cname}, {fname}));')
        lines.append(f'printf(",\\"{cname}.__size__\\": %zu", sizeof({cname}));')
    lines += ['printf("}");', "return 0;}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    got = json.loads(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)
    for cname, cls in STRUCTS.items():
        for fname, _ in cls._fields_:
            assert got[f"{cname}.{fname}"] == getattr(cls, fname).offset, f"{cname}.{fname}"
        assert got[f"{cname}.__size__"] == C.sizeof(cls), cname


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU behaviour")
def test_create_without_gpu_fails_loudly():
    """No CPU fallback: without a device the context cannot be created."""
    import scenario as S
    scn = S.make_scenario(12, 10, seed=1)
    with pytest.raises(RuntimeError, match="efdc_xm_create failed"):
        X.Solver(scn.grid)


def test_missing_library_fails_loudly(tmp_path):
    """No CPU fallback: a missing libefdc_xm.so is an error, not a slower path."""
    with pytest.raises(X.CudaLibraryMissing, match="no CPU fallback"):
        X.load(tmp_path / "libefdc_xm.so")


def test_fortran_shim_binds_declared_symbols():
    """The Fortran binding module names exactly the C entry points it uses."""
    f90 = (REPO / "efdcplus8.5_b200" / "fortran" / "efdc_xm_bind.f90").read_text()
    bound = set(re.findall(r"BIND\(C,\s*NAME='(efdc_xm_\w+)'\)", f90, flags=re.I))
    assert bound and bound <= set(declared_functions())


FORTRAN_TYPES = {
    "EFDC_XM_OBC_T": X.Obc, "EFDC_XM_GRID_T": X.Grid, "EFDC_XM_PARAMS_T": X.Params,
    "EFDC_XM_FIELDS_T": X.Fields, "EFDC_XM_BED_T": X.Bed,
    "EFDC_XM_DRAG_PARAMS_T": X.DragParams, "EFDC_XM_DRAG_FIELDS_T": X.DragFields,
    "EFDC_XM_LAYERS_T": X.Layers, "EFDC_XM_CHANNELS_T": X.Channels, "EFDC_XM_STATS_T": X.Stats,
    "EFDC_XM_MOMENTUM_T": X.Momentum, "EFDC_XM_EXPLICIT_PARAMS_T": X.ExplicitParams,
    "EFDC_XM_EXPLICIT_FIELDS_T": X.ExplicitFields,
}


def _fortran_members(f90: str, tname: str):
    """(name, kind, count) of the members of a BIND(C) derived type, in order."""
    m = re.search(rf"TYPE,\s*BIND\(C\)\s*::\s*{tname}\s*\n(.*?)\n\s*END TYPE", f90, flags=re.S | re.I)
    assert m, tname
    out = []
    for line in m.group(1).splitlines():
        line = line.split("!")[0].strip()
        if not line:
            continue
        decl, names = line.split("::")
        decl = decl.strip().upper()
        kind = ("double" if "C_DOUBLE" in decl else "int32" if "C_INT32_T" in decl else
                "ptr" if "C_PTR" in decl else decl[decl.index("(") + 1:decl.index(")")].lower())
        for nm in re.findall(r"(\w+)(?:\((\d+)\))?", names):
            out.append((nm[0].lower(), kind, int(nm[1]) if nm[1] else 1))
    return out


def _ctypes_members(cls):
    out = []
    for name, t in cls._fields_:
        n = 1
        if issubclass(t, C.Array):
            n, t = t._length_, t._type_
        kind = ("double" if t is C.c_double else "int32" if t is C.c_int32 else
                "ptr" if issubclass(t, C._Pointer) or t is C.c_void_p else
                "efdc_xm_" + t.__name__.lower() + "_t")
        out.append((name.lower(), kind, n))
    return out


def test_fortran_types_mirror_the_header():
    """Every BIND(C) type of the Fortran module lists the C struct's members in
    order, with matching kinds and array lengths (checked against the ctypes
    mirror, whose layout test_ctypes_layout_matches_header checks)."""
    f90 = (REPO / "efdcplus8.5_b200" / "fortran" / "efdc_xm_bind.f90").read_text()
    for tname, cls in FORTRAN_TYPES.items():
        assert _fortran_members(f90, tname) == _ctypes_members(cls), tname
