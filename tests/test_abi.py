"""The C ABI library loads, exports every entry point the header declares, and
its struct layouts match the ctypes mirrors. No device calls."""
import ctypes as C
import os
import re
import subprocess

import pytest

from garmentcraft_b200 import _abi
from garmentcraft_b200._lib import EXPORTS, LIB_PATH, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "klon3d_step.h")
MESH_HEADER = os.path.join(ROOT, "include", "klon3d_mesh.h")


def header_functions():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names.update(re.findall(r"\b(k3d_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_header_names_every_export():
    assert sorted(EXPORTS) == header_functions()


def test_library_exports_every_symbol():
    L = lib()
    for name in header_functions():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True).stdout
    for name in header_functions():
        assert re.search(rf"\bT {name}$", out, re.M), name


STRUCTS = {
    "k3d_params": _abi.K3dParams, "k3d_simparams": _abi.K3dSimparams, "k3d_body": _abi.K3dBody,
    "k3d_scene": _abi.K3dScene, "k3d_stats": _abi.K3dStats, "k3d_cg_result": _abi.K3dCgResult,
    "k3d_system_readback": _abi.K3dSystemReadback, "k3d_material": _abi.K3dMaterial,
    "k3d_piece": _abi.K3dPiece, "k3d_seam_part": _abi.K3dSeamPart, "k3d_seam": _abi.K3dSeam,
    "k3d_pattern": _abi.K3dPattern, "k3d_mesh_info": _abi.K3dMeshInfo,
}


def test_struct_layouts_match(tmp_path):
    src = tmp_path / "sizes.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', f'#include "{MESH_HEADER}"',
             "int main(void){"]
    for name, cls in STRUCTS.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for name, cls in STRUCTS.items():
        assert int(got[name]) == C.sizeof(cls), name
        for f, _ in cls._fields_:
            assert int(got[f"{name}.{f}"]) == getattr(cls, f).offset, f"{name}.{f}"


def test_defaults_match_reference():
    # ImplizitParameter::default (implizit.rs:505-531), Simparameter::default (szene.rs:115-126)
    p = _abi.K3dParams()
    lib().k3d_params_default(C.byref(p))
    assert (p.schritte_je_bild, p.cg_max, p.cg_toleranz, p.naht_k, p.kontakt_rand) == (5, 50, 1e-5, 500.0, 1e-4)
    assert p.normalkraft_aus_last == 0 and p.durchstoss_pruefen == 1 and p.selbstkollision == 0
    from garmentcraft_b200.params import ImplizitParameter
    q = ImplizitParameter().to_c()
    for f, _ in _abi.K3dParams._fields_:
        if f != "reserved":
            assert getattr(p, f) == getattr(q, f), f
    s = _abi.K3dSimparams()
    lib().k3d_simparams_default(C.byref(s))
    assert s.bild_dt == 1.0 / 60.0 and tuple(s.schwerkraft) == (0.0, 0.0, -9.81) and s.daempfung == 0.0


def test_solver_without_device_reports_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    L = lib()
    h = L.k3d_solver_create(None, 0)
    assert h
    s = _abi.K3dScene()
    assert L.k3d_upload_scene(h, C.byref(s)) == _abi.K3D_DEVICE_ERROR
    assert L.k3d_last_error(h)
    L.k3d_solver_destroy(h)
