"""k3d_operator_noalloc against k3d_operator.

The no-allocation entry point serves callers that may not allocate device
memory themselves — an application that owns the whole device budget in its
own pool, a real-time loop that must not wait in the driver's allocator. It
must give the same A p as the handle-based operator and as the oracle's (FP64,
tolerance 1e-12 relative in norm, as the operator parity tests use), twice in
a row on the same static scratch, also on the sheared state whose PSD
projection needs the build's rounding.

This file is collected last on purpose, so a run that stops at the first
failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import _abi, synth
from garmentcraft_b200._lib import lib
from garmentcraft_b200.implizit import ImplizitCg, build_scene
from garmentcraft_b200.params import ImplizitParameter
from garmentcraft_b200.szene import _ARRAYS

def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def device_scene(s, torch):
    """k3d_scene whose every array is a CUDA copy (kept alive in `keep`)."""
    keep = {}
    cs = _abi.K3dScene()
    cs.n_punkte = s.x.shape[0]
    cs.n_abstand = s.abstand_punkte.shape[0]
    cs.n_naht = s.naht_punkte.shape[0]
    cs.n_biegung = s.biegung_punkte.shape[0]
    cs.n_membran = s.membran_punkte.shape[0]
    cs.n_dreiecke = s.dreiecke.shape[0]
    ctype = {np.float64: C.c_double, np.uint32: C.c_uint32, np.uint8: C.c_uint8, np.int64: C.c_int64,
             np.int32: C.c_int32}
    for name, (dt, _) in _ARRAYS.items():
        a = np.ascontiguousarray(getattr(s, name), dtype=dt)
        raw = np.frombuffer(a.tobytes(), dtype=np.uint8).copy() if a.size else np.zeros(8, np.uint8)
        t = torch.from_numpy(raw).cuda()
        keep[name] = t
        setattr(cs, name, C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ctype[dt])))
    cs.n_koerper = 0
    cs.param = s.param.to_c()
    return cs, keep


def call(cs, prm, pd, out, torch):
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib().k3d_operator_noalloc(C.byref(prm), C.byref(cs), C.c_void_p(pd.data_ptr()),
                                      C.c_void_p(out.data_ptr()), stream)


@pytest.mark.gpu
def test_operator_noalloc_matches_operator_twice():
    torch = pytest.importorskip("torch")
    m, body = synth.tube()
    s = build_scene(m, [body])
    par = ImplizitParameter()
    orc = O.OracleSim(s, par.to_c())
    orc.frames(3)  # a strained state, v != 0
    x, v = orc.state()
    s.x[:], s.v[:] = x, v
    cg = ImplizitCg(par)
    w = np.arange(s.n)[:, None] * 0.6180339887498949 * np.array([1.0, 2.0, 3.0])
    vectors = [np.tile([1.0, 0.0, 0.0], (s.n, 1)), (w % 1.0) - 0.5, v.copy()]
    cs, keep = device_scene(s, torch)
    prm = par.to_c()
    L = lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for p in vectors:
        ref = cg.operator(s, p)
        pd = torch.from_numpy(np.ascontiguousarray(p)).cuda()
        for _ in range(2):  # the scratch keeps the last call's contents
            out = torch.full((s.n, 3), float("nan"), dtype=torch.float64, device="cuda")
            st = L.k3d_operator_noalloc(C.byref(prm), C.byref(cs), C.c_void_p(pd.data_ptr()),
                                        C.c_void_p(out.data_ptr()), stream)
            assert st == _abi.K3D_OK
            got = out.cpu().numpy()
            assert rel(got, ref) <= 1e-12, rel(got, ref)
    del keep


@pytest.mark.gpu
def test_operator_noalloc_sheared_state_matches_oracle():
    # the sheared sheet of test_operator_gescherter_zustand: warp strain clamped,
    # shear small, where the PSD projection of the geometric stress cancels
    torch = pytest.importorskip("torch")
    p, tri = synth.rechteck_netz(200.0, 200.0, 20, 20)
    lage = np.stack([p[:, 0] * 1e-3, p[:, 1] * 1e-3, np.zeros(p.shape[0])], axis=1)
    m = synth.Muster([synth.Teil(p, tri, (1.0, 0.0), synth.RADICAL_RUBBER_04, lage)], [],
                     synth.Simparameter(bild_dt=1.0 / 30.0, daempfung=1.0))
    s = build_scene(m)
    rng = np.random.default_rng(5)
    s.x[:, :2] += rng.uniform(-2e-4, 2e-4, size=(s.n, 2))
    s.x[:, 2] += rng.uniform(-1e-4, 1e-4, size=s.n)
    par = ImplizitParameter()
    orc = O.OracleSim(s, par.to_c())
    cs, keep = device_scene(s, torch)
    prm = par.to_c()
    for q in [rng.normal(size=(s.n, 3)), (np.arange(3 * s.n).reshape(s.n, 3) * 0.7548776662466927) % 1.0 - 0.5]:
        ref = orc.operator(q)
        pd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
        for _ in range(2):
            out = torch.full((s.n, 3), float("nan"), dtype=torch.float64, device="cuda")
            assert call(cs, prm, pd, out, torch) == _abi.K3D_OK
            got = out.cpu().numpy()
            assert rel(got, ref) <= 1e-12, rel(got, ref)
    del keep


@pytest.mark.gpu
def test_operator_noalloc_non_finite_input():
    torch = pytest.importorskip("torch")
    m, body = synth.tube()
    s = build_scene(m, [body])
    par = ImplizitParameter()
    cs, keep = device_scene(s, torch)
    prm = par.to_c()
    q = np.ones((s.n, 3))
    q[7, 1] = np.nan
    pd = torch.from_numpy(q).cuda()
    out = torch.zeros((s.n, 3), dtype=torch.float64, device="cuda")
    assert call(cs, prm, pd, out, torch) == _abi.K3D_NON_FINITE
    assert torch.isnan(out).all()
    # the next call on the same scratch is clean again
    pd = torch.ones((s.n, 3), dtype=torch.float64, device="cuda")
    assert call(cs, prm, pd, out, torch) == _abi.K3D_OK
    assert torch.isfinite(out).all()
    del keep


def test_operator_noalloc_rejects_self_collision():
    # no device work: the call refuses before it touches a pointer
    m, body = synth.tube()
    s = build_scene(m, [body])
    cs, keep = s.to_c()
    prm = ImplizitParameter(selbstkollision=True).to_c()
    dummy = np.zeros(3)
    st = lib().k3d_operator_noalloc(C.byref(prm), C.byref(cs), C.c_void_p(dummy.ctypes.data),
                                    C.c_void_p(dummy.ctypes.data), None)
    assert st == _abi.K3D_BAD_ARGUMENT


def test_operator_noalloc_rejects_too_many_points():
    m, body = synth.tube()
    s = build_scene(m, [body])
    cs, keep = s.to_c()
    cs.n_punkte = 131073
    prm = ImplizitParameter().to_c()
    dummy = np.zeros(3)
    st = lib().k3d_operator_noalloc(C.byref(prm), C.byref(cs), C.c_void_p(dummy.ctypes.data),
                                    C.c_void_p(dummy.ctypes.data), None)
    assert st == _abi.K3D_BAD_ARGUMENT
