"""Device step against the FP64 oracle, through the C ABI.

Tolerances: FP64 operator 1e-12 relative (norm), FP64 states after several
frames 1e-9 of the bounding-box diagonal (summation order differs from the
oracle's), mixed FP32/FP64 operator 2e-5 relative.
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import _abi, synth
from garmentcraft_b200.implizit import ImplizitCg, build_scene
from garmentcraft_b200.params import ImplizitParameter

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def diag(x):
    return float(np.linalg.norm(x.max(0) - x.min(0)))


def tube_scene():
    m, body = synth.tube()
    return build_scene(m, [body])


def small_sheet(n=33, seed=3):
    m, body = synth.sheet_over_sphere(n=n, seed=seed, fall_m=0.02)
    return build_scene(m, [body])


def streuung(n):
    w = np.arange(n)[:, None] * 0.6180339887498949 * np.array([1.0, 2.0, 3.0])
    return (w % 1.0) - 0.5


@pytest.mark.parametrize("prec,tol", [(_abi.K3D_FP64, 1e-12), (_abi.K3D_MIXED, 2e-5)])
def test_operator_wie_cpu(prec, tol):
    # sim/tests/gpu.rs:66-110, at the tolerance of each arithmetic
    s = tube_scene()
    par = ImplizitParameter()
    orc = O.OracleSim(s, par.to_c())
    orc.frames(3)
    x, v = orc.state()
    s.x[:], s.v[:] = x, v
    cg = ImplizitCg(ImplizitParameter(precision=prec))
    for p in [np.tile([1.0, 0.0, 0.0], (s.n, 1)), streuung(s.n), v.copy()]:
        a = orc.operator(p)
        b = cg.operator(s, p)
        assert rel(b, a) <= tol


@pytest.mark.parametrize("prec,tol", [(_abi.K3D_FP64, 1e-12), (_abi.K3D_MIXED, 2e-5)])
def test_operator_gescherter_zustand(prec, tol):
    # In-plane distortion with shear stiffness: elements whose warp strain is
    # clamped and whose shear is small sit where the PSD projection of the
    # geometric stress (kontinuum.rs:158-177) cancels; the device's build has
    # to round exactly like the reference there.
    p, tri = synth.rechteck_netz(200.0, 200.0, 20, 20)
    lage = np.stack([p[:, 0] * 1e-3, p[:, 1] * 1e-3, np.zeros(p.shape[0])], axis=1)
    m = synth.Muster([synth.Teil(p, tri, (1.0, 0.0), synth.RADICAL_RUBBER_04, lage)], [],
                     synth.Simparameter(bild_dt=1.0 / 30.0, daempfung=1.0))
    s = build_scene(m)
    rng = np.random.default_rng(5)
    s.x[:, :2] += rng.uniform(-2e-4, 2e-4, size=(s.n, 2))
    s.x[:, 2] += rng.uniform(-1e-4, 1e-4, size=s.n)
    orc = O.OracleSim(s, ImplizitParameter().to_c())
    cg = ImplizitCg(ImplizitParameter(precision=prec))
    for q in [rng.normal(size=(s.n, 3)), streuung(s.n)]:
        assert rel(cg.operator(s, q), orc.operator(q)) <= tol
    if prec == _abi.K3D_FP64:
        g, o = cg.system_fuer(s), orc.system()
        assert rel(g["rhs"], o["rhs"]) <= 1e-11
        assert np.max(np.abs(g["pinv"] - o["pinv"]) / np.abs(o["pinv"]).max(axis=(1, 2))[:, None, None]) <= 1e-10


def test_system_wie_cpu():
    s = small_sheet()
    par = ImplizitParameter(schritte_je_bild=1)
    orc = O.OracleSim(s, par.to_c())
    orc.frames(8)  # the sheet is on the sphere now: contacts exist
    x, v = orc.state()
    s.x[:], s.v[:] = x, v
    cg = ImplizitCg(par)
    g, o = cg.system_fuer(s), orc.system()
    assert np.array_equal(g["fest"], o["fest"])
    assert g["fest"].sum() > 0
    assert rel(g["rhs"], o["rhs"]) <= 1e-11
    assert rel(g["f"], o["f"]) <= 1e-11
    assert rel(g["last"], o["last"]) <= 1e-11
    assert np.max(np.abs(g["pinv"] - o["pinv"]) / np.abs(o["pinv"]).max(axis=(1, 2))[:, None, None]) <= 1e-10
    assert np.max(np.abs(g["normale"] - o["normale"])) <= 1e-12
    assert np.max(np.abs(g["vn_soll"] - o["vn_soll"])) <= 1e-9 * max(1.0, np.abs(o["vn_soll"]).max())


def test_loese_wie_cpu():
    # well conditioned (tube, solved to 1e-12): the two solutions agree to 1e-9
    s = tube_scene()
    par = ImplizitParameter(schritte_je_bild=1, cg_max=4000, cg_toleranz=1e-12)
    orc = O.OracleSim(s, par.to_c())
    orc.frames(3)
    x, v = orc.state()
    s.x[:], s.v[:] = x, v
    dv0 = orc.dv_warm()
    a, la = orc.solve(dv0)
    b, lb = ImplizitCg(par).loese(s, dv0)
    assert abs(la.iterationen - lb.iterationen) <= 2
    assert rel(b, a) <= 1e-9
    r_o = O.OracleSim(s, par.to_c())
    assert rel(ImplizitCg(par).rest_geloest(s, a), r_o.operator(a) - r_o.system()["rhs"]) <= 1e-10


def test_loese_mit_vorgegebenem_kontaktsatz():
    # Loeser::loese takes the contact set from its caller (implizit.rs:308,
    # 870-883). The tube's own set gives the device's own solve; a changed set
    # (every third held point released, the others' normal velocity shifted)
    # is honoured, and both match the oracle's solve with the same set to 1e-9.
    s = tube_scene()
    par = ImplizitParameter(schritte_je_bild=1, cg_max=4000, cg_toleranz=1e-12)
    orc = O.OracleSim(s, par.to_c())
    orc.frames(3)
    x, v = orc.state()
    s.x[:], s.v[:] = x, v
    dv0 = orc.dv_warm()
    sysr = orc.system()
    eigen = {"fest": sysr["fest"], "normale": sysr["normale"], "vn_soll": sysr["vn_soll"]}
    assert eigen["fest"].sum() > 10
    cg = ImplizitCg(par)
    a, _ = cg.loese(s, dv0, fest=eigen)
    b, _ = cg.loese(s, dv0)
    assert rel(a, b) <= 1e-12
    ao, _ = orc.solve_contacts(dv0, eigen)
    assert rel(a, ao) <= 1e-9
    held = np.flatnonzero(eigen["fest"])
    anders = {k: v.copy() for k, v in eigen.items()}
    anders["fest"][held[::3]] = 0
    anders["normale"][held[::3]] = 0.0
    anders["vn_soll"][held[1::3]] += 0.01
    c, lc = cg.loese(s, dv0, fest=anders)
    co, lo = orc.solve_contacts(dv0, anders)
    assert abs(lc.iterationen - lo.iterationen) <= 2
    assert rel(c, co) <= 1e-9
    assert rel(c, a) > 1e-6  # the set is honoured


def test_loese_sheet_innerhalb_der_toleranz():
    # ill conditioned (sheet on the sphere, tol 1e-8): the solutions differ by
    # rounding amplified by the condition number; both meet the tolerance and
    # agree far inside the step's own accuracy
    s = small_sheet()
    par = ImplizitParameter(schritte_je_bild=1, cg_max=4000, cg_toleranz=1e-8)
    orc = O.OracleSim(s, par.to_c())
    orc.frames(8)
    x, v = orc.state()
    s.x[:], s.v[:] = x, v
    dv0 = np.tile([0.0, 0.0, -9.81 / 120.0], (s.n, 1))
    a, la = orc.solve(dv0)
    b, lb = ImplizitCg(par).loese(s, dv0)
    assert not la.nicht_konvergiert and not lb.nicht_konvergiert
    assert abs(la.iterationen - lb.iterationen) <= max(2, la.iterationen // 20)
    assert rel(b, a) <= 1e-5


def test_tube_frames_wie_cpu():
    s = tube_scene()
    par = ImplizitParameter(schritte_je_bild=1, cg_max=2000, cg_toleranz=1e-6)
    orc = O.OracleSim(s, par.to_c())
    cg = ImplizitCg(par)
    for _ in range(10):
        orc.frames(1)
        cg.bild(s)
    x, v = orc.state()
    assert np.max(np.abs(s.x - x)) <= 1e-9 * diag(x)
    assert cg.statistik.kontakte > 0


def test_sheet_frames_wie_cpu():
    # solved to 1e-12 so the solver's own error is at rounding level; the
    # sheet lands on the sphere within these frames (contacts, release test,
    # friction)
    s = small_sheet()
    par = ImplizitParameter(schritte_je_bild=1, cg_max=20000, cg_toleranz=1e-12)
    orc = O.OracleSim(s, par.to_c())
    cg = ImplizitCg(par)
    kontakte = 0
    for _ in range(15):
        st_o = orc.frames(1)
        cg.bild(s)
        assert cg.statistik.kontakte == st_o.kontakte
        kontakte += st_o.kontakte
    x, _ = orc.state()
    assert kontakte > 0
    assert np.max(np.abs(s.x - x)) <= 1e-9 * diag(x)


def test_naht_mit_ruhelaenge_gpu():
    # sim/src/implizit.rs:1067-1120 on the device
    import test_oracle_golden as G
    s = G.zwei_punkte(0.04)
    cg = ImplizitCg(ImplizitParameter())
    for _ in range(60):
        cg.bild(s)
    assert abs(np.linalg.norm(s.x[1] - s.x[0]) - 0.04) < 1e-6
    s = G.zwei_punkte(0.0)
    s.naht_offen()
    cg = ImplizitCg(ImplizitParameter())
    groesster = 0.0
    for bild in range(1, 121):
        vorher = np.linalg.norm(s.x[1] - s.x[0])
        s.naht_kuerzen(1e-3)
        cg.bild(s)
        d = np.linalg.norm(s.x[1] - s.x[0])
        groesster = max(groesster, vorher - d)
        if bild == 30:
            assert abs(d - 0.07) < 1e-4
    assert np.linalg.norm(s.x[1] - s.x[0]) < 1e-6
    assert groesster < 1.1e-3


def test_tube_analytic_gpu():
    s = tube_scene()
    cg = ImplizitCg(ImplizitParameter(schritte_je_bild=1, cg_max=2000, cg_toleranz=1e-6))
    for _ in range(60):
        cg.bild(s)
    orc = O.OracleSim(s, ImplizitParameter().to_c())
    u = orc.umfang([0, 0, -0.10], [0, 0, 1])
    soll = 2 * math.pi * (0.08 + 0.25e-3) / 0.40 - 1.0
    assert abs(u / 0.40 - 1.0 - soll) <= 0.005
    assert orc.nahtspalt() < 1e-3


def test_mixed_step_error_against_fp64():
    """One step of the mixed form against one FP64 step from the same state,
    at eight states along a drop onto the sphere (converged solves, tol 1e-5).

    A solve that stops at tol 1e-5 is accurate to that tolerance, so two
    correct FP64 implementations already differ after one step (here: the
    device FP64 form against the oracle). The mixed form must stay within a
    small multiple of that spread, and under 1e-5 of the bounding-box
    diagonal per step."""
    ref = small_sheet(n=65)
    par64 = ImplizitParameter(schritte_je_bild=1, cg_max=4000)
    par32 = ImplizitParameter(schritte_je_bild=1, cg_max=4000, precision=_abi.K3D_MIXED)
    traj = ImplizitCg(par64)
    worst32, worst64 = 0.0, 0.0
    for _ in range(8):
        traj.bilder_resident(ref, 6)
        s64, s32 = ref.copy(), ref.copy()
        ImplizitCg(par64).bild(s64)
        ImplizitCg(par32).bild(s32)
        orc = O.OracleSim(ref, par64.to_c())
        orc.frames(1)
        xo, _ = orc.state()
        d = diag(s64.x)
        worst32 = max(worst32, float(np.max(np.linalg.norm(s32.x - s64.x, axis=1)) / d))
        worst64 = max(worst64, float(np.max(np.linalg.norm(s64.x - xo, axis=1)) / d))
    assert worst32 <= 1e-5, (worst32, worst64)
    assert worst32 <= 10.0 * worst64 + 1e-8, (worst32, worst64)


def test_deterministic():
    a, b = small_sheet(), small_sheet()
    for s in (a, b):
        ImplizitCg(ImplizitParameter(schritte_je_bild=1)).bilder_resident(s, 10)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.v, b.v)


def test_nonfinite_is_reported():
    s = small_sheet()
    s.x[5, 2] = np.nan
    cg = ImplizitCg(ImplizitParameter(schritte_je_bild=1))
    with pytest.raises(Exception) as e:
        cg.bild(s)
    assert "NON_FINITE" in str(e.value)


def test_bad_index_is_rejected():
    s = small_sheet()
    s.membran_punkte[0, 0] = s.n + 5
    cg = ImplizitCg(ImplizitParameter())
    with pytest.raises(Exception) as e:
        cg.bild(s)
    assert "BAD_ARGUMENT" in str(e.value)
