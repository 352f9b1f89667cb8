"""Pins the FP64 oracle to the reference's own known-answer tests.

Each test restates one test of viktoschi/GarmentCraft (crates/klon3d-sim),
with the values and tolerances that test asserts. The reference is Rust and
cannot run here, so these known answers are what ties the oracle to it.
"""
import math

import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import _abi, synth
from garmentcraft_b200.params import ImplizitParameter
from garmentcraft_b200.szene import Szene
from garmentcraft_b200.synth import RADICAL_RUBBER_04, Simparameter

import ctypes as C

D = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def steif(weft, warp, bias, theta):
    return O.lib().orc_steifigkeit(weft, warp, bias, theta)


WEFT, WARP, BIAS = 2482.2424e-9, 2486.4924e-9, 2486.4924e-9


# ---------------------------------------------------------------- sim/src/biegung.rs:186-309
def test_biegung_isotrop_bitgleich():
    # biegung.rs:186-199
    for d in [WEFT, 1.0e-12, 0.0, 6.0361e-8, 1.0e9]:
        for i in range(73):
            theta = i * (math.pi / 2) / 72.0
            assert steif(d, d, d, theta) == d


def test_biegung_drei_richtungen():
    # biegung.rs:202-218
    assert steif(WEFT, WARP, BIAS, 0.0) == WARP
    assert steif(WEFT, WARP, BIAS, math.pi / 2) == WEFT
    assert abs(steif(WEFT, WARP, BIAS, math.pi / 4) - BIAS) <= 1e-15 * BIAS


def test_biegung_weiche_schraege_minimum():
    # biegung.rs:229-262: D = (2, 3, 0.8), minimum 519/680 at 49.228260 deg
    weft, warp, bias = 2.0, 3.0, 0.8
    a = 2.0 * (weft + warp - 2.0 * bias)
    b = 4.0 * bias - warp - 3.0 * weft
    u = -b / (2.0 * a)
    theta = math.acos(math.sqrt(u))
    assert abs(math.degrees(theta) - 49.228260) < 1e-5
    m = steif(weft, warp, bias, theta)
    assert abs(m - 519.0 / 680.0) <= 1e-13 * (519.0 / 680.0)
    for i in range(3601):
        th = i * (math.pi / 2) / 3600.0
        assert steif(weft, warp, bias, th) >= m - 2e-7 * (519.0 / 680.0)


def test_biegung_acht_stoffe_nur_steifer():
    # biegung.rs:269-287: min = weft, max +0.1926 % near 30 deg
    vals = [steif(WEFT, WARP, BIAS, i * (math.pi / 2) / 1800.0) for i in range(1801)]
    assert abs(min(vals) - WEFT) < 1e-18
    rel = (max(vals) - WEFT) / WEFT
    assert abs(rel - 0.001926) < 2e-6
    assert max(vals) > WARP


def test_biegung_negative_boden():
    # biegung.rs:293-309: floor 1e-3 * softest direction
    weft, warp, bias = 1.0e-6, 10.0e-6, 1.0e-8
    hits = 0
    for i in range(3601):
        d = steif(weft, warp, bias, i * (math.pi / 2) / 3600.0)
        assert d > 0.0 and d >= 1.0e-3 * bias * (1.0 - 1e-12)
        if d <= 1.0e-3 * bias * 1.000001:
            hits += 1
    assert hits > 0
    assert steif(weft, warp, bias, 1.0) > 0.0


# ---------------------------------------------------------------- sim/src/cpu.rs:343-361
def dieder(q):
    th = C.c_double()
    g = np.zeros(12)
    ok = O.lib().orc_dieder(D(np.asarray(q, float).ravel()), C.byref(th), D(g))
    return (th.value, g.reshape(4, 3)) if ok else None


def test_dieder_gradient_wie_differenzen():
    q = np.array([[0.0, 0.0, 0.0], [1.0, 0.1, 0.0], [0.4, 0.9, 0.3], [0.6, -0.8, 0.5]])
    t, g = dieder(q)
    eps = 1e-7
    for k in range(4):
        for a in range(3):
            qp = q.copy(); qp[k, a] += eps
            qm = q.copy(); qm[k, a] -= eps
            d = (dieder(qp)[0] - dieder(qm)[0]) / (2 * eps)
            assert abs(d - g[k, a]) < 1e-5
    f = [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.5, 1.0, 0.0], [0.5, -1.0, 0.0]]
    assert abs(dieder(f)[0]) < 1e-12
    assert abs(t) > 0.1


def test_winkel_fehler_wrap():
    # cpu.rs:271-282: the difference is taken the short way round
    wf = O.lib().orc_winkel_fehler
    assert abs(wf(math.radians(-179.99), math.radians(179.99)) - math.radians(0.02)) < 1e-12
    assert wf(0.3, 0.0) == 0.3


# ---------------------------------------------------------------- sim/src/implizit.rs:1122-1132
def test_inverse_3x3():
    m = np.array([[4.0, 1.0, 0.5], [1.0, 3.0, 0.2], [0.5, 0.2, 2.0]])
    out = np.zeros(9)
    O.lib().orc_m3_inv(D(m.ravel()), D(out))
    assert np.all(np.abs(m @ out.reshape(3, 3) - np.eye(3)) < 1e-12)


# ---------------------------------------------------------------- sim/src/faerbung.rs:59-82
def test_faerbung_keine_farbe_teilt_punkt():
    c = np.array([[0, 1], [1, 2], [2, 3], [3, 4], [5, 0], [5, 1], [5, 2], [5, 3]], dtype=np.uint32)
    farbe = np.zeros(8, dtype=np.uint32)
    ordn = np.zeros(8, dtype=np.int64)
    n = O.lib().orc_faerbe(8, 2, 6, c.ctypes.data_as(C.POINTER(C.c_uint32)),
                           farbe.ctypes.data_as(C.POINTER(C.c_uint32)),
                           ordn.ctypes.data_as(C.POINTER(C.c_int64)))
    assert n >= 4
    for a in range(8):
        for b in range(a + 1, 8):
            if farbe[a] == farbe[b]:
                assert not set(c[a]) & set(c[b])
    assert sorted(ordn.tolist()) == list(range(8))
    assert all(farbe[ordn[i]] <= farbe[ordn[i + 1]] for i in range(7))


# ---------------------------------------------------------------- sim/src/koerper.rs:136-147
def test_zylinder_kontakt():
    body = synth.body_to_c(dict(art=_abi.K3D_BODY_CYLINDER, radius=0.1))
    n = np.zeros(3)
    t = C.c_double()
    assert O.lib().orc_kontakt(C.byref(body), D([0.2, 0.0, 5.0]), 0.001, D(n), C.byref(t)) == 0
    assert O.lib().orc_kontakt(C.byref(body), D([0.0, 0.05, -3.0]), 0.001, D(n), C.byref(t)) == 1
    assert abs(t.value - 0.051) < 1e-12
    assert abs(n[1] - 1.0) < 1e-12


def test_sdf_grid_kugel_kontakt():
    # The sampled grid has no reference counterpart; its ground truth is the
    # analytic sphere. Trilinear value within the grid's interpolation error.
    body = synth.sphere_sdf_grid(0.3, 128, 0.01)
    kb = synth.body_to_c(body)
    rng = np.random.default_rng(5)
    for _ in range(200):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        r = rng.uniform(0.25, 0.35)
        x = d * r
        n = np.zeros(3)
        t = C.c_double()
        hit = O.lib().orc_kontakt(C.byref(kb), D(x), 0.001, D(n), C.byref(t))
        if r < 0.3 + 0.001 - 1e-3:
            assert hit == 1
            assert abs(t.value - (0.301 - r)) < 2e-4
            assert np.dot(n, d) > 0.999
        elif r > 0.301 + 1e-3:
            assert hit == 0


# ---------------------------------------------------------------- membrane, sim/tests/kontinuum.rs
TOL = 0.05


def bauen(ruhe, kanten, dir2, e):
    out = np.zeros(12)
    ok = O.lib().orc_membran_bauen(D(np.asarray(ruhe, float).ravel()), D(kanten), D(dir2), D(e), D(out))
    assert ok
    return out


def einheit(e, dir2):
    ruhe = [[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]
    return bauen(ruhe, [1.0, math.sqrt(2.0), 1.0], dir2, e)


def meval(m, p):
    p = np.asarray(p, float).ravel()
    d3, s3, e, f9, z9, h9 = np.zeros(3), np.zeros(3), C.c_double(), np.zeros(9), np.zeros(9), np.zeros(9)
    O.lib().orc_membran_eval(D(m), D(p), D(d3), D(s3), C.byref(e), D(f9), D(z9), D(h9))
    return dict(dehnung=d3, spannung=s3, energie=e.value, krafte=f9.reshape(3, 3), zug=z9.reshape(3, 3))


def mal_h(m, p, d):
    out = np.zeros(9)
    O.lib().orc_membran_mal_h(D(m), D(np.asarray(p, float).ravel()), D(np.asarray(d, float).ravel()), D(out))
    return out.reshape(3, 3)


def diag_bloecke(m, p):
    out = np.zeros(27)
    O.lib().orc_membran_diag(D(m), D(np.asarray(p, float).ravel()), D(out))
    return out.reshape(3, 3, 3)


RR = (RADICAL_RUBBER_04.kette_n_m, RADICAL_RUBBER_04.dehnung_n_m, RADICAL_RUBBER_04.schub_n_m)


def test_membran_zug_liest_kette():
    # kontinuum.rs tests :100-120
    m = einheit(RR, [1.0, 0.0])
    for lam in [1.02, 1.05]:
        s = meval(m, [[0, 0, 0], [lam, 0, 0], [0, 1, 0]])["spannung"]
        assert abs(s[0] / (lam - 1.0) / RR[0] - 1.0) <= TOL


def test_membran_schub_liest_schub():
    # kontinuum.rs tests :122-142
    m = einheit(RR, [1.0, 0.0])
    for g in [0.02, 0.05]:
        s = meval(m, [[0, 0, 0], [1, 0, 0], [g, 1, 0]])["spannung"]
        assert abs(s[2] / g / RR[2] - 1.0) <= TOL


def test_membran_ni_folgt():
    # kontinuum.rs tests :147-160
    e, g = RR[0], RR[2]
    assert abs(e / (2 * g) - 1.0) < 0.01
    m = einheit(RR, [1.0, 0.0])
    s = meval(m, [[0, 0, 0], [1.05, 0, 0], [0, 1, 0]])["spannung"]
    assert abs(s[1]) < 1e-9


def test_membran_anisotrop():
    # kontinuum.rs tests :165-216
    st = (500.0, 200.0, 150.0)
    m = einheit(st, [1.0, 0.0])
    lam = 1.05
    px = [[0, 0, 0], [lam, 0, 0], [0, 1, 0]]
    py = [[0, 0, 0], [1, 0, 0], [0, lam, 0]]
    sx, sy = meval(m, px)["spannung"], meval(m, py)["spannung"]
    assert abs(sx[0] / (lam - 1) / st[0] - 1) <= TOL
    assert abs(sy[1] / (lam - 1) / st[1] - 1) <= TOL
    assert abs((sx[0] / sy[1]) / (st[0] / st[1]) - 1) <= TOL
    g = einheit(st, [0.0, 1.0])
    assert abs(meval(g, px)["spannung"][1] / (lam - 1) / st[1] - 1) <= TOL
    assert abs(meval(g, py)["spannung"][0] / (lam - 1) / st[0] - 1) <= TOL


def test_membran_starre_drehung():
    # kontinuum.rs tests :220-241
    m = einheit((348.0, 348.0, 174.0), [1.0, 0.0])
    p = np.array([[0, 0, 0], [1.04, 0, 0], [0, 1, 0]], float)
    w = math.pi / 5
    R = np.array([[math.cos(w), -math.sin(w), 0], [math.sin(w), math.cos(w), 0], [0, 0, 1]])
    a, b = meval(m, p), meval(m, p @ R.T)
    assert abs(b["energie"] - a["energie"]) <= 1e-12 * max(abs(a["energie"]), 1.0)
    assert np.all(np.abs(b["dehnung"] - a["dehnung"]) < 1e-12)


def test_membran_tangente_ist_ableitung():
    # kontinuum.rs tests :247-303
    m = einheit((348.0, 300.0, 174.0), [1.0, 0.0])
    p = np.array([[0, 0, 0], [1.04, 0.002, 0.01], [0.003, 1.02, -0.008]])
    d = np.array([[-0.7, 0.4, 0.9], [0.3, 0.1, 0.4], [1.3, -0.2, -0.1]])
    hd = mal_h(m, p, d)
    eps = 1e-7
    fp, fm = meval(m, p + eps * d)["krafte"], meval(m, p - eps * d)["krafte"]
    fd = -(fp - fm) / (2 * eps)
    skala = np.maximum(np.maximum(np.abs(hd), np.abs(fd)), 1.0)
    assert np.all(np.abs(hd - fd) <= 2e-5 * skala)
    flach = [[0, 0, 0], [1.04, 0, 0], [0, 1.02, 0]]
    quer = mal_h(m, flach, [[0, 0, 1], [0, 0, 0], [0, 0, 0]])
    assert abs(quer[0, 2]) > 1e-3
    dg = diag_bloecke(m, p)
    for k in range(3):
        for c in range(3):
            e = np.zeros((3, 3)); e[k, c] = 1.0
            spalte = mal_h(m, p, e)
            assert abs(dg[k, c, c] - spalte[k, c]) <= 1e-9 * max(abs(spalte[k, c]), 1.0)


def test_membran_kraft_ist_gradient():
    # kontinuum.rs tests :306-333
    m = einheit((348.0, 300.0, 174.0), [1.0, 0.0])
    p = np.array([[0, 0, 0], [1.04, 0.002, 0.0], [0.003, 0.99, 0.001]])
    f = meval(m, p)["krafte"]
    eps = 1e-7
    for k in range(3):
        for c in range(3):
            pp = p.copy(); pp[k, c] += eps
            pm = p.copy(); pm[k, c] -= eps
            fd = -(meval(m, pp)["energie"] - meval(m, pm)["energie"]) / (2 * eps)
            assert abs(fd - f[k, c]) <= 1e-5 * max(abs(f[k, c]), 1.0)
    assert np.all(np.abs(f.sum(axis=0)) < 1e-12)


def test_membran_basis_nicht_einheit():
    # kontinuum.rs tests :587-645
    ruhe = np.array([[0.0, 0.0], [0.2, 0.0], [0.05, 0.04]])
    l = lambda a, b: float(np.linalg.norm(b - a))
    kanten = [l(ruhe[0], ruhe[1]), l(ruhe[1], ruhe[2]), l(ruhe[2], ruhe[0])]
    st = (348.0, 348.0, 174.0)
    m = bauen(ruhe, kanten, [1.0, 1.0], st)
    kette, schuss = m[5:7], m[7:9]
    w = math.sqrt(0.5)
    assert np.all(np.abs(kette - [w, w]) < 1e-12)
    assert abs(np.dot(kette, schuss)) < 1e-12
    assert abs(np.linalg.norm(schuss) - 1.0) < 1e-12
    lam = 1.05
    F = np.eye(2) + (lam - 1.0) * np.outer(kette, kette)
    d1, d2 = ruhe[1] - ruhe[0], ruhe[2] - ruhe[0]
    p = [[0, 0, 0], [*(F @ d1), 0.0], [*(F @ d2), 0.0]]
    r = meval(m, p)
    assert abs(r["dehnung"][0] - 0.5 * (lam * lam - 1)) < 1e-12
    assert abs(r["dehnung"][1]) < 1e-12 and abs(r["dehnung"][2]) < 1e-12
    assert abs(r["spannung"][0] / (lam - 1) / st[0] - 1) <= TOL
    assert abs(r["spannung"][1]) < 1e-9 and abs(r["spannung"][2]) < 1e-9


# ---------------------------------------------------------------- sim/src/implizit.rs:1067-1120
def zwei_punkte(ruhe):
    z = np.zeros(0)
    e = lambda *s: np.zeros(s)
    s = Szene(x=np.array([[0.0, 0.0, 0.0], [0.1, 0.0, 0.0]]), v=e(2, 3), masse=np.full(2, 1e-5),
              w=np.full(2, 1e5), kollisionsabstand=np.full(2, 2e-4), reibung=np.zeros(2),
              abstand_punkte=np.zeros((0, 2), np.uint32), abstand_ruhe=z, abstand_nachgiebigkeit=z,
              membran_kante=np.zeros(0, np.uint8), naht_punkte=np.array([[0, 1]], np.uint32),
              naht_ruhe=np.array([ruhe]), biegung_punkte=np.zeros((0, 4), np.uint32), biegung_ruhe=z,
              biegung_nachgiebigkeit=z, membran_punkte=np.zeros((0, 3), np.uint32), membran_flaeche=z,
              membran_ruhe_inv=e(0, 4), membran_kette=e(0, 2), membran_schuss=e(0, 2),
              membran_steif=e(0, 3), dreiecke=np.zeros((0, 3), np.uint32), ruhe_inv=e(0, 4),
              param=Simparameter(schwerkraft=(0.0, 0.0, 0.0), daempfung=5.0))
    return s


def abstand(sim):
    x, _ = sim.state()
    return float(np.linalg.norm(x[1] - x[0]))


def test_naht_mit_ruhelaenge_und_kuerzen():
    sim = O.OracleSim(zwei_punkte(0.04), ImplizitParameter().to_c())
    sim.frames(60)
    assert abs(abstand(sim) - 0.04) < 1e-6
    sim = O.OracleSim(zwei_punkte(0.0), ImplizitParameter().to_c())
    sim.naht_offen()
    groesster = 0.0
    for bild in range(1, 121):
        vorher = abstand(sim)
        sim.naht_kuerzen(1e-3)
        sim.frames(1)
        groesster = max(groesster, vorher - abstand(sim))
        if bild == 30:
            assert abs(abstand(sim) - 0.07) < 1e-4
    assert abstand(sim) < 1e-6
    assert groesster < 1.1e-3


# ---------------------------------------------------------------- tube, analytic hoop strain
def tube_sim(params=None):
    muster, body = synth.tube()
    s = O.build_scene(muster, [body])
    p = params or ImplizitParameter(schritte_je_bild=1, cg_max=2000, cg_toleranz=1e-6)
    return s, O.OracleSim(s, p.to_c())


def test_tube_scene_build():
    s, _ = tube_sim()
    assert s.n == 41 * 21
    assert s.membran_punkte.shape[0] == 1600
    assert s.naht_punkte.shape[0] == 21
    assert s.oracle_counts["membran_entartet"] == 0
    assert s.oracle_counts["naht_biegung_ohne"] == 0
    # interior edges + the 20 seam hinges
    n_inner = 40 * 21 + 41 * 20 + 40 * 20 - (2 * 40 + 2 * 20)
    assert s.biegung_punkte.shape[0] == n_inner + 20
    assert np.all(s.membran_kante == 1)


def test_tube_hoop_strain_analytic():
    """Tube acceptance (sim/tests/roehre.rs:15-20, sim/tests/implizit.rs:41-58):
    circumferential strain within 0.5 pp of the analytic value, seam gap under
    1 mm, lift under 0.5 mm, after 60 implicit steps of 1/60 s."""
    s, sim = tube_sim()
    sim.frames(60)
    R, t = 0.08, synth.TUBE_MATERIAL.dicke_m
    soll = 2 * math.pi * (R + t / 2) / 0.40 - 1.0  # 26.06 %
    u = sim.umfang([0, 0, -0.10], [0, 0, 1])
    dehnung = u / 0.40 - 1.0
    assert abs(dehnung - soll) <= 0.005, (dehnung, soll)
    assert sim.nahtspalt() < 1.0e-3
    x, _ = sim.state()
    abheben = np.max(np.hypot(x[:, 0], x[:, 1]) - (R + t / 2))
    assert abheben < 0.5e-3
    # hoop tension per rest width: T = E_2D * (lambda^2 - 1)/2 (Green strain)
    lam = 1.0 + np.median(sim.dehnung()[:, 0])
    T = 600.0 * 0.5 * (lam * lam - 1.0)
    T_soll = 600.0 * 0.5 * ((1 + soll) ** 2 - 1.0)
    assert abs(T / T_soll - 1.0) < 0.02, (T, T_soll)


# ---------------------------------------------------------------- sim/tests/implizit.rs:7-14, free fall
def test_freier_fall_diskret():
    """Backward Euler covers a*h^2*N(N+1)/2 in N steps under a constant
    acceleration a (`weg_diskret`, sim/tests/implizit.rs:7-14). A free sheet
    at its rest shape stays undeformed (a uniform move is in the stiffness'
    null space), so every point falls exactly that far."""
    muster, _ = synth.sheet_over_sphere(n=17, groesse_m=0.3, jitter_mm=1.0, seed=2)
    s = O.build_scene(muster, [])
    x0 = s.x.copy()
    sim = O.OracleSim(s, ImplizitParameter(schritte_je_bild=1, cg_max=2000, cg_toleranz=1e-12).to_c())
    n = 30
    sim.frames(n)
    x, v = sim.state()
    h, g = muster.param.bild_dt, 9.81
    soll = g * h * h * n * (n + 1) / 2.0
    dz = x0[:, 2] - x[:, 2]
    assert np.max(np.abs(dz / soll - 1.0)) < 1e-9
    assert np.max(np.abs(x[:, :2] - x0[:, :2])) < 1e-12
    assert np.max(np.abs(v[:, 2] + g * h * n)) < 1e-9 * g * h * n
