"""Self-collision proximity stage on the device against the FP64 oracle.

Bit-exact (the stage's kernels round every operation on its own, like the
reference): hash bucket starts and entries, the proximity pairs (order,
points, weights, normals, distances, rest), the springs' forces, and the
velocities after the approach damping. Through the whole system: operator
1e-12 relative (FP64) and 2e-5 (mixed), system readback 1e-11, frames 1e-9 of
the bounding-box diagonal with identical pair counts. The reference's
two-layer test (sim/tests/selbstkollision.rs:34-64) on the device in both
forms.
"""
import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import _abi, synth
from garmentcraft_b200.implizit import ImplizitCg, build_scene
from garmentcraft_b200.params import ImplizitParameter

pytestmark = pytest.mark.gpu

# every upper point over the inside of a lower triangle (see tests/test_oracle_selbst.py)
INSET = dict(oben_groesse_m=0.18, versatz_m=(0.0073, 0.0041))


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def zwei_lagen(abstand_m=0.002, alle_frei=False):
    s = build_scene(synth.zwei_lagen(abstand_m=abstand_m, **INSET))
    if alle_frei:
        s.w[:] = 1.0 / s.masse
    else:
        synth.pin_teil(s, 0)
    return s


def bewegt(s, seed=5):
    """A state with motion in every direction (approaching and separating)."""
    rng = np.random.default_rng(seed)
    s.v[:] = rng.normal(0.0, 0.05, size=s.v.shape)
    s.x[:] = s.x + rng.uniform(-2e-4, 2e-4, size=s.x.shape)
    return s


@pytest.mark.parametrize("prec", [_abi.K3D_FP64, _abi.K3D_MIXED])
def test_hash_und_paare_bitgleich(prec):
    s = bewegt(zwei_lagen(alle_frei=True))
    par = ImplizitParameter(selbstkollision=True, precision=prec)
    cg = ImplizitCg(par)
    cg.system_fuer(s)
    orc = O.OracleSim(s, par.to_c())
    probe = O.SelbstProbe(orc)
    for kanten in (False, True):
        anf_g, ein_g = cg.selbst_hash(kanten)
        anf_o, ein_o = probe.hash(s.x, kanten)
        assert np.array_equal(anf_g, anf_o)
        assert np.array_equal(ein_g, ein_o)
    g, o = cg.selbst_paare(), probe.finde(s.x)
    assert o["punkte"].shape[0] > 100
    assert (o["art"] == 0).sum() > 0 and (o["art"] == 1).sum() > 0
    for k in ("art", "punkte"):
        assert np.array_equal(g[k], o[k]), k
    for k in ("gewichte", "normale", "abstand", "ruhe"):
        assert np.array_equal(g[k].view(np.uint64), o[k].view(np.uint64)), k


def test_federn_und_daempfung_bitgleich():
    s = bewegt(zwei_lagen(alle_frei=True), seed=9)
    x0, v0 = s.x.copy(), s.v.copy()
    par = ImplizitParameter(selbstkollision=True)
    cg = ImplizitCg(par)
    cg.system_fuer(s)
    fe = cg.selbst_federn()
    s2 = s.copy()
    cg.zustand_lesen(s2)
    orc = O.OracleSim(s, par.to_c())
    fo, vd = O.SelbstProbe(orc).federn(x0, v0)
    assert fo["kraft"].shape[0] > 100
    assert np.array_equal(fe["kraft"].view(np.uint64), fo["kraft"].view(np.uint64))
    iu = np.triu_indices(3)
    assert np.array_equal(fe["block"][:, iu[0], iu[1]].view(np.uint64), fo["block"][:, iu[0], iu[1]].view(np.uint64))
    assert np.max(np.abs(fe["block"] - fo["block"])) <= 1e-15 * np.abs(fo["block"]).max()
    assert not np.array_equal(vd, v0)  # approaching pairs were damped
    assert np.array_equal(s2.v.view(np.uint64), vd.view(np.uint64))
    assert np.array_equal(s2.x, x0)


@pytest.mark.parametrize("prec,tol", [(_abi.K3D_FP64, 1e-12), (_abi.K3D_MIXED, 2e-5)])
def test_operator_mit_federn(prec, tol):
    s = bewegt(zwei_lagen(), seed=2)
    par = ImplizitParameter(selbstkollision=True, precision=prec)
    cg = ImplizitCg(par)
    orc = O.OracleSim(s, par.to_c())
    rng = np.random.default_rng(1)
    for p in [rng.normal(size=(s.n, 3)), np.tile([0.0, 0.0, 1.0], (s.n, 1))]:
        orc.set_state(s.x, s.v)
        a = orc.operator(p)
        b = cg.operator(s, p)
        assert rel(b, a) <= tol


def test_system_mit_federn():
    s = bewegt(zwei_lagen(), seed=4)
    par = ImplizitParameter(selbstkollision=True, schritte_je_bild=1)
    orc = O.OracleSim(s, par.to_c())
    cg = ImplizitCg(par)
    g, o = cg.system_fuer(s), orc.system()
    assert rel(g["rhs"], o["rhs"]) <= 1e-11
    assert rel(g["f"], o["f"]) <= 1e-11
    assert np.max(np.abs(g["pinv"] - o["pinv"]) / np.abs(o["pinv"]).max(axis=(1, 2))[:, None, None]) <= 1e-10


def test_bilder_wie_cpu():
    # the upper layer lands on the lower one within these frames; solved
    # tightly, the device and the oracle stay within 1e-9 of the diagonal
    s = zwei_lagen(abstand_m=0.006)
    par = ImplizitParameter(selbstkollision=True, cg_max=4000, cg_toleranz=1e-12)
    orc = O.OracleSim(s, par.to_c())
    cg = ImplizitCg(par)
    d = float(np.linalg.norm(s.x.max(0) - s.x.min(0)))
    paare_g = paare_o = 0
    for _ in range(8):
        cg.bild(s)
        so = orc.frames(1)
        paare_g += cg.statistik.naehe_punkt_dreieck + cg.statistik.naehe_kante_kante
        paare_o += so.naehe_punkt_dreieck + so.naehe_kante_kante
        x, v = orc.state()
        assert np.max(np.abs(s.x - x)) <= 1e-9 * d
    assert paare_g == paare_o and paare_g > 0


@pytest.mark.parametrize("prec", [_abi.K3D_FP64, _abi.K3D_MIXED])
def test_obere_lage_bleibt_liegen(prec):
    """sim/tests/selbstkollision.rs:34-64 on the device."""
    s = zwei_lagen(abstand_m=0.01)
    oben = slice(int(s.teil_bereiche[1, 0]), int(s.teil_bereiche[1, 1]))
    cg = ImplizitCg(ImplizitParameter(precision=prec))
    for _ in range(30):
        cg.bild(s)
    assert s.x[oben, 2].min() < -0.05
    s = zwei_lagen(abstand_m=0.01)
    cg = ImplizitCg(ImplizitParameter(selbstkollision=True, precision=prec))
    paare = 0
    for _ in range(60):
        cg.bild(s)
        paare = cg.statistik.naehe_punkt_dreieck + cg.statistik.naehe_kante_kante
    z, hoechster = s.x[oben, 2].min(), s.x[oben, 2].max()
    assert paare > 0
    assert z > 2.0e-3 and hoechster < 3.2e-3, (z, hoechster)


def test_ohne_selbstkollision_kein_lauf():
    s = zwei_lagen()
    cg = ImplizitCg(ImplizitParameter())
    cg.system_fuer(s)
    with pytest.raises(Exception):
        cg.selbst_paare()
