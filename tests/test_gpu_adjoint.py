"""The device adjoint against the oracle's FP64 CPU adjoint and against
central differences of the device forward.

The oracle's adjoint takes its element and contact derivatives by local
central differences of its own functions, the device by forward-mode dual
numbers; both freeze the forward's discrete decisions. Scenes start from a
state reached by earlier frames (away from the rest state, where every
membrane strain sits on the clamp of the geometric stress).
"""
import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import _abi, synth
from garmentcraft_b200.adjoint import Drapierung, DrapeFunction, Stoff
from garmentcraft_b200.implizit import ImplizitCg, K3dError, build_scene
from garmentcraft_b200.params import ImplizitParameter

pytestmark = pytest.mark.gpu


def param(prec=_abi.K3D_FP64, tol=1e-14):
    return ImplizitParameter(schritte_je_bild=1, cg_max=100000, cg_toleranz=tol, precision=prec)


def haengend():
    m, _ = synth.sheet_over_sphere(n=9, groesse_m=0.2, jitter_mm=2.0, seed=5, fall_m=0.3)
    s = build_scene(m, [])
    s.w[0] = 0.0
    s.w[8] = 0.0
    s.param.daempfung = 0.5
    return s


def auf_kugel():
    m, body = synth.sheet_over_sphere(n=9, groesse_m=0.3, jitter_mm=2.0, seed=5, fall_m=0.002,
                                      kugel_radius_m=0.1, sdf_n=48, sdf_spacing_m=0.006)
    return build_scene(m, [body])


def vorlauf(s, n):
    o = O.OracleSim(s, param().to_c())
    o.frames(n)
    x, v = o.state()
    s.x = x.copy()
    s.v = v.copy()
    return s


def geraet(s, n, k, gx_fn, prec=_abi.K3D_FP64):
    """Device forward of n frames with checkpoints every k; the adjoint for
    the cotangents gx_fn(x_T, v_T). Returns (x_T, v_T, adjoint dict, cg)."""
    cg = ImplizitCg(param(prec))
    sc = s.copy()
    cg.hochladen(sc)
    cg.adjoint_vorwaerts(n, k)
    cg.zustand_lesen(sc)
    gx, gv = gx_fn(sc.x, sc.v)
    return sc.x.copy(), sc.v.copy(), cg.adjoint_rueckwaerts(gx, gv), cg


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def gewichte(n, seed=3):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, 3)), rng.normal(size=(n, 3))


@pytest.mark.parametrize("szene,vor,n,tol", [(haengend, 20, 6, 1e-6), (auf_kugel, 12, 3, 1e-5)],
                         ids=["haengend", "auf_kugel"])
def test_adjoint_wie_orakel(szene, vor, n, tol):
    s = vorlauf(szene(), vor)
    wx, wv = gewichte(s.n)
    xT, vT, ad, _ = geraet(s, n, 2, lambda x, v: (wx, wv))
    o = O.OracleSim(s, param().to_c())
    ao = o.adjoint(n, wx, wv)
    xo, vo = o.state()
    assert np.max(np.abs(xT - xo)) <= 1e-9 * np.linalg.norm(xo.max(0) - xo.min(0))
    assert rel(ad["x"], ao["x"]) <= tol
    assert rel(ad["v"], ao["v"]) <= tol
    assert rel(ad["membran"], ao["membran"]) <= tol
    assert rel(ad["biegung"], ao["biegung"]) <= tol
    assert ad["iterationen"] > 0 and ad["nicht_konvergiert"] == 0


def test_checkpoint_abstand_gleich():
    """The recomputation is deterministic: the spacing of the checkpoints
    does not change a bit of the result."""
    s = vorlauf(auf_kugel(), 12)
    wx, wv = gewichte(s.n)
    out = [geraet(s, 5, k, lambda x, v: (wx, wv))[2] for k in (1, 2, 5)]
    for r in out[1:]:
        for key in ("x", "v", "membran", "biegung"):
            assert np.array_equal(r[key], out[0][key]), key


def test_zustand_nach_rueckwaerts():
    s = vorlauf(haengend(), 10)
    wx, wv = gewichte(s.n)
    xT, vT, _, cg = geraet(s, 4, 3, lambda x, v: (wx, wv))
    sc = s.copy()
    cg.zustand_lesen(sc)
    assert np.array_equal(sc.x, xT) and np.array_equal(sc.v, vT)


def test_adjoint_wie_differenzen_geraet():
    """Directional derivatives of the device forward at relative step 1e-4
    for the five material parameters (Drapierung), within 1e-3."""
    basis = vorlauf(haengend(), 20)
    grain = float(np.arctan2(basis.membran_kette[0, 1], basis.membran_kette[0, 0]))  # any reference angle
    e = basis.membran_steif[0]
    bs = Stoff(float(e[0]), float(e[1]), float(e[2]), 1.0, grain)
    d = Drapierung(basis, bs, frames=6, k=3, param=param())
    p0 = bs.array()
    xT, vT = d.vorwaerts(p0)
    rng = np.random.default_rng(1)
    ziel = xT + rng.normal(size=xT.shape) * 1e-3

    def loss(x, v):
        return float(np.sum((x - ziel) ** 2) + 0.1 * np.sum(v ** 2))

    d.vorwaerts(p0)
    g = d.rueckwaerts(2.0 * (xT - ziel), 0.2 * vT)["stoff"]
    for q in range(5):
        h = 1e-4 * (abs(p0[q]) if q < 4 else 1.0)
        pp, pm = p0.copy(), p0.copy()
        pp[q] += h
        pm[q] -= h
        fd = (loss(*d.vorwaerts(pp)) - loss(*d.vorwaerts(pm))) / (2 * h)
        assert abs(fd - g[q]) <= 1e-3 * abs(fd), (q, fd, g[q])


def test_adjoint_nur_fp64():
    s = haengend()
    cg = ImplizitCg(param(_abi.K3D_MIXED))
    cg.hochladen(s)
    with pytest.raises(K3dError):
        cg.adjoint_vorwaerts(2, 1)


def test_drape_function_torch():
    import torch
    basis = vorlauf(haengend(), 20)
    e = basis.membran_steif[0]
    bs = Stoff(float(e[0]), float(e[1]), float(e[2]), 1.0, 0.0)
    d = Drapierung(basis, bs, frames=3, k=2, param=param())
    p = torch.tensor(bs.array(), dtype=torch.float64, requires_grad=True)
    x0 = torch.tensor(basis.x, dtype=torch.float64, requires_grad=True)
    v0 = torch.tensor(basis.v, dtype=torch.float64)
    x, v = DrapeFunction().apply(p, x0, v0, d)
    loss = (x ** 2).sum() + (v ** 2).sum()
    loss.backward()
    g = d.rueckwaerts(2.0 * x.detach().numpy(), 2.0 * v.detach().numpy())
    assert np.allclose(p.grad.numpy(), g["stoff"]) and np.allclose(x0.grad.numpy(), g["x"])


def test_adjoint_aufprall_wie_orakel():
    """The material-fit drop (25 x 25) over its first impact (40 frames, with
    releases after the last solve): device against oracle adjoint. Most of
    the sheet is still falling at its rest strain there, on the clamp of the
    geometric stress (max(e, 0)), where the step has no derivative: the
    oracle's central differences average both sides, the device's dual
    numbers take the side of the value. That shows in the state and
    per-element cotangents and in the five parameter sums (all 1e-3)."""
    from garmentcraft_b200.adjoint import szene_mit
    s, hid, start = synth.materialfit(n=25)
    sz = szene_mit(s, Stoff.von(hid), Stoff.von(start))
    wx, wv = gewichte(sz.n)
    xT, vT, ad, _ = geraet(sz, 40, 10, lambda x, v: (wx, wv))
    o = O.OracleSim(sz, param().to_c())
    ao = o.adjoint(40, wx, wv)
    xo, _ = o.state()
    assert np.max(np.abs(xT - xo)) <= 1e-9 * np.linalg.norm(xo.max(0) - xo.min(0))
    for key in ("x", "v", "membran", "biegung"):
        assert rel(ad[key], ao[key]) <= 1e-3, key
    k = 1.0 / sz.biegung_nachgiebigkeit
    for q in range(4):
        a, b = ad["membran"][:, q].sum(), ao["membran"][:, q].sum()
        assert abs(a - b) <= 1e-3 * abs(b), q
    a, b = np.sum(ad["biegung"] * k), np.sum(ao["biegung"] * k)
    assert abs(a - b) <= 1e-3 * abs(b)
