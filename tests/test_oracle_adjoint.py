"""The FP64 CPU adjoint of the oracle against central finite differences.

The reference has no adjoint, so the oracle's own forward (the restatement of
ImplizitCg::schritt, implizit.rs:899-1038) is the function differentiated.
Loss: sum |x_T - x*|^2 + 0.1 sum |v_T|^2 after N frames. Directional
derivatives for the initial positions and velocities, and for the five
material parameters scaled on every element at once (warp, weft and shear
stiffness, bending stiffness, grain angle), are compared with central
differences at relative step 1e-4 (1e-8 m for positions, which the stiff
membrane makes strongly nonlinear). The scenes start from a state reached
by earlier frames: at the rest state every membrane strain sits on the
max(e, 0) clamp of the geometric stress, where the step has no derivative.

Resting contacts sit on a kink of the reference's contact handling (the held
point lands exactly on the surface, so the push-out depth and the inward
normal velocity after the move are zero up to rounding); central differences
average the two sides there, while the adjoint follows the recorded side.
With contacts, the material parameters are checked (their gradients do not
cross that kink at first order); initial-state gradients are checked on the
contact-free scene.
"""
import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import synth
from garmentcraft_b200.implizit import build_scene
from garmentcraft_b200.params import ImplizitParameter

PAR = ImplizitParameter(schritte_je_bild=1, cg_max=100000, cg_toleranz=1e-14).to_c()


def haengend():
    m, _ = synth.sheet_over_sphere(n=9, groesse_m=0.2, jitter_mm=2.0, seed=5, fall_m=0.3)
    s = build_scene(m, [])
    s.w[0] = 0.0  # two corners held
    s.w[8] = 0.0
    s.param.daempfung = 0.5
    return s


def auf_kugel():
    m, body = synth.sheet_over_sphere(n=9, groesse_m=0.3, jitter_mm=2.0, seed=5, fall_m=0.002,
                                      kugel_radius_m=0.1, sdf_n=48, sdf_spacing_m=0.006)
    return build_scene(m, [body])


def vorlauf(s, n):
    o = O.OracleSim(s, PAR)
    o.frames(n)
    x, v = o.state()
    s.x = x.copy()
    s.v = v.copy()
    return s


def lauf(s, n, x0=None, v0=None):
    o = O.OracleSim(s, PAR)
    if x0 is not None or v0 is not None:
        o.set_state(x0, v0)
    st = o.frames(n)
    x, v = o.state()
    return x, v, (st.kontakte, st.haftend, st.freigegeben)


def gedreht(s, e):
    c, sn = np.cos(e), np.sin(e)
    for nm in ("membran_kette", "membran_schuss"):
        a = getattr(s, nm)
        b = a.copy()
        b[:, 0] = c * a[:, 0] - sn * a[:, 1]
        b[:, 1] = sn * a[:, 0] + c * a[:, 1]
        setattr(s, nm, b)
    return s


def faelle(s0, n, ad, rng, mit_zustand):
    """(name, run(eps) -> (x, v, counts), adjoint directional derivative, eps)."""
    E = s0.membran_steif[0]
    k = 1.0 / s0.biegung_nachgiebigkeit
    out = []
    if mit_zustand:
        d = rng.normal(size=s0.x.shape)
        d[s0.w <= 0] = 0.0
        dv = rng.normal(size=s0.x.shape)
        out.append(("x0", lambda e: lauf(s0, n, s0.x + e * d, None), np.sum(ad["x"] * d), 1e-8))
        out.append(("v0", lambda e: lauf(s0, n, None, s0.v + e * dv), np.sum(ad["v"] * dv), 1e-4))

    def steif(col):
        def f(e):
            s = s0.copy()
            s.membran_steif[:, col] *= 1.0 + e
            return lauf(s, n)
        return f

    def biegung(e):
        s = s0.copy()
        s.biegung_nachgiebigkeit = s.biegung_nachgiebigkeit / (1.0 + e)
        return lauf(s, n)

    for col, name in enumerate(("warp", "weft", "shear")):
        out.append((name, steif(col), np.sum(ad["membran"][:, col]) * E[col], 1e-4))
    out.append(("grain", lambda e: lauf(gedreht(s0.copy(), e), n), np.sum(ad["membran"][:, 3]), 1e-4))
    out.append(("bend", biegung, np.sum(ad["biegung"] * k), 1e-4))
    return out


@pytest.mark.parametrize("szene,vor,n,mit_zustand", [(haengend, 20, 6, True), (auf_kugel, 12, 3, False)],
                         ids=["haengend", "auf_kugel"])
def test_adjoint_wie_differenzen(szene, vor, n, mit_zustand):
    s0 = vorlauf(szene(), vor)
    rng = np.random.default_rng(1)
    xT, vT, st0 = lauf(s0, n)
    ziel = xT + rng.normal(size=xT.shape) * 1e-3

    def loss(x, v):
        return float(np.sum((x - ziel) ** 2) + 0.1 * np.sum(v ** 2))

    ad = O.OracleSim(s0, PAR).adjoint(n, 2.0 * (xT - ziel), 0.2 * vT)
    assert ad["iterationen"] > 0
    for name, f, a, eps in faelle(s0, n, ad, rng, mit_zustand):
        xp, vp, sp = f(eps)
        xm, vm, sm = f(-eps)
        assert sp == st0 and sm == st0, name  # same contact and friction counts
        fd = (loss(xp, vp) - loss(xm, vm)) / (2.0 * eps)
        assert abs(fd - a) <= 1e-3 * abs(fd), (name, fd, a)


def test_adjoint_eines_schritts_exakt():
    """One frame with contacts, against a step of 1e-4 in v0: agreement to 1e-5."""
    s0 = vorlauf(auf_kugel(), 12)
    rng = np.random.default_rng(2)
    xT, vT, _ = lauf(s0, 1)
    wx = rng.normal(size=xT.shape)
    wv = rng.normal(size=xT.shape)
    ad = O.OracleSim(s0, PAR).adjoint(1, wx, wv)
    dv = rng.normal(size=xT.shape)
    xp, vp, _ = lauf(s0, 1, None, s0.v + 1e-4 * dv)
    xm, vm, _ = lauf(s0, 1, None, s0.v - 1e-4 * dv)
    fd = (np.sum(wx * (xp - xm)) + np.sum(wv * (vp - vm))) / 2e-4
    assert abs(fd - np.sum(ad["v"] * dv)) <= 1e-5 * abs(fd)


def test_adjoint_erster_aufprall():
    """The material-fit drop (coarse: 25 x 25) over its first impact, 40
    frames: contacts, sticking and points released by the release pass, some
    of them after the last solve. Loss against the drop at the hidden
    parameters; the five parameters at relative step 1e-4, within 1e-3."""
    from garmentcraft_b200.adjoint import Stoff, szene_mit
    s, hid, start = synth.materialfit(n=25)
    bs = Stoff.von(hid)
    par = ImplizitParameter(schritte_je_bild=1, cg_max=100000, cg_toleranz=1e-12).to_c()

    def lauf_p(p):
        o = O.OracleSim(szene_mit(s, bs, Stoff.von(p)), par)
        st = o.frames(40)
        return o.state()[0], (st.kontakte, st.haftend, st.freigegeben)

    ziel, _ = lauf_p(hid)
    x, st0 = lauf_p(start)
    assert st0[0] > 0 and st0[2] > 0  # contacts and releases
    sz = szene_mit(s, bs, Stoff.von(start))
    ad = O.OracleSim(sz, par).adjoint(40, 2.0 * (x - ziel), np.zeros_like(x))
    k = 1.0 / sz.biegung_nachgiebigkeit
    g = [ad["membran"][:, 0].sum(), ad["membran"][:, 1].sum(), ad["membran"][:, 2].sum(),
         float(np.sum(ad["biegung"] * k)) / start[3], ad["membran"][:, 3].sum()]
    for q in range(5):
        h = 1e-4 * abs(start[q])
        pp, pm = start.copy(), start.copy()
        pp[q] += h
        pm[q] -= h
        (xp, sp), (xm, sm) = lauf_p(pp), lauf_p(pm)
        assert sp == st0 and sm == st0, q
        fd = (np.sum((xp - ziel) ** 2) - np.sum((xm - ziel) ** 2)) / (2 * h)
        assert abs(fd - g[q]) <= 1e-3 * abs(fd), (q, fd, g[q])
