"""The device's self-collision response (selbstkollision.rs:810-1343: edges
through triangles, their regions and push springs; impacts on the way and
their position response) against the oracle, on the reference's tilted-layer
scene (sim/tests/selbstkollision.rs:69-95): the upper layer starts through the
lower one."""
import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import _abi, synth
from garmentcraft_b200.implizit import ImplizitCg, build_scene
from garmentcraft_b200.params import ImplizitParameter

pytestmark = pytest.mark.gpu

INSET = dict(oben_groesse_m=0.18, versatz_m=(0.0073, 0.0041))


def schraeg():
    m = synth.zwei_lagen(abstand_m=-0.005, neigung=0.1, **INSET)
    s = build_scene(m)
    synth.pin_teil(s, 0)
    return s


def diag(x):
    return float(np.linalg.norm(x.max(0) - x.min(0)))


def test_antwort_wie_orakel():
    """FP64, tight tolerance: per frame the same intersection, region and
    impact counts as the oracle, positions to 1e-8 of the bbox diagonal (the
    push springs are stiff, k = 2 s (E + E)(A + A) / 1 mm^2, so the order of
    the device's reductions shows a little more than without them)."""
    s = schraeg()
    p = ImplizitParameter(selbstkollision=True, cg_max=100000, cg_toleranz=1e-12)
    o = O.OracleSim(s.copy(), p.to_c())
    assert o.schnitte().shape[0] > 10
    cg = ImplizitCg(p)
    for _ in range(4):
        cg.bild(s)
        st = o.frames(1)
        a = cg.statistik
        assert (a.durchdringungen, a.durchdringungsgebiete) == (st.durchdringungen, st.durchdringungsgebiete)
        assert a.selbst_stoesse == st.selbst_stoesse
        assert (a.naehe_punkt_dreieck, a.naehe_kante_kante) == (st.naehe_punkt_dreieck, st.naehe_kante_kante)
    xo, _ = o.state()
    assert np.max(np.abs(s.x - xo)) <= 1e-8 * diag(xo)


@pytest.mark.parametrize("prec", [_abi.K3D_FP64, _abi.K3D_MIXED])
def test_schraege_lage_loest_sich_geraet(prec):
    """The reference's acceptance test on the device: more than 10 edges
    pierce the other layer at the start, none after 90 frames (default
    parameters with self-collision)."""
    s = schraeg()
    p = ImplizitParameter(selbstkollision=True, precision=prec)
    cg = ImplizitCg(p)
    for _ in range(90):
        cg.bild(s)
    o = O.OracleSim(s, ImplizitParameter(selbstkollision=True).to_c())
    assert o.schnitte().shape[0] == 0
