"""Batched drapes: independent scenes in one launch against each scene alone.

Each instance of a batch scene gets its own blocks, barrier and reductions
in the PCG launch, so it converges on its own. Its reductions run over fewer
blocks than when the scene runs alone, so the sums round in another order:
the states agree to 1e-9 of the bounding-box diagonal (FP64) after several
frames, and the FP64 form is checked against the oracle per instance too.
"""
import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import _abi, synth
from garmentcraft_b200.implizit import ImplizitCg, build_scene
from garmentcraft_b200.params import ImplizitParameter
from garmentcraft_b200.szene import Szene

pytestmark = pytest.mark.gpu


def diag(x):
    return float(np.linalg.norm(x.max(0) - x.min(0)))


def szenen():
    m, body = synth.tube()
    tube = build_scene(m, [body])
    m, kugel = synth.sheet_over_sphere(n=33, seed=3, fall_m=0.02)
    blatt = build_scene(m, [kugel])
    m2, kugel2 = synth.sheet_over_sphere(n=21, seed=7, fall_m=0.01, groesse_m=0.6, kugel_radius_m=0.2, sdf_n=48)
    blatt2 = build_scene(m2, [kugel2])
    # one frame length, gravity and air damping for every instance of a batch
    for sz in (tube, blatt, blatt2):
        sz.param = synth.Simparameter(bild_dt=1.0 / 120.0, schwerkraft=(0.0, 0.0, -9.81), daempfung=1.0)
    return [tube, blatt, blatt2]


def param(prec):
    return ImplizitParameter(schritte_je_bild=1, cg_max=4000, cg_toleranz=1e-12, precision=prec)


@pytest.mark.parametrize("prec,tol", [(_abi.K3D_FP64, 1e-9), (_abi.K3D_MIXED, 1e-5)])
def test_batch_wie_einzeln(prec, tol):
    einzeln = szenen()
    batch = Szene.verbinden([s.copy() for s in einzeln])
    cg = ImplizitCg(param(prec))
    allein = [ImplizitCg(param(prec)) for _ in einzeln]
    its_b = its_e = 0
    for _ in range(12):
        cg.bild(batch)
        its_b += cg.statistik.cg_iterationen
        for s, c in zip(einzeln, allein):
            c.bild(s)
            its_e += c.statistik.cg_iterationen
    for k, s in enumerate(einzeln):
        xb = batch.x[batch.instanz(k)]
        assert np.max(np.abs(xb - s.x)) <= tol * diag(s.x), k
    assert its_b > 0 and abs(its_b - its_e) <= 0.1 * its_e


def test_batch_wie_orakel():
    einzeln = szenen()
    batch = Szene.verbinden([s.copy() for s in einzeln])
    orks = [O.OracleSim(s, param(_abi.K3D_FP64).to_c()) for s in einzeln]
    cg = ImplizitCg(param(_abi.K3D_FP64))
    for _ in range(8):
        cg.bild(batch)
        for o in orks:
            o.frames(1)
    for k, o in enumerate(orks):
        x, _ = o.state()
        assert np.max(np.abs(batch.x[batch.instanz(k)] - x)) <= 1e-9 * diag(x), k


def test_batch_abgelehnt():
    einzeln = szenen()
    batch = Szene.verbinden(einzeln)
    # an element that spans two instances
    batch.abstand_punkte[0, 1] = batch.instanz_punkte[1]
    cg = ImplizitCg(ImplizitParameter())
    with pytest.raises(Exception):
        cg.bild(batch)
