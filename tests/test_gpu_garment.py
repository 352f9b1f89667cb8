"""The sewn-garment workload at a reduced size (~20k points; 28 panels,
seams, the 15-capsule body SDF, latex, 2 mm collision thickness, the
self-collision proximity stage on) against the oracle: the device FP64 step
agrees with the oracle to 1e-9 of the bbox diagonal over three frames with
the same proximity pair counts, and one mixed step agrees with the FP64 step
to 1e-5."""
import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import _abi, synth
from garmentcraft_b200.implizit import ImplizitCg
from garmentcraft_b200.params import ImplizitParameter

pytestmark = pytest.mark.gpu


def param(prec):
    return ImplizitParameter(schritte_je_bild=1, cg_max=20000, cg_toleranz=1e-12, precision=prec,
                             selbstkollision=True)


def diag(x):
    return float(np.linalg.norm(x.max(0) - x.min(0)))


@pytest.fixture(scope="module")
def szene():
    s, _ = synth.garment_szene(ziel_punkte=20_000)
    return s


def test_garment_wie_orakel(szene):
    s = szene.copy()
    o = O.OracleSim(szene.copy(), param(_abi.K3D_FP64).to_c())
    cg = ImplizitCg(param(_abi.K3D_FP64))
    for _ in range(3):
        cg.bild(s)
        st_o = o.frames(1)
        assert cg.statistik.naehe_punkt_dreieck == st_o.naehe_punkt_dreieck
        assert cg.statistik.naehe_kante_kante == st_o.naehe_kante_kante
    xo, _ = o.state()
    assert cg.statistik.naehe_punkt_dreieck + cg.statistik.naehe_kante_kante > 0
    assert np.max(np.abs(s.x - xo)) <= 1e-9 * diag(xo)


def test_garment_mixed_wie_fp64(szene):
    a, b = szene.copy(), szene.copy()
    ImplizitCg(param(_abi.K3D_FP64)).bild(a)
    pm = param(_abi.K3D_MIXED)
    pm.cg_toleranz = 1e-6
    ImplizitCg(pm).bild(b)
    assert np.max(np.abs(a.x - b.x)) <= 1e-5 * diag(a.x)
