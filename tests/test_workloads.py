"""The synthetic workloads against the configurations they stand in for
(no dataset exists for this path; every input comes from a seed): sizes,
materials, bodies and time steps of the tube, the 257 x 257 sheet over the
sphere, the sewn garment, the 64 batched drapes and the material fit."""
import math

import numpy as np
import pytest

from garmentcraft_b200 import _abi, synth


def test_tube():
    m, body = synth.tube()
    t = m.teile[0]
    assert len(t.punkte_mm) == 41 * 21 and len(t.dreiecke) == 1600  # 0.40 x 0.20 m at 10 mm
    assert np.ptp(t.punkte_mm[:, 0]) == pytest.approx(400.0) and np.ptp(t.punkte_mm[:, 1]) == pytest.approx(200.0)
    mat = t.material
    assert (mat.kette_n_m, mat.dehnung_n_m, mat.schub_n_m) == (600.0, 600.0, 300.0)  # E*t, G = E/2
    assert mat.biegung_nm == mat.biegung_kette_nm == mat.biegung_schraege_nm == 1e-7
    assert mat.dicke_m == 0.5e-3 and mat.flaechengewicht_kg_m2 == pytest.approx(1000.0 * 0.5e-3)
    assert body["art"] == _abi.K3D_BODY_CYLINDER and body["radius"] == 0.08
    assert m.param.schwerkraft == (0.0, 0.0, 0.0) and m.param.bild_dt == pytest.approx(1 / 60)
    # the two 0.20 m sides keep their own points and are sewn
    assert m.naehte[0].teilnaehte[0].paare.shape == (21, 2)


def test_sheet_over_sphere():
    m, body = synth.sheet_over_sphere()
    t = m.teile[0]
    assert len(t.punkte_mm) == 66049 and len(t.dreiecke) == 131072
    regel = np.stack(np.meshgrid(np.linspace(0, 1000, 257), np.linspace(0, 1000, 257)), -1).reshape(-1, 2)
    assert np.abs(t.punkte_mm - regel).max() <= 1.0  # +/-1 mm in-plane jitter
    mat = t.material
    assert (mat.kette_n_m, mat.dehnung_n_m, mat.schub_n_m) == (2000.0, 1000.0, 50.0)
    assert mat.biegung_nm == mat.biegung_kette_nm == mat.biegung_schraege_nm == 5e-6
    assert mat.flaechengewicht_kg_m2 == 0.2 and mat.reibung == 0.3
    winkel = math.atan2(t.fadenlauf[1], t.fadenlauf[0]) % math.pi
    assert 0.0 <= winkel < math.pi
    assert body["dims"] == (128, 128, 128) and body["spacing"] == 0.01
    # the sphere of radius 0.3 m sampled exactly at the nodes (float32)
    sdf = np.asarray(body["sdf"], dtype=np.float64).reshape(128, 128, 128)
    o = body["ursprung"]
    gz, gy, gx = np.meshgrid(*(np.arange(128) * 0.01 + o[k] for k in (2, 1, 0)), indexing="ij")
    c = body.get("punkt", (0.0, 0.0, 0.0))
    d = np.sqrt((gx - c[0]) ** 2 + (gy - c[1]) ** 2 + (gz - c[2]) ** 2) - 0.3
    assert np.abs(sdf - d).max() < 1e-6
    assert np.min(t.lage[:, 2]) == pytest.approx(0.3 + 0.5)  # 0.5 m above the sphere top
    assert m.param.bild_dt == pytest.approx(1 / 120) and m.param.schwerkraft == (0.0, 0.0, -9.81)


def test_garment():
    m, body = synth.garment()
    assert len(m.teile) == 28
    n = sum(len(t.punkte_mm) for t in m.teile)
    assert 195_000 <= n <= 215_000
    for t in m.teile:
        b, h = np.ptp(t.punkte_mm[:, 0]), np.ptp(t.punkte_mm[:, 1])
        assert 80.0 <= min(b, h) and max(b, h) <= 600.0
        mat = t.material
        assert 1.0e6 <= mat.dehnung_n_m / 0.5e-3 <= 1.5e6  # E U(1.0, 1.5) MPa at 0.5 mm
        assert mat.kette_n_m == mat.dehnung_n_m and mat.schub_n_m == 0.5 * mat.dehnung_n_m  # G = E/2
        assert mat.dicke_m == 0.5e-3 and mat.reibung == 0.4
    assert len({t.material.dehnung_n_m for t in m.teile}) == 28
    assert body["dims"] == (256, 256, 384) and body["spacing"] == 0.005
    assert m.param.bild_dt == pytest.approx(1 / 120)
    s, _ = synth.garment_szene()
    assert np.all(s.kollisionsabstand == 2e-3)


def test_drape_batch():
    batch = synth.drape_batch()
    assert len(batch) == 64
    punkte = np.array([len(m.teile[0].punkte_mm) for m, _ in batch])
    assert punkte.min() >= 0.9 * 2000 and punkte.max() <= 1.1 * 60000
    # log-uniform: about half of them below the geometric mean
    assert 16 <= np.sum(punkte < math.sqrt(2000 * 60000)) <= 48
    for m, body in batch:
        t = m.teile[0]
        asp = np.ptp(t.punkte_mm[:, 0]) / np.ptp(t.punkte_mm[:, 1])
        assert 0.9 <= asp <= 3.3
        mat = t.material
        assert 1000 <= mat.kette_n_m <= 2000 and 500 <= mat.dehnung_n_m <= 1000 and 25 <= mat.schub_n_m <= 50
        assert 2.5e-6 <= mat.biegung_nm <= 5e-6
        assert body["dims"] == (64, 64, 64)
        assert m.param.bild_dt == pytest.approx(1 / 120)


def test_materialfit():
    s, verdeckt, start = synth.materialfit()
    assert s.n == 129 * 129
    assert 1000 <= verdeckt[0] <= 2000 and 500 <= verdeckt[1] <= 1000 and 25 <= verdeckt[2] <= 50
    assert 2.5e-6 <= verdeckt[3] <= 5e-6 and 0.0 <= verdeckt[4] < math.pi
    assert np.all((start / verdeckt >= 0.5) & (start / verdeckt <= 2.0))
    body = s.koerper[0]
    assert body["dims"] == (128, 128, 128) and body["spacing"] == 0.01  # the sheet workload's sphere
