"""The library's scene builder against the oracle's restatement of
Szene::bauen (sim/src/szene.rs:320-715): topology, colour order and every
value bit for bit."""
import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import synth
from garmentcraft_b200.implizit import build_scene
from garmentcraft_b200.szene import _ARRAYS

FIELDS = list(_ARRAYS)


def same(a, b):
    for f in FIELDS:
        x, y = getattr(a, f), getattr(b, f)
        assert x.shape == y.shape, f
        assert x.dtype == y.dtype, f
        # bit-exact, NaN/inf included
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), f


def test_tube_bitgleich():
    m, body = synth.tube()
    same(build_scene(m, [body]), O.build_scene(m, [body]))


def test_sheet_jitter_grain_bitgleich():
    mat = synth.Material(1000.0, 2000.0, 50.0, 5e-6, 7e-6, 3e-6, 0.2, 0.5e-3, 0.3)
    m, body = synth.sheet_over_sphere(n=33, seed=7, material=mat)
    a, b = build_scene(m, [body]), O.build_scene(m, [body])
    same(a, b)
    # anisotropic bending: stiffness follows the edge direction
    assert len(np.unique(b.biegung_nachgiebigkeit)) > 10


def test_reduction_and_ease():
    m, body = synth.tube(umfang_m=0.2, hoehe_m=0.1)
    m.teile[0].reduktion = 0.055
    m.einhalteweite = True
    m.naehte[0].laenge_a_mm, m.naehte[0].laenge_b_mm = 100.0, 96.0
    a, b = build_scene(m, [body]), O.build_scene(m, [body])
    same(a, b)
    assert b.oracle_counts["einhalte_kanten"] > 0


def test_two_pieces_with_seam_hinges():
    p1, t1 = synth.rechteck_netz(100.0, 50.0, 10, 5)
    p2, t2 = synth.rechteck_netz(100.0, 50.0, 10, 5)
    lage1 = np.c_[p1 * 1e-3, np.zeros(len(p1))]
    lage2 = np.c_[p2 * 1e-3 + [0.0, 0.05], np.full(len(p2), 1e-3)]
    mat = synth.RADICAL_RUBBER_04
    oben = np.arange(11) + 5 * 11
    unten = np.arange(11)
    m = synth.Muster([synth.Teil(p1, t1, (1.0, 0.0), mat, lage1), synth.Teil(p2, t2, (0.0, 1.0), mat, lage2)],
                     [synth.Naht([synth.Teilnaht(0, 1, np.stack([oben, unten], 1).astype(np.uint32))],
                                 100.0, 100.0)])
    a, b = build_scene(m), O.build_scene(m)
    same(a, b)
    assert a.naht_punkte.shape[0] == 11
    assert b.oracle_counts["naht_biegung_ohne"] == 0
    # 10 seam hinges on top of the interior edges of both pieces
    inner = 2 * (10 * 6 + 11 * 5 + 10 * 5 - (2 * 10 + 2 * 5))
    assert a.biegung_punkte.shape[0] == inner + 10


def test_garment_205k_bitgleich():
    # the sewn garment at full size: 28 panels, ~205k points, seams by length
    # fraction (both builders, every field bit for bit)
    m, body = synth.garment(ziel_punkte=200_000)
    a, b = build_scene(m, [body]), O.build_scene(m, [body])
    same(a, b)
    assert a.n > 200_000 and a.teil_bereiche.shape[0] == 28
    assert b.oracle_counts["membran_entartet"] == 0
    assert a.membran_punkte.shape[0] == sum(t.dreiecke.shape[0] for t in m.teile)
