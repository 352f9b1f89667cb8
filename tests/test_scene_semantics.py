"""What Szene::bauen promises, checked on both scene builders (the library's
and the oracle's) from the reference's own statements, not by comparing the
two with each other:

* the ease (sim/src/szene.rs:556-592) shortens exactly the surplus of the
  longer seam side: the summed rest lengths drop by l_long - l_short, and only
  when the switch is on (the reference's test
  sim/tests/einhalteweite.rs:376-390, 112 mm against 100 mm, 1e-9 m);
* the lumped mass (szene.rs:387-389, `gesamtmasse` :785-787) is the reduced
  pattern area times the areal density, a third of each triangle's on each
  corner, and w = 1/m (:682);
* collision distance and friction per point are the material's half
  thickness and friction (:377-378);
* a spring's rest length is its pattern edge times the piece's scale
  1 - reduction (:362, :426-427), and the seam springs rest at zero
  (:542-543);
* every triangle gets a membrane whose rest area is the reduced pattern area
  (:602-647), and every pattern edge is flagged as a membrane edge.
"""
import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import synth
from garmentcraft_b200.implizit import build_scene

BUILDERS = {"library": build_scene, "oracle": O.build_scene}

KURZ_MM, LANG_MM = 100.0, 112.0


def zwei_teile(einhalteweite: bool, reduktion_a: float = 0.0, naht_nachgiebigkeit: float = 0.0):
    """A 100 x 50 mm piece sewn along its bottom edge to the 112 mm top edge
    of a 112 x 50 mm piece, 11 points on each side: the shorter side is a."""
    pa, ta = synth.rechteck_netz(KURZ_MM, 50.0, 10, 5)
    pb, tb = synth.rechteck_netz(LANG_MM, 50.0, 10, 5)
    lage_a = np.c_[pa * 1e-3, np.zeros(len(pa))]
    lage_b = np.c_[pb * 1e-3 - [0.0, 0.05], np.full(len(pb), 1e-3)]
    unten_a = np.arange(11)
    oben_b = np.arange(11) + 5 * 11
    mat_a = synth.RADICAL_RUBBER_04
    mat_b = synth.RETIFIST_NR_040
    m = synth.Muster(
        [synth.Teil(pa, ta, (1.0, 0.0), mat_a, lage_a, reduktion_a),
         synth.Teil(pb, tb, (0.0, 1.0), mat_b, lage_b)],
        [synth.Naht([synth.Teilnaht(0, 1, np.stack([unten_a, oben_b], 1).astype(np.uint32))], KURZ_MM, LANG_MM)],
        naht_nachgiebigkeit=naht_nachgiebigkeit, einhalteweite=einhalteweite)
    return m, (pa, pb), (mat_a, mat_b)


def dreiecksflaeche(p, t):
    a, b, c = p[t[:, 0]], p[t[:, 1]], p[t[:, 2]]
    return 0.5 * np.abs((b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0]))


@pytest.mark.parametrize("wer", list(BUILDERS))
def test_ease_shortens_exactly_the_surplus(wer):
    bauen = BUILDERS[wer]
    ohne = bauen(zwei_teile(False)[0])
    mit = bauen(zwei_teile(True)[0])
    weg = ohne.abstand_ruhe.sum() - mit.abstand_ruhe.sum()
    assert abs(weg - (LANG_MM - KURZ_MM) * 1e-3) < 1e-9, weg
    # exactly the ten boundary springs of the longer side, each by 100/112
    geaendert = np.flatnonzero(ohne.abstand_ruhe != mit.abstand_ruhe)
    assert geaendert.size == 10
    np.testing.assert_allclose(mit.abstand_ruhe[geaendert], ohne.abstand_ruhe[geaendert] * (KURZ_MM / LANG_MM),
                               rtol=1e-15, atol=0)
    np.testing.assert_allclose(ohne.abstand_ruhe[geaendert], LANG_MM / 10 * 1e-3, rtol=1e-12)
    # the springs belong to the longer piece (b), on its sewn top row
    b0, b1 = ohne.teil_bereiche[1, 0], ohne.teil_bereiche[1, 1]
    pts = ohne.abstand_punkte[geaendert]
    assert np.all((pts >= b0 + 5 * 11) & (pts < b1))
    # switched off, equal seam lengths ease nothing either
    m, _, _ = zwei_teile(True)
    m.naehte[0].laenge_b_mm = KURZ_MM
    gleich = bauen(m)
    assert np.array_equal(gleich.abstand_ruhe, ohne.abstand_ruhe)


@pytest.mark.parametrize("wer", list(BUILDERS))
def test_mass_is_reduced_area_times_density(wer):
    red = 0.05
    m, (pa, pb), (ma, mb) = zwei_teile(False, reduktion_a=red)
    s = BUILDERS[wer](m)
    ta, tb = m.teile[0].dreiecke, m.teile[1].dreiecke
    fa = dreiecksflaeche(pa * 1e-3, ta) * (1 - red) ** 2
    fb = dreiecksflaeche(pb * 1e-3, tb)
    erwartet = fa.sum() * ma.flaechengewicht_kg_m2 + fb.sum() * mb.flaechengewicht_kg_m2
    assert abs(s.masse.sum() - erwartet) < 1e-13 * erwartet
    # a third of every triangle on each corner, piece by piece
    for k, (p, t, f, mat) in enumerate([(pa, ta, fa, ma), (pb, tb, fb, mb)]):
        lo, hi = s.teil_bereiche[k, 0], s.teil_bereiche[k, 1]
        eck = np.zeros(len(p))
        for c in range(3):
            np.add.at(eck, t[:, c], f * mat.flaechengewicht_kg_m2 / 3.0)
        np.testing.assert_allclose(s.masse[lo:hi], eck, rtol=1e-13)
        assert np.all(s.kollisionsabstand[lo:hi] == mat.dicke_m / 2.0)
        assert np.all(s.reibung[lo:hi] == mat.reibung)
    assert np.all(s.masse > 0)
    assert np.array_equal(s.w, 1.0 / s.masse)


@pytest.mark.parametrize("wer", list(BUILDERS))
def test_rest_lengths_and_membranes_follow_the_reduced_pattern(wer):
    red = 0.05
    m, (pa, pb), _ = zwei_teile(False, reduktion_a=red, naht_nachgiebigkeit=2.5e-4)
    s = BUILDERS[wer](m)
    # every pattern point in metres on the reduced piece, in global order
    lo_b = s.teil_bereiche[1, 0]
    p2 = np.concatenate([pa * 1e-3 * (1 - red), pb * 1e-3])
    i, j = s.abstand_punkte[:, 0], s.abstand_punkte[:, 1]
    np.testing.assert_allclose(s.abstand_ruhe, np.linalg.norm(p2[i] - p2[j], axis=1), rtol=1e-13)
    # springs stay within their piece
    assert np.all((i < lo_b) == (j < lo_b))
    # seams: 11 pairs at rest length zero
    assert s.naht_punkte.shape[0] == 11
    assert np.all(s.naht_ruhe == 0.0)
    # one membrane per triangle, rest area = reduced pattern area
    tri = np.concatenate([m.teile[0].dreiecke, m.teile[1].dreiecke + lo_b])
    assert s.membran_punkte.shape[0] == tri.shape[0]
    np.testing.assert_allclose(np.sort(s.membran_flaeche), np.sort(dreiecksflaeche(p2, tri)), rtol=1e-12)
    assert s.membran_flaeche.sum() == pytest.approx(dreiecksflaeche(p2, tri).sum(), rel=1e-13)
    assert np.all(s.membran_kante == 1)
