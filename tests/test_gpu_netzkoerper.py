"""The device body mesh (include/klon3d_mesh.h) against the oracle's
restatement of sim/src/netzkoerper.rs: the point-dependent tables, the
nearest query over the grid and over every triangle, the segment
penetration, nachfuehren, the refusals, and the voxelised grid. Distances,
nearest points, regions and triangles are bit-identical (both round every
product and sum on its own); the point normals go through atan2, whose last
bit may differ between the device and the host library (1e-15)."""
import math

import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import synth
from garmentcraft_b200._lib import K3dError
from garmentcraft_b200.netzkoerper import Koerpernetz
from test_oracle_netzkoerper import Xorshift, abstand_wuerfel, wuerfel_punkte, zylinder_punkte

pytestmark = pytest.mark.gpu


def beide(p, d, suchtiefe):
    return Koerpernetz(p, d, suchtiefe), O.Koerpernetz(p, d, suchtiefe)


def gleich(a, b, felder=("abstand", "punkt", "dreieck", "region")):
    for f in felder:
        assert np.array_equal(a[f], b[f]), f
    assert np.max(np.abs(a["normale"] - b["normale"])) <= 1e-15


def test_wuerfel_wie_orakel_und_analytisch():
    p, d = synth.wuerfel_netz(1.0)
    g, o = beide(p, d, 0.5)
    assert g.randkanten == 0 and abs(g.volumen - 8.0) < 1e-12
    x = wuerfel_punkte()
    r = g.naechster_alle(x)
    gleich(r, o.naechster(x))
    assert np.max(np.abs(r["abstand"] - abstand_wuerfel(x, 1.0))) < 1e-12
    zurueck = x - r["normale"] * r["abstand"][:, None]
    assert np.max(np.linalg.norm(zurueck - r["punkt"], axis=1)) < 1e-9
    # the grid query within the search depth agrees where it finds something
    rg = g.naechster(x, 0.5)
    hit = rg["dreieck"] >= 0
    assert hit.sum() > 1000
    assert np.array_equal(rg["abstand"][hit], r["abstand"][hit])
    assert np.all(np.abs(r["abstand"][~hit]) >= 0.5)


def test_tabellen_wie_orakel():
    p, d = synth.koerper_netz(segmente=64, ringe=25)
    g, o = beide(p, d, 0.01)
    tg, to = g.tabellen(), o.tabellen()
    assert np.array_equal(tg["flaechennormale"], to["flaechennormale"])
    assert np.array_equal(tg["nachbar"], to["nachbar"])
    assert np.array_equal(tg["kugel"], to["kugel"])
    assert np.max(np.abs(tg["punktnormale"] - to["punktnormale"])) <= 1e-15
    ig, io = g.info(), o.info()
    assert ig.randkanten == io["randkanten"] == 0
    assert abs(ig.volumen - io["volumen"]) <= 1e-14 * io["volumen"]
    assert tuple(ig.gitter_zahl) == tuple(io["zahl"]) and ig.gitter_eintraege == io["eintraege"]
    assert tuple(ig.gitter_ursprung) == tuple(io["ursprung"]) and ig.gitter_zelle == io["zelle"]


def test_gitter_wie_alle_dreiecke():
    # netzkoerper.rs:1032-1059 on the device: the grid query equals the
    # all-triangle query within the search depth, nothing beyond it
    p, d = synth.zylinder_netz(0.09, -0.3, 0.1, 96, 20)
    g, o = beide(p, d, 0.01)
    x = zylinder_punkte()
    alle = g.naechster_alle(x)
    gleich(alle, o.naechster(x))
    r = g.naechster(x, 0.01)
    gleich(r, o.naechster(x, 0.01))
    hit = r["dreieck"] >= 0
    assert np.max(np.abs(r["abstand"][hit] - alle["abstand"][hit])) < 1e-12
    assert np.max(np.linalg.norm(r["punkt"][hit] - alle["punkt"][hit], axis=1)) < 1e-12
    assert np.all(np.abs(alle["abstand"][~hit]) >= 0.01)
    assert min(int(np.sum(r["abstand"][hit] < 0)), int(np.sum(r["abstand"][hit] >= 0)), int(np.sum(~hit))) > 1000


def koerper_proben(p, n, seed):
    rng = np.random.default_rng(seed)
    return p[rng.integers(0, p.shape[0], n)] + rng.normal(0.0, 0.02, (n, 3))


def test_koerper_wie_orakel():
    # both queries keep the reference's choice among equal distances: the
    # grid query the first in its cell order, the other the smallest index
    p, d = synth.koerper_netz()
    g, o = beide(p, d, 0.01)
    x = koerper_proben(p, 4000, 1)
    gleich(g.naechster_alle(x), o.naechster(x))
    rg = g.naechster(x, 0.03)
    gleich(rg, o.naechster(x, 0.03))
    assert (rg["dreieck"] >= 0).sum() > 1000


def test_durchstoss_wie_referenz_und_orakel():
    # netzkoerper.rs:1063-1079, then random segments against the oracle
    p, d = synth.wuerfel_netz(1.0)
    g, o = beide(p, d, 0.5)
    a = np.array([[0.2, 0.3, 3.0], [0.2, 0.3, 0.0], [0.2, 0.3, 3.0], [0.5, 0.5, 2.0]])
    b = np.array([[0.2, 0.3, -3.0], [0.2, 0.3, -3.0], [0.2, 0.3, 1.5], [0.5, 0.5, 0.0]])
    r = g.durchstoss(a, b)
    assert r["dreieck"][0] >= 0 and np.linalg.norm(r["punkt"][0] - [0.2, 0.3, 1.0]) < 1e-12
    assert abs(r["normale"][0][2] - 1.0) < 1e-12
    assert r["dreieck"][1] < 0 and r["dreieck"][2] < 0
    assert r["dreieck"][3] >= 0 and abs(r["punkt"][3][2] - 1.0) < 1e-12
    q, dd = synth.zylinder_netz(0.05, -0.001, 0.001, 64, 1)
    r = Koerpernetz(q, dd, 0.01).durchstoss([[0.01, 0.0, 0.05]], [[0.01, 0.0, -0.05]])
    assert r["dreieck"][0] >= 0 and abs(r["punkt"][0][2] - 0.001) < 1e-12 and r["normale"][0][2] > 0.999
    p, d = synth.koerper_netz()
    g, o = beide(p, d, 0.01)
    rng = np.random.default_rng(2)
    a = koerper_proben(p, 3000, 3)
    b = a + rng.normal(0.0, 0.03, a.shape)
    rg, ro = g.durchstoss(a, b), o.durchstoss(a, b)
    assert np.array_equal(rg["dreieck"], ro["dreieck"])
    hit = rg["dreieck"] >= 0
    assert hit.sum() > 100
    assert np.array_equal(rg["punkt"][hit], ro["punkt"][hit])
    assert np.array_equal(rg["normale"][hit], ro["normale"][hit])


def test_nachfuehren_wie_orakel():
    p, d = synth.koerper_netz(segmente=96, ringe=33)
    g, o = beide(p, d, 0.01)
    q = p * [1.1, 0.9, 1.0] + [0.05, 0.0, 0.02]
    g.nachfuehren(q)
    o.nachfuehren(q)
    ig, io = g.info(), o.info()
    assert tuple(ig.gitter_zahl) == tuple(io["zahl"]) and tuple(ig.gitter_ursprung) == tuple(io["ursprung"])
    x = koerper_proben(q, 2000, 4)
    gleich(g.naechster_alle(x), o.naechster(x))
    with pytest.raises(K3dError, match="volume"):
        g.nachfuehren(q * [-1.0, 1.0, 1.0])
    gleich(g.naechster_alle(x), o.naechster(x))  # the previous positions stay


def test_neu_weist_ab_wie_orakel():
    p, d = synth.wuerfel_netz(1.0)
    faelle = [(p, d[:0], 0.5, "without triangles"), (p, d, 0.0, "search depth")]
    bad = d.copy()
    bad[3, 1] = 8
    faelle.append((p, bad, 0.5, "out of range"))
    flip = d.copy()
    flip[0] = flip[0][[0, 2, 1]]
    faelle += [(p, flip, 0.5, "inconsistent"), (p, d[:, [0, 2, 1]], 0.5, "volume"),
               (p, np.concatenate([d, d[:1]]), 0.5, "more than two")]
    for pp, dd, s, grund in faelle:
        with pytest.raises(K3dError, match=grund):
            Koerpernetz(pp, dd, s)
        with pytest.raises(ValueError, match=grund):
            O.Koerpernetz(pp, dd, s)
    assert Koerpernetz(p, d[:-1], 0.5).randkanten == 3


def test_sdf_wie_orakel():
    p, d = synth.koerper_netz(segmente=64, ringe=25)
    g, o = beide(p, d, 0.01)
    dims, urs, s = (28, 20, 70), np.array([-0.25, -0.17, 0.0]), 0.026
    exakt = g.sdf(dims, urs, s)
    assert np.array_equal(exakt, o.sdf(dims, urs, s))
    band = g.sdf(dims, urs, s, band=0.06)
    assert np.array_equal(band, o.sdf(dims, urs, s, band=0.06))
    assert g.info().ungeklaert == 0
    # a grid that misses the body: every node beyond the band, the exact query decides
    weit = g.sdf((6, 5, 4), [2.0, 2.0, 2.0], 0.05, band=0.06)
    assert g.info().ungeklaert == 6 * 5 * 4
    assert np.array_equal(weit, o.sdf((6, 5, 4), [2.0, 2.0, 2.0], 0.05, band=0.06))
    with pytest.raises(K3dError, match="band must exceed"):
        g.sdf(dims, urs, s, band=0.02)


def test_sdf_koerper_voll_gegen_stichprobe():
    # the body-size mesh (36,864 triangles) at 5 mm with a 3 cm band: nodes in
    # the band equal the oracle's exact distance, every other node has the
    # oracle's sign
    p, d = synth.koerper_netz()
    g, o = beide(p, d, 0.01)
    body = g.sdf_body(0.005, 0.03)
    nx, ny, nz = body["dims"]
    sdf = body["sdf"].reshape(nz, ny, nx)
    rng = np.random.default_rng(5)
    idx = rng.integers(0, sdf.size, 3000)
    k, rest = np.divmod(idx, nx * ny)
    j, i = np.divmod(rest, nx)
    urs, s = np.array(body["ursprung"]), body["spacing"]
    x = np.stack([urs[0] + s * i, urs[1] + s * j, urs[2] + s * k], axis=1)
    soll = o.naechster(x)["abstand"]
    got = sdf.ravel()[idx].astype(np.float64)
    nah = np.abs(soll) < 0.03
    assert nah.sum() > 50
    assert np.array_equal(got[nah], soll[nah].astype(np.float32).astype(np.float64))
    assert np.array_equal(np.sign(got[~nah]), np.sign(soll[~nah]))
    assert np.all(np.abs(got[~nah]) == np.float32(0.03))
    assert (sdf < 0).sum() > 0.05 * sdf.size


def test_geschwindigkeitsfeld_wie_orakel():
    # netzkoerper.rs:1116-1215 on the device, and a random field against the oracle
    p, d = synth.wuerfel_netz(1.0)
    g, o = beide(p, d, 0.5)
    feld = np.zeros((8, 3))
    feld[7] = (0.0, 0.0, -1.0)
    g.setze_punktgeschwindigkeit(feld)
    r = g.naechster(np.array([[1.02, 1.0, 1.0], [1.02, 0.0, 1.0], [-1.02, 0.5, 0.5]]), 0.05)
    v = g.geschwindigkeit_an(r["dreieck"], r["punkt"])
    assert np.array_equal(v[0], [0.0, 0.0, -1.0]) and abs(v[1][2] + 0.5) < 1e-12
    assert np.array_equal(v[2], [0.0, 0.0, 0.0])
    g.setze_punktgeschwindigkeit(None)
    assert np.array_equal(g.geschwindigkeit_an(r["dreieck"], r["punkt"], (0.3, -0.2, 0.1)), np.tile([0.3, -0.2, 0.1], (3, 1)))
    p, d = synth.koerper_netz(segmente=96, ringe=33)
    g, o = beide(p, d, 0.01)
    rng = np.random.default_rng(8)
    feld = rng.normal(0.0, 1.0, p.shape)
    g.setze_punktgeschwindigkeit(feld)
    o.setze_punktgeschwindigkeit(feld)
    x = koerper_proben(p, 3000, 9)
    r = o.naechster(x)
    assert np.array_equal(g.geschwindigkeit_an(r["dreieck"], r["punkt"]), o.geschwindigkeit_an(r["dreieck"], r["punkt"]))
    g.nachfuehren(p)  # clears the field, as nachfuehren does
    assert np.array_equal(g.geschwindigkeit_an(r["dreieck"][:5], r["punkt"][:5], (1.0, 2.0, 3.0)),
                          np.tile([1.0, 2.0, 3.0], (5, 1)))
