"""Synthetic pattern meshes and collider grids for the benchmark workloads.

The reference meshes real pattern files with its own mesher (klon3d-mesh,
out of scope here). These generators produce the same kind of input the
scene builder reads — pieces in pattern coordinates (mm), positively oriented
triangles, a grainline per piece, seam point pairs at equal length fraction
(crates/klon3d-mesh/src/lib.rs:178-228) and a start position per point —
from a seed, with numpy only.

Workloads (sizes as named by the benchmark configurations):
  * ``tube``: closed tube, rest circumference 40 cm, height 20 cm, ~10 mm
    edges, fitted over an analytic cylinder of radius 8 cm;
  * ``sheet_over_sphere``: 1.0 x 1.0 m sheet on a 257 x 257 vertex grid with
    +/-1 mm in-plane jitter, dropped 0.5 m onto a sphere stored as a 128^3
    signed-distance grid at 1 cm spacing.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi


@dataclass
class Material:
    """Fabric record (sim/src/material.rs:21-68), SI units."""
    dehnung_n_m: float
    kette_n_m: float
    schub_n_m: float
    biegung_nm: float
    biegung_kette_nm: float
    biegung_schraege_nm: float
    flaechengewicht_kg_m2: float
    dicke_m: float
    reibung: float

    def to_c(self) -> _abi.K3dMaterial:
        return _abi.K3dMaterial(self.dehnung_n_m, self.kette_n_m, self.schub_n_m, self.biegung_nm,
                                self.biegung_kette_nm, self.biegung_schraege_nm,
                                self.flaechengewicht_kg_m2, self.dicke_m, self.reibung)


# Fabric profiles shipped with the reference (sim/src/material.rs:73-102).
RADICAL_RUBBER_04 = Material(348.2741562, 348.2817188, 174.1590469, 2482.2424e-9, 2486.4924e-9,
                             2486.4924e-9, 0.3489899, 0.4e-3, 0.03)
RETIFIST_NR_040 = Material(33.333332, 33.333332, 6.6666665, 60.361e-9, 60.361e-9, 60.361e-9,
                           0.380, 0.4e-3, 0.03)


@dataclass
class Simparameter:
    """Simparameter (sim/src/szene.rs:96-126), the fields the implicit step reads."""
    bild_dt: float = 1.0 / 60.0
    schwerkraft: tuple = (0.0, 0.0, -9.81)
    daempfung: float = 0.0

    def to_c(self) -> _abi.K3dSimparams:
        return _abi.K3dSimparams(self.bild_dt, (C.c_double * 3)(*self.schwerkraft), self.daempfung)


@dataclass
class Teil:
    punkte_mm: np.ndarray            # (n, 2) float64
    dreiecke: np.ndarray             # (t, 3) uint32
    fadenlauf: tuple
    material: Material
    lage: np.ndarray                 # (n, 3) float64, metres
    reduktion: float = 0.0


@dataclass
class Teilnaht:
    teil_a: int
    teil_b: int
    paare: np.ndarray                # (k, 2) uint32, local indices on a and b


@dataclass
class Naht:
    teilnaehte: list
    laenge_a_mm: float = 0.0
    laenge_b_mm: float = 0.0


@dataclass
class Muster:
    """A pattern: pieces, seams and the scene parameters."""
    teile: list
    naehte: list = field(default_factory=list)
    param: Simparameter = field(default_factory=Simparameter)
    naht_nachgiebigkeit: float = 0.0
    einhalteweite: bool = False

    def to_c(self):
        """The k3d_pattern struct plus the objects that keep its memory alive."""
        keep = []
        pieces = (_abi.K3dPiece * max(len(self.teile), 1))()
        for k, t in enumerate(self.teile):
            pm = np.ascontiguousarray(t.punkte_mm, dtype=np.float64)
            dr = np.ascontiguousarray(t.dreiecke, dtype=np.uint32)
            la = np.ascontiguousarray(t.lage, dtype=np.float64)
            keep += [pm, dr, la]
            pieces[k] = _abi.K3dPiece(pm.shape[0], _abi.ptr(pm, C.c_double), dr.shape[0],
                                      _abi.ptr(dr, C.c_uint32),
                                      (C.c_double * 2)(*t.fadenlauf), t.material.to_c(),
                                      t.reduktion, _abi.ptr(la, C.c_double))
        seams = (_abi.K3dSeam * max(len(self.naehte), 1))()
        for k, n in enumerate(self.naehte):
            parts = (_abi.K3dSeamPart * max(len(n.teilnaehte), 1))()
            for q, tn in enumerate(n.teilnaehte):
                pr = np.ascontiguousarray(tn.paare, dtype=np.uint32)
                keep.append(pr)
                parts[q] = _abi.K3dSeamPart(tn.teil_a, tn.teil_b, pr.shape[0], _abi.ptr(pr, C.c_uint32))
            keep.append(parts)
            seams[k] = _abi.K3dSeam(len(n.teilnaehte), 0, parts, n.laenge_a_mm, n.laenge_b_mm)
        keep += [pieces, seams]
        pat = _abi.K3dPattern(len(self.teile), len(self.naehte), pieces, seams, self.param.to_c(),
                              self.naht_nachgiebigkeit, 1 if self.einhalteweite else 0, 0)
        return pat, keep


def rechteck_netz(breite_mm: float, hoehe_mm: float, nx: int, ny: int, jitter_mm: float = 0.0,
                  seed: int = 0):
    """Regular grid of (nx+1) x (ny+1) points, two positive triangles per cell.

    Point (i, j) has index j*(nx+1) + i. With ``jitter_mm`` every point moves
    by U(-jitter, jitter) in x and y (seeded)."""
    xs = np.linspace(0.0, breite_mm, nx + 1)
    ys = np.linspace(0.0, hoehe_mm, ny + 1)
    gx, gy = np.meshgrid(xs, ys)
    p = np.stack([gx.ravel(), gy.ravel()], axis=1)
    if jitter_mm > 0.0:
        rng = np.random.default_rng(seed)
        p = p + rng.uniform(-jitter_mm, jitter_mm, size=p.shape)
    i = np.arange(nx)
    j = np.arange(ny)
    ii, jj = np.meshgrid(i, j)
    a = (jj * (nx + 1) + ii).ravel()
    b = a + 1
    c = a + nx + 2
    d = a + nx + 1
    tri = np.empty((2 * a.size, 3), dtype=np.uint32)
    tri[0::2] = np.stack([a, b, c], axis=1)
    tri[1::2] = np.stack([a, c, d], axis=1)
    return p, tri


# ------------------------------------------------------------------ tube
TUBE_MATERIAL = Material(600.0, 600.0, 300.0, 1e-7, 1e-7, 1e-7, 0.5, 0.5e-3, 0.03)


def tube(umfang_m: float = 0.40, hoehe_m: float = 0.20, kante_mm: float = 10.0,
         zylinder_radius_m: float = 0.08, anfangsabstand_m: float = 0.005,
         material: Material = TUBE_MATERIAL):
    """Closed tube over a cylinder (the reference's tube acceptance case,
    sim/src/roehre.rs:197-239, built without the mesher).

    The rectangle's right side is sewn to its left side (roehre.rs:45, B->C
    against A->D), the two sides keep their own points. Start position: rolled
    all the way round at radius R + t/2 + ``anfangsabstand_m``, seam closed.
    Returns (muster, cylinder body dict)."""
    nx = int(round(umfang_m * 1e3 / kante_mm))
    ny = int(round(hoehe_m * 1e3 / kante_mm))
    p, tri = rechteck_netz(umfang_m * 1e3, hoehe_m * 1e3, nx, ny)
    r0 = zylinder_radius_m + material.dicke_m / 2.0 + anfangsabstand_m
    je_m = 2.0 * math.pi / umfang_m
    u = p[:, 0] * 1e-3
    y = p[:, 1] * 1e-3
    w = u * je_m
    lage = np.stack([r0 * np.cos(w), r0 * np.sin(w), -y], axis=1)
    rechts = np.arange(ny + 1) * (nx + 1) + nx
    links = np.arange(ny + 1) * (nx + 1)
    paare = np.stack([rechts, links], axis=1).astype(np.uint32)
    teil = Teil(p, tri, (1.0, 0.0), material, lage)
    naht = Naht([Teilnaht(0, 0, paare)], hoehe_m * 1e3, hoehe_m * 1e3)
    param = Simparameter(bild_dt=1.0 / 60.0, schwerkraft=(0.0, 0.0, 0.0), daempfung=5.0)
    body = dict(art=_abi.K3D_BODY_CYLINDER, punkt=(0.0, 0.0, 0.0), achse=(0.0, 0.0, 1.0),
                radius=zylinder_radius_m)
    return Muster([teil], [naht], param), body


# ------------------------------------------------------------------ sheet over a sphere
SHEET_MATERIAL = Material(dehnung_n_m=1000.0, kette_n_m=2000.0, schub_n_m=50.0, biegung_nm=5e-6,
                          biegung_kette_nm=5e-6, biegung_schraege_nm=5e-6,
                          flaechengewicht_kg_m2=0.2, dicke_m=0.5e-3, reibung=0.3)


def sphere_sdf_grid(radius_m: float, n: int, spacing_m: float, zentrum=(0.0, 0.0, 0.0)):
    """Signed distance of a sphere sampled at the nodes of an n^3 grid
    centred on the sphere. Returns a body dict for a K3D_BODY_SDF_GRID."""
    half = 0.5 * (n - 1) * spacing_m
    ax = np.arange(n, dtype=np.float64) * spacing_m - half
    gz, gy, gx = np.meshgrid(ax, ax, ax, indexing="ij")
    d = np.sqrt(gx * gx + gy * gy + gz * gz) - radius_m
    return dict(art=_abi.K3D_BODY_SDF_GRID, punkt=tuple(zentrum), dims=(n, n, n),
                ursprung=(-half, -half, -half), spacing=spacing_m,
                sdf=np.ascontiguousarray(d.astype(np.float32)))


def sheet_over_sphere(n: int = 257, groesse_m: float = 1.0, jitter_mm: float = 1.0, seed: int = 0,
                      fall_m: float = 0.5, kugel_radius_m: float = 0.3, sdf_n: int = 128,
                      sdf_spacing_m: float = 0.01, material: Material = SHEET_MATERIAL,
                      bild_dt: float = 1.0 / 120.0, winkel: float | None = None):
    """Woven sheet dropped onto a sphere collider.

    n x n vertices over ``groesse_m`` square, in-plane jitter U(-1, 1) mm,
    grainline angle U[0, pi) from the seed (or ``winkel``), start plane
    ``fall_m`` above the sphere top. Returns (muster, sphere SDF body dict)."""
    rng = np.random.default_rng(seed)
    w0 = float(rng.uniform(0.0, math.pi))
    winkel = w0 if winkel is None else float(winkel)
    p, tri = rechteck_netz(groesse_m * 1e3, groesse_m * 1e3, n - 1, n - 1, jitter_mm, seed + 1)
    z0 = kugel_radius_m + fall_m
    lage = np.stack([p[:, 0] * 1e-3 - 0.5 * groesse_m, p[:, 1] * 1e-3 - 0.5 * groesse_m,
                     np.full(p.shape[0], z0)], axis=1)
    teil = Teil(p, tri, (math.cos(winkel), math.sin(winkel)), material, lage)
    param = Simparameter(bild_dt=bild_dt, schwerkraft=(0.0, 0.0, -9.81), daempfung=0.0)
    body = sphere_sdf_grid(kugel_radius_m, sdf_n, sdf_spacing_m)
    return Muster([teil], [], param), body


# ------------------------------------------------------------------ sewn garment
def kapsel_sdf(segmente, dims, spacing_m: float, ursprung, band_m: float = 0.06):
    """Signed distance of a union of capsules (segments (a, b, radius)) at the
    nodes of a grid (x fastest), in float32: exact within ``band_m`` of each
    capsule, ``band_m`` beyond (contact queries only read the values near the
    surface). Returns a body dict."""
    nx, ny, nz = dims
    o = np.asarray(ursprung, dtype=np.float64)
    out = np.full((nz, ny, nx), band_m, dtype=np.float32)
    for a, b, r in segmente:
        a = np.asarray(a, dtype=np.float64)
        b = np.asarray(b, dtype=np.float64)
        lo = np.floor((np.minimum(a, b) - r - band_m - o) / spacing_m).astype(int)
        hi = np.ceil((np.maximum(a, b) + r + band_m - o) / spacing_m).astype(int) + 1
        lo = np.maximum(lo, 0)
        hi = np.minimum(hi, [nx, ny, nz])
        if np.any(hi <= lo):
            continue
        zs = o[2] + spacing_m * np.arange(lo[2], hi[2])
        ys = o[1] + spacing_m * np.arange(lo[1], hi[1])
        xs = o[0] + spacing_m * np.arange(lo[0], hi[0])
        gz, gy, gx = np.meshgrid(zs, ys, xs, indexing="ij")
        p = np.stack([gx, gy, gz], axis=-1)
        ab = b - a
        t = np.clip(((p - a) @ ab) / float(ab @ ab), 0.0, 1.0)
        d = np.linalg.norm(p - (a + t[..., None] * ab), axis=-1) - r
        sub = out[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
        np.minimum(sub, np.minimum(d, band_m).astype(np.float32), out=sub)
    return dict(art=_abi.K3D_BODY_SDF_GRID, punkt=(0.0, 0.0, 0.0), dims=(nx, ny, nz), ursprung=tuple(ursprung),
                spacing=spacing_m, sdf=np.ascontiguousarray(out.ravel()))


# Body proxy: 15 capsules (a, b, radius), metres, z up, A-pose.
KOERPER_KAPSELN = [
    ((0.0, 0.0, 0.95), (0.0, 0.0, 1.08), 0.150),    # hips
    ((0.0, 0.0, 1.08), (0.0, 0.0, 1.24), 0.125),    # waist
    ((0.0, 0.0, 1.24), (0.0, 0.0, 1.40), 0.150),    # chest
    ((0.0, 0.0, 1.44), (0.0, 0.0, 1.58), 0.055),    # neck
    ((0.0, 0.0, 0.88), (0.0, 0.0, 0.95), 0.140),    # pelvis
    ((0.09, 0.0, 0.86), (0.11, 0.0, 0.45), 0.075),  # thighs
    ((-0.09, 0.0, 0.86), (-0.11, 0.0, 0.45), 0.075),
    ((0.12, 0.0, 1.42), (0.22, 0.0, 1.40), 0.060),  # shoulders
    ((-0.12, 0.0, 1.42), (-0.22, 0.0, 1.40), 0.060),
    ((0.22, 0.0, 1.40), (0.38, 0.0, 1.16), 0.050),  # upper arms
    ((-0.22, 0.0, 1.40), (-0.38, 0.0, 1.16), 0.050),
    ((0.38, 0.0, 1.16), (0.50, 0.0, 0.92), 0.040),  # forearms
    ((-0.38, 0.0, 1.16), (-0.50, 0.0, 0.92), 0.040),
    ((0.50, 0.0, 0.92), (0.54, 0.0, 0.84), 0.035),  # hands
    ((-0.50, 0.0, 0.92), (-0.54, 0.0, 0.84), 0.035),
]


def garment(seed: int = 0, ziel_punkte: int = 200_000, sdf: bool = True):
    """The sewn-garment workload: 28 panels (rectangles or trapezoids, sides
    10-60 cm) rolled on cylinders around a body proxy of 15 capsules, voxelised
    into a 256 x 256 x 384 SDF at 5 mm. Tubes: 8 panels round the torso, 4
    round each upper arm and each forearm, 4 round the neck; neighbouring
    panels of a tube are sewn side to side (points paired at equal length
    fractions), each upper sleeve to its forearm sleeve. Latex: E U(1.0, 1.5)
    MPa per panel, G = E/2, 0.5 mm, 1000 kg/m^3, friction 0.4, collision
    thickness 2 mm (the scene's kollisionsabstand), dt 1/120 s. The mesh
    spacing is chosen so that the garment has about ``ziel_punkte`` points.
    Returns (muster, body dict or None)."""
    rng = np.random.default_rng(seed)
    # tubes: (centre of the axis start, axis end, radius of the cloth, panels, height)
    k = KOERPER_KAPSELN

    def aermel(kap, ab):  # sleeve tube along a capsule, starting a fraction `ab` down it
        a, b, r = np.asarray(kap[0]), np.asarray(kap[1]), kap[2]
        return (a + ab * (b - a), b, r + 0.025, 4)

    rohre = [((0.0, 0.0, 0.98), (0.0, 0.0, 1.30), 0.180, 8),                  # torso
             aermel(k[9], 0.3), aermel(k[10], 0.3), aermel(k[11], 0.0), aermel(k[12], 0.0),
             ((0.0, 0.0, 1.54), (0.0, 0.0, 1.62), 0.085, 4)]                   # collar
    flaeche = 0.0
    geo = []
    for a, b, r, np_ in rohre:
        a = np.asarray(a, dtype=np.float64)
        b = np.asarray(b, dtype=np.float64)
        hoehe = float(np.linalg.norm(b - a))
        breite = 2.0 * math.pi * r / np_
        # trapezoid: the panels of a tube share their height; the top edge
        # is narrower or wider by up to 15 % (the tube becomes a cone)
        konus = float(rng.uniform(-0.15, 0.15))
        geo.append((a, b, r, np_, hoehe, breite, konus))
        flaeche += np_ * hoehe * breite * (1.0 + 0.5 * konus)
    h_mm = 1e3 * math.sqrt(flaeche / ziel_punkte)
    teile, naehte = [], []
    for ri, (a, b, r, np_, hoehe, breite, konus) in enumerate(geo):
        achse = (b - a) / hoehe
        e1 = np.cross(achse, [0.0, 1.0, 0.0])
        if np.linalg.norm(e1) < 1e-6:
            e1 = np.cross(achse, [1.0, 0.0, 0.0])
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(achse, e1)
        nx = max(int(round(breite * 1e3 / h_mm)), 2)
        ny = max(int(round(hoehe * 1e3 / h_mm)), 2)
        erst = len(teile)
        for q in range(np_):
            p, tri = rechteck_netz(breite * 1e3, hoehe * 1e3, nx, ny)
            # trapezoid in the pattern plane: width scales with the height
            sk = 1.0 + konus * p[:, 1] / (hoehe * 1e3)
            p2 = np.stack([(p[:, 0] - 0.5 * breite * 1e3) * sk + 0.5 * breite * 1e3, p[:, 1]], axis=1)
            E = float(rng.uniform(1.0e6, 1.5e6)) * 0.5e-3
            mat = Material(dehnung_n_m=E, kette_n_m=E, schub_n_m=0.5 * E, biegung_nm=1e-7, biegung_kette_nm=1e-7,
                           biegung_schraege_nm=1e-7, flaechengewicht_kg_m2=0.5, dicke_m=0.5e-3, reibung=0.4)
            # roll onto the tube: the panel's u runs round the axis
            u = p2[:, 0] * 1e-3 + q * breite
            v = p2[:, 1] * 1e-3
            rr = r * (1.0 + konus * v / hoehe)
            w = u / r
            lage = a + np.outer(v, achse) + (rr * np.cos(w))[:, None] * e1 + (rr * np.sin(w))[:, None] * e2
            teile.append(Teil(p2, tri, (1.0, 0.0), mat, lage))
        links = np.arange(ny + 1) * (nx + 1)
        rechts = links + nx
        for q in range(np_):
            ta, tb = erst + q, erst + (q + 1) % np_
            paare = np.stack([rechts, links], axis=1).astype(np.uint32)
            naehte.append(Naht([Teilnaht(ta, tb, paare)], hoehe * 1e3, hoehe * 1e3))
        geo[ri] = geo[ri] + (erst, nx, ny)
    # each upper sleeve's far end (its top row) to the forearm sleeve's near
    # end (bottom row), panel by panel; the shorter edge's points pair with
    # the points at the same length fraction of the longer one
    for ob, un in ((1, 3), (2, 4)):
        _, _, _, np_a, _, _, _, ea, nxa, nya = geo[ob]
        _, _, _, np_b, _, _, _, eb, nxb, nyb = geo[un]
        oben = nya * (nxa + 1) + np.arange(nxa + 1)
        unten = np.arange(nxb + 1)
        if nxa <= nxb:
            ib = np.rint(np.arange(nxa + 1) * (nxb / nxa)).astype(np.int64)
            paare = np.stack([oben, unten[ib]], axis=1)
        else:
            ia = np.rint(np.arange(nxb + 1) * (nxa / nxb)).astype(np.int64)
            paare = np.stack([oben[ia], unten], axis=1)
        for q in range(min(np_a, np_b)):
            naehte.append(Naht([Teilnaht(ea + q, eb + q, paare.astype(np.uint32))], 1.0, 1.0))
    param = Simparameter(bild_dt=1.0 / 120.0, schwerkraft=(0.0, 0.0, -9.81), daempfung=0.0)
    body = None
    if sdf:
        body = kapsel_sdf(KOERPER_KAPSELN, (256, 256, 384), 0.005, (-0.6375, -0.6375, 0.0))
    return Muster(teile, naehte, param), body


def garment_szene(seed: int = 0, ziel_punkte: int = 200_000, sdf: bool = True):
    """The garment workload as a scene: ``garment`` built with the library's
    scene builder, collision thickness 2 mm on every point. Returns (szene,
    body dict or None)."""
    from .implizit import build_scene
    m, body = garment(seed, ziel_punkte, sdf)
    s = build_scene(m, [body] if body is not None else [])
    s.kollisionsabstand[:] = 2e-3
    return s, body


# ------------------------------------------------------------------ material fit
def materialfit(n: int = 129, seed: int = 0):
    """The material-fit workload: an n x n sheet (1 x 1 m) dropped onto the
    sphere of the sheet workload (R 0.3 m, 128^3 SDF at 1 cm). Hidden
    parameters from the seed, uniform in warp 1000-2000, weft 500-1000, shear
    25-50 N/m, bending 2.5e-6-5e-6 N m (all three directions), grain angle
    [0, pi); the fit starts from them scaled by U(0.5, 2) each. Returns
    (szene at the hidden parameters, hidden (warp, weft, shear, bend, grain),
    start parameters)."""
    from .implizit import build_scene
    rng = np.random.default_rng(seed + 7919)
    verdeckt = np.array([rng.uniform(1000.0, 2000.0), rng.uniform(500.0, 1000.0), rng.uniform(25.0, 50.0),
                         rng.uniform(2.5e-6, 5e-6), rng.uniform(0.0, math.pi)])
    start = verdeckt * rng.uniform(0.5, 2.0, size=5)
    b = float(verdeckt[3])
    mat = Material(dehnung_n_m=float(verdeckt[1]), kette_n_m=float(verdeckt[0]), schub_n_m=float(verdeckt[2]),
                   biegung_nm=b, biegung_kette_nm=b, biegung_schraege_nm=b, flaechengewicht_kg_m2=0.2,
                   dicke_m=0.5e-3, reibung=0.3)
    m, body = sheet_over_sphere(n=n, seed=seed, material=mat, winkel=float(verdeckt[4]))
    return build_scene(m, [body]), verdeckt, start


# ------------------------------------------------------------------ batched drapes
def capsule_sdf_grid(radius_m: float, halbe_laenge_m: float, n: int, zentrum=(0.0, 0.0, 0.0)):
    """Signed distance of a capsule (segment along x of half length
    ``halbe_laenge_m``, radius ``radius_m``) sampled on an n^3 grid that holds
    it with a margin. Returns a body dict for a K3D_BODY_SDF_GRID."""
    ausdehnung = 2.0 * (halbe_laenge_m + radius_m) * 1.2
    spacing = ausdehnung / (n - 1)
    half = 0.5 * (n - 1) * spacing
    ax = np.arange(n, dtype=np.float64) * spacing - half
    gz, gy, gx = np.meshgrid(ax, ax, ax, indexing="ij")
    px = np.clip(gx, -halbe_laenge_m, halbe_laenge_m)
    d = np.sqrt((gx - px) ** 2 + gy * gy + gz * gz) - radius_m
    return dict(art=_abi.K3D_BODY_SDF_GRID, punkt=tuple(zentrum), dims=(n, n, n),
                ursprung=(-half, -half, -half), spacing=spacing, sdf=np.ascontiguousarray(d.astype(np.float32)))


def drape(nx: int, ny: int, kante_m: float, material: Material, winkel: float, body: dict, fall_m: float,
          koerper_oben_m: float, seed: int, jitter_frac: float = 0.25, bild_dt: float = 1.0 / 120.0):
    """A rectangular sheet of (nx + 1) x (ny + 1) vertices at spacing
    ``kante_m``, centred over the body, ``fall_m`` above the body's top, with
    in-plane jitter of ``jitter_frac`` of the spacing. Returns (muster, body)."""
    rng_j = jitter_frac * kante_m * 1e3
    p, tri = rechteck_netz(nx * kante_m * 1e3, ny * kante_m * 1e3, nx, ny, rng_j, seed)
    z0 = koerper_oben_m + fall_m
    lage = np.stack([p[:, 0] * 1e-3 - 0.5 * nx * kante_m, p[:, 1] * 1e-3 - 0.5 * ny * kante_m,
                     np.full(p.shape[0], z0)], axis=1)
    teil = Teil(p, tri, (math.cos(winkel), math.sin(winkel)), material, lage)
    param = Simparameter(bild_dt=bild_dt, schwerkraft=(0.0, 0.0, -9.81), daempfung=0.0)
    return Muster([teil], [], param), body


def drape_batch(anzahl: int = 64, seed: int = 0, n_min: int = 2000, n_max: int = 60000, kante_m: float = 1.0 / 256,
                fall_m: float = 0.1):
    """The batched-drape workload: ``anzahl`` sheets with vertex counts
    log-uniform in [n_min, n_max], aspect ratio U(1, 3), the C2 sheet's
    spacing and areal density, warp U(1000, 2000), weft U(500, 1000), shear
    U(25, 50) N/m, bending U(2.5e-6, 5e-6) N m, grain angle U[0, pi), each
    falling onto its own sphere or capsule sampled on a 64^3 grid. Returns a
    list of (muster, body)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(anzahl):
        nv = float(np.exp(rng.uniform(math.log(n_min), math.log(n_max))))
        asp = float(rng.uniform(1.0, 3.0))
        ny = max(int(round(math.sqrt(nv / asp))) - 1, 2)
        nx = max(int(round(asp * (ny + 1))) - 1, 2)
        bend = float(rng.uniform(2.5e-6, 5e-6))
        mat = Material(dehnung_n_m=float(rng.uniform(500.0, 1000.0)), kette_n_m=float(rng.uniform(1000.0, 2000.0)),
                       schub_n_m=float(rng.uniform(25.0, 50.0)), biegung_nm=bend, biegung_kette_nm=bend,
                       biegung_schraege_nm=bend, flaechengewicht_kg_m2=0.2, dicke_m=0.5e-3, reibung=0.3)
        winkel = float(rng.uniform(0.0, math.pi))
        laenge = max(nx, ny) * kante_m
        if rng.uniform() < 0.5:
            r = 0.3 * laenge
            body = sphere_sdf_grid(r, 64, 2.4 * r / 63)
            oben = r
        else:
            r = 0.15 * laenge
            body = capsule_sdf_grid(r, 0.3 * nx * kante_m, 64)
            oben = r
        out.append(drape(nx, ny, kante_m, mat, winkel, body, fall_m, oben, seed * 1000 + k))
    return out


# ------------------------------------------------------------------ two layers
def zwei_lagen(groesse_m: float = 0.2, kante_mm: float = 10.0, abstand_m: float = 0.01,
               material: Material = RADICAL_RUBBER_04, neigung: float = 0.0, z_unten: float = 0.0,
               oben_groesse_m: float | None = None, versatz_m=(0.0, 0.0)):
    """Two square pieces, the upper one ``abstand_m`` above the lower (the
    reference's self-collision scene, sim/tests/selbstkollision.rs:15-32,
    meshed as a regular grid instead of by the mesher). The upper piece has
    side ``oben_groesse_m`` (default: the same) and is shifted by
    ``versatz_m`` in x and y. With ``neigung`` it is tilted:
    z = z_unten + abstand_m + neigung * x. Frame 1/30 s, air damping 1. Pin
    the lower piece's points (w = 0) with ``pin_teil(szene, 0)``. Returns the
    pattern."""
    nk = int(round(groesse_m * 1e3 / kante_mm))
    p, tri = rechteck_netz(groesse_m * 1e3, groesse_m * 1e3, nk, nk)
    xm, ym = p[:, 0] * 1e-3, p[:, 1] * 1e-3
    unten = np.stack([xm, ym, np.full(xm.shape, z_unten)], axis=1)
    go = groesse_m if oben_groesse_m is None else oben_groesse_m
    no = int(round(go * 1e3 / kante_mm))
    q, tq = rechteck_netz(go * 1e3, go * 1e3, no, no)
    xo, yo = q[:, 0] * 1e-3 + versatz_m[0], q[:, 1] * 1e-3 + versatz_m[1]
    oben = np.stack([xo, yo, z_unten + abstand_m + neigung * xo], axis=1)
    teile = [Teil(p, tri, (1.0, 0.0), material, unten), Teil(q, tq, (1.0, 0.0), material, oben)]
    param = Simparameter(bild_dt=1.0 / 30.0, schwerkraft=(0.0, 0.0, -9.81), daempfung=1.0)
    return Muster(teile, [], param)


def pin_teil(szene, teil: int) -> None:
    """Holds every point of one piece (w = 0), as the reference's tests do."""
    a, b = int(szene.teil_bereiche[teil, 0]), int(szene.teil_bereiche[teil, 1])
    szene.w[a:b] = 0.0


def body_to_c(body: dict) -> _abi.K3dBody:
    """k3d_body from a body dict; the dict keeps the SDF array alive."""
    kb = _abi.K3dBody()
    kb.art = body["art"]
    for a in range(3):
        kb.dims[a] = body.get("dims", (0, 0, 0))[a]
        kb.punkt[a] = body.get("punkt", (0.0, 0.0, 0.0))[a]
        kb.achse[a] = body.get("achse", (0.0, 0.0, 1.0))[a]
        kb.geschwindigkeit[a] = body.get("geschwindigkeit", (0.0, 0.0, 0.0))[a]
        kb.ursprung[a] = body.get("ursprung", (0.0, 0.0, 0.0))[a]
    kb.radius = body.get("radius", 0.0)
    kb.spacing = body.get("spacing", 1.0)
    kb.instanz = int(body.get("instanz", -1))
    sdf = body.get("sdf")
    kb.sdf = _abi.ptr(sdf, C.c_float) if sdf is not None else None
    netz = body.get("netz")
    kb.netz = netz.c_handle if netz is not None else None
    return kb


# ------------------------------------------------------------------ body meshes
def wuerfel_netz(h: float = 1.0):
    """The cube [-h, h]^3 as 12 triangles, counter-clockwise from outside.
    Corner i has the signs of its bits (x: 1, y: 2, z: 4); each face splits
    along its diagonal from the (-, -) to the (+, +) corner of its two
    in-plane axes. Returns (points (8, 3), triangles (12, 3))."""
    p = np.array([[h if i & 1 else -h, h if i & 2 else -h, h if i & 4 else -h] for i in range(8)], dtype=np.float64)
    d = []
    for a in range(3):
        b, c = (a + 1) % 3, (a + 2) % 3
        for s in (-1, 1):
            def ecke(u, v):
                bits = {a: s > 0, b: u > 0, c: v > 0}
                return sum(1 << k for k in range(3) if bits[k])
            q = [ecke(-1, -1), ecke(1, -1), ecke(1, 1), ecke(-1, 1)]  # counter-clockwise about +e_a
            if s < 0:
                q = [q[0], q[3], q[2], q[1]]
            d += [[q[0], q[1], q[2]], [q[0], q[2], q[3]]]
    return p, np.asarray(d, dtype=np.uint32)


def zylinder_netz(radius: float, z_unten: float, z_oben: float, segmente: int, ringe: int):
    """A closed cylinder about the z axis (netzkoerper.rs:934-962): `segmente`
    points per ring, `ringe` bands between z_unten and z_oben, each cap a fan
    about its centre point, outward normals."""
    s, r = max(segmente, 3), max(ringe, 1)
    w = 2.0 * math.pi * np.arange(s) / s
    z = z_unten + (z_oben - z_unten) * np.arange(r + 1) / r
    ring = np.stack([radius * np.cos(w), radius * np.sin(w)], axis=1)
    p = np.concatenate([np.column_stack([ring, np.full(s, zi)]) for zi in z]
                       + [np.array([[0.0, 0.0, z_unten], [0.0, 0.0, z_oben]])])
    unten, oben = (r + 1) * s, (r + 1) * s + 1

    def idx(i, j):
        return i * s + j % s
    d = []
    for i in range(r):
        for j in range(s):
            a, b, c, e = idx(i, j), idx(i, j + 1), idx(i + 1, j + 1), idx(i + 1, j)
            d += [[a, b, c], [a, c, e]]
    for j in range(s):
        d.append([unten, idx(0, j + 1), idx(0, j)])
        d.append([oben, idx(r, j), idx(r, j + 1)])
    return p, np.asarray(d, dtype=np.uint32)


def koerper_netz(segmente: int = 256, ringe: int = 73, halbachsen=(0.18, 0.12, 0.85), mitte=(0.0, 0.0, 0.9),
                 seed: int = 0):
    """A closed, star-shaped body surface standing in for a scanned body
    mesh: a latitude-longitude ellipsoid with the given half axes whose radius
    is modulated by low-order waves (amplitudes from the seed, radius factor
    in [0.7, 1.3]), `ringe - 1` rings of `segmente` points plus two poles,
    2 * segmente * (ringe - 1) triangles (36,864 at the defaults, the size of
    a human base mesh split into triangles). Outward normals."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(-0.05, 0.05, size=(4, 4))
    th = math.pi * np.arange(1, ringe) / ringe
    ph = 2.0 * math.pi * np.arange(segmente) / segmente
    T, Ph = np.meshgrid(th, ph, indexing="ij")
    f = np.ones_like(T)
    for m in range(4):
        for k in range(4):
            f += amp[m, k] * np.sin((m + 1) * T) * np.cos(k * Ph + m)
    f = np.clip(f, 0.7, 1.3)
    x = halbachsen[0] * f * np.sin(T) * np.cos(Ph)
    y = halbachsen[1] * f * np.sin(T) * np.sin(Ph)
    z = halbachsen[2] * f * np.cos(T)
    p = np.column_stack([x.ravel(), y.ravel(), z.ravel()])
    p = np.concatenate([p, [[0.0, 0.0, halbachsen[2]], [0.0, 0.0, -halbachsen[2]]]]) + np.asarray(mitte)
    nord, sued = p.shape[0] - 2, p.shape[0] - 1
    s = segmente

    def idx(i, j):
        return i * s + j % s
    d = []
    for i in range(ringe - 2):
        for j in range(s):
            a, b, c, e = idx(i, j), idx(i, j + 1), idx(i + 1, j + 1), idx(i + 1, j)
            d += [[a, c, b], [a, e, c]]
    for j in range(s):
        d.append([nord, idx(0, j), idx(0, j + 1)])
        d.append([sued, idx(ringe - 2, j + 1), idx(ringe - 2, j)])
    d = np.asarray(d, dtype=np.uint32)
    q = p[d.astype(np.int64)]
    if np.einsum("ij,ij->i", q[:, 0], np.cross(q[:, 1], q[:, 2])).sum() < 0.0:
        d = d[:, [0, 2, 1]]
    return p, np.ascontiguousarray(d)


def punkteregen(netz_punkte, kante_m: float = 0.01, hoehe_m: float = 0.05, rand_m: float = 0.02):
    """Loose points raining onto a body mesh: a grid at `kante_m` spacing
    over the mesh's footprint grown by `rand_m`, `hoehe_m` above its top, at
    rest; mass 1e-5 kg, collision distance 0.2 mm, friction 0.6, gravity
    only (the point rain of the reference's mesh-body tests,
    sim/tests/band/mod.rs:279-315, over a synthetic body). No body is
    attached; add one to the scene's koerper."""
    from .szene import Szene
    p = np.asarray(netz_punkte, dtype=np.float64)
    lo, hi = p.min(axis=0) - rand_m, p.max(axis=0) + rand_m
    xs = np.arange(lo[0], hi[0] + 0.5 * kante_m, kante_m)
    ys = np.arange(lo[1], hi[1] + 0.5 * kante_m, kante_m)
    gx, gy = np.meshgrid(xs, ys, indexing="ij")
    x = np.column_stack([gx.ravel(), gy.ravel(), np.full(gx.size, hi[2] - rand_m + hoehe_m)])
    n = x.shape[0]
    m = 1e-5

    def leer(cols, dt=np.float64):
        return np.zeros((0, cols) if cols else 0, dtype=dt)
    return Szene(x=x, v=np.zeros((n, 3)), masse=np.full(n, m), w=np.full(n, 1.0 / m),
                 kollisionsabstand=np.full(n, 0.2e-3), reibung=np.full(n, 0.6),
                 abstand_punkte=leer(2, np.uint32), abstand_ruhe=leer(0), abstand_nachgiebigkeit=leer(0),
                 membran_kante=leer(0, np.uint8), naht_punkte=leer(2, np.uint32), naht_ruhe=leer(0),
                 biegung_punkte=leer(4, np.uint32), biegung_ruhe=leer(0), biegung_nachgiebigkeit=leer(0),
                 membran_punkte=leer(3, np.uint32), membran_flaeche=leer(0), membran_ruhe_inv=leer(4),
                 membran_kette=leer(2), membran_schuss=leer(2), membran_steif=leer(3),
                 dreiecke=leer(3, np.uint32), ruhe_inv=leer(4),
                 param=Simparameter(bild_dt=1.0 / 60.0, schwerkraft=(0.0, 0.0, -9.81), daempfung=0.0))
