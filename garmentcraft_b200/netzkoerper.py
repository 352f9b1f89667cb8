"""The body mesh as a signed-distance collider on the device: the host-side
mirror of ``Koerpernetz`` (sim/src/netzkoerper.rs:145-800) over the C ABI of
include/klon3d_mesh.h.

Names and argument meaning follow the reference: ``Koerpernetz(punkte,
dreiecke, suchtiefe)`` refuses what ``Koerpernetz::neu`` refuses (the reason
in the raised error), ``nachfuehren`` moves the points, ``naechster`` answers
within a radius, ``naechster_alle`` over every triangle, ``durchstoss`` tests
segments. The queries take a batch of points (shape (m, 3)) and return arrays.
``sdf`` voxelises the mesh into the sampled grid a K3D_BODY_SDF_GRID body
reads. There is no CPU path: without the device library this module raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._lib import K3dError, lib

SUCHTIEFE = 0.01  # netzkoerper.rs:46
REGION_NAMEN = {0: "Ecke(0)", 1: "Ecke(1)", 2: "Ecke(2)", 3: "Kante(0)", 4: "Kante(1)", 5: "Kante(2)",
                6: "Flaeche", -1: None}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def _d(a):
    return a.ctypes.data_as(_dp)


def _f64(a, form=(-1, 3)):
    return np.ascontiguousarray(a, dtype=np.float64).reshape(form)


class Koerpernetz:
    def __init__(self, punkte, dreiecke, suchtiefe: float = SUCHTIEFE, device: int = 0):
        self._L = lib()
        p = _f64(punkte)
        d = np.ascontiguousarray(dreiecke, dtype=np.uint32).reshape(-1, 3)
        self.n_punkte, self.n_dreiecke = p.shape[0], d.shape[0]
        self.suchtiefe = float(suchtiefe)
        self._punkte = p.copy()
        self._h = C.c_void_p()
        err = C.create_string_buffer(256)
        s = self._L.k3d_mesh_create(_d(p), p.shape[0], d.ctypes.data_as(C.POINTER(C.c_uint32)), d.shape[0],
                                    float(suchtiefe), int(device), C.byref(self._h), err, 256)
        if s != _abi.K3D_OK:
            self._h = None
            raise K3dError(s, err.value.decode())

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.k3d_mesh_destroy(self._h)
            self._h = None

    def _check(self, s):
        if s != _abi.K3D_OK:
            raise K3dError(s, self._L.k3d_mesh_last_error(self._h).decode())

    # ------------------------------------------------------------------ state
    def nachfuehren(self, punkte) -> None:
        """Koerpernetz::nachfuehren (:390-411)."""
        p = _f64(punkte)
        if p.shape[0] != self.n_punkte:
            raise K3dError(_abi.K3D_BAD_ARGUMENT, f"nachfuehren: {p.shape[0]} points instead of {self.n_punkte}")
        self._check(self._L.k3d_mesh_update(self._h, _d(p)))
        self._punkte = p.copy()

    def info(self) -> _abi.K3dMeshInfo:
        i = _abi.K3dMeshInfo()
        self._check(self._L.k3d_mesh_get_info(self._h, C.byref(i)))
        return i

    @property
    def randkanten(self) -> int:
        return int(self.info().randkanten)

    @property
    def volumen(self) -> float:
        return float(self.info().volumen)

    def tabellen(self) -> dict:
        """Face normals, point normals, edge neighbours, bounding spheres."""
        fn, pn = np.zeros((self.n_dreiecke, 3)), np.zeros((self.n_punkte, 3))
        nb, kg = np.zeros((self.n_dreiecke, 3), dtype=np.uint32), np.zeros((self.n_dreiecke, 4))
        self._check(self._L.k3d_mesh_tables(self._h, _d(fn), _d(pn), nb.ctypes.data_as(C.POINTER(C.c_uint32)),
                                            _d(kg)))
        return dict(flaechennormale=fn, punktnormale=pn, nachbar=nb, kugel=kg)

    def setze_punktgeschwindigkeit(self, v=None) -> None:
        """Koerpernetz::setze_punktgeschwindigkeit (:454-463): the velocity
        per point of a deforming body; None clears it (rigid again)."""
        if v is None or len(v) == 0:
            self._check(self._L.k3d_mesh_set_velocity(self._h, None))
            return
        a = _f64(v)
        if a.shape[0] != self.n_punkte:
            raise K3dError(_abi.K3D_BAD_ARGUMENT, f"velocity for {a.shape[0]} points, the mesh has {self.n_punkte}")
        self._check(self._L.k3d_mesh_set_velocity(self._h, _d(a)))

    def geschwindigkeit_an(self, dreieck, punkt, starr=(0.0, 0.0, 0.0)) -> np.ndarray:
        """Koerpernetz::geschwindigkeit_an (:474-489) per (triangle, point)."""
        dr = np.ascontiguousarray(dreieck, dtype=np.int32).reshape(-1)
        p = _f64(punkt)
        out = np.zeros((dr.shape[0], 3))
        self._check(self._L.k3d_mesh_velocity_at(self._h, dr.ctypes.data_as(_ip), _d(p), dr.shape[0],
                                                 _d(_f64(starr, (3,))), _d(out)))
        return out

    # ------------------------------------------------------------------ queries
    def _nearest(self, x, radius: float) -> dict:
        x = _f64(x)
        m = x.shape[0]
        ab, pu, no = np.zeros(m), np.zeros((m, 3)), np.zeros((m, 3))
        dr, rg = np.zeros(m, dtype=np.int32), np.zeros(m, dtype=np.int32)
        self._check(self._L.k3d_mesh_nearest(self._h, _d(x), m, float(radius), _d(ab), _d(pu), _d(no),
                                             dr.ctypes.data_as(_ip), rg.ctypes.data_as(_ip)))
        return dict(abstand=ab, punkt=pu, normale=no, dreieck=dr, region=rg)

    def naechster(self, x, radius: float) -> dict:
        """Koerpernetz::naechster (:503-539) per point: signed distance,
        nearest point, outward normal, triangle and region; dreieck and
        region -1 where no surface point is closer than ``radius``."""
        if not radius > 0.0:
            raise K3dError(_abi.K3D_BAD_ARGUMENT, "naechster: radius must be positive")
        return self._nearest(x, radius)

    def naechster_alle(self, x) -> dict:
        """Koerpernetz::naechster_alle (:770-782) per point."""
        return self._nearest(x, 0.0)

    def durchstoss(self, a, b) -> dict:
        """Koerpernetz::durchstoss (:541-593) per segment a -> b: dreieck
        (-1 = none), entry point, face normal."""
        a, b = _f64(a), _f64(b)
        m = a.shape[0]
        if b.shape[0] != m:
            raise K3dError(_abi.K3D_BAD_ARGUMENT, "durchstoss: a and b differ in length")
        dr, pu, no = np.zeros(m, dtype=np.int32), np.zeros((m, 3)), np.zeros((m, 3))
        self._check(self._L.k3d_mesh_penetration(self._h, _d(a), _d(b), m, dr.ctypes.data_as(_ip), _d(pu), _d(no)))
        return dict(dreieck=dr, punkt=pu, normale=no)

    # ------------------------------------------------------------------ voxelisation
    def sdf(self, dims, ursprung, spacing: float, band: float = 0.0) -> np.ndarray:
        """Signed distance at the nodes ursprung + spacing * (i, j, k), float32
        of shape (dims[2], dims[1], dims[0]). band <= 0: exact at every node;
        band > spacing: exact within the band, +-band beyond."""
        dm = np.ascontiguousarray(dims, dtype=np.int32)
        out = np.empty((int(dm[2]), int(dm[1]), int(dm[0])), dtype=np.float32)
        self._check(self._L.k3d_mesh_sdf(self._h, dm.ctypes.data_as(_ip), _d(_f64(ursprung, (3,))), float(spacing),
                                         float(band), out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def sdf_body(self, spacing: float, band: float, rand: float | None = None, versatz=(0.0, 0.0, 0.0),
                 geschwindigkeit=(0.0, 0.0, 0.0)) -> dict:
        """The mesh as a K3D_BODY_SDF_GRID body dict: a grid over the mesh's
        hull grown by ``rand`` (default band + 2 spacing) on each side; the
        body sits at ``versatz``."""
        lo, hi = self._punkte.min(axis=0), self._punkte.max(axis=0)
        r = (band + 2.0 * spacing) if rand is None else float(rand)
        o = lo - r
        dims = tuple(int(np.ceil((hi[a] + r - o[a]) / spacing)) + 1 for a in range(3))
        g = self.sdf(dims, o, spacing, band)
        return dict(art=_abi.K3D_BODY_SDF_GRID, punkt=tuple(float(v) for v in versatz), dims=dims,
                    ursprung=tuple(float(v) for v in o), spacing=float(spacing),
                    geschwindigkeit=tuple(float(v) for v in geschwindigkeit), sdf=np.ascontiguousarray(g.ravel()))

    @property
    def c_handle(self):
        """The k3d_mesh pointer for k3d_body.netz."""
        return self._h.value if self._h is not None else None

    def body(self, versatz=(0.0, 0.0, 0.0), geschwindigkeit=(0.0, 0.0, 0.0), instanz: int = -1) -> dict:
        """Koerper::Netz (koerper.rs:20-24) as a body dict for a scene; the
        dict holds this mesh, which must outlive the solver's use of it."""
        return dict(art=_abi.K3D_BODY_MESH, punkt=tuple(float(v) for v in versatz),
                    geschwindigkeit=tuple(float(v) for v in geschwindigkeit), instanz=int(instanz), netz=self)

    @property
    def letzte_ms(self) -> float:
        """Device time of the last call's kernels (CUDA events), ms."""
        return float(self.info().ms_letzter_aufruf)
