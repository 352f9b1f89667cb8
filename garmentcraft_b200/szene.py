"""The scene as the implicit step sees it (Szene, sim/src/szene.rs:198-269).

Host-side numpy arrays in the layout of the k3d_scene C struct. The groups
(abstand, naht, biegung) are in the scene's colour order, which fixes the
summation order of the reference CPU solver.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .synth import Simparameter, body_to_c

_ARRAYS = {
    # name: (dtype, columns)
    "x": (np.float64, 3), "v": (np.float64, 3), "masse": (np.float64, 0), "w": (np.float64, 0),
    "kollisionsabstand": (np.float64, 0), "reibung": (np.float64, 0),
    "abstand_punkte": (np.uint32, 2), "abstand_ruhe": (np.float64, 0),
    "abstand_nachgiebigkeit": (np.float64, 0), "membran_kante": (np.uint8, 0),
    "naht_punkte": (np.uint32, 2), "naht_ruhe": (np.float64, 0),
    "biegung_punkte": (np.uint32, 4), "biegung_ruhe": (np.float64, 0),
    "biegung_nachgiebigkeit": (np.float64, 0),
    "membran_punkte": (np.uint32, 3), "membran_flaeche": (np.float64, 0),
    "membran_ruhe_inv": (np.float64, 4), "membran_kette": (np.float64, 2),
    "membran_schuss": (np.float64, 2), "membran_steif": (np.float64, 3),
    "dreiecke": (np.uint32, 3), "ruhe_inv": (np.float64, 4),
    "teil_bereiche": (np.int64, 4), "teil_dehnung": (np.float64, 0), "teil_band_von": (np.int32, 0),
}
_COUNT = {
    "x": "n_punkte", "v": "n_punkte", "masse": "n_punkte", "w": "n_punkte",
    "kollisionsabstand": "n_punkte", "reibung": "n_punkte",
    "abstand_punkte": "n_abstand", "abstand_ruhe": "n_abstand", "abstand_nachgiebigkeit": "n_abstand",
    "membran_kante": "n_abstand", "naht_punkte": "n_naht", "naht_ruhe": "n_naht",
    "biegung_punkte": "n_biegung", "biegung_ruhe": "n_biegung", "biegung_nachgiebigkeit": "n_biegung",
    "membran_punkte": "n_membran", "membran_flaeche": "n_membran", "membran_ruhe_inv": "n_membran",
    "membran_kette": "n_membran", "membran_schuss": "n_membran", "membran_steif": "n_membran",
    "dreiecke": "n_dreiecke", "ruhe_inv": "n_dreiecke",
    "teil_bereiche": "n_teile", "teil_dehnung": "n_teile", "teil_band_von": "n_teile",
}
_CTYPE = {np.float64: C.c_double, np.uint32: C.c_uint32, np.uint8: C.c_uint8, np.int64: C.c_int64,
          np.int32: C.c_int32}


@dataclass
class Szene:
    x: np.ndarray
    v: np.ndarray
    masse: np.ndarray
    w: np.ndarray
    kollisionsabstand: np.ndarray
    reibung: np.ndarray
    abstand_punkte: np.ndarray
    abstand_ruhe: np.ndarray
    abstand_nachgiebigkeit: np.ndarray
    membran_kante: np.ndarray
    naht_punkte: np.ndarray
    naht_ruhe: np.ndarray
    biegung_punkte: np.ndarray
    biegung_ruhe: np.ndarray
    biegung_nachgiebigkeit: np.ndarray
    membran_punkte: np.ndarray
    membran_flaeche: np.ndarray
    membran_ruhe_inv: np.ndarray
    membran_kette: np.ndarray
    membran_schuss: np.ndarray
    membran_steif: np.ndarray
    dreiecke: np.ndarray
    ruhe_inv: np.ndarray
    # Teilinfo (szene.rs:181-194): per part its point and triangle ranges
    # (start, end, start, end), stretch stiffness and folded-band carrier (-1)
    teil_bereiche: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), dtype=np.int64))
    teil_dehnung: np.ndarray = field(default_factory=lambda: np.zeros(0))
    teil_band_von: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int32))
    # batch of independent drapes: n_instanzen + 1 point offsets (empty: one drape)
    instanz_punkte: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int64))
    koerper: list = field(default_factory=list)
    param: Simparameter = field(default_factory=Simparameter)
    zeit: float = 0.0

    @property
    def n(self) -> int:
        return self.x.shape[0]

    @classmethod
    def from_view(cls, view: _abi.K3dScene, koerper=None) -> "Szene":
        """Copies a k3d_scene view into numpy arrays."""
        kw = {}
        for name, (dt, cols) in _ARRAYS.items():
            cnt = getattr(view, _COUNT[name])
            size = cnt * (cols if cols else 1)
            p = getattr(view, name)
            if cnt == 0 or not p:
                a = np.zeros(size, dtype=dt)
            else:
                a = np.ctypeslib.as_array(p, shape=(size,)).astype(dt, copy=True)
            kw[name] = a.reshape(cnt, cols) if cols else a
        prm = view.param
        kw["param"] = Simparameter(prm.bild_dt, tuple(prm.schwerkraft), prm.daempfung)
        kw["zeit"] = view.zeit
        kw["koerper"] = list(koerper or [])
        return cls(**kw)

    def copy(self) -> "Szene":
        kw = {name: getattr(self, name).copy() for name in _ARRAYS}
        return Szene(**kw, instanz_punkte=self.instanz_punkte.copy(), koerper=list(self.koerper),
                     param=self.param, zeit=self.zeit)

    @classmethod
    def verbinden(cls, szenen: list) -> "Szene":
        """A batch scene of independent drapes: the scenes' points, elements and
        parts one after another (each element group instance by instance),
        bodies tagged with their instance. All scenes share one frame length
        and substep count; the first scene's Simparameter apply."""
        off = 0
        tri_off = 0
        parts = {name: [] for name in _ARRAYS}
        koerper = []
        io = [0]
        for k, s in enumerate(szenen):
            for name, (dt, cols) in _ARRAYS.items():
                a = np.asarray(getattr(s, name))
                if name in ("abstand_punkte", "naht_punkte", "biegung_punkte", "membran_punkte", "dreiecke"):
                    a = a.astype(np.uint32) + np.uint32(off)
                elif name == "teil_bereiche":
                    a = a.astype(np.int64) + np.array([off, off, tri_off, tri_off], dtype=np.int64)
                parts[name].append(a)
            for b in s.koerper:
                d = dict(b)
                d["instanz"] = k
                koerper.append(d)
            off += s.n
            tri_off += s.dreiecke.shape[0]
            io.append(off)
        kw = {}
        for name, (dt, cols) in _ARRAYS.items():
            kw[name] = np.ascontiguousarray(np.concatenate(parts[name], axis=0), dtype=dt)
        return cls(**kw, instanz_punkte=np.array(io, dtype=np.int64), koerper=koerper,
                   param=szenen[0].param, zeit=szenen[0].zeit)

    def instanz(self, k: int):
        """Point slice of instance k of a batch scene."""
        if self.instanz_punkte.shape[0] == 0:
            return slice(0, self.n)
        return slice(int(self.instanz_punkte[k]), int(self.instanz_punkte[k + 1]))

    def to_c(self):
        """(k3d_scene, keepalive). x and v point at this scene's own arrays, so
        a call that writes them writes this scene."""
        for name in _ARRAYS:
            a = getattr(self, name)
            if not a.flags["C_CONTIGUOUS"] or a.dtype != _ARRAYS[name][0]:
                setattr(self, name, np.ascontiguousarray(a, dtype=_ARRAYS[name][0]))
        s = _abi.K3dScene()
        s.n_punkte = self.x.shape[0]
        s.n_abstand = self.abstand_punkte.shape[0]
        s.n_naht = self.naht_punkte.shape[0]
        s.n_biegung = self.biegung_punkte.shape[0]
        s.n_membran = self.membran_punkte.shape[0]
        s.n_dreiecke = self.dreiecke.shape[0]
        s.n_teile = self.teil_dehnung.shape[0]
        self.instanz_punkte = np.ascontiguousarray(self.instanz_punkte, dtype=np.int64)
        s.n_instanzen = max(self.instanz_punkte.shape[0] - 1, 0)
        s.instanz_punkte = _abi.ptr(self.instanz_punkte, C.c_int64) if s.n_instanzen > 0 else None
        for name, (dt, _) in _ARRAYS.items():
            setattr(s, name, _abi.ptr(getattr(self, name), _CTYPE[dt]))
        bodies = (_abi.K3dBody * max(len(self.koerper), 1))()
        for k, b in enumerate(self.koerper):
            bodies[k] = body_to_c(b)
        s.n_koerper = len(self.koerper)
        s.koerper = bodies
        s.param = self.param.to_c()
        s.zeit = self.zeit
        return s, [bodies]

    # sim/src/szene.rs:768-774
    def naht_kuerzen(self, schritt: float) -> None:
        i, j = self.naht_punkte[:, 0], self.naht_punkte[:, 1]
        l = np.sqrt(np.sum((self.x[i] - self.x[j]) ** 2, axis=1))
        self.naht_ruhe = np.maximum(np.minimum(self.naht_ruhe, l) - schritt, 0.0)

    # sim/src/szene.rs:778-782
    def naht_offen(self) -> None:
        self.naht_ruhe = np.full_like(self.naht_ruhe, math.inf)

    def gesamtmasse(self) -> float:
        return float(np.sum(self.masse))
