"""ImplizitCg on the B200: the reference's implicit solver API over the C ABI.

Mirrors sim/src/implizit.rs:570-657 and the Rechenweg trait (sim/src/cpu.rs:
58-60): ``bild`` advances a scene by one frame, ``operator`` and
``system_fuer`` are the parity probes, ``loese`` / ``rest_geloest`` /
``last_lesen`` are the Loeser backend calls (implizit.rs:304-351). The scene
stays a host object (numpy arrays); the device keeps its own copy between
calls, and ``bild`` moves x and v across the boundary every frame.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._lib import K3dError, lib
from .params import ImplizitParameter, ImplizitStatistik
from .szene import Szene


@dataclass
class CgLauf:
    """CgLauf (implizit.rs:294-299)."""
    iterationen: int
    nicht_konvergiert: bool
    rest: float
    breakdown: bool = False


def _d(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def build_scene(muster, koerper=None) -> Szene:
    """Szene::aus_netz (sim/src/szene.rs:284-292) on the host, by the library."""
    L = lib()
    pat, keep = muster.to_c()
    h = C.c_void_p()
    st = L.k3d_build_scene(C.byref(pat), C.byref(h))
    if st != _abi.K3D_OK:
        raise K3dError(st, "scene build failed")
    view = _abi.K3dScene()
    L.k3d_built_scene_view(h, C.byref(view))
    s = Szene.from_view(view, koerper)
    s.param = muster.param
    L.k3d_built_scene_free(h)
    del keep
    return s


class ImplizitCg:
    """The implicit path with the B200 backend (ImplizitCg::mit_loeser)."""

    def __init__(self, param: ImplizitParameter | None = None, device: int = 0):
        self.param = param or ImplizitParameter()
        self._L = lib()
        cp = self.param.to_c()
        self._h = self._L.k3d_solver_create(C.byref(cp), device)
        self.statistik = ImplizitStatistik()
        self._szene = None
        self._c = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.k3d_solver_destroy(h)
            self._h = None

    def _check(self, st: int, what: str):
        if st not in (_abi.K3D_OK, _abi.K3D_NOT_CONVERGED):
            raise K3dError(st, f"{what}: {self._L.k3d_last_error(self._h).decode()}")

    def loeser_name(self) -> str:
        """Loeser::name (implizit.rs:306)."""
        return self._L.k3d_solver_name(self._h).decode()

    def hochladen(self, s: Szene) -> None:
        """Uploads the scene (topology, material, bodies, state) and resets the
        warm start. Called automatically when ``bild`` sees another scene."""
        cs, keep = s.to_c()
        self._check(self._L.k3d_upload_scene(self._h, C.byref(cs)), "upload")
        self._szene = s
        self._c = (cs, keep)

    def _ensure(self, s: Szene):
        if self._szene is not s:
            self.hochladen(s)
        else:
            cs, keep = s.to_c()
            self._c = (cs, keep)
        return self._c[0]

    def bild(self, s: Szene) -> None:
        """Rechenweg::bild (implizit.rs:1042-1057): one frame of
        ``schritte_je_bild`` substeps on the device; writes s.x, s.v."""
        cs = self._ensure(s)
        st = _abi.K3dStats()
        self._check(self._L.k3d_frame(self._h, C.byref(cs), C.byref(st)), "frame")
        s.zeit = cs.zeit
        for b in s.koerper:
            g = b.get("geschwindigkeit", (0.0, 0.0, 0.0))
            p = b.get("punkt", (0.0, 0.0, 0.0))
            b["punkt"] = tuple(p[k] + g[k] * s.param.bild_dt for k in range(3))
        self.statistik = ImplizitStatistik.from_c(st)

    def bilder_resident(self, s: Szene, n: int) -> ImplizitStatistik:
        """``n`` frames with the state kept on the device; s.x / s.v are read
        back once at the end."""
        self._ensure(s)
        self._check(self._L.k3d_upload_state(self._h, _d(s.x), _d(s.v)), "upload state")
        st = _abi.K3dStats()
        self._check(self._L.k3d_frames_resident(self._h, n, C.byref(st)), "frames")
        self._check(self._L.k3d_download_state(self._h, _d(s.x), _d(s.v)), "download state")
        s.zeit += n * s.param.bild_dt
        for b in s.koerper:
            g = b.get("geschwindigkeit", (0.0, 0.0, 0.0))
            p = b.get("punkt", (0.0, 0.0, 0.0))
            b["punkt"] = tuple(p[k] + g[k] * s.param.bild_dt * n for k in range(3))
        return ImplizitStatistik.from_c(st)

    def zustand_hochladen(self, s: Szene) -> None:
        """Copies s.x and s.v to the device-resident state."""
        self._ensure(s)
        self._check(self._L.k3d_upload_state(self._h, _d(s.x), _d(s.v)), "upload state")

    def zustand_lesen(self, s: Szene) -> None:
        """Copies the device-resident state into s.x and s.v."""
        self._check(self._L.k3d_download_state(self._h, _d(s.x), _d(s.v)), "download state")

    def bilder_auf_geraet(self, n: int) -> ImplizitStatistik:
        """``n`` frames on the device-resident state, no host copies. The
        frame's device time is ``letzte_bild_ms()``."""
        st = _abi.K3dStats()
        self._check(self._L.k3d_frames_resident(self._h, n, C.byref(st)), "frames")
        return ImplizitStatistik.from_c(st)

    def _sync_state(self, s: Szene):
        self._ensure(s)
        self._check(self._L.k3d_upload_state(self._h, _d(s.x), _d(s.v)), "upload state")

    def operator(self, s: Szene, p: np.ndarray) -> np.ndarray:
        """ImplizitCg::operator (implizit.rs:637-643)."""
        self._sync_state(s)
        p = np.ascontiguousarray(p, dtype=np.float64)
        out = np.zeros((s.n, 3))
        self._check(self._L.k3d_operator(self._h, _d(p), _d(out)), "operator")
        return out

    def system_fuer(self, s: Szene) -> dict:
        """ImplizitCg::system_fuer (implizit.rs:651-654) as a readback."""
        self._sync_state(s)
        n = s.n
        out = dict(rhs=np.zeros((n, 3)), f=np.zeros((n, 3)), last=np.zeros((n, 3)),
                   pinv=np.zeros((n, 3, 3)), normale=np.zeros((n, 3)), vn_soll=np.zeros(n),
                   fest=np.zeros(n, dtype=np.uint8))
        rb = _abi.K3dSystemReadback(_d(out["rhs"]), _d(out["f"]), _d(out["last"]), _d(out["pinv"]),
                                    _d(out["normale"]), _d(out["vn_soll"]),
                                    out["fest"].ctypes.data_as(C.POINTER(C.c_uint8)))
        self._check(self._L.k3d_system_for(self._h, C.byref(rb)), "system")
        return out

    def loese(self, s: Szene, dv: np.ndarray, fest: dict | None = None):
        """Loeser::loese (implizit.rs:308, 370-426) on the system of the
        scene's state. ``fest`` is the contact set the reference hands every
        backend (implizit.rs:870-883): a dict of ``fest`` (held flag per
        point), ``normale`` (unit normal, 3 per point) and ``vn_soll``
        (required normal velocity); None solves with the contact set the
        device finds against the bodies."""
        self._sync_state(s)
        dv = np.ascontiguousarray(dv, dtype=np.float64).copy()
        res = _abi.K3dCgResult()
        if fest is None:
            self._check(self._L.k3d_solve(self._h, _d(dv), C.byref(res)), "solve")
        else:
            on = np.ascontiguousarray(fest["fest"], dtype=np.uint8)
            nrm = np.ascontiguousarray(fest["normale"], dtype=np.float64)
            soll = np.ascontiguousarray(fest["vn_soll"], dtype=np.float64)
            if on.shape != (s.n,) or nrm.shape != (s.n, 3) or soll.shape != (s.n,):
                raise ValueError("contact set does not match the scene's points")
            cs = _abi.K3dContactSet(on.ctypes.data_as(C.POINTER(C.c_uint8)), _d(nrm), _d(soll))
            self._check(self._L.k3d_solve_contacts(self._h, C.byref(cs), _d(dv), C.byref(res)), "solve")
        return dv, CgLauf(res.iterationen, bool(res.nicht_konvergiert), res.rest, bool(res.breakdown))

    def rest_geloest(self, s: Szene, dv: np.ndarray) -> np.ndarray:
        """Loeser::rest_geloest (implizit.rs:337-342): A dv - b."""
        self._sync_state(s)
        dv = np.ascontiguousarray(dv, dtype=np.float64)
        out = np.zeros((s.n, 3))
        self._check(self._L.k3d_residual(self._h, _d(dv), _d(out)), "residual")
        return out

    def last_lesen(self) -> np.ndarray:
        """Loeser::last_lesen (implizit.rs:348-350)."""
        out = np.zeros((self._szene.n, 3))
        self._check(self._L.k3d_read_load(self._h, _d(out)), "load")
        return out

    def warmstart_lesen(self) -> np.ndarray:
        """The CG warm start of the next substep (ImplizitCg's dv_vorher,
        implizit.rs:906, 945), 3 per point."""
        out = np.zeros((self._szene.n, 3))
        self._check(self._L.k3d_read_warm_start(self._h, _d(out)), "warm start")
        return out

    # ---- self-collision probes: the proximity stage's last run
    def _selbst_check(self, n: int, what: str) -> int:
        if n < 0:
            raise K3dError(_abi.K3D_BAD_ARGUMENT, f"{what}: {self._L.k3d_last_error(self._h).decode()}")
        return n

    def selbst_paare(self) -> dict:
        """selbstkollision::finde (selbstkollision.rs:387-398) of the last run:
        art (0 point-triangle, 1 edge-edge), punkte, gewichte, normale,
        abstand, ruhe, in the reference's order."""
        L = self._L
        n = self._selbst_check(L.k3d_selfcollision_pairs(self._h, 0, None, None, None, None, None, None), "pairs")
        m = max(n, 1)
        art = np.zeros(m, dtype=np.int32)
        pk = np.zeros((m, 4), dtype=np.uint32)
        gw = np.zeros((m, 4))
        nr = np.zeros((m, 3))
        ab = np.zeros(m)
        ru = np.zeros(m)
        L.k3d_selfcollision_pairs(self._h, n, art.ctypes.data_as(C.POINTER(C.c_int32)),
                                  pk.ctypes.data_as(C.POINTER(C.c_uint32)), _d(gw), _d(nr), _d(ab), _d(ru))
        return dict(art=art[:n], punkte=pk[:n], gewichte=gw[:n], normale=nr[:n], abstand=ab[:n], ruhe=ru[:n])

    def selbst_hash(self, kanten: bool):
        """Hashgitter (selbstkollision.rs:256-345) of the last run's point or
        edge boxes: (bucket starts, entries)."""
        L = self._L
        ne = C.c_int64()
        eimer = self._selbst_check(L.k3d_selfcollision_hash(self._h, int(kanten), 0, None, 0, None, C.byref(ne)),
                                   "hash")
        anf = np.zeros(eimer + 1, dtype=np.uint32)
        ein = np.zeros(max(ne.value, 1), dtype=np.uint32)
        L.k3d_selfcollision_hash(self._h, int(kanten), eimer + 1, anf.ctypes.data_as(C.POINTER(C.c_uint32)),
                                 ne.value, ein.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(ne))
        return anf, ein[:ne.value]

    def selbst_federn(self) -> dict:
        """selbstkollision::federn (selbstkollision.rs:713-787) of the last run:
        force on the first side and the 3x3 block per pair."""
        L = self._L
        n = self._selbst_check(L.k3d_selfcollision_springs(self._h, 0, None, None), "springs")
        kr = np.zeros((max(n, 1), 3))
        bl = np.zeros((max(n, 1), 3, 3))
        L.k3d_selfcollision_springs(self._h, n, _d(kr), _d(bl))
        return dict(kraft=kr[:n], block=bl[:n])

    def adjoint_vorwaerts(self, n: int, k: int = 10) -> ImplizitStatistik:
        """``n`` frames on the device-resident state (as ``bilder_auf_geraet``)
        that keep x, v and the warm start every ``k`` substeps for
        ``adjoint_rueckwaerts``."""
        st = _abi.K3dStats()
        self._check(self._L.k3d_adjoint_forward(self._h, n, k, C.byref(st)), "adjoint forward")
        return ImplizitStatistik.from_c(st)

    def adjoint_rueckwaerts(self, gx: np.ndarray, gv: np.ndarray) -> dict:
        """The adjoint of the last ``adjoint_vorwaerts``: for the cotangents
        ``gx``, ``gv`` of the final x, v, those of the initial x, v, per
        membrane of (E_warp, E_weft, G, grain rotation) and per hinge of k,
        with the adjoint solve's statistics and device times."""
        sz = self._szene
        if sz is None:
            raise K3dError(_abi.K3D_BAD_ARGUMENT, "no scene uploaded")
        n, nt, nb = sz.n, sz.membran_punkte.shape[0], sz.biegung_punkte.shape[0]
        gx = np.ascontiguousarray(gx, dtype=np.float64).reshape(n, 3)
        gv = np.ascontiguousarray(gv, dtype=np.float64).reshape(n, 3)
        ox = np.zeros((n, 3))
        ov = np.zeros((n, 3))
        gm = np.zeros((max(nt, 1), 4))
        gb = np.zeros(max(nb, 1))
        st = _abi.K3dAdjointStats()
        self._check(self._L.k3d_adjoint_backward(self._h, _d(gx), _d(gv), _d(ox), _d(ov), _d(gm), _d(gb),
                                                 C.byref(st)), "adjoint backward")
        return dict(x=ox, v=ov, membran=gm[:nt], biegung=gb[:nb], iterationen=st.cg_iterationen,
                    loesungen=st.loesungen, nicht_konvergiert=st.nicht_konvergiert,
                    zusammenbrueche=st.zusammenbrueche, ms_vorwaerts=st.ms_vorwaerts,
                    ms_rueckwaerts=st.ms_rueckwaerts, ms_neuberechnung=st.ms_neuberechnung)

    def letzte_bild_ms(self) -> float:
        return self._L.k3d_last_frame_ms(self._h)

    def letzte_loesung_ms(self) -> float:
        """Device time of the PCG launches of the last frame call (ms)."""
        return self._L.k3d_last_solve_ms(self._h)

    def kernel_starts(self) -> int:
        return self._L.k3d_kernel_launches(self._h)

    def pcg_bloecke(self) -> int:
        """CTAs of the persistent PCG launch (``ImplizitParameter.pcg_bloecke``,
        capped at the most that can be resident at once)."""
        return self._L.k3d_pcg_blocks(self._h)
