"""ORACLE (test infrastructure): ctypes access to the FP64 CPU restatement.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py load
this module, as the checker or as the timed CPU baseline. The product package
never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from garmentcraft_b200 import _abi
from garmentcraft_b200.szene import Szene

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libk3d_oracle.so")

_lib = None


def build() -> str:
    """Compiles the oracle with its Makefile (g++ only, no GPU)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    L.orc_build_scene.argtypes = [C.POINTER(_abi.K3dPattern)]
    L.orc_build_scene.restype = P
    L.orc_built_scene_view.argtypes = [P, C.POINTER(_abi.K3dScene)]
    L.orc_built_scene_counts.argtypes = [P, C.POINTER(C.c_int64)]
    L.orc_built_scene_free.argtypes = [P]
    L.orc_sim_create.argtypes = [C.POINTER(_abi.K3dScene), C.POINTER(_abi.K3dParams)]
    L.orc_sim_create.restype = P
    L.orc_sim_free.argtypes = [P]
    L.orc_sim_frames.argtypes = [P, C.c_int32, C.POINTER(_abi.K3dStats)]
    L.orc_sim_adjoint.argtypes = [P, C.c_int32, dp, dp, dp, dp, dp, dp, C.c_double, C.POINTER(C.c_int64)]
    up = C.POINTER(C.c_uint32)
    L.orc_stoesse.argtypes = [C.c_int64, dp, dp, dp, dp, C.c_int64, up, C.c_int64, up, C.c_int32, C.c_int32,
                              C.c_int32, dp, C.c_int64, C.POINTER(C.c_int64)]
    L.orc_stoesse.restype = C.c_int64
    L.orc_sim_schnitte.argtypes = [P, C.c_int32, C.c_int64, C.POINTER(C.c_int64)]
    L.orc_sim_schnitte.restype = C.c_int64
    L.orc_sim_get_state.argtypes = [P, dp, dp]
    L.orc_sim_set_state.argtypes = [P, dp, dp]
    L.orc_sim_set_naht_ruhe.argtypes = [P, dp]
    L.orc_sim_get_naht_ruhe.argtypes = [P, dp]
    L.orc_sim_naht_kuerzen.argtypes = [P, C.c_double]
    L.orc_sim_naht_offen.argtypes = [P]
    L.orc_sim_set_reibung.argtypes = [P, C.c_double]
    L.orc_sim_get_dv_warm.argtypes = [P, dp]
    L.orc_sim_set_dv_warm.argtypes = [P, dp]
    L.orc_sim_operator.argtypes = [P, dp, dp]
    L.orc_sim_system.argtypes = [P, C.POINTER(_abi.K3dSystemReadback)]
    L.orc_sim_solve.argtypes = [P, dp, C.POINTER(_abi.K3dCgResult)]
    L.orc_sim_solve_contacts.argtypes = [P, C.POINTER(C.c_uint8), dp, dp, dp, C.POINTER(_abi.K3dCgResult)]
    L.orc_sim_umfang.argtypes = [P, dp, dp]
    L.orc_sim_umfang.restype = C.c_double
    L.orc_sim_nahtspalt.argtypes = [P]
    L.orc_sim_nahtspalt.restype = C.c_double
    L.orc_sim_mittlere_geschwindigkeit.argtypes = [P]
    L.orc_sim_mittlere_geschwindigkeit.restype = C.c_double
    L.orc_sim_dehnung.argtypes = [P, dp]
    L.orc_sim_schwerpunkt.argtypes = [P, dp]
    L.orc_membran_bauen.argtypes = [dp, dp, dp, dp, dp]
    L.orc_membran_bauen.restype = C.c_int32
    L.orc_membran_eval.argtypes = [dp, dp, dp, dp, dp, dp, dp, dp]
    L.orc_membran_zuege.argtypes = [dp, dp, dp, dp, dp]
    L.orc_sim_xpbd_frames.argtypes = [P, C.c_int32, C.c_int32, dp]
    L.orc_xpbd_abstand.argtypes = [dp, dp, dp, dp, C.c_double, C.c_double]
    L.orc_membran_mal_h.argtypes = [dp, dp, dp, dp]
    L.orc_membran_diag.argtypes = [dp, dp, dp]
    L.orc_psd2.argtypes = [C.c_double, C.c_double, C.c_double, dp]
    L.orc_steifigkeit.argtypes = [C.c_double] * 4
    L.orc_steifigkeit.restype = C.c_double
    L.orc_cos2_sin2.argtypes = [dp, dp, dp]
    L.orc_cos2_sin2.restype = C.c_int32
    L.orc_dieder.argtypes = [dp, dp, dp]
    L.orc_dieder.restype = C.c_int32
    L.orc_winkel_fehler.argtypes = [C.c_double, C.c_double]
    L.orc_winkel_fehler.restype = C.c_double
    L.orc_m3_inv.argtypes = [dp, dp]
    L.orc_faerbe.argtypes = [C.c_int64, C.c_int32, C.c_int64, C.POINTER(C.c_uint32),
                             C.POINTER(C.c_uint32), C.POINTER(C.c_int64)]
    L.orc_faerbe.restype = C.c_int64
    L.orc_kontakt.argtypes = [C.POINTER(_abi.K3dBody), dp, C.c_double, dp, dp]
    L.orc_kontakt.restype = C.c_int32
    u32p = C.POINTER(C.c_uint32)
    i32p = C.POINTER(C.c_int32)
    i64p = C.POINTER(C.c_int64)
    L.orc_zellindex.argtypes = [C.c_double, C.c_double]
    L.orc_zellindex.restype = C.c_int64
    L.orc_streue.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_uint64]
    L.orc_streue.restype = C.c_uint64
    L.orc_finde_roh.argtypes = [C.c_int64, dp, dp, C.c_int64, u32p, dp, C.c_int32, C.c_int32, C.c_int64,
                                i32p, u32p, dp, dp, dp, dp]
    L.orc_finde_roh.restype = C.c_int64
    L.orc_selbst_finde.argtypes = [P, dp, C.c_int32, C.c_int32, C.c_int64, i32p, u32p, dp, dp, dp, dp]
    L.orc_selbst_finde.restype = C.c_int64
    L.orc_selbst_kanten.argtypes = [P, C.c_int64, u32p, dp]
    L.orc_selbst_kanten.restype = C.c_int64
    L.orc_selbst_hash.argtypes = [P, dp, C.c_int32, C.c_int64, u32p, C.c_int64, u32p, i64p]
    L.orc_selbst_hash.restype = C.c_int64
    L.orc_selbst_federn.argtypes = [P, dp, dp, C.c_int64, u32p, dp, dp, dp]
    L.orc_selbst_federn.restype = C.c_int64
    cp = C.c_char_p
    L.orc_netz_neu.argtypes = [dp, C.c_int64, u32p, C.c_int64, C.c_double, cp, C.c_int64]
    L.orc_netz_neu.restype = P
    L.orc_netz_free.argtypes = [P]
    L.orc_netz_nachfuehren.argtypes = [P, dp, cp, C.c_int64]
    L.orc_netz_nachfuehren.restype = C.c_int32
    L.orc_netz_info.argtypes = [P, i64p, dp, dp, dp, i64p, i64p]
    L.orc_netz_tabellen.argtypes = [P, dp, dp, u32p, dp]
    L.orc_netz_naechster.argtypes = [P, dp, C.c_int64, C.c_double, dp, dp, dp, i32p, i32p]
    L.orc_netz_durchstoss.argtypes = [P, dp, dp, C.c_int64, i32p, dp, dp]
    L.orc_netz_sdf.argtypes = [P, i32p, dp, C.c_double, C.c_double, C.POINTER(C.c_float)]
    L.orc_netz_setze_geschwindigkeit.argtypes = [P, dp, C.c_int64, cp, C.c_int64]
    L.orc_netz_setze_geschwindigkeit.restype = C.c_int32
    L.orc_netz_geschwindigkeit_an.argtypes = [P, i32p, dp, C.c_int64, dp, dp]
    L.orc_netz_punkte_gegen_dreiecke.argtypes = [P, C.c_double, dp, dp, u32p, C.c_int64, dp, dp, dp, C.c_int64]
    L.orc_netz_punkte_gegen_dreiecke.restype = C.c_int64
    _lib = L
    return L


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def build_scene(muster, koerper=None) -> Szene:
    """Szene::aus_netz restated (oracle side)."""
    L = lib()
    pat, keep = muster.to_c()
    h = L.orc_build_scene(C.byref(pat))
    view = _abi.K3dScene()
    L.orc_built_scene_view(h, C.byref(view))
    s = Szene.from_view(view, koerper)
    s.param = muster.param
    counts = (C.c_int64 * 6)()
    L.orc_built_scene_counts(h, counts)
    s.oracle_counts = dict(membran_entartet=counts[0], naht_biegung_ohne=counts[1],
                           einhalte_kanten=counts[2], farben_abstand=counts[3],
                           farben_biegung=counts[4], farben_naht=counts[5])
    L.orc_built_scene_free(h)
    del keep
    return s


class OracleSim:
    """ImplizitCg with CpuLoeser over one scene (FP64, single thread)."""

    def __init__(self, szene: Szene, params: _abi.K3dParams):
        self.L = lib()
        self.n = szene.n
        self.n_naht = szene.naht_punkte.shape[0]
        self.n_tri = szene.dreiecke.shape[0]
        self.n_membran = szene.membran_punkte.shape[0]
        self.n_biegung = szene.biegung_punkte.shape[0]
        cs, keep = szene.to_c()
        self.h = self.L.orc_sim_create(C.byref(cs), C.byref(params))
        del keep

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_sim_free(self.h)
            self.h = None

    def frames(self, n: int = 1) -> _abi.K3dStats:
        st = _abi.K3dStats()
        self.L.orc_sim_frames(self.h, n, C.byref(st))
        return st

    def xpbd_frames(self, n: int = 1, unterschritte: int = 20) -> dict:
        """n frames of the XPBD cross-check (CpuReferenz, cpu.rs:222-245) on
        this scene; the last frame's Kontaktstatistik."""
        out = np.zeros(4)
        self.L.orc_sim_xpbd_frames(self.h, n, unterschritte, out.ctypes.data_as(C.POINTER(C.c_double)))
        return dict(kontakte=int(out[0]), haftend=int(out[1]), tiefe=out[2], tangential=out[3])

    def adjoint(self, n: int, gx, gv, toleranz: float = 1e-12) -> dict:
        """``n`` frames from the current state, then the adjoint back through
        them: cotangents of the initial x, v and of the element parameters
        (per membrane E_warp, E_weft, G, grain rotation; per hinge k) for the
        cotangents ``gx``, ``gv`` of the final x, v."""
        gx = f64(gx)
        gv = f64(gv)
        ox = np.zeros((self.n, 3))
        ov = np.zeros((self.n, 3))
        gm = np.zeros((self.n_membran, 4))
        gb = np.zeros(self.n_biegung)
        it = C.c_int64(0)
        self.L.orc_sim_adjoint(self.h, n, _d(gx), _d(gv), _d(ox), _d(ov), _d(gm), _d(gb), toleranz, C.byref(it))
        return dict(x=ox, v=ov, membran=gm, biegung=gb, iterationen=int(it.value))

    def schnitte(self, an_naehten: bool = True):
        """finde_schnitte and gebiete at the current state: the region root of
        each intersection (selbstkollision.rs:858-1009)."""
        cap = 1 << 20
        r = np.zeros(cap, dtype=np.int64)
        n = self.L.orc_sim_schnitte(self.h, int(an_naehten), cap,
                                    r.ctypes.data_as(C.POINTER(C.c_int64)))
        return r[:n]

    def state(self):
        x = np.zeros((self.n, 3))
        v = np.zeros((self.n, 3))
        self.L.orc_sim_get_state(self.h, _d(x), _d(v))
        return x, v

    def set_state(self, x=None, v=None):
        xa = f64(x) if x is not None else None
        va = f64(v) if v is not None else None
        self.L.orc_sim_set_state(self.h, _d(xa) if xa is not None else None,
                                 _d(va) if va is not None else None)

    def naht_ruhe(self):
        r = np.zeros(self.n_naht)
        self.L.orc_sim_get_naht_ruhe(self.h, _d(r))
        return r

    def set_naht_ruhe(self, r):
        r = f64(r)
        self.L.orc_sim_set_naht_ruhe(self.h, _d(r))

    def naht_kuerzen(self, schritt):
        self.L.orc_sim_naht_kuerzen(self.h, schritt)

    def naht_offen(self):
        self.L.orc_sim_naht_offen(self.h)

    def set_reibung(self, mu):
        self.L.orc_sim_set_reibung(self.h, mu)

    def dv_warm(self):
        dv = np.zeros((self.n, 3))
        self.L.orc_sim_get_dv_warm(self.h, _d(dv))
        return dv

    def set_dv_warm(self, dv):
        """Sets the warm start of the next substep (dv_vorher)."""
        dv = f64(dv)
        self.L.orc_sim_set_dv_warm(self.h, _d(dv))

    def operator(self, p):
        p = f64(p)
        out = np.zeros((self.n, 3))
        self.L.orc_sim_operator(self.h, _d(p), _d(out))
        return out

    def system(self):
        n = self.n
        out = dict(rhs=np.zeros((n, 3)), f=np.zeros((n, 3)), last=np.zeros((n, 3)),
                   pinv=np.zeros((n, 3, 3)), normale=np.zeros((n, 3)), vn_soll=np.zeros(n),
                   fest=np.zeros(n, dtype=np.uint8))
        rb = _abi.K3dSystemReadback(_d(out["rhs"]), _d(out["f"]), _d(out["last"]), _d(out["pinv"]),
                                    _d(out["normale"]), _d(out["vn_soll"]),
                                    out["fest"].ctypes.data_as(C.POINTER(C.c_uint8)))
        self.L.orc_sim_system(self.h, C.byref(rb))
        return out

    def solve_contacts(self, dv, fest):
        """Loeser::loese with the given contact set (dict of fest, normale,
        vn_soll as ImplizitCg.loese takes it)."""
        dv = f64(dv).copy()
        on = np.ascontiguousarray(fest["fest"], dtype=np.uint8)
        nrm, soll = f64(fest["normale"]), f64(fest["vn_soll"])
        res = _abi.K3dCgResult()
        self.L.orc_sim_solve_contacts(self.h, on.ctypes.data_as(C.POINTER(C.c_uint8)), _d(nrm), _d(soll), _d(dv),
                                      C.byref(res))
        return dv, res

    def solve(self, dv):
        dv = f64(dv).copy()
        res = _abi.K3dCgResult()
        self.L.orc_sim_solve(self.h, _d(dv), C.byref(res))
        return dv, res

    def umfang(self, punkt, normale):
        return self.L.orc_sim_umfang(self.h, _d(f64(punkt)), _d(f64(normale)))

    def nahtspalt(self):
        return self.L.orc_sim_nahtspalt(self.h)

    def mittlere_geschwindigkeit(self):
        return self.L.orc_sim_mittlere_geschwindigkeit(self.h)

    def dehnung(self):
        out = np.zeros((self.n_tri, 2))
        self.L.orc_sim_dehnung(self.h, _d(out))
        return out

    def schwerpunkt(self):
        out = np.zeros(3)
        self.L.orc_sim_schwerpunkt(self.h, _d(out))
        return out


def _naehe(call, cap=0):
    """Runs a pair query twice (count, then fill) and returns the pairs as arrays."""
    n = call(0, None, None, None, None, None, None)
    art = np.zeros(max(n, 1), dtype=np.int32)
    pk = np.zeros((max(n, 1), 4), dtype=np.uint32)
    gw = np.zeros((max(n, 1), 4))
    nr = np.zeros((max(n, 1), 3))
    ab = np.zeros(max(n, 1))
    ru = np.zeros(max(n, 1))
    call(n, art.ctypes.data_as(C.POINTER(C.c_int32)), pk.ctypes.data_as(C.POINTER(C.c_uint32)), _d(gw), _d(nr),
         _d(ab), _d(ru))
    return dict(art=art[:n], punkte=pk[:n], gewichte=gw[:n], normale=nr[:n], abstand=ab[:n], ruhe=ru[:n])


def finde_roh(x, w, dreiecke, r_punkt, punkt_dreieck=True, kante_kante=True):
    """Stoffnetz::neu + finde (selbstkollision.rs:159-187, 387-398) on a bare mesh."""
    L = lib()
    x, w, r = f64(x), f64(w), f64(r_punkt)
    d = np.ascontiguousarray(dreiecke, dtype=np.uint32)
    return _naehe(lambda cap, *o: L.orc_finde_roh(x.shape[0], _d(x), _d(w), d.shape[0],
                                                  d.ctypes.data_as(C.POINTER(C.c_uint32)), _d(r),
                                                  int(punkt_dreieck), int(kante_kante), cap, *o))


class SelbstProbe:
    """Self-collision probes on an OracleSim's scene (aus_szene with its params)."""

    def __init__(self, sim: "OracleSim"):
        self.sim = sim
        self.L = sim.L

    def finde(self, x, punkt_dreieck=True, kante_kante=True):
        x = f64(x)
        return _naehe(lambda cap, *o: self.L.orc_selbst_finde(self.sim.h, _d(x), int(punkt_dreieck),
                                                              int(kante_kante), cap, *o))

    def kanten(self):
        z = C.c_double()
        n = self.L.orc_selbst_kanten(self.sim.h, 0, None, C.byref(z))
        k = np.zeros((max(n, 1), 2), dtype=np.uint32)
        self.L.orc_selbst_kanten(self.sim.h, n, k.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(z))
        return k[:n], z.value

    def hash(self, x, kanten: bool):
        """(anfang, eintraege) of Hashgitter::neu over the point or edge boxes."""
        x = f64(x)
        ne = C.c_int64()
        eimer = self.L.orc_selbst_hash(self.sim.h, _d(x), int(kanten), 0, None, 0, None, C.byref(ne))
        anf = np.zeros(eimer + 1, dtype=np.uint32)
        ein = np.zeros(max(ne.value, 1), dtype=np.uint32)
        self.L.orc_selbst_hash(self.sim.h, _d(x), int(kanten), eimer + 1, anf.ctypes.data_as(C.POINTER(C.c_uint32)),
                               ne.value, ein.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(ne))
        return anf, ein[:ne.value]

    def federn(self, x, v):
        """Springs and the damped velocities (selbstkollision.rs:713-787)."""
        x = f64(x)
        vv = f64(v).copy()
        n = self.L.orc_selbst_federn(self.sim.h, _d(x), _d(vv.copy()), 0, None, None, None, None)
        pk = np.zeros((max(n, 1), 5), dtype=np.uint32)
        gw = np.zeros((max(n, 1), 5))
        kr = np.zeros((max(n, 1), 3))
        bl = np.zeros((max(n, 1), 3, 3))
        self.L.orc_selbst_federn(self.sim.h, _d(x), _d(vv), n, pk.ctypes.data_as(C.POINTER(C.c_uint32)), _d(gw),
                                 _d(kr), _d(bl))
        return dict(punkte=pk[:n], gewichte=gw[:n], kraft=kr[:n], block=bl[:n]), vv


def stoesse(x0, x1, w, masse, dreiecke=None, kanten=None, pd=True, kk=True, iterationen=1):
    """finde_stoesse and stossantwort on a small mesh (oracle): returns
    (impacts as rows (art, zeit, seite), responses, x1 after the response)."""
    L = lib()
    x0 = f64(x0)
    x1 = f64(x1).copy()
    w = f64(w)
    m = f64(masse)
    tri = np.ascontiguousarray(np.zeros((0, 3)) if dreiecke is None else dreiecke, dtype=np.uint32)
    ka = np.ascontiguousarray(np.zeros((0, 2)) if kanten is None else kanten, dtype=np.uint32)
    out = np.zeros((64, 3))
    z = C.c_int64(0)
    up = C.POINTER(C.c_uint32)
    n = L.orc_stoesse(x0.shape[0], _d(x0), _d(x1), _d(w), _d(m), tri.shape[0], tri.ctypes.data_as(up),
                      ka.shape[0], ka.ctypes.data_as(up), int(pd), int(kk), iterationen, _d(out), 64, C.byref(z))
    return out[:n], int(z.value), x1


class Koerpernetz:
    """The body mesh as a signed-distance collider (netzkoerper.rs:145-800),
    oracle side. Raises ValueError with the reference's reason where
    Koerpernetz::neu refuses the mesh."""

    def __init__(self, punkte, dreiecke, suchtiefe: float = 0.01):
        self.L = lib()
        p = f64(punkte).reshape(-1, 3)
        d = np.ascontiguousarray(dreiecke, dtype=np.uint32).reshape(-1, 3)
        self.n, self.nd = p.shape[0], d.shape[0]
        err = C.create_string_buffer(256)
        self.h = self.L.orc_netz_neu(_d(p), self.n, d.ctypes.data_as(C.POINTER(C.c_uint32)), self.nd, suchtiefe,
                                     err, 256)
        if not self.h:
            raise ValueError(err.value.decode())
        self.suchtiefe = suchtiefe

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_netz_free(self.h)
            self.h = None

    @property
    def c_handle(self):
        """The oracle mesh pointer, passed as k3d_body.netz to the oracle."""
        return self.h

    def body(self, versatz=(0.0, 0.0, 0.0), geschwindigkeit=(0.0, 0.0, 0.0), instanz: int = -1) -> dict:
        return dict(art=_abi.K3D_BODY_MESH, punkt=tuple(float(v) for v in versatz),
                    geschwindigkeit=tuple(float(v) for v in geschwindigkeit), instanz=int(instanz), netz=self)

    def nachfuehren(self, punkte):
        p = f64(punkte).reshape(-1, 3)
        err = C.create_string_buffer(256)
        if self.L.orc_netz_nachfuehren(self.h, _d(p), err, 256):
            raise ValueError(err.value.decode())

    def info(self) -> dict:
        rk, zahl, ein = C.c_int64(), np.zeros(3, dtype=np.int64), C.c_int64()
        vol, urs, zelle = C.c_double(), np.zeros(3), C.c_double()
        self.L.orc_netz_info(self.h, C.byref(rk), C.byref(vol), _d(urs), C.byref(zelle),
                             zahl.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(ein))
        return dict(randkanten=rk.value, volumen=vol.value, ursprung=urs, zelle=zelle.value, zahl=zahl,
                    eintraege=ein.value)

    def tabellen(self) -> dict:
        fn, pn = np.zeros((self.nd, 3)), np.zeros((self.n, 3))
        nb, kg = np.zeros((self.nd, 3), dtype=np.uint32), np.zeros((self.nd, 4))
        self.L.orc_netz_tabellen(self.h, _d(fn), _d(pn), nb.ctypes.data_as(C.POINTER(C.c_uint32)), _d(kg))
        return dict(flaechennormale=fn, punktnormale=pn, nachbar=nb, kugel=kg)

    def naechster(self, x, radius: float = 0.0) -> dict:
        """radius > 0: naechster (:503-539), dreieck -1 where nothing is
        closer; otherwise naechster_alle (:770-782)."""
        x = f64(x).reshape(-1, 3)
        m = x.shape[0]
        ab, pu, no = np.zeros(m), np.zeros((m, 3)), np.zeros((m, 3))
        dr, rg = np.zeros(m, dtype=np.int32), np.zeros(m, dtype=np.int32)
        i32 = C.POINTER(C.c_int32)
        self.L.orc_netz_naechster(self.h, _d(x), m, radius, _d(ab), _d(pu), _d(no), dr.ctypes.data_as(i32),
                                  rg.ctypes.data_as(i32))
        return dict(abstand=ab, punkt=pu, normale=no, dreieck=dr, region=rg)

    def durchstoss(self, a, b) -> dict:
        a, b = f64(a).reshape(-1, 3), f64(b).reshape(-1, 3)
        m = a.shape[0]
        dr, pu, no = np.zeros(m, dtype=np.int32), np.zeros((m, 3)), np.zeros((m, 3))
        self.L.orc_netz_durchstoss(self.h, _d(a), _d(b), m, dr.ctypes.data_as(C.POINTER(C.c_int32)), _d(pu),
                                   _d(no))
        return dict(dreieck=dr, punkt=pu, normale=no)

    def setze_punktgeschwindigkeit(self, v=None):
        """netzkoerper.rs:454-463; None or empty clears the field."""
        err = C.create_string_buffer(256)
        if v is None or len(v) == 0:
            rc = self.L.orc_netz_setze_geschwindigkeit(self.h, None, 0, err, 256)
        else:
            a = f64(v).reshape(-1, 3)
            rc = self.L.orc_netz_setze_geschwindigkeit(self.h, _d(a), a.shape[0], err, 256)
        if rc:
            raise ValueError(err.value.decode())

    def geschwindigkeit_an(self, dreieck, punkt, starr=(0.0, 0.0, 0.0)):
        """netzkoerper.rs:474-489 per (triangle, point)."""
        dr = np.ascontiguousarray(dreieck, dtype=np.int32).reshape(-1)
        p = f64(punkt).reshape(-1, 3)
        out = np.zeros((dr.shape[0], 3))
        self.L.orc_netz_geschwindigkeit_an(self.h, dr.ctypes.data_as(C.POINTER(C.c_int32)), _d(p), dr.shape[0],
                                           _d(f64(starr)), _d(out))
        return out

    def punkte_gegen_dreiecke(self, tief, dreiecke, w, x, v, versatz=(0.0, 0.0, 0.0), geschwindigkeit=(0.0, 0.0, 0.0)):
        """netzkoerper.rs:612-665 on raw cloth arrays: returns (count, x, v)."""
        d = np.ascontiguousarray(dreiecke, dtype=np.uint32).reshape(-1, 3)
        xs, vs = f64(x).reshape(-1, 3).copy(), f64(v).reshape(-1, 3).copy()
        n = self.L.orc_netz_punkte_gegen_dreiecke(self.h, tief, _d(f64(versatz)), _d(f64(geschwindigkeit)),
                                                  d.ctypes.data_as(C.POINTER(C.c_uint32)), d.shape[0],
                                                  _d(f64(w)), _d(xs), _d(vs), xs.shape[0])
        return int(n), xs, vs

    def sdf(self, dims, ursprung, spacing: float, band: float = 0.0):
        """naechster_alle at every node, clamped to +-band when band > 0;
        float32 array of shape (dims[2], dims[1], dims[0])."""
        dm = np.ascontiguousarray(dims, dtype=np.int32)
        out = np.zeros((dims[2], dims[1], dims[0]), dtype=np.float32)
        self.L.orc_netz_sdf(self.h, dm.ctypes.data_as(C.POINTER(C.c_int32)), _d(f64(ursprung)), spacing, band,
                            out.ctypes.data_as(C.POINTER(C.c_float)))
        return out
