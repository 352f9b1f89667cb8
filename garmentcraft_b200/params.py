"""ImplizitParameter / ImplizitStatistik (sim/src/implizit.rs:457-561)."""
from __future__ import annotations

from dataclasses import dataclass, fields

from . import _abi


@dataclass
class ImplizitParameter:
    """Settings of the implicit path, same meaning and defaults as the
    reference (implizit.rs:505-531). ``precision`` picks the device form:
    K3D_FP64 mirrors the reference, K3D_MIXED is the FP32/FP64 form,
    K3D_MIXED_STORAGE stores the operator and preconditioner in FP32 and runs
    the CG vectors in FP64."""
    schritte_je_bild: int = 5
    cg_max: int = 50
    cg_toleranz: float = 1e-5
    naht_k: float = 500.0
    kontakt_rand: float = 1e-4
    normalkraft_aus_last: bool = False
    durchstoss_pruefen: bool = True
    selbstkollision: bool = False
    selbst_zusatzdicke: float = 2.5e-3
    selbst_steifigkeit: float = 1e-3
    selbst_stoss_iterationen: int = 1
    selbst_schnitte_an_naehten: bool = False
    koerperpunkt_durchgaenge: int = 0
    koerperpunkt_tiefe: float = 0.01
    precision: int = _abi.K3D_FP64
    pcg_bloecke: int = 0
    graph: bool = False
    pcg_threads: int = 0

    def to_c(self) -> _abi.K3dParams:
        p = _abi.K3dParams()
        p.schritte_je_bild = self.schritte_je_bild
        p.cg_max = self.cg_max
        p.cg_toleranz = self.cg_toleranz
        p.naht_k = self.naht_k
        p.kontakt_rand = self.kontakt_rand
        p.normalkraft_aus_last = int(self.normalkraft_aus_last)
        p.durchstoss_pruefen = int(self.durchstoss_pruefen)
        p.selbstkollision = int(self.selbstkollision)
        p.precision = self.precision
        p.selbst_zusatzdicke = self.selbst_zusatzdicke
        p.selbst_steifigkeit = self.selbst_steifigkeit
        p.selbst_stoss_iterationen = self.selbst_stoss_iterationen
        p.selbst_schnitte_an_naehten = int(self.selbst_schnitte_an_naehten)
        p.koerperpunkt_durchgaenge = self.koerperpunkt_durchgaenge
        p.koerperpunkt_tiefe = self.koerperpunkt_tiefe
        p.pcg_bloecke = self.pcg_bloecke
        p.graph = int(self.graph)
        p.pcg_threads = self.pcg_threads
        return p


@dataclass
class ImplizitStatistik:
    """Counters of the last frame (implizit.rs:535-561)."""
    cg_iterationen: int = 0
    loesungen: int = 0
    nicht_konvergiert: int = 0
    kontakte: int = 0
    haftend: int = 0
    freigegeben: int = 0
    durchstoesse: int = 0
    koerperpunkte: int = 0
    rest_max: float = 0.0
    naehe_punkt_dreieck: int = 0
    naehe_kante_kante: int = 0
    selbst_stoesse: int = 0
    durchdringungen: int = 0
    durchdringungsgebiete: int = 0
    zusammenbrueche: int = 0
    dv_max: float = 0.0

    @classmethod
    def from_c(cls, st: _abi.K3dStats) -> "ImplizitStatistik":
        return cls(**{f.name: getattr(st, f.name) for f in fields(cls)})
