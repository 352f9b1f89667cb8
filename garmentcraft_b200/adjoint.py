"""Forward/backward pair of a drape over the material parameters.

The reference has no differentiation (klon3d-sim steps forward only); this is
new API on top of the device adjoint (``k3d_adjoint_forward`` /
``k3d_adjoint_backward``). ``Drapierung`` runs n frames of a scene at given
material parameters and returns the final state; its ``rueckwaerts`` maps the
per-element cotangents of the device to the five parameters of the scene's
one material: warp, weft and shear stiffness (N/m), bending stiffness (N m)
and the grain angle (rad). ``DrapeFunction`` is the same pair as a
``torch.autograd.Function``.

Parameter map (one material, isotropic bending as in the sheet workloads):
every membrane has (E_warp, E_weft, G) = (warp, weft, shear) and its grain
basis rotated by the angle's change; every hinge has k = k_0 * bend / bend_0
(implizit.rs:774-796 with biegung.rs:111-173, where the hinge stiffness is
linear in the bending stiffness when all three directions are equal).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _abi
from .implizit import ImplizitCg
from .params import ImplizitParameter
from .szene import Szene

NAMEN = ("warp", "weft", "shear", "bend", "grain")


@dataclass
class Stoff:
    """The five parameters (warp, weft, shear N/m; bend N m; grain rad)."""
    warp: float
    weft: float
    shear: float
    bend: float
    grain: float

    def array(self) -> np.ndarray:
        return np.array([self.warp, self.weft, self.shear, self.bend, self.grain])

    @staticmethod
    def von(a) -> "Stoff":
        a = [float(v) for v in a]
        return Stoff(*a)


def stoff_der_szene(s: Szene, bend: float, grain: float) -> Stoff:
    """The parameters a one-material scene was built with (bend and grain as
    given to the builder, which the element arrays do not keep)."""
    e = s.membran_steif[0]
    return Stoff(float(e[0]), float(e[1]), float(e[2]), bend, grain)


def szene_mit(basis: Szene, basis_stoff: Stoff, p: Stoff) -> Szene:
    """A copy of ``basis`` with the element constants of parameters ``p``."""
    s = basis.copy()
    s.membran_steif = np.repeat(np.array([[p.warp, p.weft, p.shear]]), s.membran_steif.shape[0], axis=0)
    d = p.grain - basis_stoff.grain
    c, sn = math.cos(d), math.sin(d)
    for nm in ("membran_kette", "membran_schuss"):
        a = getattr(basis, nm)
        b = np.empty_like(a)
        b[:, 0] = c * a[:, 0] - sn * a[:, 1]
        b[:, 1] = sn * a[:, 0] + c * a[:, 1]
        setattr(s, nm, b)
    s.biegung_nachgiebigkeit = basis.biegung_nachgiebigkeit * (basis_stoff.bend / p.bend)
    return s


class Drapierung:
    """n frames of one scene from (x0, v0) at parameters p, differentiable.

    ``vorwaerts`` keeps checkpoints every ``k`` substeps on the device;
    ``rueckwaerts`` recomputes between them and returns the cotangents of the
    parameters and of x0, v0 for those of the final x, v."""

    def __init__(self, basis: Szene, basis_stoff: Stoff, frames: int, k: int = 10,
                 param: ImplizitParameter | None = None, device: int = 0):
        self.basis = basis
        self.basis_stoff = basis_stoff
        self.frames = frames
        self.k = k
        self.param = param or ImplizitParameter(schritte_je_bild=1, cg_max=4000, cg_toleranz=1e-8)
        if self.param.precision != _abi.K3D_FP64:
            raise ValueError("the adjoint runs in FP64")
        self.cg = ImplizitCg(self.param, device=device)
        self.p: Stoff | None = None
        self.letzte: dict = {}

    def vorwaerts(self, p, x0: np.ndarray | None = None, v0: np.ndarray | None = None):
        self.p = p if isinstance(p, Stoff) else Stoff.von(p)
        s = szene_mit(self.basis, self.basis_stoff, self.p)
        if x0 is not None:
            s.x = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1, 3).copy()
        if v0 is not None:
            s.v = np.ascontiguousarray(v0, dtype=np.float64).reshape(-1, 3).copy()
        self.szene = s
        self.cg.hochladen(s)
        st = self.cg.adjoint_vorwaerts(self.frames, self.k)
        self.cg.zustand_lesen(s)
        self.letzte = dict(vorwaerts=st)
        return s.x.copy(), s.v.copy()

    def rueckwaerts(self, gx: np.ndarray, gv: np.ndarray | None = None) -> dict:
        if gv is None:
            gv = np.zeros_like(gx)
        r = self.cg.adjoint_rueckwaerts(gx, gv)
        k = 1.0 / self.szene.biegung_nachgiebigkeit
        gm, gb = r["membran"], r["biegung"]
        g = np.array([gm[:, 0].sum(), gm[:, 1].sum(), gm[:, 2].sum(), float(np.sum(gb * k)) / self.p.bend,
                      gm[:, 3].sum()])
        self.letzte.update(r)
        return dict(stoff=g, x=r["x"], v=r["v"], roh=r)


def DrapeFunction():
    """The torch.autograd.Function of a Drapierung:
    ``x, v = DrapeFunction().apply(p, x0, v0, drapierung)`` with p a tensor of
    the five parameters and x0, v0 (N, 3) float64 tensors."""
    import torch

    class _Drape(torch.autograd.Function):
        @staticmethod
        def forward(ctx, p, x0, v0, d: Drapierung):
            x, v = d.vorwaerts(p.detach().cpu().numpy(), x0.detach().cpu().numpy(), v0.detach().cpu().numpy())
            ctx.d = d
            ctx.dev = p.device
            return torch.from_numpy(x).to(x0.device), torch.from_numpy(v).to(v0.device)

        @staticmethod
        def backward(ctx, gx, gv):
            gxn = gx.detach().cpu().numpy() if gx is not None else None
            gvn = gv.detach().cpu().numpy() if gv is not None else np.zeros_like(gxn)
            if gxn is None:
                gxn = np.zeros_like(gvn)
            g = ctx.d.rueckwaerts(gxn, gvn)
            dev = ctx.dev
            return (torch.from_numpy(g["stoff"]).to(dev), torch.from_numpy(g["x"]).to(gx.device if gx is not None else dev),
                    torch.from_numpy(g["v"]).to(dev), None)

    return _Drape
