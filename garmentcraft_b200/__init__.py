"""B200 implicit cloth step: a drop-in for klon3d-sim's ImplizitCg / Loeser.

The hot path is hand-written sm_100a CUDA (garmentcraft_b200/csrc) behind the
C ABI in include/klon3d_step.h; this package is the host-side mirror of the
reference's solver API for Python callers and the tests.
"""
from . import _abi, synth
from ._abi import K3D_FP64, K3D_MIXED, K3D_MIXED_STORAGE
from .params import ImplizitParameter, ImplizitStatistik
from .szene import Szene

__all__ = ["ImplizitCg", "ImplizitParameter", "ImplizitStatistik", "Szene", "build_scene", "synth",
           "K3D_FP64", "K3D_MIXED", "K3D_MIXED_STORAGE", "CgLauf"]


def __getattr__(name):
    # the device solver loads the native library on first use
    if name in ("ImplizitCg", "build_scene", "CgLauf"):
        from . import implizit
        return getattr(implizit, name)
    raise AttributeError(name)
