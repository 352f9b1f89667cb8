"""Launch shapes of the device step (no reference counterpart): the frame
replayed as a CUDA graph, fewer CTAs in the persistent PCG launch, and the
tuner that picks between them. The graph runs the same kernels with the same
arguments, so its states are bit-identical to direct launches; fewer CTAs
change only the summation order of the grid reductions, so those states match
the oracle to the batched tests' 1e-9 of the bounding-box diagonal."""
import numpy as np
import pytest

import oracle_py as O
from garmentcraft_b200 import _abi, autotune
from garmentcraft_b200.implizit import ImplizitCg
from garmentcraft_b200.params import ImplizitParameter
from garmentcraft_b200.szene import Szene
from test_gpu_batch import diag, param, szenen

pytestmark = pytest.mark.gpu


def _bewegt(s):
    """The scene's body moving sideways, so every frame's launch arguments
    differ (the graph is captured again each frame)."""
    t = s.copy()
    k = dict(t.koerper[0])
    k["geschwindigkeit"] = (0.05, 0.0, 0.0)
    t.koerper = [k]
    return t


@pytest.mark.parametrize("prec", [_abi.K3D_FP64, _abi.K3D_MIXED])
@pytest.mark.parametrize("bewegt", [False, True])
def test_graph_wie_direkt(prec, bewegt):
    tube, blatt, _ = szenen()
    for s0 in (tube, blatt):
        s0 = _bewegt(s0) if bewegt else s0
        p = param(prec)
        p.schritte_je_bild = 3
        a, b = s0.copy(), s0.copy()
        for t in (a, b):  # each copy moves its own bodies
            t.koerper = [dict(k) for k in t.koerper]
        ca = ImplizitCg(p)
        cb = ImplizitCg(ImplizitParameter(**{**p.__dict__, "graph": True}))
        for f in range(6):
            ca.bild(a)
            cb.bild(b)
            assert np.array_equal(a.x, b.x) and np.array_equal(a.v, b.v), f
            assert ca.statistik == cb.statistik, f
        assert ca.kernel_starts() == cb.kernel_starts()
        assert cb.letzte_loesung_ms() == 0.0 and cb.letzte_bild_ms() > 0.0
        # resident frames replay the graph captured by the frames above
        ca.bilder_auf_geraet(4)
        cb.bilder_auf_geraet(4)
        ca.zustand_lesen(a)
        cb.zustand_lesen(b)
        assert np.array_equal(a.x, b.x)


def test_wenige_bloecke_wie_orakel():
    einzeln = szenen()
    for k, s in enumerate(einzeln):
        for bl in (8, 37):
            p = param(_abi.K3D_FP64)
            p.pcg_bloecke = bl
            cg = ImplizitCg(p)
            t = s.copy()
            o = O.OracleSim(s, param(_abi.K3D_FP64).to_c())
            for _ in range(6):
                cg.bild(t)
                o.frames(1)
            assert cg.pcg_bloecke() == bl
            x, _ = o.state()
            assert np.max(np.abs(t.x - x)) <= 1e-9 * diag(x), (k, bl)


def test_batch_mit_wenigen_bloecken():
    """Three instances on 8 CTAs against the oracle; fewer CTAs than
    instances are refused."""
    einzeln = szenen()
    batch = Szene.verbinden([s.copy() for s in einzeln])
    p = param(_abi.K3D_FP64)
    p.pcg_bloecke = 8
    cg = ImplizitCg(p)
    orks = [O.OracleSim(s, param(_abi.K3D_FP64).to_c()) for s in einzeln]
    for _ in range(5):
        cg.bild(batch)
        for o in orks:
            o.frames(1)
    for k, o in enumerate(orks):
        x, _ = o.state()
        assert np.max(np.abs(batch.x[batch.instanz(k)] - x)) <= 1e-9 * diag(x), k
    p.pcg_bloecke = 2
    with pytest.raises(RuntimeError):
        ImplizitCg(p).bild(Szene.verbinden([s.copy() for s in einzeln]))


def test_abstimmen_schreibt_und_liest(tmp_path):
    _, blatt, _ = szenen()
    pfad = str(tmp_path / "abstimmung.json")
    p = param(_abi.K3D_MIXED)
    p.schritte_je_bild = 2
    q, rec = autotune.abstimmen(blatt, p, bilder=2, runden=1, cache=pfad)
    assert (q.pcg_bloecke, q.graph) == (rec["pcg_bloecke"], rec["graph"])
    assert len(rec["kandidaten"]) >= 4 and all(z["ms_je_bild"] > 0 for z in rec["kandidaten"])
    assert rec["ms_je_bild"] == min(z["ms_je_bild"] for z in rec["kandidaten"])
    q2, rec2 = autotune.abstimmen(blatt, p, cache=pfad)
    assert rec2 == rec and q2 == q
    # the chosen shape steps the scene like the default one
    a, b = blatt.copy(), blatt.copy()
    ca, cb = ImplizitCg(p), ImplizitCg(q)
    for _ in range(3):
        ca.bild(a)
        cb.bild(b)
    assert np.max(np.abs(a.x - b.x)) <= 1e-5 * diag(a.x)
