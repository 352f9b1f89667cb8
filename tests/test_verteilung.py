"""Batched drapes partitioned over ranks (garmentcraft_b200.verteilung).

The split is checked for its properties (disjoint, complete, balanced,
deterministic), and two gloo ranks on the CPU run a small batch with the
oracle as each rank's step: the states gathered on rank 0 equal, bit for bit,
those of one process that steps every drape alone.
"""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle_py as O
from garmentcraft_b200 import synth
from garmentcraft_b200.params import ImplizitParameter
from garmentcraft_b200.verteilung import VerteilteDrapierung, instanzen_teilen

FRAMES = 6


def test_teilen_eigenschaften():
    rng = np.random.default_rng(1)
    punkte = [int(p) for p in np.exp(rng.uniform(np.log(2000), np.log(60000), 64))]
    for welt in (1, 2, 3, 8):
        teile = instanzen_teilen(punkte, welt)
        alle = sorted(k for t in teile for k in t)
        assert alle == list(range(len(punkte)))
        assert all(t == sorted(t) for t in teile)
        last = [sum(punkte[k] ** 1.5 for k in t) for t in teile]
        assert max(last) - min(last) <= max(p ** 1.5 for p in punkte) + 1e-6
        assert teile == instanzen_teilen(punkte, welt)
    assert instanzen_teilen([5, 5], 4)[2:] == [[], []]


def szenen():
    return [O.build_scene(m, [b]) for m, b in synth.drape_batch(5, seed=2, n_min=60, n_max=400, fall_m=0.01)]


def param():
    return ImplizitParameter(schritte_je_bild=1, cg_max=2000, cg_toleranz=1e-8)


def oracle_schritt(instanzen):
    """Steps a batch scene instance by instance with the oracle (CPU)."""
    sims = [O.OracleSim(s, param().to_c()) for s in instanzen]

    def schritt(batch, n):
        for q, sim in enumerate(sims):
            sl = batch.instanz(q)
            sim.set_state(batch.x[sl], batch.v[sl])
            sim.frames(n)
            x, v = sim.state()
            batch.x[sl], batch.v[sl] = x, v
    return schritt


def _rang(rang, welt, port, pfad):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rang, world_size=welt)
    try:
        alle = szenen()
        teile = instanzen_teilen([s.n for s in alle], welt)
        d = VerteilteDrapierung(alle, oracle_schritt([alle[k] for k in teile[rang]]), rang, welt, dist)
        d.bilder(FRAMES)
        got = d.zustand_sammeln()
        if rang == 0:
            np.savez(pfad, x=got[0], v=got[1], teile=np.array([len(t) for t in teile]))
        else:
            assert got is None
    finally:
        dist.destroy_process_group()


def test_zwei_gloo_raenge_wie_ein_prozess():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    with tempfile.TemporaryDirectory() as tmp:
        pfad = os.path.join(tmp, "rang0.npz")
        mp.start_processes(_rang, args=(2, port, pfad), nprocs=2, join=True, start_method="spawn")
        got = np.load(pfad)
    assert got["teile"].min() >= 1  # both ranks had work
    alle = szenen()
    ein = VerteilteDrapierung(alle, oracle_schritt(alle))
    ein.bilder(FRAMES)
    x, v = ein.zustand_sammeln()
    assert np.array_equal(got["x"], x) and np.array_equal(got["v"], v)
    assert float(np.max(np.abs(x - np.concatenate([s.x for s in alle])))) > 0.0  # the drapes moved
