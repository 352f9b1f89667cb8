"""Independent drapes of a batch spread over ranks (one process per GPU).

A batch of drapes has no coupling between its instances: each is its own
implicit step with its own Krylov solve. Across GPUs the batch is therefore
partitioned, not sharded: every rank takes a disjoint subset of the
instances, runs them as one batch scene on its own device (one persistent
PCG launch per substep, Szene.verbinden), and the host gathers the
instances' states back in the batch's order. No collective touches the data
path; the only exchange is the final gather of positions and velocities.

The split balances the same work estimate the PCG launch uses for its block
groups: an instance's PCG work per step grows as points^1.5 (points times an
iteration count that grows with the mesh width).
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np

from .szene import Szene


def instanzen_teilen(punkte: Sequence[int], welt: int) -> list[list[int]]:
    """Instance indices per rank: the heaviest remaining instance goes to the
    rank with the least work so far (the lowest rank among equals); each
    rank's list is in batch order. Deterministic: every rank computes the
    same split without talking to the others."""
    if welt < 1:
        raise ValueError("at least one rank")
    gewicht = [float(p) ** 1.5 for p in punkte]
    reihenfolge = sorted(range(len(punkte)), key=lambda k: (-gewicht[k], k))
    last = [0.0] * welt
    teile: list[list[int]] = [[] for _ in range(welt)]
    for k in reihenfolge:
        r = min(range(welt), key=lambda q: (last[q], q))
        teile[r].append(k)
        last[r] += gewicht[k]
    return [sorted(t) for t in teile]


class VerteilteDrapierung:
    """One rank's share of a batch of drapes.

    ``szenen`` is the whole batch (every rank passes the same list);
    ``schritt(szene, n)`` advances a scene by n frames in place, e.g.
    ``ImplizitCg(param, device).bilder_resident`` on this rank's GPU. With
    ``dist`` (torch.distributed, initialised) the ranks gather their states
    on rank 0; without it the object serves one process (welt = 1)."""

    def __init__(self, szenen: Sequence[Szene], schritt: Callable[[Szene, int], object], rang: int = 0,
                 welt: int = 1, dist=None):
        self.rang, self.welt, self.dist = rang, welt, dist
        self.teile = instanzen_teilen([s.n for s in szenen], welt)
        self.meine = self.teile[rang]
        self.punkte = [s.n for s in szenen]
        self.szene = Szene.verbinden([szenen[k].copy() for k in self.meine]) if self.meine else None
        self.schritt = schritt

    def bilder(self, n: int):
        """n frames of this rank's instances (none: nothing to do)."""
        if self.szene is not None:
            return self.schritt(self.szene, n)
        return None

    def _eigene(self) -> dict:
        if self.szene is None:
            return {}
        return {k: (self.szene.x[self.szene.instanz(q)].copy(), self.szene.v[self.szene.instanz(q)].copy())
                for q, k in enumerate(self.meine)}

    def zustand_sammeln(self):
        """(x, v) of the whole batch in batch order on rank 0 (None on the
        other ranks): each rank sends its instances' states once."""
        eigene = self._eigene()
        if self.dist is None or self.welt == 1:
            alle = [eigene]
        else:
            alle = [None] * self.welt if self.rang == 0 else None
            self.dist.gather_object(eigene, alle, dst=0)
            if self.rang != 0:
                return None
        teile = {}
        for d in alle:
            teile.update(d)
        if sorted(teile) != list(range(len(self.punkte))):
            raise RuntimeError("an instance is missing or doubled in the gather")
        x = np.concatenate([teile[k][0] for k in range(len(self.punkte))], axis=0)
        v = np.concatenate([teile[k][1] for k in range(len(self.punkte))], axis=0)
        return x, v
