"""Launch-shape tuner for the device step (no counterpart in the reference,
whose solver has a single CPU form).

The step has three launch choices that change its speed but not its
arithmetic beyond the summation order of the grid reductions:

* ``pcg_threads`` -- the CTA size of the persistent PCG launch: 512 threads
  (one CTA per SM, 128 registers a thread), 256 (two CTAs per SM, the same
  registers; twice the CTAs at every grid barrier) or 1024 (one CTA per SM,
  64 registers a thread, so the kernel spills; twice the warps to hide the
  row products' load latency).
* ``pcg_bloecke`` -- CTAs of the persistent PCG launch. Every PCG iteration
  passes two grid barriers whose cost grows with the CTAs that arrive; a
  small drape has too little work per iteration to hide it, so fewer CTAs
  win there, while a large drape needs every SM for its row products.
* ``graph`` -- replaying a frame's launches as one CUDA graph, which removes
  the host launch cost between the short kernels of a substep (not with
  self-collision, whose stage reads counts back between launches).

``abstimmen`` times every candidate (CTA size x CTA count x graph) on the
caller's own scene (the same
frames from the same state, device time from CUDA events), keeps the fastest
and caches it in a JSON file keyed by the device, the precision and the
scene's size, so the sweep runs once per shape.
"""
from __future__ import annotations

import json
import os
from dataclasses import replace

from .implizit import ImplizitCg
from .params import ImplizitParameter
from .szene import Szene

CACHE_ENV = "GARMENTCRAFT_B200_TUNE"
THREADS = (512, 256, 1024)  # CTA sizes the library is built for


def cache_pfad() -> str:
    """The cache file: $GARMENTCRAFT_B200_TUNE, else
    ~/.cache/garmentcraft_b200/abstimmung.json."""
    return os.environ.get(CACHE_ENV) or os.path.join(
        os.path.expanduser("~"), ".cache", "garmentcraft_b200", "abstimmung.json")


def _instanzen(s: Szene) -> int:
    """Instances of a batch scene (its point offsets hold one more entry)."""
    return max(int(s.instanz_punkte.shape[0]) - 1, 1)


def schluessel(geraet: str, param: ImplizitParameter, s: Szene) -> str:
    """Cache key: device, precision, points, triangles, instances, substeps
    and whether self-collision runs."""
    inst = _instanzen(s)
    return (f"{geraet}|p{param.precision}|n{s.n}|t{len(s.dreiecke)}|i{inst}"
            f"|s{param.schritte_je_bild}|sk{int(param.selbstkollision)}")


def kandidaten(max_bloecke: int, instanzen: int = 1) -> list[int]:
    """CTA counts to try: the full grid, then halvings down to 8, each at
    least the instance count (every instance needs a CTA of its own)."""
    out, b = [], max_bloecke
    while b >= max(8, instanzen):
        out.append(b)
        b //= 2
    if not out:
        out.append(max_bloecke)
    return out


def _lesen(pfad: str) -> dict:
    try:
        with open(pfad) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _schreiben(pfad: str, daten: dict) -> None:
    os.makedirs(os.path.dirname(pfad) or ".", exist_ok=True)
    tmp = pfad + ".tmp"
    with open(tmp, "w") as f:
        json.dump(daten, f, indent=1, sort_keys=True)
    os.replace(tmp, pfad)


def _gewaehlt(param: ImplizitParameter, rec: dict) -> ImplizitParameter:
    return replace(param, pcg_bloecke=rec["pcg_bloecke"], graph=rec["graph"],
                   pcg_threads=rec.get("pcg_threads", 0))


def abstimmen(s: Szene, param: ImplizitParameter | None = None, bilder: int = 3, runden: int = 2,
              cache: str | None = None, device: int = 0, neu: bool = False,
              threads: tuple[int, ...] = THREADS) -> tuple[ImplizitParameter, dict]:
    """The fastest launch shape for ``s`` under ``param``: returns the
    parameters with ``pcg_threads``, ``pcg_bloecke`` and ``graph`` set, and
    the record (the time per frame of every candidate). ``s`` is not changed.
    A cached record for the same key is used unless ``neu``."""
    param = param or ImplizitParameter()
    pfad = cache or cache_pfad()
    probe = ImplizitCg(param, device)
    geraet = probe.loeser_name()
    del probe
    key = schluessel(geraet, param, s)
    daten = _lesen(pfad)
    if not neu and key in daten:
        rec = daten[key]
        return _gewaehlt(param, rec), rec
    inst = _instanzen(s)
    graphen = (False,) if param.selbstkollision else (False, True)
    formen = []
    for nt in threads:
        probe = ImplizitCg(replace(param, pcg_threads=nt), device)
        probe.hochladen(s.copy())
        voll = probe.pcg_bloecke()
        del probe
        formen += [(nt, b) for b in kandidaten(voll, inst)]
    zeiten = []
    for nt, b in formen:
        for g in graphen:
            p = replace(param, pcg_bloecke=b, graph=g, pcg_threads=nt)
            cg = ImplizitCg(p, device)
            t = s.copy()
            cg.hochladen(t)
            cg.bilder_auf_geraet(2)  # warm-up; the graph is captured here
            best = float("inf")
            for _ in range(max(runden, 1)):
                cg.zustand_hochladen(s)
                cg.bilder_auf_geraet(bilder)
                best = min(best, cg.letzte_bild_ms() / bilder)
            zeiten.append({"pcg_threads": nt, "pcg_bloecke": b, "graph": g, "ms_je_bild": best})
            del cg
    sieger = min(zeiten, key=lambda z: z["ms_je_bild"])
    rec = {"pcg_threads": sieger["pcg_threads"], "pcg_bloecke": sieger["pcg_bloecke"], "graph": sieger["graph"],
           "ms_je_bild": sieger["ms_je_bild"], "kandidaten": zeiten, "bilder": bilder}
    daten[key] = rec
    _schreiben(pfad, daten)
    return _gewaehlt(param, rec), rec
