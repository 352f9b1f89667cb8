#!/usr/bin/env python
"""Benchmark of the implicit cloth step: vertex-steps/s.

Workload: a woven sheet of 257 x 257 vertices (66,049 points, 131,072
membrane triangles, ~196k bending hinges), 1 x 1 m with +/-1 mm jitter,
warp/weft/shear 2000/1000/50 N/m, dropped 0.5 m onto a sphere of radius
0.3 m stored as a 128^3 signed-distance grid at 1 cm; friction 0.3,
dt = 1/120 s, one implicit step per frame, PCG tolerance 1e-5 with a cap of
4000 iterations (the reference's default cap of 50 leaves this mesh's solves
far from converged and the drop diverges; converged solves take ~500-1800
iterations per step at impact). Synthetic, generated from a seed.

The first 34 steps are free fall (the warm start solves them exactly, no CG
iterations). Timing starts at step 34, just before first contact; the W
warm-up steps are the last W steps of the free fall (more than 34 extend the
start), the steps before them are an untimed pre-roll. Both arms time the same
window from the same state.

A step is one implicit backward-Euler step (build, PCG with release pass,
friction, integration) of the whole sheet. ``value`` is the chosen form,
K3D_MIXED_STORAGE (operator blocks and preconditioner stored in FP32, CG
vectors and sums in FP64), measured on the device-resident state with CUDA
events around the step kernels, L2 flushed (256 MiB write) before every timed
step; ``e2e`` is the same step through the public API (ImplizitCg.bild) with x
and v copied from pinned host memory to the device and back every step.
``fp64`` (the drop-in form) and ``mixed_fp32_vectors`` (K3D_MIXED) are timed
on the same window; ``mixed_vs_fp64`` gives the speed ratios and the
position error of each form against FP64 after one step from the same state,
after 100 steps of the drop, and after 10, 25, 50 and 100 steps of the same
sheet hanging from two corners with no body (see no_contact_leg).

``cpu_baseline`` is the FP64 oracle (the reference's CPU step restated, one
thread) on steps sampled across the timed window, each started from the FP64
device state at that step with its CG warm start, so it sees the window's
iteration counts. ``--impl reference`` runs the oracle alone over exactly the
K timed steps of the window, with the scene built by the oracle's own scene
builder; it loads no part of the device library.

``adjoint`` is the backward/forward time of the step's adjoint on the
material-fit workload (see adjoint_leg), with its gradient check.
``garment`` is the same step on the ~205k-point sewn garment with the
self-collision proximity stage on and off (see garment_leg). ``mesh`` is the
body mesh as a collider: voxelisation, nearest queries, segment tests and the
sheet step on an exact mesh body (see mesh_leg).

Multi-GPU: the step of one drape does not shard (a global Krylov solve), so
``--gpus N`` runs N independent replicas, one per rank, with no collective on
the data path; value = total vertex-steps / max over ranks of the time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CG_MAX = 4000
FREE_FALL = 34  # steps before the first contact
START = FREE_FALL


def window(warmup):
    """(pre-roll steps, warm-up steps) before the first timed step."""
    start = max(FREE_FALL, warmup)
    return start - warmup, warmup


METRIC = "vertex-steps/s, mixed vs FP64 GPU at <=1e-4 rel pos err; backward/forward time"
UNIT = "vertex-steps/s"


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=257, help="vertices per side of the sheet")
    p.add_argument("--cpu-seconds", type=float, default=25.0)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-compare", action="store_true")
    p.add_argument("--capture", type=int, default=0,
                   help="profiling case: run this many mixed-form steps of the drop on cuda:0 and exit")
    p.add_argument("--precision", default="storage", choices=["storage", "mixed", "fp64"],
                   help="form used by --capture: storage (K3D_MIXED_STORAGE), mixed (K3D_MIXED) or fp64")
    p.add_argument("--workload", default="sheet", choices=["sheet", "garment", "adjoint", "mesh"],
                   help="case of --capture: the sheet drop, the garment with self-collision (frames), the "
                        "material-fit drop's adjoint (frames forward, then the backward), or the body mesh "
                        "(rounds of voxelisation at a 3 and a 6 cm band)")
    p.add_argument("--garment-points", type=int, default=200_000,
                   help="points of the garment for --capture --workload garment (a smaller case for full captures)")
    p.add_argument("--no-batch", action="store_true", help="skip the batched-drape comparison")
    p.add_argument("--no-adjoint", action="store_true", help="skip the adjoint (material-fit) leg")
    p.add_argument("--no-garment", action="store_true", help="skip the sewn-garment leg")
    p.add_argument("--no-mesh", action="store_true", help="skip the body-mesh leg")
    p.add_argument("--no-shapes", action="store_true", help="skip the launch-shape (tuner, graph) leg")
    p.add_argument("--batch-steps", type=int, default=5)
    return p.parse_args()


BATCH_PRE = 15  # free-fall steps of the batched drapes (0.1 m drop) before the timed window


ADJ_N = 129        # material-fit sheet: 129 x 129 points
ADJ_FRAMES = 120
ADJ_K = 10         # checkpoint spacing (substeps)
ADJ_FD_FRAMES = 40  # horizon of the gradient check: through first impact


def adjoint_leg(torch):
    """Backward/forward time of the adjoint on the material-fit workload:
    a 129 x 129 sheet (16,641 points) dropped onto the sheet workload's
    sphere (128^3 SDF at 1 cm), 120 frames, FP64 (the adjoint's form), PCG
    tolerance 1e-5 as the main workload, checkpoints every 10 substeps.
    Hidden parameters (warp, weft, shear, bend, grain) from the seed, the
    target is the drop at them, the loss sum |x - x*|^2 at the start
    parameters (hidden x U(0.5, 2)). backward = device time of
    k3d_adjoint_backward, recomputation of the segments included; forward =
    that of k3d_adjoint_forward (the frames with checkpoints).

    Gradient check: the five parameter gradients against central differences
    of the device forward (relative steps 1e-3 and 1e-4, PCG tolerance 1e-8)
    over the first 40 frames, through first impact. Over the whole drop the
    central differences do not converge as the step shrinks (contact and
    friction decisions make the drop chaotic after impact), so the check
    uses the horizon where they do."""
    import numpy as np
    from garmentcraft_b200 import _abi, synth
    from garmentcraft_b200.adjoint import NAMEN, Drapierung, Stoff
    from garmentcraft_b200.params import ImplizitParameter
    s, hid, start = synth.materialfit(n=ADJ_N)
    bs = Stoff.von(hid)
    par = ImplizitParameter(schritte_je_bild=1, cg_max=CG_MAX, cg_toleranz=1e-5, precision=_abi.K3D_FP64)
    d = Drapierung(s, bs, frames=ADJ_FRAMES, k=ADJ_K, param=par)
    ziel, _ = d.vorwaerts(hid)
    x, _ = d.vorwaerts(start)  # warm-up pass
    d.rueckwaerts(2.0 * (x - ziel))
    x, _ = d.vorwaerts(start)
    fst = d.letzte["vorwaerts"]
    g = d.rueckwaerts(2.0 * (x - ziel))
    r = g["roh"]
    out = {"workload": f"material fit: {ADJ_N}x{ADJ_N} sheet ({s.n} points) onto the sphere SDF, "
                       f"{ADJ_FRAMES} frames, FP64, tol 1e-5",
           "frames": ADJ_FRAMES, "checkpoint_every": ADJ_K, "forward_ms": r["ms_vorwaerts"],
           "backward_ms": r["ms_rueckwaerts"], "recompute_ms": r["ms_neuberechnung"],
           "backward_forward": r["ms_rueckwaerts"] / r["ms_vorwaerts"],
           "forward_cg_iterations": fst.cg_iterationen, "adjoint_cg_iterations": r["iterationen"],
           "adjoint_unconverged_solves": r["nicht_konvergiert"],
           "definition": "device time of the backward (recomputation included) / device time of the forward"}
    par2 = ImplizitParameter(schritte_je_bild=1, cg_max=20000, cg_toleranz=1e-8, precision=_abi.K3D_FP64)
    d2 = Drapierung(s, bs, frames=ADJ_FD_FRAMES, k=ADJ_K, param=par2)
    ziel2, _ = d2.vorwaerts(hid)

    def loss(p):
        xx, _ = d2.vorwaerts(p)
        return float(np.sum((xx - ziel2) ** 2))

    x2, _ = d2.vorwaerts(start)
    g2 = d2.rueckwaerts(2.0 * (x2 - ziel2))["stoff"]
    chk = {}
    for q, name in enumerate(NAMEN):
        fd = {}
        for rel in (1e-3, 1e-4):
            h = rel * abs(start[q])
            pp, pm = start.copy(), start.copy()
            pp[q] += h
            pm[q] -= h
            fd[f"{rel:g}"] = (loss(pp) - loss(pm)) / (2.0 * h)
        errs = {k: abs(v - g2[q]) / abs(v) for k, v in fd.items()}
        chk[name] = {"adjoint": float(g2[q]), "fd": fd, "rel_err": errs, "best_rel_err": min(errs.values())}
    out["gradient_check"] = {"frames": ADJ_FD_FRAMES, "tol": 1e-8, "params": chk,
                             "max_best_rel_err": max(c["best_rel_err"] for c in chk.values())}
    return out


GARMENT_PRE = 10    # untimed frames of the garment before its window
GARMENT_STEPS = 5


def garment_leg(flush, torch, peaks, cpu=True):
    """The sewn-garment workload (synth.garment_szene: 28 panels, ~205k
    points, 15-capsule body SDF 256x256x384 at 5 mm, latex, 2 mm collision
    thickness, dt 1/120): frames GARMENT_PRE .. GARMENT_PRE + GARMENT_STEPS of
    the drop, device-resident, L2 flushed before every timed frame, in the
    three forms, with the self-collision stage on (the workload) and off (the
    step alone). For the chosen form with self-collision on: the PCG
    roofline, e2e through ImplizitCg.bild with host buffers (pinned, copied
    in and out every frame), and a cpu_baseline of one oracle step (FP64, one
    thread) from the FP64 device state at the window's first frame, warm
    start included. One-step position error of each form against FP64 from
    that state."""
    import numpy as np
    from garmentcraft_b200 import _abi, synth
    from garmentcraft_b200.implizit import ImplizitCg
    from garmentcraft_b200.params import ImplizitParameter
    s0, _ = synth.garment_szene()
    out = {"workload": f"sewn garment: 28 panels, {s0.n} points, {s0.membran_punkte.shape[0]} membranes, "
                       f"{s0.naht_punkte.shape[0]} seam pairs, 15-capsule SDF 256x256x384 at 5 mm",
           "window": f"frames {GARMENT_PRE}-{GARMENT_PRE + GARMENT_STEPS - 1}", "unit": UNIT}

    def par(prec, selbst):
        return ImplizitParameter(schritte_je_bild=1, cg_max=CG_MAX, cg_toleranz=1e-5, precision=prec,
                                 selbstkollision=selbst)
    for selbst in (True, False):
        for prec in (HEADLINE, 0, 1):
            name = FORMS[prec][0]
            s = s0.copy()
            cg = ImplizitCg(par(prec, selbst), device=torch.cuda.current_device())
            cg.zustand_hochladen(s)
            cg.bilder_auf_geraet(GARMENT_PRE)
            ms, sms, its, solves, pairs = [], 0.0, 0, 0, 0
            for k in range(GARMENT_STEPS):
                flush.fill_(float(k))
                torch.cuda.synchronize()
                st = cg.bilder_auf_geraet(1)
                ms.append(cg.letzte_bild_ms())
                sms += cg.letzte_loesung_ms()
                its += st.cg_iterationen
                solves += st.loesungen
                pairs += st.naehe_punkt_dreieck + st.naehe_kante_kante
            key = f"{'selfcollision' if selbst else 'no_selfcollision'}_{name}"
            out[key] = {"value": s.n * GARMENT_STEPS / (sum(ms) * 1e-3), "ms_per_step": float(np.mean(ms)),
                        "cg_iterations_per_step": its / GARMENT_STEPS, "proximity_pairs_per_step": pairs / GARMENT_STEPS,
                        "pcg_ms_per_step": sms / GARMENT_STEPS}
            if selbst and prec == HEADLINE:
                out["roofline"] = roofline_of(s, prec, its, solves, sms, sum(ms), GARMENT_STEPS, peaks,
                                              "k3d::solve_kernel<float, double, true>")
            del cg
    for tag in ("selfcollision", "no_selfcollision"):
        for prec in (HEADLINE, 1):
            out[f"{tag}_{FORMS[prec][0]}_vs_fp64"] = out[f"{tag}_{FORMS[prec][0]}"]["value"] / out[f"{tag}_fp64"]["value"]
    # e2e: the public call with host buffers
    s = s0.copy()
    for nm in ("x", "v"):
        t = torch.empty(getattr(s, nm).shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = getattr(s, nm)
        setattr(s, nm, t.numpy())
    cg = ImplizitCg(par(HEADLINE, True), device=torch.cuda.current_device())
    cg.bilder_resident(s, GARMENT_PRE)
    tot = 0.0
    for k in range(GARMENT_STEPS):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cg.bild(s)
        tot += time.perf_counter() - t0
    out["e2e"] = {"value": s.n * GARMENT_STEPS / tot, "unit": UNIT, "h2d_bytes_per_step": 48 * s.n,
                  "d2h_bytes_per_step": 48 * s.n + 144, "form": FORMS[HEADLINE][0], "selfcollision": True}
    del cg
    # one step of each form from the FP64 state at the window's start; the CPU sample from it
    s = s0.copy()
    cg = ImplizitCg(par(0, True), device=torch.cuda.current_device())
    cg.zustand_hochladen(s)
    cg.bilder_auf_geraet(GARMENT_PRE)
    cg.zustand_lesen(s)
    warm = cg.warmstart_lesen()
    ref = s.copy()
    cr = ImplizitCg(par(0, True), device=torch.cuda.current_device())
    cr.zustand_hochladen(ref)
    cr.bilder_auf_geraet(1)
    cr.zustand_lesen(ref)
    del cr
    d = float(np.linalg.norm(ref.x.max(0) - ref.x.min(0)))
    err = {}
    for prec in (HEADLINE, 1):
        t = s.copy()
        c = ImplizitCg(par(prec, True), device=torch.cuda.current_device())
        c.zustand_hochladen(t)
        c.bilder_auf_geraet(1)
        c.zustand_lesen(t)
        dx = np.linalg.norm(t.x - ref.x, axis=1)
        err[FORMS[prec][0]] = {"max": float(dx.max() / d), "rms": float(np.sqrt(np.mean(dx ** 2)) / d)}
        del c
    out["one_step_error_vs_fp64"] = {"from": f"the FP64 state at frame {GARMENT_PRE}", "errors": err,
                                     "definition": "|x_form - x_fp64| / bbox diagonal after one step from the "
                                                   "same state, every form on a new solver (no warm start)"}
    if cpu:
        O = oracle_mod()
        m, body = synth.garment(ziel_punkte=200_000)
        so = O.build_scene(m, [body])
        so.kollisionsabstand[:] = 2e-3  # as synth.garment_szene
        sim = O.OracleSim(so, par(0, True).to_c())
        sim.set_state(s.x, s.v)
        sim.set_dv_warm(warm)
        t0 = time.perf_counter()
        st = sim.frames(1)
        el = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": s.n / el, "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": f"one step (frame {GARMENT_PRE}) from the FP64 device state with its warm "
                                         f"start, self-collision on, {el:.1f} s, FP64 C++ restatement, one thread",
                               "cg_iterations_per_step": st.cg_iterationen}
    return out


MESH_REPS = 5


def mesh_leg(flush, torch):
    """The body mesh as a collider (include/klon3d_mesh.h) on a synthetic
    body of 36,864 triangles / 18,434 points (synth.koerper_netz, the size of
    a human base mesh split into triangles): voxelisation into the SDF grid at
    5 mm with a 3 cm and a 6 cm band, 200k nearest queries within the 1 cm
    search depth, 200k segment tests, nachfuehren; then the 257x257 sheet
    step on the mesh body against the same step on the 128^3 sphere grid.
    Device times are the library's CUDA events around its kernels, L2
    flushed before each; e2e is the C-ABI call with host arrays (copies
    included), wall clock."""
    import numpy as np
    from garmentcraft_b200 import synth
    from garmentcraft_b200.implizit import ImplizitCg
    from garmentcraft_b200.netzkoerper import Koerpernetz
    from garmentcraft_b200._abi import K3D_MIXED
    dev = torch.cuda.current_device()
    p, d = synth.koerper_netz()
    k = Koerpernetz(p, d, 0.01, device=dev)
    out = {"workload": f"synthetic body mesh, {d.shape[0]} triangles, {p.shape[0]} points, search depth 1 cm",
           "create_ms_device": k.letzte_ms}

    def timed(call):
        dms, wms = [], []
        call()
        for r in range(MESH_REPS):
            flush.fill_(float(r))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            call()
            wms.append(1e3 * (time.perf_counter() - t0))
            dms.append(k.letzte_ms)
        return statistics.median(dms), statistics.median(wms)

    for band in (0.03, 0.06):
        body = {}

        def vox():
            body["b"] = k.sdf_body(0.005, band)
        dm, wm = timed(vox)
        nn = int(np.prod(body["b"]["dims"]))
        out[f"sdf_band_{int(round(band * 100))}cm"] = {
            "dims": list(body["b"]["dims"]), "nodes": nn, "ms_device": dm, "value": nn / (dm * 1e-3),
            "unit": "nodes/s", "e2e": {"value": nn / (wm * 1e-3), "unit": "nodes/s", "ms": wm,
                                       "d2h_bytes": 4 * nn}, "unresolved_nodes": int(k.info().ungeklaert)}
    rng = np.random.default_rng(0)
    q = 200_000
    x = p[rng.integers(0, p.shape[0], q)] + rng.normal(0.0, 0.01, (q, 3))
    y = x + rng.normal(0.0, 0.01, (q, 3))
    dm, wm = timed(lambda: k.naechster(x, 0.01))
    out["nearest"] = {"queries": q, "radius_m": 0.01, "ms_device": dm, "value": q / (dm * 1e-3), "unit": "queries/s",
                      "e2e": {"value": q / (wm * 1e-3), "unit": "queries/s", "ms": wm}}
    dm, wm = timed(lambda: k.durchstoss(x, y))
    out["penetration"] = {"segments": q, "ms_device": dm, "value": q / (dm * 1e-3), "unit": "segments/s",
                          "e2e": {"value": q / (wm * 1e-3), "unit": "segments/s", "ms": wm}}
    flip = [p * 1.001, p]
    state = {"i": 0}

    def move():
        state["i"] ^= 1
        k.nachfuehren(flip[state["i"]])
    dm, wm = timed(move)
    out["nachfuehren"] = {"ms_device": dm, "ms_e2e": wm}
    # the sheet step on the mesh body against the sphere grid
    kugel_p, kugel_d = synth.koerper_netz(halbachsen=(0.3, 0.3, 0.3), mitte=(0.0, 0.0, 0.0))
    kugel = Koerpernetz(kugel_p, kugel_d, 0.01, device=dev)
    gitter = kugel.sdf_body(0.005, 0.03)
    for name, body in (("step_mesh_body", kugel.body()), ("step_grid_body", gitter)):
        s = make_scene(257)
        s.koerper = [body]
        cg = ImplizitCg(params(K3D_MIXED), device=dev)
        cg.zustand_hochladen(s)
        cg.bilder_auf_geraet(FREE_FALL + 6)
        ms, its = [], 0
        for r in range(MESH_REPS):
            flush.fill_(float(r))
            torch.cuda.synchronize()
            its += cg.bilder_auf_geraet(1).cg_iterationen
            ms.append(cg.letzte_bild_ms())
        out[name] = {"ms_per_step": statistics.median(ms), "value": s.n / (statistics.median(ms) * 1e-3),
                     "unit": UNIT, "cg_iterations_per_step": its / MESH_REPS}
    out["step_mesh_body"]["body"] = f"bumpy sphere mesh r 0.3 m, {kugel_d.shape[0]} triangles, exact query"
    out["step_grid_body"]["body"] = f"the same mesh voxelised, {'x'.join(map(str, gitter['dims']))} at 5 mm, trilinear"
    return out


def shapes_leg():
    """Launch shapes picked by the tuner (garmentcraft_b200.autotune): for a
    small drape (33x33 sheet, 5 substeps per frame), the 64-drape batch and
    the 257x257 sheet, every candidate (CTAs of the persistent PCG launch x
    frame replayed as a CUDA graph or launched directly) timed on the same
    frames from the drop's start, mixed form, device time per frame with CUDA
    events. 'default' is the full grid with direct launches."""
    import tempfile
    from garmentcraft_b200 import _abi, autotune, synth
    from garmentcraft_b200.implizit import build_scene
    from garmentcraft_b200.params import ImplizitParameter
    from garmentcraft_b200.szene import Szene
    m, k = synth.sheet_over_sphere(n=33, seed=3, fall_m=0.02)
    klein = build_scene(m, [k])
    batch = Szene.verbinden([build_scene(mm, [b]) for mm, b in synth.drape_batch(64)])
    gross = make_scene(257)
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for name, s, sub in (("sheet_33x33_5_substeps", klein, 5), ("batch_64_drapes", batch, 1),
                             ("sheet_257x257", gross, 1)):
            par = ImplizitParameter(schritte_je_bild=sub, cg_max=CG_MAX, precision=_abi.K3D_MIXED)
            q, rec = autotune.abstimmen(s, par, bilder=3, runden=2, cache=f"{d}/t.json", neu=True)
            voll = max(z["pcg_bloecke"] for z in rec["kandidaten"] if z["pcg_threads"] == 512)
            dflt = next(z for z in rec["kandidaten"]
                        if z["pcg_threads"] == 512 and z["pcg_bloecke"] == voll and not z["graph"])
            steps = 3 * sub
            out[name] = {"vertices": s.n, "substeps_per_frame": sub,
                         "default": {"pcg_threads": 512, "pcg_blocks": voll, "graph": False,
                                     "ms_per_frame": dflt["ms_je_bild"],
                                     "value": s.n * sub / (dflt["ms_je_bild"] * 1e-3)},
                         "tuned": {"pcg_threads": q.pcg_threads, "pcg_blocks": q.pcg_bloecke, "graph": bool(q.graph),
                                   "ms_per_frame": rec["ms_je_bild"],
                                   "value": s.n * sub / (rec["ms_je_bild"] * 1e-3)},
                         "tuned_vs_default": dflt["ms_je_bild"] / rec["ms_je_bild"],
                         "candidates": rec["kandidaten"], "frames_timed": 3, "steps_timed": steps}
    out["unit"] = UNIT
    return out


def batch_leg(steps, flush, torch):
    """Batched drapes: 64 sheets of 2k-60k vertices (log-uniform), aspect
    1:1 to 1:3, per-instance materials, each over its own sphere or capsule
    SDF (64^3). The same window (steps BATCH_PRE .. BATCH_PRE + steps) timed
    as one batch scene (one launch per kernel for all 64) and as 64 solvers
    run one after another (the per-instance launches), mixed form; the batch
    also in FP64. Device time per step with CUDA events, L2 flushed first."""
    from garmentcraft_b200 import _abi, synth
    from garmentcraft_b200.implizit import ImplizitCg, build_scene
    from garmentcraft_b200.params import ImplizitParameter
    from garmentcraft_b200.szene import Szene
    scenes = [build_scene(m, [b]) for m, b in synth.drape_batch(64)]
    nv = sum(s.n for s in scenes)

    def timed(cg, k):
        ms, its = 0.0, 0
        for _ in range(k):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            st = cg.bilder_auf_geraet(1)
            ms += cg.letzte_bild_ms()
            its += st.cg_iterationen
        return ms, its

    out = {"workload": "64 sheets, 2k-60k vertices log-uniform, aspect U(1,3), sphere or capsule SDF 64^3 each",
           "vertices": nv, "instances": len(scenes), "window": f"steps {BATCH_PRE}-{BATCH_PRE + steps} of the drop"}
    for prec, name in ((_abi.K3D_MIXED, "mixed"), (_abi.K3D_FP64, "fp64")):
        par = ImplizitParameter(schritte_je_bild=1, cg_max=CG_MAX, precision=prec)
        cg = ImplizitCg(par)
        cg.zustand_hochladen(Szene.verbinden([s.copy() for s in scenes]))
        cg.bilder_auf_geraet(BATCH_PRE)
        ms, its = timed(cg, steps)
        out[f"batched_{name}"] = {"value": nv * steps / (ms * 1e-3), "ms_per_step": ms / steps,
                                  "cg_iterations_per_step": its / steps}
        del cg
    par = ImplizitParameter(schritte_je_bild=1, cg_max=CG_MAX, precision=_abi.K3D_MIXED)
    ms_all, its_all = 0.0, 0
    for s in scenes:
        c = ImplizitCg(par)
        c.zustand_hochladen(s.copy())
        c.bilder_auf_geraet(BATCH_PRE)
        ms, its = timed(c, steps)
        ms_all += ms
        its_all += its
        del c
    out["per_instance_mixed"] = {"value": nv * steps / (ms_all * 1e-3), "ms_per_step": ms_all / steps,
                                 "cg_iterations_per_step": its_all / steps}
    out["batched_vs_per_instance"] = out["batched_mixed"]["value"] / out["per_instance_mixed"]["value"]
    out["unit"] = UNIT
    return out


def workload_config(n, s, extra=None):
    cfg = {
        "workload": f"sheet over sphere SDF, {n}x{n} vertices",
        "vertices": int(s.n), "membranes": int(s.membran_punkte.shape[0]),
        "bends": int(s.biegung_punkte.shape[0]), "springs": int(s.naht_punkte.shape[0]),
        "sdf": "128^3 at 1 cm", "dt": "1/120", "substeps_per_frame": 1, "cg_max": CG_MAX, "cg_tol": 1e-5,
        "window": f"steps {START}+ of the drop (impact and drape)",
        "l2": "flushed before every timed step (256 MiB write)", "parallelism": "replicas",
    }
    if extra:
        cfg.update(extra)
    return cfg


def make_scene(n, pinned=False, jitter_mm=1.0):
    from garmentcraft_b200 import synth
    from garmentcraft_b200.implizit import build_scene
    m, body = synth.sheet_over_sphere(n=n, jitter_mm=jitter_mm)
    s = build_scene(m, [body])
    if pinned:
        import torch
        for name in ("x", "v"):
            a = getattr(s, name)
            t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
            t.numpy()[:] = a
            setattr(s, name, t.numpy())
    return s


def make_hanging(n, jitter_mm=1.0):
    """The bench sheet with no body, its two corners of the first row held
    (w = 0): it swings from rest under gravity."""
    from garmentcraft_b200 import synth
    from garmentcraft_b200.implizit import build_scene
    m, _ = synth.sheet_over_sphere(n=n, jitter_mm=jitter_mm)
    s = build_scene(m, [])
    s.w[0] = 0.0
    s.w[n - 1] = 0.0
    return s


NO_CONTACT_TOL = 1e-10
NO_CONTACT_AT = (10, 25, 50, 100)


def no_contact_leg(n):
    """The bench sheet hanging from two corners with no body, from rest, for
    100 steps: every form against FP64 with all of them solved to
    NO_CONTACT_TOL (cap 20000), so what remains is each form's rounding
    (the FP32-vector form clamps its tolerance at 1e-6); and FP64 and the
    chosen form solved to 1e-5 against FP64 at NO_CONTACT_TOL. Errors (max
    and rms of |x - x_fp64| / bbox diagonal) after NO_CONTACT_AT steps show
    how a difference grows: no contact decision is taken, yet the swinging
    sheet buckles and amplifies any perturbation, that of the solver
    tolerance as much as that of the FP32 operator."""
    import numpy as np
    from garmentcraft_b200.implizit import ImplizitCg
    from garmentcraft_b200.params import ImplizitParameter

    def run(prec, tol):
        s = make_hanging(n)
        par = ImplizitParameter(schritte_je_bild=1, cg_max=20000, cg_toleranz=tol, precision=prec)
        cg = ImplizitCg(par)
        cg.zustand_hochladen(s)
        xs, its, done = [], 0, 0
        for k in NO_CONTACT_AT:
            its += cg.bilder_auf_geraet(k - done).cg_iterationen
            done = k
            cg.zustand_lesen(s)
            xs.append(s.x.copy())
        return xs, its / done

    ref, its_ref = run(0, NO_CONTACT_TOL)

    def err(prec, tol):
        xs, its = run(prec, tol)
        out = {"cg_iterations_per_step": its}
        for k, x, r in zip(NO_CONTACT_AT, xs, ref):
            d = float(np.linalg.norm(r.max(0) - r.min(0)))
            dx = np.linalg.norm(x - r, axis=1)
            out[f"after_{k}_steps"] = {"max": float(dx.max() / d), "rms": float(np.sqrt(np.mean(dx ** 2)) / d)}
        return out
    return {"workload": f"the {n}x{n} sheet without the sphere, held at the two corners of its first row, "
                        "100 steps from rest", "tol": NO_CONTACT_TOL,
            "fp64_cg_iterations_per_step": its_ref,
            "errors": {FORMS[p][0]: err(p, NO_CONTACT_TOL) for p in (HEADLINE, 1)},
            "at_bench_tol_1e-5": {FORMS[p][0]: err(p, 1e-5) for p in (0, HEADLINE)}}


def oracle_mod():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    return oracle_py


def make_scene_oracle(n, jitter_mm=1.0):
    """The same sheet built by the oracle's own scene builder (oracle/szene.cpp,
    Szene::aus_netz restated): no part of the device library is loaded."""
    from garmentcraft_b200 import synth
    m, body = synth.sheet_over_sphere(n=n, jitter_mm=jitter_mm)
    return oracle_mod().build_scene(m, [body])


HEADLINE = 2  # K3D_MIXED_STORAGE: the chosen form
FORMS = {0: ("fp64", 8, 8), 1: ("mixed_fp32_vectors", 4, 4), 2: ("mixed_storage", 4, 8)}


def params(prec):
    from garmentcraft_b200.params import ImplizitParameter
    return ImplizitParameter(schritte_je_bild=1, cg_max=CG_MAX, cg_toleranz=1e-5, precision=prec)


def element_counts(s):
    import numpy as np
    N, T, B = s.n, s.membran_punkte.shape[0], s.biegung_punkte.shape[0]
    S = s.naht_punkte.shape[0] + int(np.sum(s.membran_kante == 0))
    return N, T, B, S


def algorithmic_solve_bytes(s, s_op, s_vec, iters, solves):
    """Algorithmic bytes of the PCG launches alone (the dominant kernel), with
    the per-unit figures of algorithmic_bytes: operator records at s_op bytes
    per value, vectors at s_vec (FP64 form 8/8, mixed 4/4, storage form 4/8;
    the preconditioner is an operator value)."""
    N, T, B, S = element_counts(s)
    per_app = N * 10 * s_vec + T * (12 + 21 * s_op) + B * (16 + 13 * s_op) + S * (8 + 5 * s_op)
    per_it = N * (25 * s_vec + 6 * s_op)
    return (iters + 2 * solves) * per_app + iters * per_it


def algorithmic_bytes(s, s_op, s_vec, steps, iters, solves):
    """Minimal streamed bytes of the step (each datum once per pass), per
    unit: per operator application N*10s + T*(12+21s) + B*(16+13s) +
    S*(8+5s); per CG iteration the vector update N*31s (of which the
    preconditioner 6s); per step the build and integration 48N + T*(12+21s) +
    B*(16+13s) + S*(8+5s) + 18s*N + 96N + 32N. Operator applications per step =
    CG iterations + 2 per solve (the start residual and the release test)."""
    N, T, B, S = element_counts(s)
    elem = T * (12 + 21 * s_op) + B * (16 + 13 * s_op) + S * (8 + 5 * s_op)
    build = 48 * N + elem + 18 * s_op * N + 96 * N + 32 * N
    return algorithmic_solve_bytes(s, s_op, s_vec, iters, solves) + steps * build


def roofline_of(s, prec, iters, solves, solve_ms, step_ms, steps, peaks, kernel):
    _, s_op, s_vec = FORMS[prec]
    alg = algorithmic_solve_bytes(s, s_op, s_vec, iters, solves)
    achieved = alg / (solve_ms / 1e3) / 1e9
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": None, "peak_source": "measured" if peaks else "fallback", "kernel": kernel,
            "algorithmic_bytes_per_launch": alg / steps, "kernel_share_of_step": solve_ms / step_ms,
            "cg_iterations_per_launch": iters / steps,
            "note": "achieved = algorithmic PCG bytes / PCG launch time (CUDA events on the launching stream); "
                    "traffic (ncu DRAM bytes) is not measured in this run"}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id=None):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        cmd = ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200"]
        if bus_id:
            cmd += ["-i", bus_id]
        try:
            self.p = subprocess.Popen(cmd, stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [l.split(", ") for l in open(self.f.name).read().splitlines() if l.strip()]
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if len(r) > 5 + k and r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def read_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


def reference_leg(n, warmup, steps):
    """The FP64 oracle (single thread, the reference's CPU step restated) over
    exactly the timed window: the untimed steps up to the window, then the K
    window steps timed. The scene comes from the oracle's scene builder."""
    O = oracle_mod()
    from garmentcraft_b200 import _abi
    s = make_scene_oracle(n)
    sim = O.OracleSim(s, params(_abi.K3D_FP64).to_c())
    pre, wu = window(warmup)
    sim.frames(pre + wu)
    its, t0 = 0, time.perf_counter()
    for _ in range(steps):
        its += sim.frames(1).cg_iterationen
    el = time.perf_counter() - t0
    out = {"value": s.n * steps / el, "unit": UNIT, "cores": 1, "kind": "port",
           "sample": f"all {steps} timed steps (steps {pre + wu}-{pre + wu + steps - 1}) of the {n}x{n} drop, "
                     f"{el:.1f} s, FP64 C++ restatement of CpuLoeser/ImplizitCg, one thread",
           "cg_iterations_per_step": its / steps}
    out["mesh"] = cpu_mesh_leg(O)
    return s, out


def cpu_sample(n, warmup, steps, seconds, torch):
    """cpu_baseline of the device arm: the oracle on steps spread over the
    timed window. The FP64 device form runs the window; before each sampled
    step its state (x, v and the CG warm start) goes to the oracle, which
    takes that one step, timed. Reported beside the device FP64 form's
    iterations on the same steps."""
    O = oracle_mod()
    from garmentcraft_b200 import _abi
    from garmentcraft_b200.implizit import ImplizitCg
    s = make_scene(n)
    so = make_scene_oracle(n)
    cg = ImplizitCg(params(_abi.K3D_FP64), device=torch.cuda.current_device())
    cg.zustand_hochladen(s)
    pre, wu = window(warmup)
    cg.bilder_auf_geraet(pre + wu)
    picks = sorted({int(round(q * (steps - 1) / 3.0)) for q in range(4)})
    sim = O.OracleSim(so, params(_abi.K3D_FP64).to_c())
    cpu_s, cpu_its, dev_its, done = 0.0, 0, 0, []
    for k in range(steps):
        if k in picks and cpu_s < seconds:
            cg.zustand_lesen(s)
            sim.set_state(s.x, s.v)
            sim.set_dv_warm(cg.warmstart_lesen())
            t0 = time.perf_counter()
            cpu_its += sim.frames(1).cg_iterationen
            cpu_s += time.perf_counter() - t0
            dev_its += cg.bilder_auf_geraet(1).cg_iterationen
            done.append(k)
        else:
            cg.bilder_auf_geraet(1)
    start = pre + wu
    out = {"value": s.n * len(done) / cpu_s, "unit": UNIT, "cores": 1, "kind": "port",
           "sample": f"steps {[start + k for k in done]} of the timed window ({start}-{start + steps - 1}) of the "
                     f"same {n}x{n} drop, each from the FP64 device state at that step (x, v, CG warm start), "
                     f"{cpu_s:.1f} s, FP64 C++ restatement of CpuLoeser/ImplizitCg, one thread",
           "cg_iterations_per_step": cpu_its / len(done),
           "device_fp64_cg_iterations_per_step_same_states": dev_its / len(done)}
    out["mesh"] = cpu_mesh_leg(O)
    return out


def cpu_mesh_leg(oracle_py):
    """The restated Koerpernetz queries (grid query within the search depth,
    segment test; one thread) on 20k of the mesh leg's 200k points."""
    import numpy as np
    from garmentcraft_b200 import synth
    p, d = synth.koerper_netz()
    k = oracle_py.Koerpernetz(p, d, 0.01)
    rng = np.random.default_rng(0)
    q = 200_000
    x = p[rng.integers(0, p.shape[0], q)] + rng.normal(0.0, 0.01, (q, 3))
    y = x + rng.normal(0.0, 0.01, (q, 3))
    m = 20_000
    t0 = time.perf_counter()
    k.naechster(x[:m], 0.01)
    t1 = time.perf_counter()
    k.durchstoss(x[:m], y[:m])
    t2 = time.perf_counter()
    return {"nearest": {"value": m / (t1 - t0), "unit": "queries/s"},
            "penetration": {"value": m / (t2 - t1), "unit": "segments/s"}, "cores": 1, "kind": "port",
            "sample": f"the first {m} of the mesh leg's 200k points, the same body mesh"}


def dev_timed(n, prec, warmup, steps, flush, torch):
    """Device-resident steps: returns (ms list, stats sum, launches, scene, cg)."""
    from garmentcraft_b200.implizit import ImplizitCg
    s = make_scene(n)
    cg = ImplizitCg(params(prec), device=torch.cuda.current_device())
    cg.zustand_hochladen(s)
    pre, wu = window(warmup)
    cg.bilder_auf_geraet(pre + wu)
    torch.cuda.synchronize()
    ms, its, solves, solve_ms = [], 0, 0, 0.0
    l0 = cg.kernel_starts()
    for k in range(steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        st = cg.bilder_auf_geraet(1)
        ms.append(cg.letzte_bild_ms())
        solve_ms += cg.letzte_loesung_ms()
        its += st.cg_iterationen
        solves += st.loesungen
    launches = cg.kernel_starts() - l0
    cg.zustand_lesen(s)
    cg.solve_ms_total = solve_ms
    return ms, its, solves, launches, s, cg


def e2e_timed(n, prec, warmup, steps, flush, torch):
    from garmentcraft_b200.implizit import ImplizitCg
    s = make_scene(n, pinned=True)
    cg = ImplizitCg(params(prec), device=torch.cuda.current_device())
    pre, wu = window(warmup)
    cg.bilder_resident(s, pre)
    for _ in range(wu):
        cg.bild(s)
    torch.cuda.synchronize()
    tot = 0.0
    for k in range(steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cg.bild(s)  # H2D x,v (pinned) -> step -> D2H x,v, synchronised
        tot += time.perf_counter() - t0
    return tot, s


def main():
    import numpy as np
    a = args_()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if a.capture:
        # a fixed case for ncu: no timing, no flush
        from garmentcraft_b200 import _abi
        from garmentcraft_b200.implizit import ImplizitCg
        prec = {"mixed": _abi.K3D_MIXED, "fp64": _abi.K3D_FP64, "storage": _abi.K3D_MIXED_STORAGE}[a.precision]
        if a.workload == "adjoint":
            from garmentcraft_b200 import synth
            from garmentcraft_b200.adjoint import Drapierung, Stoff
            from garmentcraft_b200.params import ImplizitParameter
            s, hid, start = synth.materialfit(n=ADJ_N)
            par = ImplizitParameter(schritte_je_bild=1, cg_max=CG_MAX, cg_toleranz=1e-5, precision=_abi.K3D_FP64)
            d = Drapierung(s, Stoff.von(hid), frames=a.capture, k=ADJ_K, param=par)
            x, _ = d.vorwaerts(start)
            g = d.rueckwaerts(2.0 * x)["roh"]
            print(json.dumps({"capture_frames": a.capture, "forward_ms": g["ms_vorwaerts"],
                              "backward_ms": g["ms_rueckwaerts"], "adjoint_cg_iterations": g["iterationen"]}))
            return
        if a.workload == "mesh":
            from garmentcraft_b200 import synth
            from garmentcraft_b200.netzkoerper import Koerpernetz
            p, d = synth.koerper_netz()
            k = Koerpernetz(p, d, 0.01)
            ms = {"create": k.letzte_ms}
            for r in range(a.capture):
                for band in (0.03, 0.06):
                    k.sdf_body(0.005, band)
                    ms[f"sdf_{band}"] = k.letzte_ms
            print(json.dumps({"capture_rounds": a.capture, "ms_device": ms}))
            return
        if a.workload == "garment":
            from garmentcraft_b200 import synth
            from garmentcraft_b200.params import ImplizitParameter
            s, _ = synth.garment_szene(ziel_punkte=a.garment_points)
            cg = ImplizitCg(ImplizitParameter(schritte_je_bild=1, cg_max=CG_MAX, cg_toleranz=1e-5, precision=prec,
                                              selbstkollision=True))
            cg.zustand_hochladen(s)
            cg.bilder_auf_geraet(a.capture - 1)
            st = cg.bilder_auf_geraet(1)
            print(json.dumps({"capture_frames": a.capture, "last_frame_cg_iterations": st.cg_iterationen,
                              "last_frame_ms": cg.letzte_bild_ms(), "last_frame_solve_ms": cg.letzte_loesung_ms(),
                              "proximity_pairs": st.naehe_punkt_dreieck + st.naehe_kante_kante,
                              "intersections": st.durchdringungen, "impacts": st.selbst_stoesse}))
            return
        s = make_scene(a.n)
        cg = ImplizitCg(params(prec))
        cg.zustand_hochladen(s)
        st = cg.bilder_auf_geraet(a.capture - 1)
        st = cg.bilder_auf_geraet(1)
        print(json.dumps({"capture_steps": a.capture, "last_step_cg_iterations": st.cg_iterationen,
                          "last_step_ms": cg.letzte_bild_ms()}))
        return

    if a.impl == "reference":
        if rank != 0:
            return
        s, cpu = reference_leg(a.n, a.warmup, a.steps)
        line = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": a.gpus,
                "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": workload_config(a.n, s, {"precision": "fp64 (CPU)",
                                                   "l2": "not applicable: one host thread, no device"}),
                "cpu_baseline": cpu,
                "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import numpy as np_
    globals()["np"] = np_
    import torch
    import torch.distributed as dist
    from garmentcraft_b200 import _abi

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    bus = None
    try:
        pr = torch.cuda.get_device_properties(local)
        bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
    except Exception:
        pass

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(bus)
    ms, its, solves, launches, s_h, cg = dev_timed(a.n, HEADLINE, a.warmup, a.steps, flush, torch)
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_dev = sum(ms) / 1e3
    if world > 1:
        t = torch.tensor([t_dev], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_dev = float(t.item())
    nv = s_h.n
    value = world * nv * a.steps / t_dev

    # the same steps through the public API with host buffers
    t_e2e, _ = e2e_timed(a.n, HEADLINE, a.warmup, a.steps, flush, torch)
    if world > 1:
        t = torch.tensor([t_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())
    e2e = {"value": world * nv * a.steps / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 48 * nv,
           "d2h_bytes_per_step": 48 * nv + 144}

    extra = {}
    if not a.no_compare:
        from garmentcraft_b200.implizit import ImplizitCg
        t_form = {HEADLINE: t_dev}
        for prec in (0, 1):
            msf, itsf, solvesf, _, _, cgf = dev_timed(a.n, prec, a.warmup, a.steps, flush, torch)
            t_form[prec] = sum(msf) / 1e3
            extra[FORMS[prec][0]] = {"value": nv * a.steps / t_form[prec], "ms_per_step": 1e3 * t_form[prec] / a.steps,
                                     "cg_iterations_per_step": itsf / a.steps,
                                     "pcg_us_per_iteration": 1e3 * cgf.solve_ms_total / max(itsf, 1)}
            del cgf
        # one step of each form from the FP64 state at steps of the window, and 100 steps of the drop
        pre, wu = window(a.warmup)
        s0 = make_scene(a.n)
        c64 = ImplizitCg(params(0))
        c64.zustand_hochladen(s0)
        c64.bilder_auf_geraet(pre + wu)
        one = {FORMS[p][0]: [] for p in (HEADLINE, 1)}
        at = []
        for k in range(0, a.steps, max(1, a.steps // 4)):
            st0 = s0.copy()
            c64.zustand_lesen(st0)
            ref = st0.copy()
            cr = ImplizitCg(params(0))
            cr.zustand_hochladen(ref)
            cr.bilder_auf_geraet(1)
            cr.zustand_lesen(ref)
            del cr
            c64.bilder_auf_geraet(1)
            d = float(np.linalg.norm(ref.x.max(0) - ref.x.min(0)))
            for prec in (HEADLINE, 1):
                t = st0.copy()
                cf = ImplizitCg(params(prec))
                cf.zustand_hochladen(t)
                cf.bilder_auf_geraet(1)
                cf.zustand_lesen(t)
                dx = np.linalg.norm(t.x - ref.x, axis=1)
                one[FORMS[prec][0]].append({"max": float(dx.max() / d), "rms": float(np.sqrt(np.mean(dx ** 2)) / d)})
                del cf
            at.append(pre + wu + k)
            c64.bilder_auf_geraet(max(1, a.steps // 4) - 1)
        del c64
        sa = make_scene(a.n)
        ImplizitCg(params(0)).bilder_resident(sa, 100)
        err100 = {}
        for prec in (HEADLINE, 1):
            sb = make_scene(a.n)
            ImplizitCg(params(prec)).bilder_resident(sb, 100)
            d = float(np.linalg.norm(sa.x.max(0) - sa.x.min(0)))
            err100[FORMS[prec][0]] = float(np.max(np.linalg.norm(sa.x - sb.x, axis=1)) / d)
        try:
            free = no_contact_leg(a.n)
        except Exception as e:  # a figure beside the headline: its failure must not take the line with it
            free = {"error": f"{type(e).__name__}: {e}"}
        extra["mixed_vs_fp64"] = {
            "speedup": {FORMS[p][0]: t_form[0] / t_form[p] for p in (HEADLINE, 1)} if world == 1 else None,
            "one_step_error": {"at_steps": at, "errors": one,
                               "definition": "|x_form - x_fp64| / bbox diagonal after one step from the same FP64 "
                                             "state, every form on a new solver (no warm start)"},
            "rel_pos_err_after_100_steps": err100,
            "rel_pos_err_after_100_steps_no_contact": free,
            "definition": "max_i |x_form - x_fp64| / bbox diagonal"}

    peaks = read_peaks()
    roofline = roofline_of(s_h, HEADLINE, its, solves, cg.solve_ms_total, sum(ms), a.steps, peaks,
                           "k3d::solve_kernel<float, double, false>")

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * t_dev / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": workload_config(a.n, s_h, {"precision": "mixed storage (FP32 operator blocks and "
                                                              "preconditioner, FP64 CG vectors, sums and state)"}),
            "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline,
            "cg_iterations_per_step": its / a.steps,
            "pcg_us_per_iteration": 1e3 * cg.solve_ms_total / max(its, 1), "clocks": clk}
    line.update(extra)
    if world == 1 and not a.no_batch:
        line["batched"] = batch_leg(a.batch_steps, flush, torch)
    if world == 1 and not a.no_shapes:
        line["launch_shapes"] = shapes_leg()
    if world == 1 and not a.no_adjoint:
        line["adjoint"] = adjoint_leg(torch)
    if world == 1 and not a.no_garment:
        line["garment"] = garment_leg(flush, torch, peaks, cpu=not a.no_cpu)
    if world == 1 and not a.no_mesh:
        line["mesh"] = mesh_leg(flush, torch)
    if rank == 0 and world == 1 and not a.no_cpu:
        line["cpu_baseline"] = cpu_sample(a.n, a.warmup, a.steps, a.cpu_seconds, torch)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
