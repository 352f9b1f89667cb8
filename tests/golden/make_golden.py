"""Writes tests/golden/oracle_frames.npz: the FP64 oracle (oracle/, the
reference's CPU step restated) on small seeded scenes, frame by frame.

  tube   the closed tube over its cylinder (sim/src/roehre.rs:197-239 built
         without the mesher), 10 frames, PCG tolerance 1e-6, cap 2000;
  sheet  a 33 x 33 sheet (seed 3) dropped 2 cm onto the sphere grid,
         15 frames solved to 1e-12 (cap 20000): it lands within them, so
         contacts, the release test and friction all enter.

Per case: the final positions and velocities, and per frame the contact
count and CG iterations. Each scene is built by the oracle's own scene
builder. Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import oracle_py as O  # noqa: E402
from garmentcraft_b200 import synth  # noqa: E402
from garmentcraft_b200.params import ImplizitParameter  # noqa: E402

PATH = os.path.join(HERE, "oracle_frames.npz")

CASES = {
    "tube": dict(frames=10, cg_max=2000, tol=1e-6),
    "sheet": dict(frames=15, cg_max=20000, tol=1e-12),
}


def muster(name):
    """The pattern and body of a case, as the device tests build them."""
    if name == "tube":
        return synth.tube()
    return synth.sheet_over_sphere(n=33, seed=3, fall_m=0.02)


def params(name):
    c = CASES[name]
    return ImplizitParameter(schritte_je_bild=1, cg_max=c["cg_max"], cg_toleranz=c["tol"])


def run(name):
    m, body = muster(name)
    s = O.build_scene(m, [body])
    sim = O.OracleSim(s, params(name).to_c())
    kontakte, its = [], []
    for _ in range(CASES[name]["frames"]):
        st = sim.frames(1)
        kontakte.append(st.kontakte)
        its.append(st.cg_iterationen)
    x, v = sim.state()
    return {f"{name}_x": x, f"{name}_v": v, f"{name}_kontakte": np.array(kontakte, dtype=np.int64),
            f"{name}_iterationen": np.array(its, dtype=np.int64)}


def main():
    out = {}
    for name in CASES:
        out.update(run(name))
    np.savez_compressed(PATH, **out)
    print(PATH, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
