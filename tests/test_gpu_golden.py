"""The device step against the oracle's committed golden frames
(tests/golden/oracle_frames.npz): the same scenes and parameters as
tests/golden/make_golden.py, built by the library, stepped frame by frame in
FP64 through the C ABI. Per frame the contact count equals the oracle's; the
final positions agree to 1e-9 of the bounding-box diagonal (the device sums
in another order than the oracle), as in the live comparisons of
tests/test_gpu_parity.py."""
import os
import sys

import numpy as np
import pytest

from garmentcraft_b200.implizit import ImplizitCg, build_scene

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(HERE, "golden", "oracle_frames.npz"))


@pytest.mark.parametrize("name", list(G.CASES))
def test_frames_wie_golden(name):
    m, body = G.muster(name)
    s = build_scene(m, [body])
    cg = ImplizitCg(G.params(name))
    kontakte = []
    for _ in range(G.CASES[name]["frames"]):
        cg.bild(s)
        kontakte.append(cg.statistik.kontakte)
    x = GOLD[f"{name}_x"]
    assert np.array_equal(np.array(kontakte), GOLD[f"{name}_kontakte"])
    assert np.max(np.abs(s.x - x)) <= 1e-9 * float(np.linalg.norm(x.max(0) - x.min(0)))
