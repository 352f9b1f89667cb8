"""The oracle against its committed golden frames (tests/golden/, written by
tests/golden/make_golden.py): the tube and the 33 x 33 sheet landing on the
sphere, frame by frame. A change in the oracle's arithmetic, its scene
builder or its loop order shows here first; the device is held to the same
vectors in tests/test_gpu_golden.py."""
import os
import sys

import numpy as np
import pytest

import oracle_py as O

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as G  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "oracle_frames.npz"))


def diag(x):
    return float(np.linalg.norm(x.max(0) - x.min(0)))


@pytest.mark.parametrize("name", list(G.CASES))
def test_oracle_reproduces_golden_frames(name):
    r = G.run(name)
    x = GOLD[f"{name}_x"]
    assert np.array_equal(r[f"{name}_kontakte"], GOLD[f"{name}_kontakte"])
    assert np.max(np.abs(r[f"{name}_iterationen"] - GOLD[f"{name}_iterationen"])) <= 1
    assert np.max(np.abs(r[f"{name}_x"] - x)) <= 1e-12 * diag(x)
    assert np.max(np.abs(r[f"{name}_v"] - GOLD[f"{name}_v"])) <= 1e-9 * max(1.0, np.abs(GOLD[f"{name}_v"]).max())


def test_golden_frames_are_what_they_claim():
    # the tube holds its cylinder, the sheet lands within its frames
    assert GOLD["tube_kontakte"][-1] > 0
    assert GOLD["sheet_kontakte"][0] == 0 and GOLD["sheet_kontakte"][-1] > 0
    assert np.all(np.isfinite(GOLD["sheet_x"])) and np.all(np.isfinite(GOLD["tube_x"]))
