"""The bench's roofline numerator: the algorithmic bytes per CG iteration
that bench.algorithmic_solve_bytes counts on the 257 x 257 sheet, against the
per-unit figures (per point 10 s_vec for the operator's vectors and
25 s_vec + 6 s_op for the update, per membrane 12 + 21 s_op, per hinge
16 + 13 s_op): about 560 B per point and iteration with FP32 operator and
vectors, 700 B for FP32 operator values with FP64 vectors, 1,048 B in FP64
for a regular grid (two membranes and three hinges per point)."""
import pytest

import bench


@pytest.fixture(scope="module")
def sheet():
    return bench.make_scene(257)


@pytest.mark.parametrize("prec,per_point", [(1, 560.0), (2, 700.0), (0, 1048.0)])
def test_bytes_per_point_and_iteration(sheet, prec, per_point):
    _, s_op, s_vec = bench.FORMS[prec]
    N, T, B, S = bench.element_counts(sheet)
    assert (N, T, B, S) == (257 * 257, 2 * 256 * 256, 196096, 0)
    one = bench.algorithmic_solve_bytes(sheet, s_op, s_vec, 1, 0)
    # the grid's border has fewer elements per point than T = 2N, B = 3N
    assert one / N == pytest.approx(per_point, rel=0.01)
    # a solve adds two operator applications (start residual, release test)
    two = bench.algorithmic_solve_bytes(sheet, s_op, s_vec, 1, 1)
    per_app = N * 10 * s_vec + T * (12 + 21 * s_op) + B * (16 + 13 * s_op)
    assert two - one == 2 * per_app


def test_roofline_arithmetic(sheet):
    peaks = {"hbm_gbs": 6505.3}
    its, solves, steps = 786 * 20, 20, 20
    r = bench.roofline_of(sheet, 2, its, solves, 188.7, 191.3, steps, peaks, "k")
    alg = bench.algorithmic_solve_bytes(sheet, 4, 8, its, solves)
    assert r["achieved"] == pytest.approx(alg / 0.1887 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / 6505.3)
    assert r["peak_source"] == "measured" and r["traffic"] is None
    assert r["algorithmic_bytes_per_launch"] == pytest.approx(alg / steps)
    assert bench.roofline_of(sheet, 2, its, solves, 188.7, 191.3, steps, None, "k")["peak"] == 6650.0
