"""Host helpers of bench.py (CPU): the near-field pair count from the
occupancy map, which the roofline divides by the stage time."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, ROOT)


@pytest.mark.parametrize("X,Y,Z,s", [(16, 16, 3, 8), (20, 13, 2, 4), (9, 7, 1, 2)])
def test_near_pairs_counts_charged_sources_in_the_box_neighbourhood(X, Y, Z, s):
    import bench
    rng = np.random.default_rng(X * Y + s)
    rho = rng.standard_normal((Z, Y, X)) * (rng.random((Z, Y, X)) < 0.4)
    brute = 0
    for z in range(Z):
        for y in range(Y):
            for x in range(X):
                bx, by = x // s, y // s
                for zs in range(Z):
                    for ys in range(max(0, (by - 1) * s), min(Y, (by + 2) * s)):
                        for xs in range(max(0, (bx - 1) * s), min(X, (bx + 2) * s)):
                            brute += rho[zs, ys, xs] != 0
    assert bench.near_pairs_occupied(rho.ravel(), X, Y, Z, s) == brute


def test_near_pairs_with_every_cell_charged_is_the_plan_count():
    import bench
    # every cell charged: the count of all pairs, as mms_fmm_info reports it
    X = Y = 64
    Z, s = 3, 8
    nb = X // s
    want = 0
    for by in range(nb):
        for bx in range(nb):
            sx = min(X, (bx + 2) * s) - max(0, (bx - 1) * s)
            sy = min(Y, (by + 2) * s) - max(0, (by - 1) * s)
            want += s * s * Z * sx * sy * Z
    assert bench.near_pairs_occupied(np.ones(Z * Y * X), X, Y, Z, s) == want
