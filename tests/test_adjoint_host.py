"""Host side of the adjoint: design boxes and the eps pullback (no GPU).

The scene compiler sets every design node to the cell's eps_r and averages
node permittivities onto the Yee components (eps = eps0 (n_a + n_b) / 2), so
dL/deps_r of a node is eps0 / 2 times the sum of dL/deps over the component
cells that average it; checked against a brute-force loop.
"""
from __future__ import annotations

import importlib

import numpy as np

from conftest import load_package


def test_design_boxes_cover_every_dependent_component_cell():
    wm = load_package()
    adj = importlib.import_module("witwin_maxwell_b200.adjoint")
    reg = wm.MaterialRegion((5, 6, 7), (9, 10, 9), np.ones((4, 4, 2)))
    boxes = adj.design_boxes(reg, (20, 20, 20))
    assert boxes == [(4, 9, 6, 10, 7, 9), (5, 9, 5, 10, 7, 9), (5, 9, 6, 10, 6, 9)]


def test_pullback_matches_brute_force():
    wm = load_package()
    adj = importlib.import_module("witwin_maxwell_b200.adjoint")
    reg = wm.MaterialRegion((5, 6, 7), (9, 10, 9), np.ones((4, 4, 2)))
    boxes = adj.design_boxes(reg, (20, 20, 20))
    rng = np.random.default_rng(0)
    grads = [rng.standard_normal((b[1] - b[0], b[3] - b[2], b[5] - b[4])) for b in boxes]
    got = adj.pullback(reg, boxes, grads)
    want = np.zeros((4, 4, 2))
    eps0 = wm.scene.EPSILON_0
    for c, (b, g) in enumerate(zip(boxes, grads)):
        for i in range(b[0], b[1]):
            for j in range(b[2], b[3]):
                for k in range(b[4], b[5]):
                    for s in (0, 1):
                        node = [i, j, k]
                        node[c] += s
                        if all(reg.lo[a] <= node[a] < reg.hi[a] for a in range(3)):
                            want[tuple(node[a] - reg.lo[a] for a in range(3))] += 0.5 * eps0 * g[i - b[0], j - b[2], k - b[4]]
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-30)
