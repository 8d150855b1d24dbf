"""The engine's adjoint gradient against the reference's own adjoint.

tests/golden/adjoint.npz holds dL/d eps (absolute permittivity, the E
components over the design boxes) of a small CPML scene with Drude, Lorentz
and Debye media, produced by the reference's frozen Torch reverse ops driven
in its native runner's order in float64 (make_adjoint_golden.py).  L is
sum |X|^2 over the six components of a point probe's 300 THz spectrum.

- CPU: the golden gradient, pulled back to the design cells, against central
  finite differences of the FP64 oracle (h = 1e-3 on eps_r of 8 seeded
  design cells).  The compiled coefficients are FP32, so a difference of
  1e-3 resolves the derivative to about 1e-4; tolerance 1e-3 relative.
- GPU: the engine's adjoint (FP32), stored-history and checkpoint-replay
  modes, against the golden gradient: relative L2 <= 1e-4 over each E
  component's design box and over the pulled-back design gradient (the
  north star's "within 1e-4 of the reference").
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import load_package
from oracle import oracle as orc

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))

import make_adjoint_golden as mag  # noqa: E402

GOLDEN = np.load(HERE / "golden" / "adjoint.npz")
COMPS = ("Ex", "Ey", "Ez")
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _rel(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _golden_design_gradient(wm, cs):
    boxes = [tuple(int(v) for v in GOLDEN[f"box_{c}"]) for c in COMPS]
    return wm.adjoint.pullback(cs.design, boxes, [GOLDEN[f"grad_{c}"] for c in COMPS])


def test_golden_scene_inputs_unchanged():
    wm = load_package()
    cs = wm.compile_scene(mag.adjoint_scene(), mag.ADJ_STEPS)
    assert float(np.abs(cs.curl["Ex"]).sum()) == pytest.approx(float(GOLDEN["check_curl_Ex"]), rel=1e-12)
    np.testing.assert_allclose([float(np.abs(p.drive).sum()) for p in cs.poles], GOLDEN["check_poles"], rtol=1e-12)
    np.testing.assert_allclose([float(np.abs(p.coeff).sum()) for p in cs.patches], GOLDEN["check_patch"], rtol=1e-12)
    np.testing.assert_array_equal(cs.design.eps_r, GOLDEN["eps_r"])
    assert {p.kind for p in cs.poles} == {0, 1, 2}
    boxes = wm.adjoint.design_boxes(cs.design, cs.nodes)
    for c, box in zip(COMPS, boxes):
        assert tuple(box) == tuple(int(v) for v in GOLDEN[f"box_{c}"])


def _oracle_loss(wm, eps_r) -> float:
    cs = wm.compile_scene(mag.adjoint_scene(eps_r), mag.ADJ_STEPS)
    sim = orc.OracleSimulation(cs, "f64").run(mag.ADJ_STEPS)
    mons = sim.monitor_results()
    sim.close()
    return float(sum(np.sum(np.abs(v) ** 2) for v in mons["probe"].values()))


def test_oracle_loss_matches_golden_and_fd_matches_golden_gradient():
    wm = load_package()
    eps_r = np.asarray(GOLDEN["eps_r"], dtype=np.float64)
    assert _oracle_loss(wm, eps_r) == pytest.approx(float(GOLDEN["loss"]), rel=1e-10)
    cs = wm.compile_scene(mag.adjoint_scene(eps_r), mag.ADJ_STEPS)
    g = _golden_design_gradient(wm, cs)
    assert np.abs(g).max() > 0
    rng = np.random.default_rng(11)
    picks = rng.choice(eps_r.size, size=8, replace=False)
    h = 1e-3
    for flat in picks:
        idx = np.unravel_index(flat, eps_r.shape)
        vals = []
        for sgn in (1.0, -1.0):
            e = eps_r.copy()
            e[idx] += sgn * h
            vals.append(_oracle_loss(wm, e))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(g[idx] - fd) <= 1e-3 * np.abs(g).max(), (idx, g[idx], fd)


@pytest.mark.gpu
@pytest.mark.parametrize("history", ["store", "replay"])
def test_engine_adjoint_matches_reference_adjoint(history):
    import torch

    wm = load_package()
    lib = wm._lib.load()
    eps_r = np.asarray(GOLDEN["eps_r"], dtype=np.float64)
    problem = wm.adjoint.DesignProblem(mag.adjoint_scene(eps_r), mag.ADJ_STEPS, stride=16, history=history)
    mons = problem.forward(eps_r)
    for c in FIELDS:
        x = complex(mons["probe"][c].cpu().numpy().ravel()[0])
        want = complex(GOLDEN[f"X_{c}"])
        assert abs(x - want) <= 1e-5 * max(abs(complex(GOLDEN[f"X_{k}"])) for k in FIELDS), c
    g = problem.backward({"probe": {c: 2.0 * v for c, v in mons["probe"].items()}})
    solver = problem.solver
    for comp, name in enumerate(COMPS):
        box = problem.boxes[comp]
        out = torch.empty((box[1] - box[0], box[3] - box[2], box[5] - box[4]), device=solver.device)
        wm._lib.check(lib.fdtd_engine_adjoint_grad(solver.handle, comp, wm._lib.ptr(out)), "adjoint_grad")
        assert _rel(out.cpu().numpy(), GOLDEN[f"grad_{name}"]) <= 1e-4, name
    want = _golden_design_gradient(wm, solver.compiled)
    assert _rel(g, want) <= 1e-4
    problem.close()
