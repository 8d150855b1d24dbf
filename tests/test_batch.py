"""Batched scenes (fdtd_batch_*): independent engines stepped together through
graph-captured step blocks give exactly the fields and monitor spectra of the
same engines stepped one by one (same kernels, same per-scene order)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _scenes(wm):
    return wm.workloads.batched_designs(n_scenes=4, seed=3, size_range=(24, 40), pml=4, n_freq=3)


def _state(solver):
    fields = {n: solver.field(n).cpu().numpy() for n in FIELDS}
    mons = {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in solver.monitor_results().items()}
    return fields, mons


def test_batch_equals_individual_runs():
    wm = load_package()
    steps = 70  # two graph blocks of 32 steps and a 6-step tail
    compiled = [wm.compile_scene(sc, steps) for sc in _scenes(wm)]
    ref = []
    for cs in compiled:
        s = wm.solver.B200FDTD(cs).init_field()
        # same call split as the batch below, so the monitor samples are
        # flushed into the DFT sums in the same groups
        s.step_range(0, 40)
        s.step_range(40, steps)
        ref.append(_state(s))
        s.close()
    solvers = [wm.solver.B200FDTD(cs).init_field() for cs in compiled]
    batch = wm.solver.B200Batch(solvers)
    batch.step_range(0, 40)
    batch.step_range(40, steps)
    info = batch.info()
    assert info["scenes"] == 4 and info["block_steps"] == 32 and info["graph_launches"] == 1
    for s, (rf, rm) in zip(solvers, ref):
        f, m = _state(s)
        for n in FIELDS:
            np.testing.assert_array_equal(f[n], rf[n])
        for mon, comps in rm.items():
            for c, v in comps.items():
                np.testing.assert_array_equal(m[mon][c], v)
    batch.close()
    for s in solvers:
        s.close()


def test_batch_autotune_keeps_results():
    wm = load_package()
    steps = 64
    compiled = [wm.compile_scene(sc, steps) for sc in _scenes(wm)[:2]]
    ref = []
    for cs in compiled:
        s = wm.solver.B200FDTD(cs).init_field()
        s.step_range(0, steps)
        ref.append(_state(s)[1])
        s.close()
    solvers = [wm.solver.B200FDTD(cs).init_field() for cs in compiled]
    batch = wm.solver.B200Batch(solvers)
    batch.autotune()  # picks launch shapes; the state is restored
    batch.step_range(0, steps)
    for s, rm in zip(solvers, ref):
        m = _state(s)[1]
        for mon, comps in rm.items():
            for c, v in comps.items():
                # another launch variant may contract a different multiply-add pair
                assert np.linalg.norm(m[mon][c] - v) <= 1e-5 * max(np.linalg.norm(v), 1e-30)
    batch.close()
    for s in solvers:
        s.close()


def test_batch_rejects_mismatched_sample_blocks():
    wm = load_package()
    compiled = [wm.compile_scene(sc, 10) for sc in _scenes(wm)[:2]]
    a = wm.solver.B200FDTD(compiled[0]).init_field()
    b = wm.solver.B200FDTD(compiled[1], sample_block=16).init_field()
    with pytest.raises(wm._lib.FdtdError):
        wm.solver.B200Batch([a, b])
    a.close()
    b.close()


def test_batch_adjoint_equals_individual_problems():
    """Per-scene adjoint gradients of a batched forward run (checkpoints every 40
    steps, graph-captured batch steps) equal one DesignProblem per scene."""
    wm = load_package()
    adj = wm.adjoint
    steps, stride = 120, 40
    scenes = wm.workloads.batched_designs(n_scenes=3, seed=5, size_range=(36, 44), pml=4, n_freq=3, design=True)
    eps = [sc.material_regions[0].eps_r for sc in scenes]

    def seeds(mons):
        return {"probe": {c: 2.0 * v for c, v in mons["probe"].items()}}

    ref = []
    for sc, e in zip(scenes, eps):
        p = adj.DesignProblem(sc, steps, stride=stride, history="replay")
        ref.append((p.forward(e), None))
        ref[-1] = (ref[-1][0], p.backward(seeds(ref[-1][0])))
        p.close()
    batch = adj.BatchDesignProblem(scenes, steps, stride=stride)
    mons = batch.forward(eps)
    grads = batch.backward([seeds(m) for m in mons])
    assert set(batch.timings) == {"forward_ms", "backward_ms"}
    for (rm, rg), m, g in zip(ref, mons, grads):
        for c, v in rm["probe"].items():
            np.testing.assert_allclose(m["probe"][c].cpu().numpy(), v.cpu().numpy(), rtol=1e-6, atol=0)
        assert np.abs(rg).max() > 0
        np.testing.assert_allclose(g, rg, rtol=1e-5, atol=1e-6 * np.abs(rg).max())
    batch.close()
