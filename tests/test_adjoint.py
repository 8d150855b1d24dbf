"""Reverse-time adjoint (GPU): exact transpose of the fused step and
permittivity gradients against central finite differences.

- Dot-product test: for random states x (E, H, CPML psi) and y (their
  adjoints), <F x, y> = <x, F^T y> where F is one source-free forward step and
  F^T one adjoint step; relative tolerance 1e-5 (FP32 sums of ~1e5 terms).
- dL/deps_r of a design region for L = sum |X|^2 over a point monitor's
  spectrum, against central differences (h = 1e-2 on eps_r, FP32 fields);
  relative tolerance 1e-2 per checked cell, and the adjoint must be the same
  through torch.autograd.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import load_package
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _psi_shapes(cs):
    shapes = {}
    axes = {0: (1, 2), 1: (0, 2), 2: (0, 1)}
    for comp, name in enumerate(FIELDS):
        c = comp % 3
        nx, ny, nz = cs.nodes
        ext = {
            "Ex": (nx - 1, ny, nz), "Ey": (nx, ny - 1, nz), "Ez": (nx, ny, nz - 1),
            "Hx": (nx, ny - 1, nz - 1), "Hy": (nx - 1, ny, nz - 1), "Hz": (nx - 1, ny - 1, nz),
        }[name]
        for which, axis in enumerate(axes[c]):
            L = cs.pml_lo[axis] + cs.pml_hi[axis]
            if L == 0:
                continue
            shape = list(ext)
            shape[axis] = L
            shapes[(comp, which)] = tuple(shape)
    return shapes


def _scene(wm, boundary=None, dispersive=False):
    sc = wm.Scene(cells=(20, 18, 16), spacing=25e-9, pml_cells=4)
    if boundary is not None:
        sc.boundary = boundary
        sc.pml_cells = 0 if all(b != wm.BOUNDARY_PML for b in boundary) else 4
    sc.structures.append(wm.Structure(wm.Box((6, 5, 5), (12, 11, 10)), wm.Medium(eps_r=3.0)))
    if dispersive:
        # one medium of each ADE kind, the Drude slab reaching into the CPML
        sc.structures.append(wm.Structure(wm.Box((13, 2, 3), (15, 16, 13)), wm.Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))))
        sc.structures.append(wm.Structure(wm.Sphere((8, 8, 11), 2.5), wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
        sc.structures.append(wm.Structure(wm.Box((4, 12, 4), (7, 15, 8)), wm.Medium.debye(2.5, 3.5, 1e-14)))
    return sc


@pytest.mark.parametrize("kind", ["cpml", "pec", "mixed", "dispersive"])
def test_adjoint_step_is_the_exact_transpose(kind):
    """<F x, y> = <x, F^T y> over E, H, CPML psi and (dispersive) the ADE pole
    state: P of Debye and Lorentz poles, J of Drude and Lorentz poles (the J a
    Debye pole stores is an output of the step, not a state it reads)."""
    wm = load_package()
    lib = wm._lib.load()
    P, E, N = wm.BOUNDARY_PML, wm.BOUNDARY_PEC, wm.BOUNDARY_NONE
    boundary = {"cpml": None, "pec": (E,) * 6, "mixed": (P, E, N, P, P, E), "dispersive": None}[kind]
    cs = wm.compile_scene(_scene(wm, boundary, dispersive=kind == "dispersive"), 4)
    if kind == "dispersive":
        assert {p.kind for p in cs.poles} == {0, 1, 2}
    solver = wm.solver.B200FDTD(cs).init_field()
    h = solver.handle
    wm._lib.check(lib.fdtd_engine_adjoint_init(h, None, 1), "adjoint_init")
    rng = np.random.default_rng(7)
    dev = solver.device
    psi = _psi_shapes(cs)
    x, y = {}, {}
    for comp, name in enumerate(FIELDS):
        shape = tuple(solver.field(name).shape)
        x[("f", comp, 0)] = torch.tensor(rng.standard_normal(shape), dtype=torch.float32, device=dev)
        y[("f", comp, 0)] = torch.tensor(rng.standard_normal(shape), dtype=torch.float32, device=dev)
    for (comp, which), shape in psi.items():
        x[("p", comp, which)] = torch.tensor(rng.standard_normal(shape), dtype=torch.float32, device=dev)
        y[("p", comp, which)] = torch.tensor(rng.standard_normal(shape), dtype=torch.float32, device=dev)
    for pid, pole in enumerate(cs.poles):
        b = pole.box
        shape = (b[1] - b[0], b[3] - b[2], b[5] - b[4])
        for which in (0, 1):  # 0: P, 1: J
            x[("a", pid, which)] = torch.tensor(rng.standard_normal(shape), dtype=torch.float32, device=dev)
            state = (which == 0 and pole.kind in (0, 2)) or (which == 1 and pole.kind in (1, 2))
            yv = rng.standard_normal(shape) if state else np.zeros(shape)
            y[("a", pid, which)] = torch.tensor(yv, dtype=torch.float32, device=dev)
    kind_code = {"f": 0, "p": 1, "a": 2}
    # forward: F x
    for (kd, comp, which), t in x.items():
        if kd == "f":
            wm._lib.check(lib.fdtd_engine_pack_field(h, comp, wm._lib.ptr(t)), "pack")
        elif kd == "p":
            wm._lib.check(lib.fdtd_engine_pack_psi(h, comp, which, wm._lib.ptr(t)), "pack_psi")
        else:
            args = (wm._lib.ptr(t), None) if which == 0 else (None, wm._lib.ptr(t))
            wm._lib.check(lib.fdtd_engine_set_pole_state(h, solver.pole_ids[comp], *args), "set_pole_state")
    solver.step_range(0, 1)
    fx = {}
    for key, t in x.items():
        out = torch.empty_like(t)
        kd, comp, which = key
        if kd == "f":
            wm._lib.check(lib.fdtd_engine_unpack_field(h, comp, wm._lib.ptr(out)), "unpack")
        elif kd == "p":
            wm._lib.check(lib.fdtd_engine_unpack_psi(h, comp, which, wm._lib.ptr(out)), "unpack_psi")
        else:
            args = (wm._lib.ptr(out), None) if which == 0 else (None, wm._lib.ptr(out))
            wm._lib.check(lib.fdtd_engine_pole_state(h, solver.pole_ids[comp], *args), "pole_state")
        fx[key] = out
    # adjoint: F^T y
    for (kd, comp, which), t in y.items():
        wm._lib.check(lib.fdtd_engine_adjoint_pack(h, kind_code[kd], comp, which, wm._lib.ptr(t)), "adj_pack")
    wm._lib.check(lib.fdtd_engine_adjoint_range(h, 1, 0), "adjoint_range")
    fty = {}
    for key, t in y.items():
        out = torch.empty_like(t)
        kd, comp, which = key
        wm._lib.check(lib.fdtd_engine_adjoint_unpack(h, kind_code[kd], comp, which, wm._lib.ptr(out)), "adj_unpack")
        fty[key] = out
    torch.cuda.synchronize()
    lhs = sum(float((fx[k].double() * y[k].double()).sum()) for k in x)
    rhs = sum(float((x[k].double() * fty[k].double()).sum()) for k in x)
    scale = sum(float(fx[k].double().abs().mul(y[k].double().abs()).sum()) for k in x)
    solver.close()
    assert abs(lhs - rhs) <= 1e-5 * scale, (lhs, rhs, scale)


def _design_scene(wm, eps_r, dispersive=False):
    sc = wm.Scene(cells=(28, 24, 24), spacing=25e-9, pml_cells=5)
    if dispersive:
        # a Lorentz block between the design region and the probe, a Drude block behind the source
        sc.structures.append(wm.Structure(wm.Box((17, 9, 9), (19, 15, 15)), wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
        sc.structures.append(wm.Structure(wm.Box((6, 8, 8), (7, 16, 16)), wm.Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))))
    sc.sources.append(wm.PointDipole((9, 12, 12), "Ez", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    sc.material_regions.append(wm.MaterialRegion((12, 10, 10), (16, 14, 13), eps_r))
    sc.monitors.append(wm.PointMonitor("probe", (20, 12, 12), frequencies=(300e12,)))
    return sc


def _loss(mons):
    return sum(float(np.sum(np.abs(np.asarray(v.cpu().numpy())) ** 2)) for v in mons["probe"].values())


@pytest.mark.parametrize("dispersive", [False, True])
def test_design_gradient_matches_finite_differences(dispersive):
    wm = load_package()
    adj = wm.adjoint
    steps = 320
    rng = np.random.default_rng(3)
    eps_r = 2.0 + 2.0 * rng.random((4, 4, 3))
    problem = adj.DesignProblem(_design_scene(wm, eps_r, dispersive), steps, stride=64, history="replay")
    mons = problem.forward(eps_r)
    grad_out = {"probe": {c: 2.0 * v for c, v in mons["probe"].items()}}  # d sum|X|^2 / dX* convention
    g = problem.backward(grad_out)
    problem.close()
    assert np.isfinite(g).all() and np.abs(g).max() > 0
    order = np.argsort(-np.abs(g).ravel())[:4]
    h = 1e-2
    for flat in order:
        idx = np.unravel_index(flat, eps_r.shape)
        vals = []
        for sgn in (1.0, -1.0):
            e = eps_r.copy()
            e[idx] += sgn * h
            p = adj.DesignProblem(_design_scene(wm, e, dispersive), steps, stride=steps)
            vals.append(_loss(p.forward(e)))
            p.close()
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(g[idx] - fd) <= 1e-2 * abs(fd), (idx, g[idx], fd)


def test_design_gradient_through_autograd():
    """torch.autograd over the stored-history path equals the checkpoint-replay path."""
    wm = load_package()
    adj = wm.adjoint
    steps = 200
    eps_r = np.full((4, 4, 3), 3.0)
    problem = adj.DesignProblem(_design_scene(wm, eps_r), steps, history="store")
    t = torch.tensor(eps_r, dtype=torch.float32, requires_grad=True)
    mons = adj.design_monitors(t, problem, [("probe", c) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")])
    loss = sum((v.abs() ** 2).sum() for v in mons["probe"].values())
    loss.backward()
    direct = adj.DesignProblem(_design_scene(wm, eps_r), steps, stride=50, history="replay")
    m2 = direct.forward(eps_r)
    g2 = direct.backward({"probe": {c: 2.0 * v for c, v in m2["probe"].items()}})
    direct.close()
    problem.close()
    np.testing.assert_allclose(t.grad.numpy(), g2, rtol=1e-4, atol=1e-6 * np.abs(g2).max())


@pytest.mark.parametrize("medium", ["debye", "lorentz", "drude"])
def test_design_on_ade_cells_matches_finite_differences(medium):
    """A design region inside a dispersive block (its eps_inf is the design
    variable, the grating layer of the large Bloch workload is a Debye one)."""
    wm = load_package()
    adj = wm.adjoint
    media = {"debye": wm.Medium.debye(2.5, 3.5, 1e-14), "lorentz": wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12),
             "drude": wm.Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))}

    def scene(e):
        sc = _design_scene(wm, e)
        sc.structures.append(wm.Structure(wm.Box((11, 9, 9), (17, 15, 14)), media[medium]))
        return sc

    steps = 320
    rng = np.random.default_rng(11)
    eps_r = 2.0 + 2.0 * rng.random((4, 4, 3))
    cs = wm.compile_scene(scene(eps_r), steps)
    assert cs.poles  # the design region's cells carry the poles
    problem = adj.DesignProblem(scene(eps_r), steps, stride=64, history="replay")
    mons = problem.forward(eps_r)
    g = problem.backward({"probe": {c: 2.0 * v for c, v in mons["probe"].items()}})
    problem.close()
    assert np.isfinite(g).all() and np.abs(g).max() > 0
    h = 1e-2
    for flat in np.argsort(-np.abs(g).ravel())[:4]:
        idx = np.unravel_index(flat, eps_r.shape)
        vals = []
        for sgn in (1.0, -1.0):
            e = eps_r.copy()
            e[idx] += sgn * h
            p = adj.DesignProblem(scene(e), steps, stride=steps)
            vals.append(_loss(p.forward(e)))
            p.close()
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(g[idx] - fd) <= 1e-2 * abs(fd), (medium, idx, g[idx], fd)


def test_adjoint_rejects_designs_on_edges():
    wm = load_package()
    lib = wm._lib.load()
    solver = wm.solver.B200FDTD(wm.compile_scene(_design_scene(wm, np.full((4, 4, 3), 2.0)), 10)).init_field()
    bad = (ctypes.c_int * 18)(*([1, 5, 3, 6, 3, 6] + [0] * 12))  # reaches into the CPML slab
    assert lib.fdtd_engine_adjoint_init(solver.handle, bad, 4) == -1
    solver.close()


def test_design_workload_gradient_against_fp64_finite_differences():
    """The 160x160x96 design workload's layout at half size (80x80x48 cells,
    10-cell CPML, eps 2.1 substrate, 32x32x8 design block with eps_r ~ U[1, 12)
    seed 0, ramped 300 THz CW source, 8x8 patch objective), 400 steps, the
    reverse pass replaying checkpoints every 100 steps: dL/deps_r of 16 design
    cells drawn with numpy.random.default_rng(0) against central differences
    (h = 1e-3 on eps_r) of L = sum |E|^2 over the patch computed by the FP64
    oracle (FP32 forward runs are too noisy at this h: a single cell moves L by
    about 1e-6 of itself).  The scene's coefficients are FP32, which limits the
    differences to about 1e-4 relative; tolerance 2e-3 of the largest checked
    gradient."""
    wm = load_package()
    adj = wm.adjoint
    steps = 400
    scene = wm.workloads.adjoint_160(steps, scale=2)
    eps_r = scene.material_regions[0].eps_r
    problem = adj.DesignProblem(scene, steps, stride=100, history="replay")
    mons = problem.forward(eps_r)
    g = problem.backward({"patch": {c: 2.0 * v for c, v in mons["patch"].items()}})
    problem.close()
    rng = np.random.default_rng(0)
    picks = rng.choice(eps_r.size, size=16, replace=False)
    h = 1e-3

    def loss(e):
        sc = wm.workloads.adjoint_160(steps, scale=2)
        region = sc.material_regions[0]
        sc.material_regions[0] = wm.MaterialRegion(region.lo, region.hi, e)
        cs = wm.compile_scene(sc, steps)
        sim = orc.OracleSimulation(cs, "f64").run(steps)
        m = sim.monitor_results()
        sim.close()
        return float(sum(np.sum(np.abs(v) ** 2) for v in m["patch"].values()))

    fds, gs = [], []
    for flat in picks:
        idx = np.unravel_index(flat, eps_r.shape)
        vals = []
        for sgn in (1.0, -1.0):
            e = eps_r.copy()
            e[idx] += sgn * h
            vals.append(loss(e))
        fds.append((vals[0] - vals[1]) / (2 * h))
        gs.append(g[idx])
    fds, gs = np.array(fds), np.array(gs)
    scale = np.abs(fds).max()
    assert scale > 0
    np.testing.assert_allclose(gs, fds, rtol=0, atol=2e-3 * scale)


@pytest.mark.parametrize("dispersive", [False, True])
def test_region_replay_equals_full_replay(dispersive):
    """Region replay (each replayed step restricted to the design boxes' domain
    of dependence) records the full replay's design history bit for bit, so the
    gradients are identical; both agree with the stored-history gradient."""
    wm = load_package()
    adj = wm.adjoint
    rng = np.random.default_rng(21)
    eps_r = 2.0 + 2.0 * rng.random((4, 4, 3))

    def scene(e):
        sc = wm.Scene(cells=(72, 64, 56), spacing=25e-9, pml_cells=6)
        if dispersive:
            sc.structures.append(wm.Structure(wm.Box((40, 26, 22), (43, 38, 34)),
                                              wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
            sc.structures.append(wm.Structure(wm.Box((20, 10, 10), (22, 54, 46)),
                                              wm.Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))))
        sc.sources.append(wm.PointDipole((30, 32, 28), "Ez", wm.GaussianPulse(300e12, 100e12), width=25e-9))
        sc.material_regions.append(wm.MaterialRegion((34, 30, 26), (38, 34, 29), e))
        sc.monitors.append(wm.PointMonitor("probe", (46, 32, 28), frequencies=(300e12,)))
        return sc

    steps, stride = 240, 24
    grads = {}
    for key, kw in (("region", {"history": "replay", "replay_region": True}),
                    ("full", {"history": "replay", "replay_region": False}), ("store", {"history": "store"})):
        problem = adj.DesignProblem(scene(eps_r), steps, stride=stride, **kw)
        mons = problem.forward(eps_r)
        grads[key] = problem.backward({"probe": {c: 2.0 * v for c, v in mons["probe"].items()}})
        problem.close()
    assert np.abs(grads["full"]).max() > 0
    np.testing.assert_array_equal(grads["region"], grads["full"])
    np.testing.assert_allclose(grads["region"], grads["store"], rtol=0, atol=1e-5 * np.abs(grads["store"]).max())
