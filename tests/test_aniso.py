"""Full (off-diagonal) anisotropy: the per-edge inverse permittivity tensors of
the scene compile, the oracle's restatement of the coupling terms against the
reference's own CUDA ops (tests/golden/aniso.npz, written on a GPU by
tests/golden/make_aniso_golden.py from oracle/_ref), and on the GPU the per-op
kernel against the reference op and the fused engine (the coupling pass after
the step kernel) against the FP64 oracle."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import load_package

GOLDEN = Path(__file__).resolve().parent / "golden" / "aniso.npz"
EPS0 = 8.8541878128e-12
PATTERNS = (("open", (False, False, False)), ("perxz", (True, False, True)))


def _scene(wm, offdiag=(0.4, -0.3, 0.25), cells=(28, 24, 22)):
    sc = wm.Scene(cells=cells, spacing=25e-9, pml_cells=5)
    sc.structures.append(wm.Structure(wm.Box((8, 7, 7), (16, 14, 12)),
                                      wm.Medium(eps_r=2.0, eps_diag=(2.5, 2.0, 3.0), eps_offdiag=offdiag)))
    sc.sources.append(wm.PointDipole((12, 10, 9), "Ez", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    freqs = (250e12, 300e12)
    sc.monitors.append(wm.PlaneMonitor("zplane", 2, 9, ("Ex", "Ey", "Ez", "Hz"), freqs))
    sc.monitors.append(wm.PointMonitor("probe", (14, 10, 9), frequencies=freqs))
    return sc


def test_oracle_coupling_matches_reference_ops():
    from oracle import oracle as orc

    g = np.load(GOLDEN)
    h = tuple(g[n].astype(np.float64) for n in ("Hx", "Hy", "Hz"))
    inv = [g[f"inv_d{a}"].astype(np.float64) for a in "xyz"]
    for c, name in enumerate(("Ex", "Ey", "Ez")):
        for tag, per in PATTERNS:
            e = g[f"{name}_e0"].astype(np.float64)
            orc.full_aniso_correction(c, e, h, g[f"{name}_ca"].astype(np.float64), g[f"{name}_cb"].astype(np.float64),
                                      inv, per)
            want = g[f"{name}_{tag}"]
            # the reference computes in FP32
            np.testing.assert_allclose(e, want, rtol=0, atol=2e-6 * np.abs(want).max(), err_msg=f"{name} {tag}")


def test_scene_compiles_inverse_tensors():
    wm = load_package()
    cs = wm.compile_scene(_scene(wm), 10)
    assert cs.aniso is not None and set(cs.aniso) == {"Ex", "Ey", "Ez"}
    dt32 = np.float32(cs.dt)
    # inside the box every edge sees the full tensor: compare with a direct inverse
    t = np.array([[2.5, 0.4, -0.3], [0.4, 2.0, 0.25], [-0.3, 0.25, 3.0]])
    inv = np.linalg.inv(t)
    rows = {"Ex": (0, (1, 2)), "Ey": (1, (0, 2)), "Ez": (2, (0, 1))}
    for name, (r, (a, b)) in rows.items():
        box, ca, cb = cs.aniso[name]
        centre = tuple((box[2 * q] + box[2 * q + 1]) // 2 for q in range(3))
        local = tuple(centre[q] - box[2 * q] for q in range(3))
        np.testing.assert_allclose(ca[local], cs.dt / EPS0 * inv[r, a], rtol=1e-5)
        np.testing.assert_allclose(cb[local], cs.dt / EPS0 * inv[r, b], rtol=1e-5)
        np.testing.assert_allclose(cs.curl[name][centre], dt32 * inv[r, r] / EPS0, rtol=1e-5)
    # a diagonal tensor keeps the plain path
    assert wm.compile_scene(_scene(wm, offdiag=(0.0, 0.0, 0.0)), 10).aniso is None
    with pytest.raises(ValueError):
        wm.compile_scene(_scene(wm, offdiag=(3.0, 0.0, 0.0)), 10)  # not positive-definite


def test_anisotropy_changes_the_oracle_run():
    from oracle import oracle as orc

    wm = load_package()
    steps = 160
    a = orc.OracleSimulation(wm.compile_scene(_scene(wm), steps), "f64", threads=4).run(steps)
    b = orc.OracleSimulation(wm.compile_scene(_scene(wm, offdiag=(0.0, 0.0, 0.0)), steps), "f64", threads=4).run(steps)
    num = sum(float(np.sum((a.fields[n] - b.fields[n]) ** 2)) for n in a.fields) ** 0.5
    den = sum(float(np.sum(b.fields[n] ** 2)) for n in b.fields) ** 0.5
    assert num / den > 1e-2
    a.close()
    b.close()


@pytest.mark.gpu
def test_full_aniso_op_matches_reference_op():
    import torch

    from oracle import ref_gpu

    if not ref_gpu.available():
        pytest.skip("oracle/_ref not built")
    wm = load_package()
    mod = wm.backend.NativeFDTDModule()
    rng = np.random.default_rng(5)
    nodes = (11, 9, 10)
    nx, ny, nz = nodes
    shapes = {"Ex": (nx - 1, ny, nz), "Ey": (nx, ny - 1, nz), "Ez": (nx, ny, nz - 1),
              "Hx": (nx, ny - 1, nz - 1), "Hy": (nx - 1, ny, nz - 1), "Hz": (nx - 1, ny - 1, nz)}
    dev = torch.device("cuda")

    def t(x):
        return torch.tensor(np.asarray(x, dtype=np.float32), device=dev)

    h = {n: t(rng.standard_normal(shapes[n])) for n in ("Hx", "Hy", "Hz")}
    inv = {a: t(rng.uniform(0.5, 2.0, n)) for a, n in zip("xyz", nodes)}
    op = ref_gpu.ops()
    refs = {"Ex": op.update_electric_ex_full_aniso, "Ey": op.update_electric_ey_full_aniso,
            "Ez": op.update_electric_ez_full_aniso}
    keys = {"Ex": ("Y", "Z"), "Ey": ("X", "Z"), "Ez": ("X", "Y")}
    for name in ("Ex", "Ey", "Ez"):
        e0 = rng.standard_normal(shapes[name])
        ca, cb = rng.standard_normal(shapes[name]), rng.standard_normal(shapes[name])
        ca.flat[::3] = 0.0
        for per in ((0, 0, 0), (1, 0, 1), (0, 1, 0), (1, 1, 1)):
            mine, theirs = t(e0), t(e0)
            mod.__getattr__(f"updateElectricField{name}FullAniso3D")(
                **{name: mine, f"Coeff{keys[name][0]}": t(ca), f"Coeff{keys[name][1]}": t(cb)}, **h,
                invDx=inv["x"], invDy=inv["y"], invDz=inv["z"], periodicX=per[0], periodicY=per[1],
                periodicZ=per[2]).launchRaw()
            refs[name](theirs, h["Hx"], h["Hy"], h["Hz"], t(ca), t(cb), inv["x"], inv["y"], inv["z"], *per)
            np.testing.assert_allclose(mine.cpu().numpy(), theirs.cpu().numpy(), rtol=0,
                                       atol=1e-6 * float(theirs.abs().max()), err_msg=f"{name} {per}")


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [2, 10])
def test_engine_full_aniso_matches_oracle(variant):
    from oracle import oracle as orc
    from test_engine_parity import assert_fields_close, assert_monitors_close

    wm = load_package()
    steps = 240
    cs = wm.compile_scene(_scene(wm), steps)
    ref = orc.OracleSimulation(cs, "f64", threads=4).run(steps)
    eng = wm.solver.B200FDTD(cs).init_field()
    eng.set_launch(variant)
    eng.step_range(0, steps)
    fields = {n: eng.field(n).cpu().numpy() for n in ref.fields}
    mons = {k: {c: v.cpu().numpy() for c, v in m.items()} for k, m in eng.monitor_results().items()}
    eng.close()
    assert_fields_close(fields, ref.fields)
    assert_monitors_close(mons, ref.monitor_results())
    ref.close()
