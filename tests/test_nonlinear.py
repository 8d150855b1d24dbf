"""Instantaneous nonlinear media (Kerr chi3, chi2, two-photon absorption) and
static conductivity.

CPU: the oracle's restatement of the coefficient recomposition against the
reference's own outputs (tests/golden/ops.npz: torch_reference's Kerr curl ops
and the general formula of the reference's nonlinear test), the scene compile of
the channels and of the lossy fold, and the x-slab decomposition of a nonlinear
scene on gloo ranks.

GPU: the per-op kernels against the same golden outputs, and the fused engine
(which recomposes the coefficients of the nonlinear cells before every step)
against the FP64 oracle at the engine parity bars (joint relative L2 <= 1e-5,
<= 1e-4 per component)."""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from conftest import load_package

GOLDEN = Path(__file__).resolve().parent / "golden" / "ops.npz"
EPS0 = 8.8541878128e-12


def _g():
    return np.load(GOLDEN, allow_pickle=False)


def _golden_inputs(g, comp):
    return {k: g[f"nl_{comp}_{k}"] for k in ("eps", "dec", "ext", "sig", "chi2", "chi3", "tpa")}


def test_oracle_nonlinear_coefficients_match_reference():
    from oracle import oracle as orc

    g = _g()
    dt, eps0 = float(g["nl_dt"]), float(g["nl_eps0"])
    ex, ey, ez = g["nl_Ex"], g["nl_Ey"], g["nl_Ez"]
    for comp in ("Ex", "Ey", "Ez"):
        x = _golden_inputs(g, comp)
        curl = orc.kerr_curl(comp, ex, ey, ez, x["eps"], x["dec"], x["chi3"], dt, eps0)
        np.testing.assert_allclose(curl, g[f"out_kerr_{comp}"], rtol=1e-12, atol=0)
        d, c = orc.nonlinear_coefficients(comp, ex, ey, ez, x["eps"], x["ext"], x["sig"], x["chi2"], x["chi3"], x["tpa"],
                                          dt, eps0)
        np.testing.assert_allclose(d, g[f"out_nl_{comp}_decay"], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(c, g[f"out_nl_{comp}_curl"], rtol=1e-12, atol=0)
    # the golden set reaches the eps_eff floor and the zero clamp of the TPA conductivity
    floor = 4.8e-17 / (1e-12 * EPS0)
    assert any(np.isclose(g[f"out_kerr_{c}"], floor * g[f"nl_{c}_dec"], rtol=1e-12).any() for c in ("Ex", "Ey", "Ez"))
    assert any((g[f"nl_{c}_tpa"] < 0).any() for c in ("Ex", "Ey", "Ez"))


def _scene(wm, kind: str, cells=(24, 20, 18)):
    sc = wm.Scene(cells=cells, spacing=25e-9, pml_cells=5)
    if kind == "kerr":
        med = wm.Medium(eps_r=2.25, kerr_chi3=1e-4)
    elif kind == "general":
        med = wm.Medium(eps_r=2.25, kerr_chi3=1e-4, chi2=0.005, tpa_beta=5e6, sigma=2e4)
    elif kind == "kerr_lorentz":
        med = wm.Medium(eps_r=2.0, poles=(wm.scene.LorentzPole(1.5, 250e12, 20e12),), kerr_chi3=1.5e-4)
    else:  # lossy: conductivity only (no nonlinear channel)
        med = wm.Medium(eps_r=2.25, sigma=3e4)
    sc.structures.append(wm.Structure(wm.Box((8, 6, 5), (16, 14, 13)), med))
    if kind == "kerr_lorentz":
        # a conductive Kerr-free slab next to it: a lossy cell of a nonlinear scene
        sc.structures.append(wm.Structure(wm.Box((16, 6, 5), (18, 14, 13)), wm.Medium(eps_r=3.0, sigma=1e4)))
    sc.sources.append(wm.PointDipole((10, 10, 9), "Ez", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    freqs = (250e12, 300e12)
    sc.monitors.append(wm.PlaneMonitor("zplane", 2, 9, ("Ex", "Ey", "Ez", "Hz"), freqs))
    sc.monitors.append(wm.PointMonitor("probe", (14, 10, 9), frequencies=freqs))
    return sc


def test_scene_compiles_channels_and_lossy_fold():
    wm = load_package()
    # TPA scale (media.py:420-423): (4/3) beta (n0 eps0 c0)^2, n0 = sqrt(eps_r)
    m = wm.Medium(eps_r=2.25, tpa_beta=8e7)
    assert m.tpa_sigma == pytest.approx((4.0 / 3.0) * 8e7 * (1.5 * EPS0 * 299792458.0) ** 2, rel=1e-12)
    assert wm.Medium(eps_r=2.25, tpa_beta=8e7, tpa_index=2.0).tpa_sigma == pytest.approx(
        (4.0 / 3.0) * 8e7 * (2.0 * EPS0 * 299792458.0) ** 2, rel=1e-12)
    steps = 10
    cs = wm.compile_scene(_scene(wm, "lossy"), steps)
    assert cs.nonlinear is None
    dt32 = np.float32(cs.dt)
    node = 3e4 * wm.Box((8, 6, 5), (16, 14, 13)).node_mask(cs.nodes).astype(np.float64)
    for name in ("Ex", "Ey", "Ez"):
        # the semi-implicit lossy fold (materials.py:942-977) in float32, sigma
        # averaged onto the edges like eps (materials.py:399-407)
        sig = wm.scene._avg_node_to_component(node, name).astype(np.float32)
        half = (np.float32(0.5) * sig * dt32) / cs.eps[name]
        np.testing.assert_array_equal(cs.decay[name], ((1 - half) / (1 + half)).astype(np.float32))
        np.testing.assert_array_equal(cs.curl[name], ((dt32 / cs.eps[name]) / (1 + half)).astype(np.float32))
    cs = wm.compile_scene(_scene(wm, "kerr"), steps)
    nl = cs.nonlinear
    assert nl is not None and not nl.general
    for name in ("Ex", "Ey", "Ez"):
        active = nl.active(name)
        assert active.any() and not active.all()
        # Kerr form: the at-rest curl is dt / eps (lossless static decay 1)
        np.testing.assert_array_equal(cs.curl[name], (dt32 / cs.eps[name]).astype(np.float32))
        assert cs.decay[name] is None
    cs = wm.compile_scene(_scene(wm, "general"), steps)
    assert cs.nonlinear.general
    for name in ("Ex", "Ey", "Ez"):
        ch = cs.nonlinear.channels[name]
        np.testing.assert_array_equal(ch["decay"], np.ones_like(ch["decay"]))
        assert cs.decay[name] is not None and cs.curl[name] is not None


@pytest.mark.parametrize("kind", ["kerr", "general", "kerr_lorentz"])
def test_nonlinearity_changes_the_oracle_run(kind):
    """The channels are strong enough at these fields to matter far above the
    parity bars (so the engine tests below check the nonlinear terms)."""
    from oracle import oracle as orc

    wm = load_package()
    steps = 240
    a = orc.OracleSimulation(wm.compile_scene(_scene(wm, kind), steps), "f64", threads=4).run(steps)
    linear = {"kerr": wm.Medium(eps_r=2.25), "general": wm.Medium(eps_r=2.25, sigma=2e4),
              "kerr_lorentz": wm.Medium(eps_r=2.0, poles=(wm.scene.LorentzPole(1.5, 250e12, 20e12),))}[kind]
    sc = _scene(wm, kind)
    sc.structures[0] = wm.Structure(sc.structures[0].geometry, linear)
    b = orc.OracleSimulation(wm.compile_scene(sc, steps), "f64", threads=4).run(steps)
    num = math.sqrt(sum(float(np.sum((a.fields[n] - b.fields[n]) ** 2)) for n in a.fields))
    den = math.sqrt(sum(float(np.sum(b.fields[n] ** 2)) for n in b.fields))
    assert num / den > 1e-3
    a.close()
    b.close()


@pytest.mark.gpu
def test_nonlinear_ops_match_reference():
    import torch

    wm = load_package()
    mod = wm.backend.NativeFDTDModule()
    g = _g()
    dt, eps0 = float(g["nl_dt"]), float(g["nl_eps0"])
    dev = torch.device("cuda")

    def t(a):
        return torch.tensor(np.asarray(a, dtype=np.float32), device=dev)

    ex, ey, ez = t(g["nl_Ex"]), t(g["nl_Ey"]), t(g["nl_Ez"])
    for comp in ("Ex", "Ey", "Ez"):
        x = _golden_inputs(g, comp)
        curl = torch.zeros_like(t(x["eps"]))
        mod.__getattr__(f"updateKerrElectricField{comp}Curl3D")(
            DynamicCurl=curl, Ex=ex, Ey=ey, Ez=ez, LinearPermittivity=t(x["eps"]), **{f"{comp}Decay": t(x["dec"])},
            KerrChi3=t(x["chi3"]), dt=dt, eps0=eps0).launchRaw()
        want = g[f"out_kerr_{comp}"]
        # FP32 arithmetic on FP32-rounded inputs against the FP64 reference
        np.testing.assert_allclose(curl.cpu().numpy(), want, rtol=2e-5, atol=1e-6 * np.abs(want).max())
        dd, dc = torch.zeros_like(curl), torch.zeros_like(curl)
        mod.updateNonlinearElectricCoefficients3D(
            DynamicDecay=dd, DynamicCurl=dc, Ex=ex, Ey=ey, Ez=ez, LinearPermittivity=t(x["eps"]),
            ExternalDecay=t(x["ext"]), SigmaStatic=t(x["sig"]), Chi2=t(x["chi2"]), Chi3=t(x["chi3"]),
            TpaSigma=t(x["tpa"]), component=comp, dt=dt, eps0=eps0).launchRaw()
        for got, key in ((dd, "decay"), (dc, "curl")):
            want = g[f"out_nl_{comp}_{key}"]
            np.testing.assert_allclose(got.cpu().numpy(), want, rtol=2e-5, atol=1e-6 * np.abs(want).max(), err_msg=key)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["kerr", "general", "kerr_lorentz", "lossy"])
def test_engine_nonlinear_matches_oracle(kind):
    from oracle import oracle as orc
    from test_engine_parity import assert_fields_close, assert_monitors_close

    wm = load_package()
    steps = 240
    cs = wm.compile_scene(_scene(wm, kind), steps)
    ref = orc.OracleSimulation(cs, "f64", threads=4).run(steps)
    eng = wm.solver.B200FDTD(cs).init_field()
    eng.step_range(0, steps)
    fields = {n: eng.field(n).cpu().numpy() for n in ref.fields}
    mons = {k: {c: v.cpu().numpy() for c, v in m.items()} for k, m in eng.monitor_results().items()}
    eng.close()
    assert_fields_close(fields, ref.fields)
    assert_monitors_close(mons, ref.monitor_results())
    ref.close()


@pytest.mark.gpu
def test_engine_nonlinear_every_launch_variant():
    """The cells an instantaneous nonlinearity rewrites are read from the
    coefficient arrays by every kernel form (the warp class marks them)."""
    from oracle import oracle as orc
    from test_engine_parity import assert_fields_close

    wm = load_package()
    steps = 240
    cs = wm.compile_scene(_scene(wm, "general"), steps)
    ref = orc.OracleSimulation(cs, "f64", threads=4).run(steps)
    for variant in range(1, 11):
        eng = wm.solver.B200FDTD(cs).init_field()
        eng.set_launch(variant)
        eng.step_range(0, steps)
        fields = {n: eng.field(n).cpu().numpy() for n in ref.fields}
        eng.close()
        assert_fields_close(fields, ref.fields)
    ref.close()


@pytest.mark.gpu
def test_engine_refuses_nonlinear_where_unsupported():
    wm = load_package()
    cs = wm.compile_scene(_scene(wm, "kerr"), 10)
    with pytest.raises(wm._lib.FdtdError):
        wm.solver.B200FDTD(cs, storage="fp16").init_field()
    cs = wm.compile_scene(_scene(wm, "kerr_lorentz"), 10)
    eng = wm.solver.B200FDTD(cs).init_field()
    with pytest.raises(wm._lib.FdtdError):
        eng.set_launch(5)  # the vector kernels keep the poles inside: not with nonlinear cells
    eng.close()
