"""Soft GaussianBeam: the scene compiler's face terms against the reference's own
(tests/golden/beam.npz, written by tests/golden/make_beam_golden.py from
witwin/maxwell/fdtd/excitation/injection.py:807-968), and the engine against the
oracle on a beam scene (CW phased patches and time-shifted pulse patches)."""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from conftest import load_package

wm = load_package()
S = wm.scene

GOLDEN = Path(__file__).resolve().parent / "golden" / "beam.npz"


def _golden():
    return np.load(GOLDEN, allow_pickle=False)


def _scene(g, case_focus, direction, polarization, source_time):
    cells = tuple(int(v) for v in g["cells"])
    sc = S.Scene(cells=cells, spacing=float(g["spacing"]), pml_cells=int(g["pml"]))
    sub = int(g["sub_z"])
    sc.structures.append(S.Structure(S.Box((0, 0, 0), (cells[0], cells[1], sub - 1)), S.Medium(eps_r=2.1)))
    sc.sources.append(S.GaussianBeam(direction, polarization, float(g["waist"]), case_focus, source_time))
    return sc


CASES = {
    "cw_z": ((0.0, 0.0, 1.0), (0.0, 1.0, 0.0), (20.0, 18.0, 16.0), lambda f: S.CW(f)),
    "cw_obl": ((0.3, 0.0, 0.954), (-0.954, 0.0, 0.3), (18.5, 17.0, 20.0), lambda f: S.CW(f)),
    "cw_mz": ((0.0, 0.0, -1.0), (1.0, 0.0, 0.0), (21.0, 16.0, 12.0), lambda f: S.CW(f, amplitude=1.7, phase=0.4)),
    "pulse_z": ((0.0, 0.0, 1.0), (0.0, 1.0, 0.0), (20.0, 18.0, 16.0), lambda f: S.GaussianPulse(f, 100e12)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_beam_terms_match_reference(case):
    g = _golden()
    direction, pol, focus, st = CASES[case]
    freq = float(g["freq"])
    steps = 16
    sc = _scene(g, focus, direction, pol, st(freq))
    cs = S.compile_scene(sc, steps)
    n = int(g[f"{case}_n"])
    pulse = case.startswith("pulse")
    mine = cs.shifted if pulse else cs.patches
    assert len(mine) == (n if pulse else 2 * n)
    dt = cs.dt
    for i in range(n):
        key = f"{case}_{i}"
        field = str(g[f"{key}_field"])
        offs = tuple(int(v) for v in g[f"{key}_offsets"])
        if pulse:
            p = mine[i]
            assert p.component == field and (p.box[0], p.box[2], p.box[4]) == offs
            ref_patch, ref_delay = g[f"{key}_patch"], g[f"{key}_delay"]
            assert p.scale.shape == ref_patch.shape
            top = np.abs(ref_patch).max()
            np.testing.assert_allclose(p.scale, ref_patch, rtol=0, atol=2e-6 * top)
            np.testing.assert_allclose(p.delay, ref_delay, rtol=0, atol=1e-5 * np.abs(ref_delay).max() + 1e-21)
            assert p.t_offset == (0.5 * dt if field[0] == "E" else 0.0)
        else:
            pc, ps = mine[2 * i], mine[2 * i + 1]
            for p, ref in ((pc, g[f"{key}_cos"]), (ps, g[f"{key}_sin"])):
                assert p.component == field and (p.box[0], p.box[2], p.box[4]) == offs
                assert p.coeff.shape == ref.shape
                np.testing.assert_allclose(p.coeff, ref, rtol=0, atol=2e-6 * np.abs(ref).max())
            # the CW signal pair at the term's sample instant (E at (n + 1/2) dt,
            # H at n dt), temporal.py:71-74 and stepping.py:1776, 2300-2306
            src = sc.sources[0].source_time
            t = np.arange(steps) * dt + (0.5 * dt if field[0] == "E" else 0.0)
            w = 2.0 * math.pi * freq
            np.testing.assert_allclose(pc.signal, src.amplitude * np.cos(w * t + src.phase), atol=1e-6)
            np.testing.assert_allclose(ps.signal, src.amplitude * np.sin(w * t + src.phase), atol=1e-6)


def test_beam_ramp_and_checks():
    g = _golden()
    freq = float(g["freq"])
    sc = _scene(g, (20.0, 18.0, 16.0), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), S.CW(freq))
    dt = sc.resolve_dt()
    ramped = _scene(g, (20.0, 18.0, 16.0), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), S.CW(freq, ramp_time=10 * dt))
    a, b = S.compile_scene(sc, 30), S.compile_scene(ramped, 30)
    for pa, pb in zip(a.patches, b.patches):
        np.testing.assert_array_equal(pa.coeff, pb.coeff)
        t = np.arange(30) * dt + (0.5 * dt if pa.component[0] == "E" else 0.0)
        ramp = np.where(t < 10 * dt, 0.5 * (1.0 - np.cos(np.pi * t / (10 * dt))), 1.0)
        np.testing.assert_allclose(pb.signal, ramp * pa.signal, atol=1e-6)
    with pytest.raises(ValueError):
        S.compile_scene(_scene(g, (20, 18, 16), (0.0, 0.0, 1.0), (0.0, 0.6, 0.8), S.CW(freq)), 4)
    bloch = _scene(g, (20, 18, 16), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), S.CW(freq))
    bloch.boundary = (S.BOUNDARY_BLOCH,) * 4 + (S.BOUNDARY_PML,) * 2
    with pytest.raises(ValueError):
        S.compile_scene(bloch, 4)
    with pytest.raises(TypeError):
        S.compile_scene(_scene(g, (20, 18, 16), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0),
                               S.ramped_cw(freq, 10, dt, 20)), 4)


def _beam_scene(source_time, steps_hint=None):
    """36 x 32 x 40 cells, 8-cell CPML, eps 2.1 substrate below z = 14, an eps 4 block
    above the launch plane, a +z Ey beam (waist 0.25 um) focused at (18, 16, 22), a
    z-plane monitor and a point monitor at 280 / 300 THz."""
    sc = S.Scene(cells=(36, 32, 40), spacing=25e-9, pml_cells=8)
    sc.structures.append(S.Structure(S.Box((0, 0, 0), (36, 32, 13)), S.Medium(eps_r=2.1)))
    sc.structures.append(S.Structure(S.Box((14, 12, 20), (22, 20, 26)), S.Medium(eps_r=4.0)))
    sc.sources.append(S.GaussianBeam((0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 0.25e-6, (18.0, 16.0, 22.0), source_time))
    freqs = (280e12, 300e12)
    sc.monitors.append(S.PlaneMonitor("far", 2, 30, ("Ex", "Ey", "Ez"), freqs))
    sc.monitors.append(S.PointMonitor("probe", (18, 16, 28), frequencies=freqs))
    return sc


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["cw_ramped", "pulse"])
def test_engine_beam_against_oracle(kind):
    """Engine (FP32) vs the FP32 / FP64 oracle on a GaussianBeam scene: CW phased
    patches (with a ramp) or time-shifted pulse patches on both E and H faces."""
    from oracle import oracle as orc
    from test_engine_parity import assert_fields_close, assert_monitors_close, joint_rel_l2, _run_engine

    # the pulse (centre 6 sigma = 200 steps) is still inside the domain at 260 steps;
    # later its CPML-absorbed tails leave only round-off-sized fields to compare
    steps = 500 if kind == "cw_ramped" else 260
    dt = S.Scene(cells=(36, 32, 40), spacing=25e-9).resolve_dt()
    st = S.CW(300e12, ramp_time=100 * dt) if kind == "cw_ramped" else S.GaussianPulse(300e12, 100e12)
    cs = S.compile_scene(_beam_scene(st), steps)
    assert (len(cs.shifted) > 0) == (kind == "pulse")
    solver, fields, mons = _run_engine(cs, steps)
    ref32 = orc.OracleSimulation(cs, "f32").run(steps)
    ref64 = orc.OracleSimulation(cs, "f64").run(steps)
    assert_fields_close(fields, ref32.fields)
    assert joint_rel_l2(fields, ref64.fields) < 2.0 * joint_rel_l2(ref32.fields, ref64.fields) + 1e-6
    assert_monitors_close(mons, ref32.monitor_results())
    # the beam reaches the far plane: its Ey DFT is not round-off
    far = np.abs(np.asarray(mons["far"]["Ey"]))
    assert far.max() > 1e-3 * np.abs(fields["Ey"]).max()
    ref32.close()
    ref64.close()
    solver.close()
