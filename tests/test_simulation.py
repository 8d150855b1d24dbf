"""The ``Simulation.fdtd`` facade (witwin-maxwell_b200/simulation.py): the
reference's run-length rule and per-frequency spectral windows against the
reference's own functions (tests/golden/simulation.json, written by
tests/golden/make_sim_golden.py from witwin/maxwell/fdtd/solver.py:108-131 and
runtime/spectral.py:235-298), the keyword surface, and on the GPU a CW run with
Hanning windows through the facade against the FP64 oracle."""
from __future__ import annotations

import json
import types
from pathlib import Path

import numpy as np
import pytest

from conftest import load_package

GOLDEN = Path(__file__).resolve().parent / "golden" / "simulation.json"


def _g():
    return json.loads(GOLDEN.read_text())


def test_required_steps_match_reference():
    wm = load_package()
    sim = wm.simulation
    for case in _g()["steps"]:
        st = None
        if case["settling_time"] is not None:
            st = types.SimpleNamespace(kind="custom", settling_time=case["settling_time"])
        got = sim.required_steps(case["frequency"], case["dt"], num_cycles=case["num_cycles"],
                                 transient_cycles=case["transient_cycles"], domain_size=case["domain_size"],
                                 source_time=st)
        assert got == case["steps"], case


def test_spectral_windows_match_reference():
    wm = load_package()
    for case in _g()["windows"]:
        d = case["domain_range"]
        size = max(d[1] - d[0], d[3] - d[2], d[5] - d[4])
        got = wm.simulation.window_table(case["frequencies"], case["dt"], case["steps"], case["window"],
                                         pulsed=case["kind"] != "cw", domain_size=size)
        want = np.array(case["weights"]).T
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-15, err_msg=f"{case['kind']} {case['window']}")


def _cw_scene(wm, with_freqs=True):
    sc = wm.Scene(cells=(24, 20, 18), spacing=25e-9, pml_cells=5)
    sc.structures.append(wm.Structure(wm.Box((8, 6, 5), (16, 14, 13)), wm.Medium(eps_r=2.25)))
    sc.sources.append(wm.PointDipole((10, 10, 9), "Ez", wm.CW(300e12), width=25e-9))
    freqs = (280e12, 300e12) if with_freqs else ()
    sc.monitors.append(wm.PlaneMonitor("zplane", 2, 9, ("Ex", "Ey", "Ez", "Hz"), freqs))
    sc.monitors.append(wm.PointMonitor("probe", (14, 10, 9), frequencies=freqs))
    return sc


def test_facade_keywords_and_refusals():
    wm = load_package()
    sc = _cw_scene(wm, with_freqs=False)
    sim = wm.Simulation.fdtd(sc, frequencies=[300e12, 280e12], run_time=wm.TimeConfig.auto(steady_cycles=5))
    resolved = sim._resolved_scene()
    assert all(m.frequencies == (300e12, 280e12) for m in resolved.monitors)
    dt = resolved.resolve_dt()
    assert sim._steps(resolved, dt) == wm.simulation.required_steps(
        280e12, dt, num_cycles=5, domain_size=wm.simulation.physical_extent(resolved), source_time=wm.CW(300e12))
    assert wm.Simulation.fdtd(sc, frequency=3e14, time_steps=77)._steps(resolved, dt) == 77
    with pytest.raises(ValueError):
        wm.Simulation.fdtd(_cw_scene(wm, with_freqs=False))._resolved_scene()
    for kw in ({"absorber": "pml"}, {"enable_plot": True}, {"shutoff": 1e-4}, {"cpml_config": {"kappa_max": 3}}):
        with pytest.raises(NotImplementedError):
            wm.Simulation.fdtd(sc, frequencies=[3e14], **kw)
    with pytest.raises(ValueError):
        wm.SpectralSampler(window="blackman")
    full = wm.Simulation.fdtd(sc, frequencies=[3e14], full_field_dft=True)._resolved_scene()
    assert full.monitors[-1].name == "full_field"


@pytest.mark.gpu
def test_facade_cw_run_with_hanning_windows_matches_oracle():
    """A CW run through the facade: per-frequency Hanning windows, each starting
    after its own transient, on the engine (fdtd_engine_set_dft_windows) against
    the FP64 oracle stepping the same compiled scene."""
    from oracle import oracle as orc
    from test_engine_parity import assert_monitors_close

    wm = load_package()
    sim = wm.Simulation.fdtd(_cw_scene(wm, with_freqs=False), frequencies=[300e12, 280e12],
                             run_time=wm.TimeConfig(time_steps=1500), spectral_sampler=wm.SpectralSampler("hanning"))
    result = sim.run()
    cs = sim.solver.compiled
    assert cs.window.shape == (1500, 2)
    starts = [int(np.argmax(cs.window[:, f] > 0)) for f in range(2)]
    assert starts[0] != starts[1] and min(starts) > 0  # per-frequency transients
    ref = orc.OracleSimulation(cs, "f64", threads=4).run(1500)
    want = ref.monitor_results()
    got = {name: {c: v.cpu().numpy() for c, v in result.monitor(name)["components"].items()} for name in want}
    assert_monitors_close(got, want)
    one = result.monitor("probe", frequency=280e12)
    np.testing.assert_allclose(one["components"]["Ez"].cpu().numpy(), got["probe"]["Ez"][1])
    sim.solver.close()
    ref.close()
