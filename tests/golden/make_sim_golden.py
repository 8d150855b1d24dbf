"""Generate simulation.json: the reference's own run-length and spectral-window
rules on a set of cases, the golden values that pin witwin-maxwell_b200/
simulation.py (required_steps, spectral_windows).

Run from the repository root in a container where the reference checkout is
available (it is not needed anywhere else):

    python tests/golden/make_sim_golden.py [--reference CHECKOUT]

It executes, without their modules' package imports, the reference functions

  calculate_required_steps    witwin/maxwell/fdtd/solver.py:108-131
  compute_spectral_start_step witwin/maxwell/fdtd/runtime/spectral.py:250-267
  compute_window_weight       witwin/maxwell/fdtd/runtime/spectral.py:270-298

(with source_time_kind, spectral.py:235-241) and records the step counts, the
start steps and the per-step weights.
"""
from __future__ import annotations

import argparse
import ast
import json
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
C0 = 299792458.0


def _functions(path: Path, names, extra=None):
    tree = ast.parse(path.read_text())
    body = [node for node in tree.body if isinstance(node, ast.FunctionDef) and node.name in names]
    ns = {"np": np, "C_0": C0}
    ns.update(extra or {})
    exec(compile(ast.Module(body=body, type_ignores=[]), str(path), "exec"), ns)
    return ns


def run(ref: Path) -> dict:
    solver_ns = _functions(ref / "witwin/maxwell/fdtd/solver.py", {"calculate_required_steps"})
    spec_ns = _functions(ref / "witwin/maxwell/fdtd/runtime/spectral.py",
                         {"source_time_kind", "compute_spectral_start_step", "compute_window_weight"})
    out = {"steps": [], "windows": []}
    for freq, dt, cycles, transient, domain, settle in (
            (300e12, 4.8e-17, 20, 15, 1.2e-6, None), (250e12, 4.8e-17, 8, 18, 0.8e-6, 3.1e-14),
            (1e9, 5e-11, 20, 15, 2.0, 0.0), (500e12, 2.4e-17, 30, 10, 4e-6, 1e-13)):
        source = None if settle is None else types.SimpleNamespace(settling_time=settle)
        n = solver_ns["calculate_required_steps"](frequency=freq, dt=dt, c=C0, num_cycles=cycles,
                                                  transient_cycles=transient, domain_size=domain, source_time=source)
        out["steps"].append({"frequency": freq, "dt": dt, "num_cycles": cycles, "transient_cycles": transient,
                             "domain_size": domain, "settling_time": settle, "steps": int(n)})
    for kind, window, freqs, dt, domain, steps in (
            ("cw", "hanning", (300e12, 200e12), 1e-16, (0.0, 0.6e-6, 0.0, 0.5e-6, 0.0, 0.4e-6), 1200),
            ("cw", "ramp", (250e12,), 1e-16, (0.0, 0.3e-6, 0.0, 0.3e-6, 0.0, 0.3e-6), 1000),
            ("cw", "hanning", (300e12,), 1e-16, (0.0, 3.0e-6, 0.0, 0.3e-6, 0.0, 0.3e-6), 2400),
            ("cw", "none", (300e12,), 4.8e-17, (0.0, 0.3e-6, 0.0, 0.3e-6, 0.0, 0.3e-6), 300),
            ("gaussian_pulse", "hanning", (300e12, 350e12), 4.8e-17, (0.0, 0.6e-6, 0.0, 0.6e-6, 0.0, 0.6e-6), 400)):
        solver = types.SimpleNamespace(
            _source_time={"kind": kind}, dt=dt, c=C0,
            scene=types.SimpleNamespace(domain_range=domain, physical_domain_range=domain), dft_window_type=window)
        resolved = "none" if kind != "cw" else window
        cols = []
        for f in freqs:
            start = spec_ns["compute_spectral_start_step"](solver, f, window_type=window)
            cols.append([float(spec_ns["compute_window_weight"](solver, n, start_step=start, end_step=steps,
                                                                window_type=resolved)) for n in range(steps)])
        out["windows"].append({"kind": kind, "window": window, "frequencies": list(freqs), "dt": dt,
                               "domain_range": list(domain), "steps": steps, "weights": cols})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    args = ap.parse_args()
    sys.path.insert(0, str(ROOT))
    from oracle.build_ref import reference_checkout

    ref = reference_checkout(args.reference)
    if ref is None:
        sys.exit("no reference checkout: pass --reference or set WITWIN_MAXWELL_REFERENCE")
    out = run(Path(ref))
    (HERE / "simulation.json").write_text(json.dumps(out))
    print("wrote", HERE / "simulation.json")


if __name__ == "__main__":
    main()
