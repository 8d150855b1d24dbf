"""Generate beam.npz: the reference's own soft GaussianBeam face terms, the golden
vectors that pin the scene compiler's GaussianBeam (face specs, unit-power scale,
numerical phase speed, beam amplitude and delay, cos / sin phased patches and
time-shifted patches).

Run from the repository root in a container where the reference checkout is
available (it is not needed anywhere else):

    python tests/golden/make_beam_golden.py [--reference CHECKOUT]

It loads the reference's excitation modules (fdtd/excitation/injection.py,
spatial.py, tfsf_specs.py, tfsf_common.py, temporal.py, fdtd/dispersion.py,
waveforms.py, constants.py) from the checkout, with stand-ins for the imports
the beam path does not use (witwin.core's vacuum permittivity, the scene's
prepare_scene, the mode solver), and calls
_prepare_power_normalized_surface_source (injection.py:807-968) on a minimal
solver object that carries what that function reads: node and half-node
coordinates, spacings, the physical and computational domain ranges, CPML
thicknesses, dt, c, the source omega and the per-component curl coefficient
arrays (dt / eps for E with an eps 2.1 substrate below z = 12 cells, dt / mu0
for H).

Cases (cells 40 x 36 x 32, 25 nm, 8-cell CPML, waist 0.3 um, 300 THz):
  cw_z      +z, Ey, focus at the centre, CW
  cw_obl    oblique (0.3, 0, 0.954), polarization (-0.954, 0, 0.3), CW
  cw_mz     -z (the high face), Ex, CW with phase 0.4 and amplitude 1.7
  pulse_z   +z, Ey, GaussianPulse (300 THz, 100 THz): time-shifted patches
Per term: field name, offsets, the cos / sin patches (CW) or patch and delay
(pulse), and which of electric / magnetic lists it belongs to.  Coordinates:
the reference's physical domain is centred on the origin, so node i sits at
(i - cells / 2) * d; the compiler's focus is in node indices.
"""
from __future__ import annotations

import argparse
import importlib.util
import math
import sys
import types
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]

CELLS = (40, 36, 32)
D = 25e-9
PML = 8
WAIST = 0.3e-6
FREQ = 300e12
EPS0 = 8.8541878128e-12
MU0 = 1.25663706212e-6
C0 = 299792458.0
SUB_Z = 12
CASES = {
    "cw_z": dict(direction=(0.0, 0.0, 1.0), polarization=(0.0, 1.0, 0.0), focus=(20.0, 18.0, 16.0),
                 time=dict(kind="cw", amplitude=1.0, phase=0.0)),
    "cw_obl": dict(direction=(0.3, 0.0, 0.954), polarization=(-0.954, 0.0, 0.3), focus=(18.5, 17.0, 20.0),
                   time=dict(kind="cw", amplitude=1.0, phase=0.0)),
    "cw_mz": dict(direction=(0.0, 0.0, -1.0), polarization=(1.0, 0.0, 0.0), focus=(21.0, 16.0, 12.0),
                  time=dict(kind="cw", amplitude=1.7, phase=0.4)),
    "pulse_z": dict(direction=(0.0, 0.0, 1.0), polarization=(0.0, 1.0, 0.0), focus=(20.0, 18.0, 16.0),
                    time=dict(kind="gaussian_pulse", amplitude=1.0, phase=0.0, fwidth=100e12)),
}


def _module(name, path=None, **attrs):
    if path is None:
        mod = types.ModuleType(name)
        mod.__path__ = []
        mod.__dict__.update(attrs)
        sys.modules[name] = mod
        return mod
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_injection(ref: Path):
    m = ref / "witwin" / "maxwell"
    for pkg in ("witwin", "witwin.core", "witwin.maxwell", "witwin.maxwell.fdtd", "witwin.maxwell.fdtd.excitation"):
        _module(pkg)
    _module("witwin.core.material", VACUUM_PERMITTIVITY=EPS0)
    _module("witwin.maxwell.constants", m / "constants.py")
    _module("witwin.maxwell.waveforms", m / "waveforms.py")
    _module("witwin.maxwell.sources", POINT_DIPOLE_REFERENCE_WIDTH=0.02,
            evaluate_source_time=lambda *a, **k: 0.0)
    _module("witwin.maxwell.scene", prepare_scene=lambda scene: scene)
    _module("witwin.maxwell.fdtd.dispersion", m / "fdtd" / "dispersion.py")
    ex = m / "fdtd" / "excitation"
    _module("witwin.maxwell.fdtd.excitation.modes", sample_mode_source_component=None,
            solve_mode_source_profile=None)
    for name in ("spatial", "tfsf_specs", "temporal", "tfsf_common", "injection"):
        _module(f"witwin.maxwell.fdtd.excitation.{name}", ex / f"{name}.py")
    return sys.modules["witwin.maxwell.fdtd.excitation.injection"]


class _Boundary:
    def uses_kind(self, kind):
        return kind == "pml"

    def axis_kind(self, axis):
        return "pml"


class _Domain:
    def __init__(self, rng):
        self.domain_range = rng


class _Scene:
    """What the soft-surface-source path reads from a prepared scene."""

    def __init__(self):
        self.boundary = _Boundary()
        nodes = [c + 1 for c in CELLS]
        phys = []
        comp = []
        for a, c in enumerate(CELLS):
            half = 0.5 * (c - 2 * PML) * D
            phys += [-half, half]
            comp += [-half - PML * D, half + PML * D]
        self.domain = _Domain(tuple(phys))
        self.domain_range = tuple(comp)
        for a, name in enumerate("xyz"):
            n64 = (np.arange(nodes[a], dtype=np.float64) - CELLS[a] / 2) * D
            h64 = n64[:-1] + 0.5 * D
            setattr(self, name, torch.tensor(n64, dtype=torch.float32))
            setattr(self, f"{name}_half", torch.tensor(h64, dtype=torch.float32))
            setattr(self, f"d{name}_primal64", np.full(nodes[a] - 1, D))
            setattr(self, f"d{name}_dual64", np.full(nodes[a], D))
        self.Nx, self.Ny, self.Nz = nodes

    def pml_thickness_for_face(self, axis, side):
        return PML


class _Solver:
    _HALF = {"Ex": (True, False, False), "Ey": (False, True, False), "Ez": (False, False, True),
             "Hx": (False, True, True), "Hy": (True, False, True), "Hz": (True, True, False)}

    def __init__(self, eps):
        self.scene = _Scene()
        self.Nx, self.Ny, self.Nz = self.scene.Nx, self.scene.Ny, self.scene.Nz
        self.device = torch.device("cpu")
        self.c = C0
        self.dt = 0.99 / (C0 * math.sqrt(3.0 / (D * D)))
        self.source_omega = 2.0 * math.pi * FREQ
        self.Ex = torch.zeros(1, dtype=torch.float32)
        dt32 = np.float32(self.dt)
        self.cex_curl = torch.tensor(dt32 / eps["Ex"])
        self.cey_curl = torch.tensor(dt32 / eps["Ey"])
        self.cez_curl = torch.tensor(dt32 / eps["Ez"])
        hc = np.float32(dt32 / np.float32(MU0))
        nodes = (self.Nx, self.Ny, self.Nz)
        shapes = {"Hx": (nodes[0], nodes[1] - 1, nodes[2] - 1), "Hy": (nodes[0] - 1, nodes[1], nodes[2] - 1),
                  "Hz": (nodes[0] - 1, nodes[1] - 1, nodes[2])}
        self.chx_curl = torch.full(shapes["Hx"], float(hc), dtype=torch.float32)
        self.chy_curl = torch.full(shapes["Hy"], float(hc), dtype=torch.float32)
        self.chz_curl = torch.full(shapes["Hz"], float(hc), dtype=torch.float32)
        self._electric_source_terms = []
        self._magnetic_source_terms = []

    def _component_positions(self, field_name, offsets, shape, dtype):
        half_axes = self._HALF[field_name]
        s = self.scene
        coords = ((s.x, s.x_half), (s.y, s.y_half), (s.z, s.z_half))
        px, py, pz = (c[h][o:o + n].to(dtype=dtype) for c, h, o, n in zip(coords, half_axes, offsets, shape))
        px = px[:, None, None].expand(*shape)
        py = py[None, :, None].expand(*shape)
        pz = pz[None, None, :].expand(*shape)
        return torch.stack((px, py, pz), dim=-1)

    def _plane_coordinate(self, axis, plane_index):
        vals = {"x": self.scene.x, "y": self.scene.y, "z": self.scene.z}[axis]
        return float(vals[min(max(int(plane_index), 0), len(vals) - 1)].item())


def substrate_eps():
    """Absolute permittivity per E component: eps_r 2.1 on nodes with z < SUB_Z, node
    values averaged onto the components as the compiler does."""
    sys.path.insert(0, str(ROOT))
    import importlib

    spec = importlib.util.spec_from_file_location("wm", ROOT / "witwin-maxwell_b200" / "__init__.py",
                                                  submodule_search_locations=[str(ROOT / "witwin-maxwell_b200")])
    wm = importlib.util.module_from_spec(spec)
    sys.modules["wm"] = wm
    spec.loader.exec_module(wm)
    return wm, beam_scene(wm, None).structures


def beam_scene(wm, source):
    S = wm.scene
    sc = S.Scene(cells=CELLS, spacing=D, pml_cells=PML)
    sc.structures.append(S.Structure(S.Box((0, 0, 0), (CELLS[0], CELLS[1], SUB_Z - 1)), S.Medium(eps_r=2.1)))
    if source is not None:
        sc.sources.append(source)
    return sc


def run(inj, wm) -> dict:
    cs = wm.scene.compile_scene(beam_scene(wm, None), 4)
    eps = {n: cs.eps[n] for n in ("Ex", "Ey", "Ez")}
    out = {"cells": np.array(CELLS), "spacing": np.array(D), "pml": np.array(PML), "waist": np.array(WAIST),
           "freq": np.array(FREQ), "sub_z": np.array(SUB_Z)}
    for case, cfg in CASES.items():
        solver = _Solver(eps)
        tm = cfg["time"]
        source_time = {"kind": tm["kind"], "kind_code": 0 if tm["kind"] == "cw" else 1, "frequency": FREQ,
                       "fwidth": tm.get("fwidth", 0.0), "amplitude": tm["amplitude"], "phase": tm["phase"],
                       "delay": 6.0 / (2.0 * math.pi * tm["fwidth"]) if "fwidth" in tm else 0.0}
        focus = tuple((f - c / 2) * D for f, c in zip(cfg["focus"], CELLS))
        # GaussianBeam normalises both vectors (sources.py:155-166)
        direction, polarization = (tuple(v / math.sqrt(sum(x * x for x in vec)) for v in vec)
                                   for vec in (cfg["direction"], cfg["polarization"]))
        source = {"kind": "gaussian_beam", "direction": direction, "polarization": polarization,
                  "beam_waist": WAIST, "focus": focus, "source_time": source_time, "injection_axis": None}
        inj._prepare_power_normalized_surface_source(solver, source, source_index=0)
        terms = [("E", t) for t in solver._electric_source_terms] + [("H", t) for t in solver._magnetic_source_terms]
        out[f"{case}_n"] = np.array(len(terms))
        for i, (kind, term) in enumerate(terms):
            key = f"{case}_{i}"
            out[f"{key}_field"] = np.array(term["field_name"])
            out[f"{key}_offsets"] = np.array(term["offsets"])
            if term["cw_cos_patch"] is not None:
                out[f"{key}_cos"] = term["cw_cos_patch"].double().numpy()
                out[f"{key}_sin"] = term["cw_sin_patch"].double().numpy()
            else:
                out[f"{key}_patch"] = term["patch"].double().numpy()
                out[f"{key}_delay"] = term["delay_patch"].double().numpy()
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
    inj = load_injection(ref)
    wm, _ = substrate_eps()
    out = run(inj, wm)
    np.savez_compressed(HERE / "beam.npz", **out)
    print("wrote", HERE / "beam.npz", {k: int(v) for k, v in out.items() if k.endswith("_n")})


if __name__ == "__main__":
    main()
