"""Generate postprocess.npz: the reference's own diffraction-order projection and
near-to-far-field transform on seeded synthetic plane spectra, the golden
vectors that pin witwin-maxwell_b200/postprocess.py and its GPU kernels.

Run from the repository root in a container where the reference checkout is
available (it is not needed anywhere else):

    python tests/golden/make_postprocess_golden.py [--reference CHECKOUT]

It loads the reference's witwin/maxwell/constants.py and postprocess/
stratton_chu.py, modal.py, diffraction.py and nfft.py from the checkout, with
stand-ins for the imports these paths do not use (witwin.core's vacuum
permittivity, the scene compiler, the mode solver, the source classes), and
calls

  compute_diffraction_from_payload (diffraction.py:84-196) on a z-normal plane
  of 48 x 40 complex64 samples of all six components over a 1.6 x 1.2 um unit
  cell (k_bloch = (0.7, -0.4) / um, 300 THz, background index 1.2, incident
  power given), recording every order's m, n, amplitudes, power, efficiency;

  NearFieldFarFieldTransformer.transform (nfft.py:187-265) of two planar
  equivalent-current surfaces (PlanarEquivalentCurrents, stratton_chu.py:
  339-460; one trapezoidal, one cell-centred) at 250 THz over a 7 x 9
  theta-phi grid, radius 2 um, recording E, H, E_theta, E_phi and the power
  density.
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
EPS0 = 8.8541878128e-12


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


def load_postprocess(ref: Path):
    m = ref / "witwin" / "maxwell"
    for pkg in ("witwin", "witwin.core", "witwin.maxwell", "witwin.maxwell.postprocess", "witwin.maxwell.compiler",
                "witwin.maxwell.fdtd", "witwin.maxwell.fdtd.excitation"):
        _module(pkg)
    _module("witwin.core.material", VACUUM_PERMITTIVITY=EPS0)
    _module("witwin.maxwell.constants", m / "constants.py")
    _module("witwin.maxwell.compiler.sources", _compile_mode_source=None)
    _module("witwin.maxwell.fdtd.excitation.modes", sample_mode_source_component=None,
            solve_mode_source_profile=None)
    _module("witwin.maxwell.scene", prepare_scene=lambda scene: scene)
    _module("witwin.maxwell.sources", CW=object, ModeSource=object)
    pp = m / "postprocess"
    for name in ("stratton_chu", "modal", "diffraction", "nfft"):
        _module(f"witwin.maxwell.postprocess.{name}", pp / f"{name}.py")
    return sys.modules["witwin.maxwell.postprocess.diffraction"], sys.modules["witwin.maxwell.postprocess.nfft"], \
        sys.modules["witwin.maxwell.postprocess.stratton_chu"], sys.modules["witwin.maxwell.constants"]


def run(diff, nfft, sc, const) -> dict:
    rng = np.random.default_rng(20261204)
    out = {}
    # ---- diffraction ----
    na, nb = 48, 40
    period_a, period_b = 1.6e-6, 1.2e-6
    coords_a = np.linspace(0.0, period_a, na, endpoint=False) + 0.01e-6
    coords_b = np.linspace(0.0, period_b, nb, endpoint=False) - 0.2e-6
    freq = 300e12
    kb = (0.7e6, -0.4e6)
    fields = {n: (rng.standard_normal((na, nb)) + 1j * rng.standard_normal((na, nb))).astype(np.complex64)
              for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    payload = {"monitor_type": "diffraction", "axis": "z", "x": torch.tensor(coords_a, dtype=torch.float32),
               "y": torch.tensor(coords_b, dtype=torch.float32), "frequency": freq, "position": 0.5e-6,
               "normal_direction": "+", "diffraction_spec": {"orders": None}}
    for n, v in fields.items():
        payload[n] = torch.tensor(v)
    result = types.SimpleNamespace(solver=types.SimpleNamespace(
        scene=types.SimpleNamespace(domain_range=(0.0, period_a, 0.0, period_b, -1e-6, 1e-6)),
        resolved_bloch_wavevector=(kb[0], kb[1], 0.0)))
    res = diff.compute_diffraction_from_payload(result, "grating", payload, incident_power=2.5, background_index=1.2)
    out.update(dif_na=np.array(na), dif_nb=np.array(nb), dif_ca=coords_a, dif_cb=coords_b, dif_freq=np.array(freq),
               dif_periods=np.array([period_a, period_b]), dif_kb=np.array(kb))
    for n, v in fields.items():
        out[f"dif_{n}"] = v
    orders = res["orders"]
    out["dif_m"] = np.array([o["m"] for o in orders])
    out["dif_n"] = np.array([o["n"] for o in orders])
    out["dif_power"] = np.array([o["power"] for o in orders])
    out["dif_eff"] = np.array([o["efficiency"] for o in orders])
    out["dif_prop"] = np.array([o["propagating"] for o in orders])
    out["dif_amp_e"] = np.stack([o["amplitude_E"].numpy() for o in orders])
    out["dif_amp_h"] = np.stack([o["amplitude_H"].numpy() for o in orders])
    out["dif_total"] = np.array(res["total_power"])
    # ---- near-to-far field ----
    surfaces = []
    for i, (axis, pos, rule) in enumerate((("z", 0.6e-6, "trapezoidal"), ("x", -0.5e-6, "cell_centered"))):
        nu, nv = 20 + 3 * i, 18 + 2 * i
        u = np.linspace(-0.5e-6, 0.5e-6, nu)
        v = np.linspace(-0.4e-6, 0.45e-6, nv)
        J = (rng.standard_normal((nu, nv, 3)) + 1j * rng.standard_normal((nu, nv, 3))).astype(np.complex64)
        M = (rng.standard_normal((nu, nv, 3)) + 1j * rng.standard_normal((nu, nv, 3))).astype(np.complex64) * 300
        out.update({f"nf{i}_axis": np.array(axis), f"nf{i}_pos": np.array(pos), f"nf{i}_rule": np.array(rule),
                    f"nf{i}_u": u, f"nf{i}_v": v, f"nf{i}_J": J, f"nf{i}_M": M})
        surfaces.append(sc.PlanarEquivalentCurrents(axis=axis, position=pos, frequency=250e12,
                                                    u=torch.tensor(u, dtype=torch.float32),
                                                    v=torch.tensor(v, dtype=torch.float32), J=torch.tensor(J),
                                                    M=torch.tensor(M), quadrature_rule=rule))
    collection = sc.EquivalentCurrentsSurface(surfaces=tuple(surfaces)) if hasattr(sc, "EquivalentCurrentsSurface") \
        else surfaces[0]
    tr = nfft.NearFieldFarFieldTransformer(collection, c=const.C_0, eps0=const.EPSILON_0, mu0=const.MU_0,
                                           device="cpu")
    theta = np.linspace(0.1, 2.9, 7)[:, None]
    phi = np.linspace(0.0, 5.5, 9)[None, :]
    far = tr.transform(torch.tensor(theta, dtype=torch.float32), torch.tensor(phi, dtype=torch.float32), radius=2e-6)
    out.update(nf_theta=theta, nf_phi=phi, nf_radius=np.array(2e-6), nf_freq=np.array(250e12))
    for key in ("E", "H", "E_theta", "E_phi", "power_density"):
        out[f"nf_out_{key}"] = far[key].numpy()
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
    diff, nfft, sc, const = load_postprocess(ref)
    out = run(diff, nfft, sc, const)
    np.savez_compressed(HERE / "postprocess.npz", **out)
    print("wrote", HERE / "postprocess.npz", "orders", len(out["dif_m"]))


if __name__ == "__main__":
    main()
