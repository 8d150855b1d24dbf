"""Consumers of the DFT planes (witwin-maxwell_b200/postprocess.py) against the
reference's own diffraction-order projection and near-to-far-field transform
(tests/golden/postprocess.npz, written by tests/golden/make_postprocess_golden.py
from witwin/maxwell/postprocess/diffraction.py and nfft.py).

Tolerances: the reference computes in complex64 / float32; amplitudes, far
fields and powers agree to 2e-5 of the largest magnitude (FP32 inputs, FP64 sums
here against FP32 sums there)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import load_package

GOLDEN = Path(__file__).resolve().parent / "golden" / "postprocess.npz"


def _g():
    return np.load(GOLDEN, allow_pickle=False)


def test_order_enumeration_matches_reference():
    wm = load_package()
    g = _g()
    k0 = 2 * np.pi * float(g["dif_freq"]) / 299792458.0
    orders, _ = wm.postprocess.enumerate_diffraction_orders(periods=tuple(g["dif_periods"]), k_bloch=tuple(g["dif_kb"]),
                                                            k0=k0, background_index=1.2)
    assert [o["m"] for o in orders] == list(g["dif_m"])
    assert [o["n"] for o in orders] == list(g["dif_n"])
    assert [o["propagating"] for o in orders] == list(g["dif_prop"])


@pytest.mark.gpu
def test_diffraction_orders_match_reference():
    wm = load_package()
    g = _g()
    fields = {n: g[f"dif_{n}"] for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    res = wm.postprocess.compute_diffraction(fields, g["dif_ca"], g["dif_cb"], axis="z", frequency=float(g["dif_freq"]),
                                             periods=tuple(g["dif_periods"]), k_bloch=tuple(g["dif_kb"]),
                                             background_index=1.2, incident_power=2.5, position=0.5e-6)
    orders = res["orders"]
    assert [o["m"] for o in orders] == list(g["dif_m"]) and [o["n"] for o in orders] == list(g["dif_n"])
    amp_e = np.stack([o["amplitude_E"] for o in orders])
    amp_h = np.stack([o["amplitude_H"] for o in orders])
    for got, want in ((amp_e, g["dif_amp_e"]), (amp_h, g["dif_amp_h"])):
        np.testing.assert_allclose(got, want, rtol=0, atol=2e-5 * np.abs(want).max())
    power = np.array([o["power"] for o in orders])
    np.testing.assert_allclose(power, g["dif_power"], rtol=0, atol=2e-5 * np.abs(g["dif_power"]).max())
    eff = np.array([o["efficiency"] for o in orders])
    np.testing.assert_allclose(eff, g["dif_eff"], rtol=0, atol=2e-5 * np.abs(g["dif_eff"]).max())
    assert res["total_power"] == pytest.approx(float(g["dif_total"]), rel=1e-4, abs=1e-5 * np.abs(g["dif_power"]).max())


@pytest.mark.gpu
def test_near_to_far_field_matches_reference():
    wm = load_package()
    pp = wm.postprocess
    g = _g()
    surfaces = []
    for i in range(2):
        surfaces.append(pp.PlanarEquivalentCurrents(
            axis=str(g[f"nf{i}_axis"]), position=float(g[f"nf{i}_pos"]), frequency=float(g["nf_freq"]),
            u=g[f"nf{i}_u"].astype(np.float32), v=g[f"nf{i}_v"].astype(np.float32), J=g[f"nf{i}_J"],
            M=g[f"nf{i}_M"], quadrature_rule=str(g[f"nf{i}_rule"])))
    tr = pp.NearFieldFarFieldTransformer(surfaces)
    far = tr.transform(g["nf_theta"], g["nf_phi"], radius=float(g["nf_radius"]))
    for key in ("E", "H", "E_theta", "E_phi", "power_density"):
        got = far[key].cpu().numpy()
        want = g[f"nf_out_{key}"]
        assert got.shape == want.shape, key
        np.testing.assert_allclose(got, want, rtol=0, atol=2e-5 * np.abs(want).max(), err_msg=key)


def test_plane_alignment_averages_onto_cell_centres():
    wm = load_package()
    rng = np.random.default_rng(3)
    nx, ny = 9, 7
    shapes = {"Ex": (nx - 1, ny), "Ey": (nx, ny - 1), "Ez": (nx, ny), "Hx": (nx, ny - 1), "Hy": (nx - 1, ny),
              "Hz": (nx - 1, ny - 1)}
    spectra = {n: rng.standard_normal(s) + 1j * rng.standard_normal(s) for n, s in shapes.items()}
    fields, ca, cb = wm.postprocess.aligned_plane(spectra, "z", 25e-9)
    assert set(fields) == {"Ex", "Ey", "Ez", "Hx", "Hy"}  # the normal H is not aligned
    for v in fields.values():
        assert v.shape == (nx - 1, ny - 1)
    np.testing.assert_allclose(fields["Ex"], 0.5 * (spectra["Ex"][:, :-1] + spectra["Ex"][:, 1:]))
    ez = spectra["Ez"]
    np.testing.assert_allclose(fields["Ez"], 0.25 * (ez[:-1, :-1] + ez[1:, :-1] + ez[:-1, 1:] + ez[1:, 1:]))
    np.testing.assert_allclose(ca, (np.arange(nx - 1) + 0.5) * 25e-9)
