"""Consumers of the DFT planes: diffraction orders of a periodic plane and the
near-to-far-field transform of equivalent surface currents, with the
projections and radiation integrals on the GPU (fdtd_pp_diffraction,
fdtd_pp_nfft in libfdtd_b200.so).

Mirrors witwin/maxwell/postprocess/diffraction.py (enumerate_diffraction_orders
:23-68, compute_diffraction_from_payload :84-196) and
witwin/maxwell/postprocess/nfft.py (NearFieldFarFieldTransformer :47-265) with
its planar equivalent currents (stratton_chu.py:339-460): the same inputs,
outputs and order of results.  Fields are the co-located complex plane samples
the reference's payloads carry; the lossless background only (real k and eta).
There is no CPU path: the projections run through the CUDA library.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .scene import C_0, EPSILON_0, MU_0

_AXIS = {"x": 0, "y": 1, "z": 2}
_POWER_FLOOR = 1e-30


def _device(device) -> torch.device:
    dev = torch.device(device if device is not None else "cuda")
    if dev.type != "cuda" or not torch.cuda.is_available():
        raise RuntimeError("the postprocess kernels need a CUDA device; there is no CPU path")
    return dev


def _stream(dev: torch.device):
    return torch.cuda.current_stream(dev).cuda_stream


def enumerate_diffraction_orders(*, periods, k_bloch, k0, background_index=1.0, max_order=None):
    """Orders (m, n) with transverse wavevector k_bloch + (m Ga, n Gb), Ga = 2 pi / La;
    propagating when kz^2 = (k0 n)^2 - kx^2 - ky^2 > 0 (diffraction.py:23-68).
    Returns (orders, (Ga, Gb)) with the orders in m-major order."""
    pa, pb = float(periods[0]), float(periods[1])
    ga, gb = 2.0 * math.pi / pa, 2.0 * math.pi / pb
    cutoff = float(k0) * float(background_index)
    if max_order is None:
        bound_a = int(math.floor((cutoff + abs(k_bloch[0])) / ga)) + 1
        bound_b = int(math.floor((cutoff + abs(k_bloch[1])) / gb)) + 1
    else:
        bound_a = bound_b = int(max_order)
    orders = []
    for m in range(-bound_a, bound_a + 1):
        for n in range(-bound_b, bound_b + 1):
            kx = float(k_bloch[0]) + m * ga
            ky = float(k_bloch[1]) + n * gb
            kz2 = cutoff * cutoff - kx * kx - ky * ky
            orders.append({"m": m, "n": n, "kx": kx, "ky": ky, "kz_squared": kz2, "propagating": kz2 > 0.0})
    return orders, (ga, gb)


def _plane_amplitudes(field: np.ndarray, ca, cb, kx, ky, dev) -> torch.Tensor:
    """[n_m, n_n, 3] complex amplitudes of one field ([na, nb, 3] complex)."""
    na, nb = field.shape[0], field.shape[1]
    f = torch.view_as_real(torch.as_tensor(np.ascontiguousarray(field), dtype=torch.complex64)).contiguous().to(dev)
    a = torch.as_tensor(np.asarray(ca, dtype=np.float32), device=dev)
    b = torch.as_tensor(np.asarray(cb, dtype=np.float32), device=dev)
    tkx = torch.as_tensor(np.asarray(kx, dtype=np.float64), device=dev)
    tky = torch.as_tensor(np.asarray(ky, dtype=np.float64), device=dev)
    scratch = torch.empty(2 * len(ky) * na * 3, dtype=torch.float64, device=dev)
    out = torch.empty((len(kx), len(ky), 3, 2), dtype=torch.float32, device=dev)
    _lib.check(_lib.load().fdtd_pp_diffraction(na, nb, _lib.ptr(a), _lib.ptr(b), _lib.ptr(f), len(kx), _lib.ptr(tkx),
                                               len(ky), _lib.ptr(tky), _lib.ptr(scratch), _lib.ptr(out),
                                               _stream(dev)), "diffraction")
    return torch.view_as_complex(out)


# In-plane averages that bring each component of a plane monitor onto the
# plane's cell centres (witwin/maxwell/fdtd/observers.py:25-38, 126-160): the
# axes (0: first, 1: second tangential axis) along which the component's Yee
# samples are averaged; the plane-normal H component is not aligned.
_ALIGN = {
    "x": {"Ex": (0, 1), "Ey": (1,), "Ez": (0,), "Hy": (0,), "Hz": (1,)},
    "y": {"Ex": (1,), "Ey": (0, 1), "Ez": (0,), "Hx": (0,), "Hz": (1,)},
    "z": {"Ex": (1,), "Ey": (0,), "Ez": (0, 1), "Hx": (0,), "Hy": (1,)},
}


def aligned_plane(spectra: dict, axis: str, spacing: float, origin=(0.0, 0.0)) -> tuple[dict, np.ndarray, np.ndarray]:
    """Co-locate one frequency of a plane monitor's components (``spectra``: name ->
    2-D complex array over the plane, as B200FDTD.monitor_results gives them with
    the frequency and normal axes dropped) on the plane's cell centres by averaging
    adjacent Yee samples (observers.py:96-160).  Returns (fields, coords_a, coords_b)
    with the centre coordinates ``origin + (i + 1/2) * spacing`` of the two
    tangential axes."""
    rules = _ALIGN[str(axis).lower()]
    out = {}
    for name, data in spectra.items():
        axes = rules.get(name)
        if axes is None:
            continue
        v = np.asarray(data)
        for ax in axes:
            lo = [slice(None)] * 2
            hi = [slice(None)] * 2
            lo[ax], hi[ax] = slice(0, -1), slice(1, None)
            v = 0.5 * (v[tuple(lo)] + v[tuple(hi)])
        out[name] = v
    shapes = {v.shape for v in out.values()}
    if len(shapes) != 1:
        raise ValueError("the plane's components do not share the cell-centre grid")
    na, nb = shapes.pop()
    ca = float(origin[0]) + (np.arange(na) + 0.5) * float(spacing)
    cb = float(origin[1]) + (np.arange(nb) + 0.5) * float(spacing)
    return out, ca, cb


def compute_diffraction(fields: dict, coords_a, coords_b, *, axis: str, frequency: float, periods, k_bloch=(0.0, 0.0),
                        normal_direction: str = "+", position: float = 0.0, background_index: float = 1.0,
                        max_order=None, incident_power=None, device=None) -> dict:
    """Diffraction orders of one frequency's plane spectrum (diffraction.py:84-196).

    ``fields`` maps Ex .. Hz to complex arrays [len(coords_a), len(coords_b)] on
    the plane's tangential coordinates (missing components are zero);
    ``periods`` / ``k_bloch`` are the transverse unit-cell lengths and Bloch
    wavevector along the plane's two tangential axes."""
    dev = _device(device)
    axis = str(axis).lower()
    tangential = tuple(a for a in "xyz" if a != axis)
    na, nb = len(coords_a), len(coords_b)
    e = np.zeros((na, nb, 3), dtype=np.complex64)
    h = np.zeros((na, nb, 3), dtype=np.complex64)
    for c, lab in enumerate("xyz"):
        if f"E{lab}" in fields:
            e[..., c] = np.asarray(fields[f"E{lab}"])
        if f"H{lab}" in fields:
            h[..., c] = np.asarray(fields[f"H{lab}"])
    k0 = 2.0 * math.pi * float(frequency) / C_0
    orders, reciprocal = enumerate_diffraction_orders(periods=periods, k_bloch=k_bloch, k0=k0,
                                                      background_index=background_index, max_order=max_order)
    ms = sorted({o["m"] for o in orders})
    ns = sorted({o["n"] for o in orders})
    kx = [float(k_bloch[0]) + m * reciprocal[0] for m in ms]
    ky = [float(k_bloch[1]) + n * reciprocal[1] for n in ns]
    amp_e = _plane_amplitudes(e, coords_a, coords_b, kx, ky, dev).cpu().numpy().astype(np.complex128)
    amp_h = _plane_amplitudes(h, coords_a, coords_b, kx, ky, dev).cpu().numpy().astype(np.complex128)
    normal = np.zeros(3)
    normal[_AXIS[axis]] = -1.0 if str(normal_direction) == "-" else 1.0
    area = float(periods[0]) * float(periods[1])
    cutoff = k0 * float(background_index)
    records, total = [], 0.0
    for o in orders:
        ae = amp_e[ms.index(o["m"]), ns.index(o["n"])]
        ah = amp_h[ms.index(o["m"]), ns.index(o["n"])]
        power = float(np.real(np.sum(0.5 * np.cross(ae, np.conj(ah)) * normal))) * area
        total += power
        if o["propagating"]:
            kz = math.sqrt(max(o["kz_squared"], 0.0))
            theta = math.asin(min(math.hypot(o["kx"], o["ky"]) / cutoff, 1.0)) if cutoff > 0.0 else None
        else:
            kz = theta = None
        records.append({"m": o["m"], "n": o["n"], "kx": o["kx"], "ky": o["ky"], "kz": kz,
                        "propagating": o["propagating"], "power": power, "amplitude_E": ae, "amplitude_H": ah,
                        "theta": theta, "phi": math.atan2(o["ky"], o["kx"])})
    propagating_power = sum(r["power"] for r in records if r["propagating"])
    denominator = incident_power if incident_power is not None else propagating_power
    for r in records:
        r["efficiency"] = (r["power"] / denominator
                           if denominator is not None and abs(denominator) > _POWER_FLOOR else None)
    return {
        "kind": "diffraction", "frequency": float(frequency), "axis": axis, "normal_direction": normal_direction,
        "position": float(position), "tangential_axes": tangential,
        "periods": {tangential[0]: float(periods[0]), tangential[1]: float(periods[1])},
        "reciprocal_vectors": {tangential[0]: reciprocal[0], tangential[1]: reciprocal[1]},
        "background_index": float(background_index), "incident_power": incident_power, "total_power": total,
        "propagating_power": propagating_power,
        "num_propagating": sum(1 for r in records if r["propagating"]), "orders": records,
    }


def _trapz_weights(points: np.ndarray) -> np.ndarray:
    """Trapezoid widths of 1-D samples (stratton_chu.py:102-113)."""
    n = points.size
    if n <= 1:
        return np.ones(n)
    d = np.diff(points)
    w = np.empty(n)
    w[0], w[-1] = d[0] / 2.0, d[-1] / 2.0
    if n > 2:
        w[1:-1] = (d[:-1] + d[1:]) / 2.0
    return w


def _cell_centre_weights(points: np.ndarray) -> np.ndarray:
    """Control-volume widths of cell-centred samples (stratton_chu.py:116-129)."""
    n = points.size
    if n <= 1:
        return np.ones(n)
    d = np.diff(points)
    w = np.empty(n)
    w[0], w[-1] = d[0], d[-1]
    if n > 2:
        w[1:-1] = (d[:-1] + d[1:]) / 2.0
    return w


@dataclass
class PlanarEquivalentCurrents:
    """Equivalent surface currents J, M [len(u), len(v), 3] (complex) on the plane
    ``axis`` = position with tangential samples u, v (stratton_chu.py:339-460)."""

    axis: str
    position: float
    frequency: float
    u: np.ndarray
    v: np.ndarray
    J: np.ndarray
    M: np.ndarray
    background_eps_r: float = 1.0
    background_mu_r: float = 1.0
    normal_direction: str = "+"
    quadrature_rule: str = "trapezoidal"

    def quadrature(self):
        """Flattened (points, J weighted, M weighted) with the plane's area weights."""
        u, v = np.asarray(self.u, dtype=np.float64), np.asarray(self.v, dtype=np.float64)
        rule = _cell_centre_weights if self.quadrature_rule == "cell_centered" else _trapz_weights
        w = rule(u)[:, None] * rule(v)[None, :]
        a = _AXIS[str(self.axis).lower()]
        ta, tb = [i for i in range(3) if i != a]
        uu, vv = np.meshgrid(u, v, indexing="ij")
        pts = np.zeros(uu.shape + (3,))
        pts[..., a] = float(self.position)
        pts[..., ta] = uu
        pts[..., tb] = vv
        jw = np.asarray(self.J) * w[..., None]
        mw = np.asarray(self.M) * w[..., None]
        return pts.reshape(-1, 3), jw.reshape(-1, 3), mw.reshape(-1, 3)


class NearFieldFarFieldTransformer:
    """Far fields of one or more planar equivalent-current surfaces in a lossless
    homogeneous background (nfft.py:47-265): k = omega n / c, eta = eta0 sqrt(mu_r /
    eps_r); the radiation integrals run on the GPU."""

    def __init__(self, currents, *, c: float = C_0, eps0: float = EPSILON_0, mu0: float = MU_0,
                 background_eps_r=None, background_mu_r=None, device=None):
        surfaces = list(currents) if isinstance(currents, (list, tuple)) else [currents]
        if not surfaces:
            raise ValueError("no current surfaces")
        self.device = _device(device)
        self.frequency = float(surfaces[0].frequency)
        eps_r = float(surfaces[0].background_eps_r if background_eps_r is None else background_eps_r)
        mu_r = float(surfaces[0].background_mu_r if background_mu_r is None else background_mu_r)
        if eps_r <= 0.0 or mu_r <= 0.0:
            raise ValueError("a lossless background is required")
        self.omega = 2.0 * math.pi * self.frequency
        self.eta0 = math.sqrt(mu0 / eps0)
        self.k = (self.omega / c) * math.sqrt(eps_r * mu_r)
        self.eta = self.eta0 * math.sqrt(mu_r / eps_r)
        pts, jw, mw = [], [], []
        for s in surfaces:
            p, j, m = s.quadrature()
            pts.append(p)
            jw.append(j)
            mw.append(m)
        dev = self.device
        self._points = torch.as_tensor(np.concatenate(pts).astype(np.float32), device=dev).contiguous()
        self._jw = torch.view_as_real(torch.as_tensor(np.concatenate(jw), dtype=torch.complex64)).contiguous().to(dev)
        self._mw = torch.view_as_real(torch.as_tensor(np.concatenate(mw), dtype=torch.complex64)).contiguous().to(dev)

    def transform_directions(self, directions, *, radius=1.0) -> dict:
        d = np.asarray(directions, dtype=np.float64).reshape(-1, 3)
        norms = np.linalg.norm(d, axis=1, keepdims=True)
        if np.any(norms <= 0.0):
            raise ValueError("directions must be non-zero vectors")
        d = d / norms
        r = np.broadcast_to(np.asarray(radius, dtype=np.float64), (d.shape[0],)).copy()
        if np.any(r <= 0.0):
            raise ValueError("radius must be positive")
        dev = self.device
        td = torch.as_tensor(d.astype(np.float32), device=dev).contiguous()
        tr = torch.as_tensor(r.astype(np.float32), device=dev).contiguous()
        e = torch.empty((d.shape[0], 3, 2), dtype=torch.float32, device=dev)
        h = torch.empty_like(e)
        pw = torch.empty((d.shape[0],), dtype=torch.float32, device=dev)
        _lib.check(_lib.load().fdtd_pp_nfft(
            int(self._points.shape[0]), _lib.ptr(self._points), _lib.ptr(self._jw), _lib.ptr(self._mw), int(d.shape[0]),
            _lib.ptr(td), _lib.ptr(tr), float(self.k), float(self.eta), _lib.ptr(e), _lib.ptr(h), _lib.ptr(pw),
            _stream(dev)), "nfft")
        ef, hf = torch.view_as_complex(e), torch.view_as_complex(h)
        return {"directions": td, "radius": tr, "frequency": self.frequency, "E": ef, "H": hf,
                "Ex": ef[:, 0], "Ey": ef[:, 1], "Ez": ef[:, 2], "Hx": hf[:, 0], "Hy": hf[:, 1], "Hz": hf[:, 2],
                "power_density": pw}

    def transform(self, theta, phi, *, radius=1.0) -> dict:
        th, ph = np.broadcast_arrays(np.asarray(theta, dtype=np.float64), np.asarray(phi, dtype=np.float64))
        shape = th.shape
        dirs = np.stack((np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)), axis=-1)
        out = self.transform_directions(dirs.reshape(-1, 3), radius=np.broadcast_to(radius, shape).reshape(-1))
        e = out["E"].reshape(shape + (3,))
        h = out["H"].reshape(shape + (3,))
        dev = self.device
        tt = torch.as_tensor(th, device=dev, dtype=torch.float32)
        pp = torch.as_tensor(ph, device=dev, dtype=torch.float32)
        th_hat = torch.stack((torch.cos(tt) * torch.cos(pp), torch.cos(tt) * torch.sin(pp), -torch.sin(tt)),
                             dim=-1).to(torch.complex64)
        ph_hat = torch.stack((-torch.sin(pp), torch.cos(pp), torch.zeros_like(pp)), dim=-1).to(torch.complex64)
        return {"theta": tt, "phi": pp, "directions": out["directions"].reshape(shape + (3,)),
                "frequency": self.frequency, "E": e, "H": h,
                "Ex": e[..., 0], "Ey": e[..., 1], "Ez": e[..., 2], "Hx": h[..., 0], "Hy": h[..., 1], "Hz": h[..., 2],
                "E_theta": torch.sum(e * th_hat, dim=-1), "E_phi": torch.sum(e * ph_hat, dim=-1),
                "H_theta": torch.sum(h * th_hat, dim=-1), "H_phi": torch.sum(h * ph_hat, dim=-1),
                "power_density": out["power_density"].reshape(shape)}
