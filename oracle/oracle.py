"""CPU oracle for the FDTD hot path -- test infrastructure, not product code.

``OracleSimulation`` steps a compiled scene on the CPU with the reference's
per-step kernel order (witwin/maxwell/fdtd/runtime/stepping.py:1740-1815 and
:2289-2345), calling the plain-C restatements of the reference's per-op kernels
in ``fdtd_oracle.c`` on full Yee-shaped arrays:

    H update (CPML slab psi)           magnetic.cu:145-212
    TFSF H correction, aux H advance   tfsf_apply.py:228-264, sources.cu:803-839
    ADE advance from E^n               dispersive.cu:18-70, materials.py:665-703
    E update (boundary modes, CPML)    electric.cu:242-311, 647-941
    TFSF E correction, aux E advance   tfsf_apply.py:237-264
    soft sources                       sources.cu:135-154, temporal.py:408-491
    ADE subtraction E -= dt J / eps    dispersive.cu:72-83, materials.py:911
    nonlinear E coefficients           dispersive.cu:165-400, materials.py:1664-1770
    full-anisotropy coupling           aniso.cu:26-580, stepping.py:1808-1811
    monitor running DFT                observers.py:577-659, spectral.py:165-232

The DFT phase follows the reference's observer path: a float64 rotation
recurrence per frequency, H samples rotated by -omega*dt/2, result scaled by
2/sum(window).  Precision "f64" is the accuracy oracle; "f32" is the FP32
restatement used as the CPU baseline.  Only tests, smoke() and the benchmark's
CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIBS: dict = {}
_vp = ctypes.c_void_p

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def build(force: bool = False) -> None:
    """Compile the two oracle libraries with the committed Makefile."""
    libs = [HERE / "liboracle_f64.so", HERE / "liboracle_f32.so"]
    src = HERE / "fdtd_oracle.c"
    if not force and all(p.exists() and p.stat().st_mtime >= src.stat().st_mtime for p in libs):
        return
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load(precision: str = "f64") -> ctypes.CDLL:
    if precision not in ("f64", "f32"):
        raise ValueError(precision)
    if precision not in _LIBS:
        path = HERE / f"liboracle_{precision}.so"
        if not path.exists():
            build()
        lib = ctypes.CDLL(str(path))
        real = ctypes.c_double if precision == "f64" else ctypes.c_float
        i, i64 = ctypes.c_int, ctypes.c_int64
        lib.oracle_real_size.restype = i
        lib.oracle_h_update.argtypes = [i, i, i, i, i, i, i] + [_vp] * 15 + [i] * 6
        lib.oracle_e_update.argtypes = [i, i, i, i, i, i, i] + [_vp] * 7 + [i] * 4 + [_vp] * 8 + [i] * 6
        lib.oracle_debye.argtypes = [i64, i64, _vp, _vp, real, real, _vp, _vp]
        lib.oracle_drude.argtypes = [i64, i64, _vp, _vp, real, _vp]
        lib.oracle_lorentz.argtypes = [i64, i64, _vp, _vp, real, real, real, _vp, _vp]
        lib.oracle_apply_polarization.argtypes = [i64, i64, _vp, _vp, real, _vp]
        lib.oracle_add_patch.argtypes = [i, i, i, _vp, i, i, i, _vp, i, i, i, real]
        lib.oracle_add_line_patch.argtypes = [i, i, i, _vp, i, i, i, _vp, _vp, _vp, i, i, i, i, real]
        lib.oracle_aux_magnetic.argtypes = [i, _vp, _vp, _vp, _vp]
        lib.oracle_aux_electric.argtypes = [i, _vp, _vp, _vp, _vp, i, real]
        lib.oracle_point_observers.argtypes = [i, i, _vp, i, _vp, _vp, _vp, _vp, _vp, real, real]
        lib.oracle_plane_observer.argtypes = [i, i, i, _vp, i, i, _vp, _vp, real, real]
        lib.oracle_dft_volume.argtypes = [i64, i64, i64, i, _vp, _vp, _vp, _vp, _vp]
        lib.oracle_clamp_face.argtypes = [i, i, i, _vp, i, i]
        _LIBS[precision] = lib
    return _LIBS[precision]


def _p(a):
    return None if a is None else a.ctypes.data_as(_vp)


def shifted_waveform(source_time, t):
    """Waveform of a time-shifted patch (witwin/maxwell/waveforms.py:83-107) at
    times t: CW A cos(2 pi f t + phase); Gaussian pulse A exp(-(tau 2 pi fwidth)^2 / 2)
    cos(2 pi f tau + phase) with tau = t - delay (delay 6 / (2 pi fwidth) unless
    given)."""
    t = np.asarray(t, dtype=np.float64)
    f = float(source_time.frequency)
    if source_time.kind == "cw":
        return source_time.amplitude * np.cos(2.0 * np.pi * f * t + source_time.phase)
    fw = float(source_time.fwidth)
    centre = 6.0 / (2.0 * np.pi * fw) if source_time.delay is None else float(source_time.delay)
    tau = t - centre
    return source_time.amplitude * np.exp(-0.5 * (tau * 2.0 * np.pi * fw) ** 2) * np.cos(2.0 * np.pi * f * tau
                                                                                        + source_time.phase)


def component_shape(name, nodes):
    nx, ny, nz = nodes
    return {
        "Ex": (nx - 1, ny, nz), "Ey": (nx, ny - 1, nz), "Ez": (nx, ny, nz - 1),
        "Hx": (nx, ny - 1, nz - 1), "Hy": (nx - 1, ny, nz - 1), "Hz": (nx - 1, ny - 1, nz),
    }[name]


def _clamped(f, i, j, k):
    return f[np.clip(i, 0, f.shape[0] - 1), np.clip(j, 0, f.shape[1] - 1), np.clip(k, 0, f.shape[2] - 1)]


def collocate_e(comp, ex, ey, ez):
    """E collocated onto the Yee edges of ``comp`` (witwin/maxwell/fdtd/cuda/
    kernels/dispersive.cu:160-265): the own component as is, the other two as
    the mean of their four surrounding edges, indices clamped to each array."""
    own = {"Ex": ex, "Ey": ey, "Ez": ez}[comp]
    i, j, k = np.meshgrid(*(np.arange(n) for n in own.shape), indexing="ij")
    if comp == "Ex":
        vy = 0.25 * (_clamped(ey, i, j - 1, k) + _clamped(ey, i, j, k) + _clamped(ey, i + 1, j - 1, k)
                     + _clamped(ey, i + 1, j, k))
        vz = 0.25 * (_clamped(ez, i, j, k - 1) + _clamped(ez, i, j, k) + _clamped(ez, i + 1, j, k - 1)
                     + _clamped(ez, i + 1, j, k))
        return ex, vy, vz
    if comp == "Ey":
        vx = 0.25 * (_clamped(ex, i - 1, j, k) + _clamped(ex, i, j, k) + _clamped(ex, i - 1, j + 1, k)
                     + _clamped(ex, i, j + 1, k))
        vz = 0.25 * (_clamped(ez, i, j, k - 1) + _clamped(ez, i, j, k) + _clamped(ez, i, j + 1, k - 1)
                     + _clamped(ez, i, j + 1, k))
        return vx, ey, vz
    vx = 0.25 * (_clamped(ex, i - 1, j, k) + _clamped(ex, i, j, k) + _clamped(ex, i - 1, j, k + 1)
                 + _clamped(ex, i, j, k + 1))
    vy = 0.25 * (_clamped(ey, i, j - 1, k) + _clamped(ey, i, j, k) + _clamped(ey, i, j - 1, k + 1)
                 + _clamped(ey, i, j, k + 1))
    return vx, vy, ez


def _aniso_curl_at(d, s, h, inv, periodic):
    """curl(H)_d at the d-edges with index arrays s = (s0, s1, s2) (kernels/
    aniso.cu:105-215): s_d an edge coordinate, the other two node coordinates;
    returns (value, valid) with the sample skipped where a stencil leaves a
    non-periodic axis (periodic axes wrap, the last node duplicating node 0)."""
    n = [h[0].shape[0], h[1].shape[1], h[2].shape[2]]  # node counts
    s = [np.array(v) for v in s]
    valid = np.ones(np.broadcast(*s).shape, dtype=bool)
    cnt = n[d] - 1
    if periodic[d]:
        s[d] = np.where(s[d] < 0, s[d] + cnt, np.where(s[d] >= cnt, s[d] - cnt, s[d]))
    else:
        valid &= (s[d] >= 0) & (s[d] < cnt)
    pairs = {}
    for ax in range(3):
        if ax == d:
            continue
        if periodic[ax]:
            s[ax] = np.where(s[ax] == n[ax] - 1, 0, s[ax])
        hi, lo = s[ax].copy(), s[ax] - 1
        if periodic[ax]:
            hi = np.where(hi > n[ax] - 2, hi - (n[ax] - 1), hi)
            lo = np.where(lo < 0, lo + (n[ax] - 1), lo)
        else:
            valid &= (hi <= n[ax] - 2) & (lo >= 0)
        pairs[ax] = (lo, hi)
    s = [np.where(valid, v, 0) for v in s]
    pairs = {ax: (np.where(valid, lo, 0), np.where(valid, hi, 0)) for ax, (lo, hi) in pairs.items()}

    def diff(comp, ax):
        lo, hi = pairs[ax]
        a = [s[0], s[1], s[2]]
        b = [s[0], s[1], s[2]]
        a[ax], b[ax] = hi, lo
        return (h[comp][tuple(a)] - h[comp][tuple(b)]) * inv[ax][s[ax]]

    if d == 0:
        value = diff(2, 1) - diff(1, 2)  # dHz/dy - dHy/dz
    elif d == 1:
        value = diff(0, 2) - diff(2, 0)  # dHx/dz - dHz/dx
    else:
        value = diff(1, 0) - diff(0, 1)  # dHy/dx - dHx/dy
    return np.where(valid, value, 0.0), valid


def full_aniso_correction(comp, e, h, coeff_a, coeff_b, inv, periodic=(False, False, False)):
    """E_c += (coeff_a <curlH_a> + coeff_b <curlH_b>) / 4 (kernels/aniso.cu:373-580):
    <curlH_d> sums curl(H)_d over the four d-edges around each E_c edge (own
    axis offsets {0, 1}, curl axis {-1, 0}, the lower axis outermost), skipped
    samples contributing nothing; cells with both coefficients zero unchanged.
    ``h`` = (Hx, Hy, Hz), ``inv`` = per-node inverse spacings; updates e in place."""
    idx = np.meshgrid(*(np.arange(v) for v in e.shape), indexing="ij")
    da, db = (1, 2) if comp == 0 else ((0, 2) if comp == 1 else (0, 1))
    active = (coeff_a != 0) | (coeff_b != 0)
    total = np.zeros(e.shape, dtype=np.result_type(e, coeff_a))
    for coeff, d in ((coeff_a, da), (coeff_b, db)):
        outer, inner = min(comp, d), max(comp, d)
        acc = np.zeros_like(total)
        for u in range(2):
            for v in range(2):
                s = [idx[0].copy(), idx[1].copy(), idx[2].copy()]
                s[outer] += u if outer == comp else u - 1
                s[inner] += v if inner == comp else v - 1
                value, _ = _aniso_curl_at(d, s, h, inv, periodic)
                acc = acc + value
        total = total + coeff * acc
    e[active] += (0.25 * total)[active]
    return e


def kerr_curl(comp, ex, ey, ez, eps, decay, chi3, dt, eps0):
    """Kerr curl coefficient (dispersive.cu:267-321): dt / max(eps + eps0 chi3 |E|^2,
    1e-12 eps0) * decay."""
    vx, vy, vz = collocate_e(comp, ex, ey, ez)
    eff = np.maximum(eps + eps0 * chi3 * (vx * vx + vy * vy + vz * vz), 1.0e-12 * eps0)
    return (dt / eff) * decay


def nonlinear_coefficients(comp, ex, ey, ez, eps, external, sigma, chi2, chi3, tpa, dt, eps0):
    """General instantaneous-nonlinear decay / curl pair (dispersive.cu:323-400):
    eps_eff = eps + eps0 (chi2 E_own + chi3 |E|^2) (floored at 1e-12 eps0),
    sigma_eff = max(sigma + tpa |E|^2, 0), half = sigma_eff dt / (2 eps_eff),
    decay = ext (1 - half) / (1 + half), curl = ext dt / eps_eff / (1 + half)."""
    vx, vy, vz = collocate_e(comp, ex, ey, ez)
    fsq = vx * vx + vy * vy + vz * vz
    own = {"Ex": vx, "Ey": vy, "Ez": vz}[comp]
    eff = np.maximum(eps + eps0 * (chi2 * own + chi3 * fsq), 1.0e-12 * eps0)
    sig = np.maximum(sigma + tpa * fsq, 0.0)
    half = 0.5 * sig * dt / eff
    inv = 1.0 / (1.0 + half)
    return external * (1.0 - half) * inv, external * (dt / eff) * inv


# (a-axis, b-axis, first, second) per component, magnetic.cu:20-212 / electric.cu:242-941
_H_SPEC = {"Hx": (1, 2, "Ey", "Ez"), "Hy": (0, 2, "Ex", "Ez"), "Hz": (0, 1, "Ex", "Ey")}
_E_SPEC = {"Ex": (1, 2, "Hy", "Hz"), "Ey": (0, 2, "Hx", "Hz"), "Ez": (0, 1, "Hx", "Hy")}


class OracleSimulation:
    def __init__(self, compiled, precision: str = "f64", threads: int | None = None):
        self.cs = compiled
        self.precision = precision
        self.lib = load(precision)
        self.dtype = np.float64 if precision == "f64" else np.float32
        self.threads = max(1, int(threads or os.cpu_count() or 1))
        self.pool = ThreadPoolExecutor(self.threads) if self.threads > 1 else None
        cs = compiled
        dt = self.dtype
        nodes = cs.nodes
        self.fields = {n: np.zeros(component_shape(n, nodes), dt) for n in COMPONENTS}
        self.decay = {}
        self.curl = {}
        for n in COMPONENTS:
            shape = component_shape(n, nodes)
            du, cu = cs.uniform[n]
            self.decay[n] = (np.full(shape, du, dt) if cs.decay[n] is None else cs.decay[n].astype(dt))
            self.curl[n] = (np.full(shape, cu, dt) if cs.curl[n] is None else cs.curl[n].astype(dt))
        self.inv_e = [a.astype(dt) for a in cs.inv_e]
        self.inv_h = [a.astype(dt) for a in cs.inv_h]
        self.cp = {k: [a.astype(dt) for a in v] for k, v in cs.cpml.items()}
        self.cpml = any(cs.pml_lo) or any(cs.pml_hi)
        # slab psi in the reference's compressed layout (cpml.py:218-333)
        self.psi = {}
        self.slab = {}
        for n in COMPONENTS:
            spec = _H_SPEC.get(n) or _E_SPEC[n]
            shape = component_shape(n, nodes)
            for which, axis in enumerate(spec[:2]):
                size = shape[axis]
                low = min(cs.pml_lo[axis], size)
                high = min(cs.pml_hi[axis], max(size - low, 0))
                cshape = list(shape)
                cshape[axis] = low + high
                self.psi[(n, which)] = np.zeros(cshape, dt)
                self.slab[(n, which)] = (low, size - high, high)
        # ADE: full-volume drive / state per pole component (materials.py:530-662)
        self.poles = []
        for pole in cs.poles:
            shape = component_shape(pole.component, nodes)
            b = pole.box
            sl = (slice(b[0], b[1]), slice(b[2], b[3]), slice(b[4], b[5]))
            drive = np.zeros(shape, dt)
            drive[sl] = pole.drive
            inv_eps = (1.0 / cs.eps[pole.component]).astype(np.float32).astype(dt)
            inv_eps[sl] = pole.inv_eps
            self.poles.append({
                "comp": pole.component, "kind": pole.kind, "decay": pole.decay, "restoring": pole.restoring,
                "drive": drive, "inv_eps": inv_eps, "P": np.zeros(shape, dt), "J": np.zeros(shape, dt),
            })
        # full anisotropy: the off-diagonal coupling after the E update
        self.aniso = []
        for name, (box, ca, cb) in (getattr(cs, "aniso", None) or {}).items():
            shape = component_shape(name, nodes)
            fa, fb = np.zeros(shape, dt), np.zeros(shape, dt)
            sl = (slice(box[0], box[1]), slice(box[2], box[3]), slice(box[4], box[5]))
            fa[sl], fb[sl] = ca, cb
            self.aniso.append((name, fa, fb))
        # instantaneous nonlinear channels: the E coefficients are recomposed
        # from E^n over every cell before each E update (materials.py:1664-1770)
        self.nl = None
        if getattr(cs, "nonlinear", None) is not None:
            nl = cs.nonlinear
            self.nl = {"general": nl.general, "eps0": nl.eps0,
                       "eps": {n: cs.eps[n].astype(dt) for n in ("Ex", "Ey", "Ez")},
                       "ch": {n: {k: v.astype(dt) for k, v in nl.channels[n].items()} for n in ("Ex", "Ey", "Ez")}}
        self.patches = [(p.component, p.box, p.coeff.astype(dt), p.signal) for p in cs.patches]
        # time-shifted patches: scale * w(n dt + t_offset - delay) per cell, the
        # waveform evaluated in FP64 here (sources.cu:173-221)
        self.shifted = [(p.component, p.box, p.scale.astype(np.float64), p.delay.astype(np.float64), p.t_offset,
                         p.source_time) for p in getattr(cs, "shifted", [])]
        self.aux = None
        if cs.aux_line is not None:
            a = cs.aux_line
            ne = a.e_decay.size
            self.aux = {
                "e": np.zeros(ne, dt), "h": np.zeros(ne - 1, dt),
                "ed": a.e_decay.astype(dt), "ec": a.e_curl.astype(dt),
                "hd": a.h_decay.astype(dt), "hc": a.h_curl.astype(dt),
                "src": a.source_index, "signal": a.source,
            }
        self.lines = [
            (lp.component, lp.box, lp.coeff.astype(dt), lp.sample_kind, lp.sample_axis,
             lp.sample_index.astype(np.int64), lp.scale)
            for lp in cs.line_patches
        ]
        # monitor running DFT state (observers.py:409-659)
        self.freqs = np.asarray(cs.frequencies, dtype=np.float64)
        nf = self.freqs.size
        self.acc = []
        for reg in cs.regions:
            b = reg.box
            shape = (nf, b[1] - b[0], b[3] - b[2], b[5] - b[4])
            self.acc.append([np.zeros(shape, dt), np.zeros(shape, dt)])
        omega = 2.0 * np.pi * self.freqs
        self.phase_step_cos = np.cos(omega * cs.dt)
        self.phase_step_sin = np.sin(omega * cs.dt)
        self.h_off_cos = np.cos(-0.5 * omega * cs.dt)
        self.h_off_sin = np.sin(-0.5 * omega * cs.dt)
        self.phase_cos = np.ones(nf)
        self.phase_sin = np.zeros(nf)
        self.window_sum = 0.0
        self.step = 0

    # ------------------------------------------------------------------ utils
    def _split(self, nx, fn):
        if self.pool is None or nx < 2 * self.threads:
            fn(0, nx)
            return
        edges = np.linspace(0, nx, self.threads + 1).astype(int)
        futures = [self.pool.submit(fn, int(a), int(b)) for a, b in zip(edges[:-1], edges[1:]) if b > a]
        for f in futures:
            f.result()

    def _split_flat(self, n, fn):
        if self.pool is None or n < 1 << 16:
            fn(0, n)
            return
        edges = np.linspace(0, n, self.threads + 1).astype(np.int64)
        futures = [self.pool.submit(fn, int(a), int(b)) for a, b in zip(edges[:-1], edges[1:]) if b > a]
        for f in futures:
            f.result()

    # ------------------------------------------------------------------- ops
    def update_h(self):
        F = self.fields
        mode = 2 if self.cpml else 0
        for n, (A, B, first, second) in _H_SPEC.items():
            shape = F[n].shape
            pa, pb = self.psi[(n, 0)], self.psi[(n, 1)]
            sa, sb = self.slab[(n, 0)], self.slab[(n, 1)]
            cp = self.cp
            args = (n, A, B, first, second, pa, pb, sa, sb)

            def run(i0, i1, n=n, A=A, B=B, first=first, second=second, pa=pa, pb=pb, sa=sa, sb=sb, shape=shape):
                self.lib.oracle_h_update(
                    i0, i1, "xyz".index(n[1]), mode, shape[0], shape[1], shape[2], _p(F[n]), _p(F[first]),
                    _p(F[second]), _p(self.decay[n]), _p(self.curl[n]), _p(self.inv_h[A]), _p(self.inv_h[B]),
                    _p(pa), _p(pb), _p(cp["ik_h"][A]), _p(cp["b_h"][A]), _p(cp["c_h"][A]), _p(cp["ik_h"][B]),
                    _p(cp["b_h"][B]), _p(cp["c_h"][B]), sa[0], sa[1], sa[2], sb[0], sb[1], sb[2])

            del args
            self._split(shape[0], run)

    def update_e(self):
        F = self.fields
        mode = 2 if self.cpml else 0
        bnd = self.cs.boundary
        for n, (A, B, first, second) in _E_SPEC.items():
            shape = F[n].shape
            pa, pb = self.psi[(n, 0)], self.psi[(n, 1)]
            sa, sb = self.slab[(n, 0)], self.slab[(n, 1)]
            cp = self.cp

            def run(i0, i1, n=n, A=A, B=B, first=first, second=second, pa=pa, pb=pb, sa=sa, sb=sb, shape=shape):
                self.lib.oracle_e_update(
                    i0, i1, "xyz".index(n[1]), mode, shape[0], shape[1], shape[2], _p(F[n]), _p(F[first]),
                    _p(F[second]), _p(self.decay[n]), _p(self.curl[n]), _p(self.inv_e[A]), _p(self.inv_e[B]),
                    bnd[2 * A], bnd[2 * A + 1], bnd[2 * B], bnd[2 * B + 1], _p(pa), _p(pb), _p(cp["ik_e"][A]),
                    _p(cp["b_e"][A]), _p(cp["c_e"][A]), _p(cp["ik_e"][B]), _p(cp["b_e"][B]), _p(cp["c_e"][B]),
                    sa[0], sa[1], sa[2], sb[0], sb[1], sb[2])

            self._split(shape[0], run)

    def advance_ade(self):
        F = self.fields
        dt = self.cs.dt
        for p in self.poles:
            e = F[p["comp"]]
            n = e.size
            if p["kind"] == 0:
                self._split_flat(n, lambda a, b, p=p, e=e: self.lib.oracle_debye(
                    a, b, _p(e), _p(p["drive"]), p["decay"], dt, _p(p["P"]), _p(p["J"])))
            elif p["kind"] == 1:
                self._split_flat(n, lambda a, b, p=p, e=e: self.lib.oracle_drude(
                    a, b, _p(e), _p(p["drive"]), p["decay"], _p(p["J"])))
            else:
                self._split_flat(n, lambda a, b, p=p, e=e: self.lib.oracle_lorentz(
                    a, b, _p(e), _p(p["drive"]), p["decay"], p["restoring"], dt, _p(p["P"]), _p(p["J"])))

    def apply_ade(self):
        F = self.fields
        dt = self.cs.dt
        for p in self.poles:
            e = F[p["comp"]]
            # nonlinear scenes: J times this step's curl coefficient, dt 1 (materials.py:751-773)
            coef, apply_dt = (self.curl[p["comp"]], 1.0) if self.nl is not None else (p["inv_eps"], dt)
            self._split_flat(e.size, lambda a, b, p=p, e=e, coef=coef, apply_dt=apply_dt:
                             self.lib.oracle_apply_polarization(a, b, _p(p["J"]), _p(coef), apply_dt, _p(e)))

    def update_nonlinear(self):
        F = self.fields
        nl = self.nl
        # the reference's kernels take dt and eps0 as float (dispersive.cu:284-285)
        dt, eps0 = float(np.float32(self.cs.dt)), float(np.float32(nl["eps0"]))
        out = {}
        for n in ("Ex", "Ey", "Ez"):
            ch, eps = nl["ch"][n], nl["eps"][n]
            if nl["general"]:
                out[n] = nonlinear_coefficients(n, F["Ex"], F["Ey"], F["Ez"], eps, ch["decay"], ch["sigma"], ch["chi2"],
                                                ch["chi3"], ch["tpa"], dt, eps0)
            else:
                out[n] = (None, kerr_curl(n, F["Ex"], F["Ey"], F["Ez"], eps, ch["decay"], ch["chi3"], dt, eps0))
        for n, (d, c) in out.items():
            if d is not None:
                self.decay[n][...] = d
            self.curl[n][...] = c

    def _line_corrections(self, magnetic: bool):
        if self.aux is None:
            return
        sample = self.aux["e"] if magnetic else self.aux["h"]
        for comp, box, coeff, kind, axis, idx, scale in self.lines:
            if (comp[0] == "H") != magnetic:
                continue
            f = self.fields[comp]
            pshape = coeff.shape
            self.lib.oracle_add_line_patch(f.shape[0], f.shape[1], f.shape[2], _p(f), pshape[0], pshape[1], pshape[2],
                                           _p(coeff), _p(sample), _p(idx), axis, box[0], box[2], box[4], scale)

    def _soft_terms(self, n: int, magnetic: bool):
        """Soft patches of one phase: H components right after the H update
        (stepping.py:1776-1777), E components after the E update (:2300-2308)."""
        F = self.fields
        for comp, box, coeff, signal in self.patches:
            if (comp[0] == "H") != magnetic:
                continue
            f = F[comp]
            self.lib.oracle_add_patch(f.shape[0], f.shape[1], f.shape[2], _p(f), coeff.shape[0], coeff.shape[1],
                                      coeff.shape[2], _p(coeff), box[0], box[2], box[4], float(signal[n]))
        for comp, box, scale, delay, t_off, st in self.shifted:
            if (comp[0] == "H") != magnetic:
                continue
            value = np.ascontiguousarray(scale * shifted_waveform(st, n * self.cs.dt + t_off - delay), dtype=self.dtype)
            f = F[comp]
            self.lib.oracle_add_patch(f.shape[0], f.shape[1], f.shape[2], _p(f), value.shape[0], value.shape[1],
                                      value.shape[2], _p(value), box[0], box[2], box[4], 1.0)

    def step_once(self):
        n = self.step
        self.update_h()
        if self.aux is not None:
            self._line_corrections(True)
            a = self.aux
            self.lib.oracle_aux_magnetic(a["e"].size, _p(a["h"]), _p(a["e"]), _p(a["hd"]), _p(a["hc"]))
        self._soft_terms(n, True)
        self.advance_ade()
        if self.nl is not None:
            self.update_nonlinear()
        self.update_e()
        for name, fa, fb in self.aniso:  # stepping.py:1808-1811
            full_aniso_correction("xyz".index(name[1]), self.fields[name],
                                  (self.fields["Hx"], self.fields["Hy"], self.fields["Hz"]), fa, fb, self.inv_e)
        if self.aux is not None:
            self._line_corrections(False)
            a = self.aux
            self.lib.oracle_aux_electric(a["e"].size, _p(a["e"]), _p(a["h"]), _p(a["ed"]), _p(a["ec"]), a["src"],
                                         float(a["signal"][n]))
        self._soft_terms(n, False)
        self.apply_ade()
        if self.aux is None:
            self._clamp_pec()
        self._accumulate(n)
        self.step += 1

    def _clamp_pec(self):
        bnd = self.cs.boundary
        # enforce_pec_boundaries (stepping.py:1450): tangential E on PEC faces
        for n, (A, B, _, _) in _E_SPEC.items():
            f = self.fields[n]
            for axis in (A, B):
                for side in (0, 1):
                    if bnd[2 * axis + side] == 4:
                        self.lib.oracle_clamp_face(f.shape[0], f.shape[1], f.shape[2], _p(f), axis, side)

    def _accumulate(self, n):
        cs = self.cs
        if self.freqs.size == 0 or not cs.regions:
            return
        # one weight per step, or one per (step, frequency)
        w = np.broadcast_to(np.asarray(cs.window[n], dtype=np.float64), self.phase_cos.shape)
        wc = w * self.phase_cos
        ws = w * self.phase_sin
        hc = wc * self.h_off_cos - ws * self.h_off_sin
        hs = ws * self.h_off_cos + wc * self.h_off_sin
        dt = self.dtype
        for reg, (re, im) in zip(cs.regions, self.acc):
            b = reg.box
            v = self.fields[reg.component][b[0]:b[1], b[2]:b[3], b[4]:b[5]]
            ccos, csin = (wc, ws) if reg.component[0] == "E" else (hc, hs)
            for f in range(self.freqs.size):
                re[f] += v * dt(ccos[f])
                im[f] += v * dt(csin[f])
        self.window_sum += w
        nc = self.phase_cos * self.phase_step_cos - self.phase_sin * self.phase_step_sin
        ns = self.phase_sin * self.phase_step_cos + self.phase_cos * self.phase_step_sin
        self.phase_cos, self.phase_sin = nc, ns

    def run(self, steps: int):
        for _ in range(int(steps)):
            self.step_once()
        return self

    def monitor_results(self) -> dict:
        cs = self.cs
        total = np.broadcast_to(np.asarray(self.window_sum, dtype=np.float64), self.freqs.shape)
        scale = np.zeros(self.freqs.shape)
        np.divide(2.0, total, out=scale, where=total > 0)
        out: dict = {}
        for reg, (re, im) in zip(cs.regions, self.acc):
            fidx = [cs.frequencies.index(f) for f in cs.monitor_frequencies[reg.monitor]]
            sc = scale[fidx].reshape((-1,) + (1,) * (re.ndim - 1))
            data = (re[fidx].astype(np.float64) + 1j * im[fidx].astype(np.float64)) * sc
            out.setdefault(reg.monitor, {})[reg.component] = data
        return out

    def close(self):
        if self.pool is not None:
            self.pool.shutdown()
            self.pool = None
