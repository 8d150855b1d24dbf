"""Scene description and compilation into the solver-scene tensors of the hot path.

The reference compiles a ``witwin.maxwell.Scene`` (through the ``witwin.core``
geometry layer) into per-Yee-component tensors: permittivities, update
coefficients, CPML profiles, ADE drive templates, source patches and monitor
index sets (witwin/maxwell/scene.py:1260-1481, fdtd/runtime/materials.py,
fdtd/boundary/cpml.py, fdtd/excitation/*, fdtd/observers.py).  This module
produces the same tensors for scenes built from axis-aligned boxes and spheres
on a uniform grid, which is what the FDTD hot path consumes.  Geometry
rasterisation is node-based (a node is inside a structure or not) followed by
the reference's node-to-Yee-component averaging
(fdtd/runtime/materials.py:399-407); the reference's subpixel smoothing of
arbitrary geometry belongs to the scene compiler and is not part of this
package.

Everything here is host-side numpy in float64 with float32 results, as in the
reference.  Cell-index coordinates are node indices of the full grid
(CPML cells included): node i sits at x = i * dx.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Sequence

import numpy as np

# CODATA 2018 constants, witwin/maxwell/constants.py:24-36.
EPSILON_0 = 8.8541878128e-12
MU_0 = 1.25663706212e-6
C_0 = 299792458.0
ETA_0 = 376.730313668

BOUNDARY_NONE = 0
BOUNDARY_PML = 1
BOUNDARY_PERIODIC = 2
BOUNDARY_BLOCH = 3
BOUNDARY_PEC = 4
BOUNDARY_PMC = 5

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
COMP_INDEX = {name: idx for idx, name in enumerate(COMPONENTS)}

# Default CPML grading, witwin/maxwell/fdtd/boundary/cpml.py:9-21.
DEFAULT_CPML_CONFIG = {"grading_order": 3.0, "kappa_max": 1.0, "alpha_max": 0.0, "reflection": 1e-6}
# Point dipole reference width, witwin/maxwell/sources.py:21.
POINT_DIPOLE_REFERENCE_WIDTH = 0.02
# TFSF auxiliary line absorber, witwin/maxwell/fdtd/excitation/tfsf_state.py:46.
TFSF_ABSORBER_CELLS = 20


def component_shape(name: str, nodes: Sequence[int]) -> tuple[int, int, int]:
    """Yee shape of a component on a node grid (witwin/maxwell/fdtd/runtime/stepping.py:1625-1630)."""
    nx, ny, nz = (int(v) for v in nodes)
    return {
        "Ex": (nx - 1, ny, nz),
        "Ey": (nx, ny - 1, nz),
        "Ez": (nx, ny, nz - 1),
        "Hx": (nx, ny - 1, nz - 1),
        "Hy": (nx - 1, ny, nz - 1),
        "Hz": (nx - 1, ny - 1, nz),
    }[name]


# --------------------------------------------------------------------------
# Source time functions (witwin/maxwell/sources.py:181-330, waveforms.py:30-61)
# --------------------------------------------------------------------------
@dataclass(frozen=True)
class GaussianPulse:
    frequency: float
    fwidth: float
    amplitude: float = 1.0
    phase: float = 0.0
    delay: float | None = None
    kind: str = "gaussian_pulse"

    @property
    def sigma_t(self) -> float:
        return 1.0 / (2.0 * math.pi * self.fwidth)

    @property
    def resolved_delay(self) -> float:
        return 6.0 * self.sigma_t if self.delay is None else float(self.delay)

    def evaluate(self, t: float) -> float:
        tau = float(t) - self.resolved_delay
        envelope = math.exp(-0.5 * (tau / self.sigma_t) ** 2)
        return self.amplitude * envelope * math.cos(2.0 * math.pi * self.frequency * tau + self.phase)

    @property
    def characteristic_frequency(self) -> float:
        return max(self.frequency, self.frequency + 3.0 * self.fwidth)


@dataclass(frozen=True)
class CW:
    """Continuous wave A cos(2 pi f t + phase).  ``ramp_time`` > 0 multiplies it by a
    raised-cosine turn-on 0.5 (1 - cos(pi t / ramp_time)) for t < ramp_time; the
    reference's CW (ramp_time 0) starts at full amplitude."""

    frequency: float
    amplitude: float = 1.0
    phase: float = 0.0
    ramp_time: float = 0.0
    kind: str = "cw"

    def ramp(self, t: float) -> float:
        if self.ramp_time <= 0.0 or t >= self.ramp_time:
            return 1.0
        return 0.5 * (1.0 - math.cos(math.pi * max(float(t), 0.0) / self.ramp_time))

    def evaluate(self, t: float) -> float:
        return self.ramp(t) * self.amplitude * math.cos(2.0 * math.pi * self.frequency * float(t) + self.phase)

    @property
    def characteristic_frequency(self) -> float:
        return self.frequency


@dataclass(frozen=True)
class CustomSourceTime:
    """Sampled waveform table, linear interpolation, zero outside (waveforms.py:63-66)."""

    times: tuple[float, ...]
    amplitudes: tuple[float, ...]
    frequency: float = 0.0
    kind: str = "custom"

    def evaluate(self, t: float) -> float:
        return float(np.interp(float(t), self.times, self.amplitudes, left=0.0, right=0.0))

    @property
    def characteristic_frequency(self) -> float:
        return self.frequency


def ramped_cw(frequency: float, ramp_steps: int, dt: float, total_steps: int, amplitude: float = 1.0) -> CustomSourceTime:
    """CW with a raised-cosine ramp over the first ``ramp_steps`` steps, as a sampled table."""
    times = np.arange(total_steps + 1, dtype=np.float64) * dt
    ramp = np.where(
        np.arange(total_steps + 1) < ramp_steps,
        0.5 * (1.0 - np.cos(np.pi * np.arange(total_steps + 1) / max(ramp_steps, 1))),
        1.0,
    )
    values = amplitude * ramp * np.cos(2.0 * np.pi * frequency * times)
    return CustomSourceTime(tuple(times.tolist()), tuple(values.tolist()), frequency=frequency)


# --------------------------------------------------------------------------
# Media (witwin/maxwell/media.py:125-215, 1050-1113)
# --------------------------------------------------------------------------
@dataclass(frozen=True)
class DebyePole:
    delta_eps: float
    tau: float


@dataclass(frozen=True)
class DrudePole:
    plasma_frequency: float  # Hz; 2*pi applied at compile (media.py:149-155)
    gamma: float  # Hz


@dataclass(frozen=True)
class LorentzPole:
    delta_eps: float
    resonance_frequency: float  # Hz
    gamma: float  # Hz


@dataclass(frozen=True)
class Medium:
    """A material (witwin/maxwell/media.py): relative permittivity, dispersive
    poles, diagonal or full (symmetric) anisotropy, static conductivity ``sigma`` (S/m) and the
    instantaneous nonlinear channels: Kerr ``kerr_chi3`` (m^2/V^2), ``chi2``
    (m/V) and two-photon absorption ``tpa_beta`` (m/W; conductivity
    tpa_sigma |E|^2, media.py:395-423)."""

    eps_r: float = 1.0
    poles: tuple = ()
    eps_diag: tuple[float, float, float] | None = None  # diagonal anisotropy (eps_xx, eps_yy, eps_zz)
    # off-diagonal relative permittivity (eps_xy, eps_xz, eps_yz) of a full symmetric tensor
    eps_offdiag: tuple[float, float, float] | None = None
    sigma: float = 0.0
    kerr_chi3: float = 0.0
    chi2: float = 0.0
    tpa_beta: float = 0.0
    tpa_index: float | None = None  # n0 of the TPA scale; sqrt(eps_r) when None

    @property
    def tpa_sigma(self) -> float:
        """sigma_NL / |E|^2 = (4/3) beta (n0 eps0 c0)^2 (media.py:420-423, 884-893)."""
        if self.tpa_beta == 0.0:
            return 0.0
        n0 = float(self.tpa_index) if self.tpa_index is not None else math.sqrt(float(self.eps_r))
        return (4.0 / 3.0) * float(self.tpa_beta) * (n0 * EPSILON_0 * C_0) ** 2

    @staticmethod
    def debye(eps_inf: float, delta_eps: float, tau: float) -> "Medium":
        return Medium(eps_r=eps_inf, poles=(DebyePole(delta_eps, tau),))

    @staticmethod
    def drude(plasma_frequency: float, gamma: float, eps_inf: float = 1.0) -> "Medium":
        return Medium(eps_r=eps_inf, poles=(DrudePole(plasma_frequency, gamma),))

    @staticmethod
    def lorentz(eps_inf: float, delta_eps: float, resonance_frequency: float, gamma: float) -> "Medium":
        return Medium(eps_r=eps_inf, poles=(LorentzPole(delta_eps, resonance_frequency, gamma),))

    def axis_eps(self, axis: int) -> float:
        return float(self.eps_diag[axis]) if self.eps_diag is not None else float(self.eps_r)


# --------------------------------------------------------------------------
# Geometry in node-index coordinates
# --------------------------------------------------------------------------
@dataclass(frozen=True)
class Box:
    """Cells [lo, hi) per axis, i.e. nodes lo..hi inclusive."""

    lo: tuple[float, float, float]
    hi: tuple[float, float, float]

    def node_mask(self, nodes: Sequence[int]) -> np.ndarray:
        axes = [np.arange(n, dtype=np.float64) for n in nodes]
        m = [(a >= lo) & (a <= hi) for a, lo, hi in zip(axes, self.lo, self.hi)]
        return m[0][:, None, None] & m[1][None, :, None] & m[2][None, None, :]


@dataclass(frozen=True)
class Sphere:
    center: tuple[float, float, float]
    radius: float

    def node_mask(self, nodes: Sequence[int]) -> np.ndarray:
        x = np.arange(nodes[0], dtype=np.float64)[:, None, None] - self.center[0]
        y = np.arange(nodes[1], dtype=np.float64)[None, :, None] - self.center[1]
        z = np.arange(nodes[2], dtype=np.float64)[None, None, :] - self.center[2]
        return x * x + y * y + z * z <= self.radius * self.radius


@dataclass(frozen=True)
class Structure:
    geometry: object
    medium: Medium


@dataclass(frozen=True)
class MaterialRegion:
    """Design region with per-cell relative permittivity (witwin/maxwell/scene.py:567-610).

    ``eps_r`` holds one value per cell of ``box`` (shape hi - lo); node values
    take the cell's value for the cell whose low corner is the node.
    """

    lo: tuple[int, int, int]
    hi: tuple[int, int, int]
    eps_r: np.ndarray


# --------------------------------------------------------------------------
# Sources and monitors
# --------------------------------------------------------------------------
@dataclass(frozen=True)
class PointDipole:
    position: tuple[float, float, float]  # node-index coordinates
    polarization: str  # "Ex" | "Ey" | "Ez"
    source_time: object
    width: float | None = None  # metres; default POINT_DIPOLE_REFERENCE_WIDTH


@dataclass(frozen=True)
class PlaneSource:
    """Soft current sheet on the plane ``index`` normal to ``axis`` driving the
    tangential component ``polarization`` over the whole plane, with the
    transverse phase profile e^{i (k_x x + k_y y)} of the scene's Bloch
    wavevector (a uniform sheet when it is zero).  The coefficient is the
    component's -dt/eps times the inverse spacing along ``axis`` (a surface
    current J_s adds -dt J_s / (eps d) to E, as injection.py:807-970 does for
    soft surface sources)."""

    axis: int
    index: int
    polarization: str
    source_time: object


@dataclass(frozen=True)
class GaussianBeam:
    """Soft Gaussian beam (witwin/maxwell/sources.py:615-655) launched by the
    surface-equivalent currents of one face, J_s = n x H_inc on the E components and
    M_s = -n x E_inc on the H components, over the whole plane normal to the
    injection axis (excitation/injection.py:807-968), with the beam's amplitude and
    per-cell delay (excitation/spatial.py:175-251) and unit forward power.

    ``focus`` is in node-index coordinates (node i at x = i * spacing), ``beam_waist``
    in metres.  The launch plane sits 5 % of the physical span inside the CPML edge
    on the side the beam comes from (spatial.py:64-77).  A CW source time gives
    cos / sin phased patches (the delay folded into their phase), a pulse gives
    time-shifted patches (the waveform evaluated at t - delay per cell)."""

    direction: tuple[float, float, float]
    polarization: tuple[float, float, float]
    beam_waist: float
    focus: tuple[float, float, float]
    source_time: object
    injection_axis: int | None = None


@dataclass(frozen=True)
class PlaneWaveTFSF:
    """Axis-aligned plane wave injected through a TFSF box (or slab along the propagation axis)."""

    direction: tuple[int, int, int]  # e.g. (1, 0, 0)
    polarization: tuple[float, float, float]  # e.g. (0, 0, 1)
    source_time: object
    lower: tuple[int, int, int]  # TF box node indices
    upper: tuple[int, int, int]
    slab: bool = False


@dataclass(frozen=True)
class PlaneMonitor:
    name: str
    axis: int
    index: int
    components: tuple[str, ...] = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    frequencies: tuple[float, ...] = ()
    lo: tuple[int, int] | None = None  # in-plane bounds (optional finite plane)
    hi: tuple[int, int] | None = None


@dataclass(frozen=True)
class PointMonitor:
    name: str
    index: tuple[int, int, int]
    components: tuple[str, ...] = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    frequencies: tuple[float, ...] = ()


@dataclass(frozen=True)
class VolumeMonitor:
    """Running DFT of whole field components over a box of cells (the full grid
    by default): the reference's full-field DFT (runtime/spectral.py:309-652,
    kernels/spectral.cu:9-146, E components by default), accumulated through
    the engine's monitor sample ring and batched flush like every monitor."""

    name: str
    components: tuple[str, ...] = ("Ex", "Ey", "Ez")
    frequencies: tuple[float, ...] = ()
    lo: tuple[int, int, int] | None = None
    hi: tuple[int, int, int] | None = None


def tangential_components(axis: int) -> tuple[str, ...]:
    """Tangential field components of a monitor plane (witwin/maxwell/monitors.py:71-77)."""
    return {0: ("Ey", "Ez", "Hy", "Hz"), 1: ("Ex", "Ez", "Hx", "Hz"), 2: ("Ex", "Ey", "Hx", "Hy")}[axis]


def flux_monitor(name: str, axis: int, index: int, frequencies, lo=None, hi=None) -> PlaneMonitor:
    return PlaneMonitor(name, axis, index, tangential_components(axis), tuple(frequencies), lo, hi)


def closed_box_monitor(name: str, lo: Sequence[int], hi: Sequence[int], frequencies) -> list[PlaneMonitor]:
    """Six finite flux planes bounding [lo, hi] (witwin/maxwell/monitors.py:323-376)."""
    faces = []
    for axis in range(3):
        others = [a for a in range(3) if a != axis]
        plo = (int(lo[others[0]]), int(lo[others[1]]))
        phi = (int(hi[others[0]]), int(hi[others[1]]))
        for side, index in (("lo", lo[axis]), ("hi", hi[axis])):
            faces.append(flux_monitor(f"{name}_{'xyz'[axis]}{side}", axis, int(index), frequencies, plo, phi))
    return faces


@dataclass
class Scene:
    """A uniform-grid scene: cells per axis (CPML included), spacing and content."""

    cells: tuple[int, int, int]
    spacing: float
    pml_cells: int = 10
    boundary: tuple[int, int, int, int, int, int] = (BOUNDARY_PML,) * 6
    structures: list = field(default_factory=list)
    material_regions: list = field(default_factory=list)
    sources: list = field(default_factory=list)
    monitors: list = field(default_factory=list)
    courant: float = 0.99
    dt: float | None = None
    # Bloch wavevector (rad/m) of the x / y Bloch faces: the field on the high
    # face is e^{i k L} times the field on the low face
    # (witwin/maxwell/fdtd/boundary/bloch.py:79-90).
    bloch_k: tuple[float, float, float] | str = (0.0, 0.0, 0.0)  # or "auto": from the CW TFSF plane wave

    @property
    def nodes(self) -> tuple[int, int, int]:
        return tuple(int(c) + 1 for c in self.cells)

    def resolve_dt(self) -> float:
        # Courant-scaled 3-D stability limit, fdtd/solver.py:145-159 (dt2 term).
        if self.dt is not None:
            return float(self.dt)
        d = float(self.spacing)
        return float(self.courant) / (C_0 * math.sqrt(3.0 / (d * d)))

    def pml_lengths(self) -> tuple[list[int], list[int]]:
        lo = [self.pml_cells if self.boundary[2 * a] == BOUNDARY_PML else 0 for a in range(3)]
        hi = [self.pml_cells if self.boundary[2 * a + 1] == BOUNDARY_PML else 0 for a in range(3)]
        return lo, hi


# --------------------------------------------------------------------------
# Compiled scene (the hot path's inputs)
# --------------------------------------------------------------------------
@dataclass
class CompiledPole:
    component: str  # "Ex" | "Ey" | "Ez"
    kind: int  # 0 Debye, 1 Drude, 2 Lorentz
    decay: float
    restoring: float
    box: tuple[int, int, int, int, int, int]
    drive: np.ndarray  # box-dense float32
    inv_eps: np.ndarray  # box-dense float32


@dataclass
class CompiledPatch:
    component: str
    box: tuple[int, int, int, int, int, int]
    coeff: np.ndarray  # box-dense float32
    signal: np.ndarray  # float32 per step
    channel: int = 0  # 0: the (real part of the) field, 1: the imaginary part of a Bloch field


@dataclass
class CompiledShiftedPatch:
    """Time-shifted patch (witwin/maxwell/fdtd/cuda/kernels/sources.cu:173-221): comp
    gets scale[cell] * w(n * dt + t_offset - delay[cell]) at step n, w the analytic
    waveform of ``source_time`` (a GaussianPulse, or a CW without ramp)."""

    component: str
    box: tuple[int, int, int, int, int, int]
    scale: np.ndarray  # box-dense float32
    delay: np.ndarray  # box-dense float32, seconds
    t_offset: float  # 0 for H components, dt / 2 for E components
    source_time: object
    channel: int = 0  # 0 real, 1 imaginary part of a complex (Bloch) field


@dataclass
class CompiledLinePatch:
    component: str
    box: tuple[int, int, int, int, int, int]
    coeff: np.ndarray
    sample_kind: int  # 0 = incident E history, 1 = incident H history
    sample_axis: int
    sample_index: np.ndarray  # int32, one per coordinate along sample_axis
    scale: float


@dataclass
class CompiledAuxLine:
    e_decay: np.ndarray
    e_curl: np.ndarray
    h_decay: np.ndarray
    h_curl: np.ndarray
    source_index: int
    source: np.ndarray  # float32 per step


@dataclass
class CompiledRegion:
    monitor: str
    component: str
    box: tuple[int, int, int, int, int, int]


@dataclass
class CompiledScene:
    nodes: tuple[int, int, int]
    spacing: float
    dt: float
    time_steps: int
    boundary: tuple[int, ...]
    pml_lo: list[int]
    pml_hi: list[int]
    inv_e: list[np.ndarray]
    inv_h: list[np.ndarray]
    cpml: dict  # b_e, c_e, ik_e, b_h, c_h, ik_h -> list per axis
    eps: dict  # Ex, Ey, Ez absolute permittivity (float32, Yee shapes)
    decay: dict  # component -> array or None
    curl: dict
    uniform: dict  # component -> (decay_value | None, curl_value | None)
    poles: list
    patches: list
    aux_line: CompiledAuxLine | None
    line_patches: list
    regions: list
    frequencies: tuple[float, ...]
    monitor_frequencies: dict
    window: np.ndarray  # float64 per step
    design: MaterialRegion | None = None
    # Bloch faces: the field is complex (real and imaginary channels) and the
    # wrap phase of axis a is bloch_cos[a] + i bloch_sin[a] = e^{i k_a L_a}.
    complex_fields: bool = False
    bloch_cos: tuple[float, float, float] = (1.0, 1.0, 1.0)
    bloch_sin: tuple[float, float, float] = (0.0, 0.0, 0.0)
    shifted: list = field(default_factory=list)  # CompiledShiftedPatch
    nonlinear: "CompiledNonlinear | None" = None
    # full anisotropy: component -> (box, coeff_a, coeff_b), box-dense
    # off-diagonal coupling coefficients dt inv_cd / eps0 (lower axis first)
    aniso: dict | None = None

    @property
    def cells(self) -> int:
        return int(np.prod([n - 1 for n in self.nodes]))


@dataclass
class CompiledNonlinear:
    """Instantaneous nonlinear channels on the E components
    (witwin/maxwell/fdtd/runtime/materials.py:164-217): per component the
    static decay (Kerr form) or external decay (general form, ones here: CPML is
    not folded into the coefficients), the static conductivity and the chi2,
    chi3 and TPA channels, averaged onto the Yee edges (float32, Yee shapes).
    general: some chi2 or TPA channel is nonzero, and both the decay and the
    curl coefficients are recomposed every step; else only the Kerr curl."""

    general: bool
    eps0: float
    channels: dict  # component -> {"decay", "sigma", "chi2", "chi3", "tpa"}

    def active(self, name: str) -> np.ndarray:
        """Cells whose coefficients change with the field."""
        ch = self.channels[name]
        m = ch["chi3"] != 0
        if self.general:
            m = m | (ch["chi2"] != 0) | (ch["tpa"] != 0)
        return m


_ANISO_ROWS = {"Ex": ("xy", "xz"), "Ey": ("xy", "yz"), "Ez": ("xz", "yz")}
_ANISO_DIAG = {"Ex": "xx", "Ey": "yy", "Ez": "zz"}


def _full_aniso(eps_node, offdiag_node, dt):
    """Per-edge inverse permittivity tensors (witwin/maxwell/fdtd/runtime/
    materials.py:272-398, 1421-1440), in float32 like the reference: the six
    relative node tensors averaged onto each E component's edges, inverted in
    closed form; the diagonal entry gives the effective permittivity of the
    base curl coefficient (eps0 / inv_ii), the two off-diagonal entries of the
    component's row the coupling coefficients dt inv / eps0.  Returns
    ({component: eps_eff}, {component: (box, coeff_a, coeff_b)}) with the box
    the bounding box of the nonzero coefficients."""
    f32 = np.float32
    node = {"xx": eps_node[0], "yy": eps_node[1], "zz": eps_node[2], **offdiag_node}
    node = {k: v.astype(f32) for k, v in node.items()}
    scale = f32(dt / EPSILON_0)
    eps_eff, aniso = {}, {}
    for name in ("Ex", "Ey", "Ez"):
        axis = "xyz".index(name[1])
        sl0 = [slice(None)] * 3
        sl1 = [slice(None)] * 3
        sl0[axis], sl1[axis] = slice(None, -1), slice(1, None)
        e = {k: (f32(0.5) * (v[tuple(sl0)] + v[tuple(sl1)])).astype(f32) for k, v in node.items()}
        a, b, c, d, ee, f = e["xx"], e["yy"], e["zz"], e["xy"], e["xz"], e["yz"]
        det = a * (b * c - f * f) - d * (d * c - f * ee) + ee * (d * f - b * ee)
        inv_det = f32(1.0) / det
        inv = {"xx": (b * c - f * f) * inv_det, "yy": (a * c - ee * ee) * inv_det, "zz": (a * b - d * d) * inv_det,
               "xy": (ee * f - d * c) * inv_det, "xz": (d * f - b * ee) * inv_det, "yz": (d * ee - a * f) * inv_det}
        diag = inv[_ANISO_DIAG[name]]
        if np.any(det <= 0) or np.any(diag <= 0):
            raise ValueError(f"the anisotropic permittivity tensor is not positive-definite on the {name} edges")
        eps_eff[name] = (f32(EPSILON_0) / diag).astype(f32)
        ca = (scale * inv[_ANISO_ROWS[name][0]]).astype(f32)
        cb = (scale * inv[_ANISO_ROWS[name][1]]).astype(f32)
        nz = np.argwhere((ca != 0) | (cb != 0))
        if nz.size == 0:
            continue
        lo, hi = nz.min(axis=0), nz.max(axis=0) + 1
        box = (int(lo[0]), int(hi[0]), int(lo[1]), int(hi[1]), int(lo[2]), int(hi[2]))
        sl = (slice(box[0], box[1]), slice(box[2], box[3]), slice(box[4], box[5]))
        aniso[name] = (box, np.ascontiguousarray(ca[sl]), np.ascontiguousarray(cb[sl]))
    return eps_eff, aniso


def _node_bbox(mask: np.ndarray):
    """Inclusive (lo, hi) node index range per axis of the nonzero entries, or None."""
    out = []
    for a in range(3):
        other = tuple(b for b in range(3) if b != a)
        idx = np.flatnonzero(np.any(mask != 0, axis=other))
        if idx.size == 0:
            return None
        out.append((int(idx[0]), int(idx[-1])))
    return out


def window_scales(window: np.ndarray, steps: int, n_freq: int) -> np.ndarray:
    """Per-frequency spectrum scale 2 / sum(window) over the first ``steps`` steps
    (witwin/maxwell/fdtd/observers.py:236-241); ``window`` is one weight per step
    or one per (step, frequency); 0 where nothing was sampled."""
    w = np.asarray(window, dtype=np.float64)[: int(steps)]
    total = np.broadcast_to(w.sum(axis=0), (n_freq,)).astype(np.float64)
    out = np.zeros(n_freq, dtype=np.float64)
    np.divide(2.0, total, out=out, where=total > 0)
    return out


def _avg_node_to_component(node: np.ndarray, name: str) -> np.ndarray:
    """witwin/maxwell/fdtd/runtime/materials.py:399-407."""
    if name == "Ex":
        return 0.5 * (node[:-1, :, :] + node[1:, :, :])
    if name == "Ey":
        return 0.5 * (node[:, :-1, :] + node[:, 1:, :])
    return 0.5 * (node[:, :, :-1] + node[:, :, 1:])


def cpml_profile_1d(positions64, nodes64, thickness, dt, vacuum_constant, strength, impedance, config,
                    *, high_positions64=None, apply_low=True, apply_high=True):
    """(kappa, b, c) graded by physical depth, witwin/maxwell/fdtd/boundary/cpml.py:114-210."""
    length = len(positions64)
    thickness = int(thickness)
    if thickness <= 0 or not (apply_low or apply_high):
        return np.ones(length, np.float32), np.zeros(length, np.float32), np.zeros(length, np.float32)
    nodes64 = np.asarray(nodes64, dtype=np.float64)

    def interface(low):
        cell_count = len(nodes64) - 1
        if thickness <= cell_count:
            return float(nodes64[thickness]) if low else float(nodes64[-1 - thickness])
        extra = thickness - cell_count
        if low:
            return float(nodes64[-1]) + extra * float(nodes64[-1] - nodes64[-2])
        return float(nodes64[0]) - extra * float(nodes64[1] - nodes64[0])

    m = float(config["grading_order"])
    kappa_max = float(config["kappa_max"])
    alpha_max = float(config["alpha_max"])
    reflection = float(config["reflection"])
    sigma_numerator = -(m + 1.0) * math.log(reflection) / (2.0 * float(impedance))
    positions = np.asarray(positions64, dtype=np.float64)
    high_positions = positions if high_positions64 is None else np.asarray(high_positions64, dtype=np.float64)
    depth_low = np.zeros(length)
    depth_high = np.zeros(length)
    sigma_max_low = sigma_max_high = 0.0
    if apply_low:
        low_interface = interface(True)
        layer_low = low_interface - float(nodes64[0])
        depth_low = np.clip((low_interface - positions) / layer_low, 0.0, 1.0)
        sigma_max_low = sigma_numerator / layer_low * strength
    if apply_high:
        high_interface = interface(False)
        layer_high = float(nodes64[-1]) - high_interface
        depth_high = np.clip((high_positions - high_interface) / layer_high, 0.0, 1.0)
        sigma_max_high = sigma_numerator / layer_high * strength
    use_high = depth_high > depth_low
    depth = np.where(use_high, depth_high, depth_low)
    sigma_peak = np.where(use_high, sigma_max_high, sigma_max_low)
    active = depth > 0.0
    graded = np.zeros(length)
    graded[active] = depth[active] ** m
    sigma = sigma_peak * graded
    kappa = np.ones(length)
    kappa[active] = 1.0 + (kappa_max - 1.0) * graded[active]
    alpha = np.zeros(length)
    alpha[active] = alpha_max * (1.0 - depth[active])
    decay = np.exp(-(sigma / kappa + alpha) * float(dt) / float(vacuum_constant))
    denom = sigma + alpha * kappa
    c = np.zeros(length)
    mask = denom > 1e-12
    c[mask] = sigma[mask] * (decay[mask] - 1.0) / (denom[mask] * kappa[mask])
    return kappa.astype(np.float32), decay.astype(np.float32), c.astype(np.float32)


def _source_signal(source_time, dt: float, steps: int) -> np.ndarray:
    """Host-evaluated waveform per step at t_n = n*dt (excitation/temporal.py:408-491)."""
    return np.asarray([source_time.evaluate(n * dt) for n in range(steps)], dtype=np.float64).astype(np.float32)


def _dipole_patch(scene: Scene, src: PointDipole, eps: dict, dt: float):
    """Normalised Gaussian point-dipole patch, witwin/maxwell/fdtd/excitation/injection.py:36-61, 214-396.

    The reference evaluates the profile over the cutoff window (3 * max(width,
    0.01 m), which covers the whole grid at optical scales) in float32; entries
    that underflow to zero are cropped away here, which leaves the sum unchanged.
    """
    d = float(scene.spacing)
    nodes = scene.nodes
    width = POINT_DIPOLE_REFERENCE_WIDTH if src.width is None else float(src.width)
    name = src.polarization
    shape = component_shape(name, nodes)
    axis = "xyz".index(name[1])
    coords = []
    for a in range(3):
        base = np.arange(shape[a], dtype=np.float64) * d
        if a == axis:
            base = base + 0.5 * d
        coords.append(base.astype(np.float32))
    pos = [np.float32(p * d) for p in src.position]
    dist_sq = ((coords[0][:, None, None] - pos[0]) ** 2 + (coords[1][None, :, None] - pos[1]) ** 2
               + (coords[2][None, None, :] - pos[2]) ** 2).astype(np.float32)

    def widths(c):
        w = np.empty_like(c)
        diffs = c[1:] - c[:-1]
        w[0] = 0.5 * diffs[0]
        w[-1] = 0.5 * diffs[-1]
        w[1:-1] = 0.5 * (diffs[:-1] + diffs[1:])
        return w

    wv = [widths(c) for c in coords]
    volumes = wv[0][:, None, None] * wv[1][None, :, None] * wv[2][None, None, :]
    width_sq = np.float32(2.0 * width ** 2)
    profile = np.exp(-dist_sq / width_sq).astype(np.float32)
    mass = np.float32(np.sum(profile * volumes, dtype=np.float32))
    profile = profile / max(mass, np.finfo(np.float32).eps)
    patch = (np.float32(-dt) / eps[name]) * profile
    patch = patch.astype(np.float32)
    nz = np.nonzero(patch)
    box = tuple(int(v) for a in range(3) for v in (nz[a].min(), nz[a].max() + 1))
    coeff = patch[box[0]:box[1], box[2]:box[3], box[4]:box[5]].copy()
    return box, coeff


# TFSF face specs, witwin/maxwell/fdtd/excitation/tfsf_specs.py:46-333:
# (field, incident, offsets, shape, sample_offsets, delta_axis, sign) built from lower/upper.
def _tfsf_specs(lower, upper):
    ix0, iy0, iz0 = lower
    ix1, iy1, iz1 = upper
    mag = [
        ("Hy", "Ez", (ix0 - 1, iy0, iz0), (1, iy1 - iy0 + 1, iz1 - iz0), (ix0, iy0, iz0), 0, +1.0),
        ("Hz", "Ey", (ix0 - 1, iy0, iz0), (1, iy1 - iy0, iz1 - iz0 + 1), (ix0, iy0, iz0), 0, -1.0),
        ("Hy", "Ez", (ix1, iy0, iz0), (1, iy1 - iy0 + 1, iz1 - iz0), (ix1, iy0, iz0), 0, -1.0),
        ("Hz", "Ey", (ix1, iy0, iz0), (1, iy1 - iy0, iz1 - iz0 + 1), (ix1, iy0, iz0), 0, +1.0),
        ("Hx", "Ez", (ix0, iy0 - 1, iz0), (ix1 - ix0 + 1, 1, iz1 - iz0), (ix0, iy0, iz0), 1, -1.0),
        ("Hz", "Ex", (ix0, iy0 - 1, iz0), (ix1 - ix0, 1, iz1 - iz0 + 1), (ix0, iy0, iz0), 1, +1.0),
        ("Hx", "Ez", (ix0, iy1, iz0), (ix1 - ix0 + 1, 1, iz1 - iz0), (ix0, iy1, iz0), 1, +1.0),
        ("Hz", "Ex", (ix0, iy1, iz0), (ix1 - ix0, 1, iz1 - iz0 + 1), (ix0, iy1, iz0), 1, -1.0),
        ("Hx", "Ey", (ix0, iy0, iz0 - 1), (ix1 - ix0 + 1, iy1 - iy0, 1), (ix0, iy0, iz0), 2, +1.0),
        ("Hy", "Ex", (ix0, iy0, iz0 - 1), (ix1 - ix0, iy1 - iy0 + 1, 1), (ix0, iy0, iz0), 2, -1.0),
        ("Hx", "Ey", (ix0, iy0, iz1), (ix1 - ix0 + 1, iy1 - iy0, 1), (ix0, iy0, iz1), 2, -1.0),
        ("Hy", "Ex", (ix0, iy0, iz1), (ix1 - ix0, iy1 - iy0 + 1, 1), (ix0, iy0, iz1), 2, +1.0),
    ]
    ele = [
        ("Ey", "Hz", (ix0, iy0, iz0), (1, iy1 - iy0, iz1 - iz0 + 1), (ix0 - 1, iy0, iz0), 0, +1.0),
        ("Ez", "Hy", (ix0, iy0, iz0), (1, iy1 - iy0 + 1, iz1 - iz0), (ix0 - 1, iy0, iz0), 0, -1.0),
        ("Ey", "Hz", (ix1, iy0, iz0), (1, iy1 - iy0, iz1 - iz0 + 1), (ix1, iy0, iz0), 0, -1.0),
        ("Ez", "Hy", (ix1, iy0, iz0), (1, iy1 - iy0 + 1, iz1 - iz0), (ix1, iy0, iz0), 0, +1.0),
        ("Ex", "Hz", (ix0, iy0, iz0), (ix1 - ix0, 1, iz1 - iz0 + 1), (ix0, iy0 - 1, iz0), 1, -1.0),
        ("Ez", "Hx", (ix0, iy0, iz0), (ix1 - ix0 + 1, 1, iz1 - iz0), (ix0, iy0 - 1, iz0), 1, +1.0),
        ("Ex", "Hz", (ix0, iy1, iz0), (ix1 - ix0, 1, iz1 - iz0 + 1), (ix0, iy1, iz0), 1, +1.0),
        ("Ez", "Hx", (ix0, iy1, iz0), (ix1 - ix0 + 1, 1, iz1 - iz0), (ix0, iy1, iz0), 1, -1.0),
        ("Ex", "Hy", (ix0, iy0, iz0), (ix1 - ix0, iy1 - iy0 + 1, 1), (ix0, iy0, iz0 - 1), 2, +1.0),
        ("Ey", "Hx", (ix0, iy0, iz0), (ix1 - ix0 + 1, iy1 - iy0, 1), (ix0, iy0, iz0 - 1), 2, -1.0),
        ("Ex", "Hy", (ix0, iy0, iz1), (ix1 - ix0, iy1 - iy0 + 1, 1), (ix0, iy0, iz1), 2, -1.0),
        ("Ey", "Hx", (ix0, iy0, iz1), (ix1 - ix0 + 1, iy1 - iy0, 1), (ix0, iy0, iz1), 2, +1.0),
    ]
    return ele, mag


def _magnetic_unit_vector(direction, polarization):
    """witwin/maxwell/fdtd/excitation/tfsf_specs.py:335-346."""
    d, p = direction, polarization
    mx = -(d[1] * p[2] - d[2] * p[1])
    my = -(d[2] * p[0] - d[0] * p[2])
    mz = -(d[0] * p[1] - d[1] * p[0])
    mag = math.sqrt(mx * mx + my * my + mz * mz)
    return {"Hx": mx / mag, "Hy": my / mag, "Hz": mz / mag}


def _compile_tfsf(scene: Scene, src: PlaneWaveTFSF, curl: dict, dt: float, steps: int):
    """Axis-aligned plane-wave TFSF (excitation/tfsf_state.py:293-357, spatial.py:311-469)."""
    d = float(scene.spacing)
    nodes = scene.nodes
    axis = int(np.argmax(np.abs(src.direction)))
    sign = 1 if src.direction[axis] > 0 else -1
    if any(src.direction[a] != 0 for a in range(3) if a != axis):
        raise ValueError("only axis-aligned plane waves are supported")
    # 1-D incident line over the domain extent along the axis plus the absorber
    # (tfsf_state.py:57-76): s_min = 0, ds = d.
    s_span = (nodes[axis] - 1) * d
    s_max = s_span + TFSF_ABSORBER_CELLS * d
    ne = max(int(math.ceil(s_max / d)) + 1, 4)
    eps_line = 1.0 / (ETA_0 * C_0)
    mu_line = ETA_0 / C_0
    sigma_e = np.zeros(ne, np.float32)
    sigma_h = np.zeros(ne - 1, np.float32)
    edge_e = min(TFSF_ABSORBER_CELLS, ne - 1)
    edge_h = min(TFSF_ABSORBER_CELLS, ne - 1)
    sigma_e[-edge_e:] = np.float32(0.35) * ((np.arange(edge_e, dtype=np.float32) + 1.0) / edge_e) ** 2
    sigma_h[-edge_h:] = np.float32(0.35) * ((np.arange(edge_h, dtype=np.float32) + 0.5) / edge_h) ** 2
    sf_e = (np.float32(0.5 * dt) * sigma_e / np.float32(eps_line)).astype(np.float32)
    sf_h = (np.float32(0.5 * dt) * sigma_h / np.float32(mu_line)).astype(np.float32)
    aux = CompiledAuxLine(
        e_decay=((1.0 - sf_e) / (1.0 + sf_e)).astype(np.float32),
        e_curl=(np.float32(dt / (eps_line * d)) / (1.0 + sf_e)).astype(np.float32),
        h_decay=((1.0 - sf_h) / (1.0 + sf_h)).astype(np.float32),
        h_curl=(np.float32(dt / (mu_line * d)) / (1.0 + sf_h)).astype(np.float32),
        source_index=0,
        source=_source_signal(src.source_time, dt, steps),
    )
    electric_vector = {"Ex": src.polarization[0], "Ey": src.polarization[1], "Ez": src.polarization[2]}
    magnetic_vector = _magnetic_unit_vector(src.direction, src.polarization)
    ele, mag = _tfsf_specs(src.lower, src.upper)
    if src.slab:
        # Slab injection keeps the two faces normal to the propagation axis
        # (tfsf_specs.py:322-332).
        ele = [s for s in ele if s[5] == axis]
        mag = [s for s in mag if s[5] == axis]
    out = []
    for specs, vector, kind in ((mag, electric_vector, 0), (ele, magnetic_vector, 1)):
        for fname, iname, offs, shape, soffs, delta_axis, sgn in specs:
            scale = float(vector[iname])
            if abs(sgn * scale) <= 1e-12:
                continue
            box = (offs[0], offs[0] + shape[0], offs[1], offs[1] + shape[1], offs[2], offs[2] + shape[2])
            c = curl[fname]
            c_arr = np.broadcast_to(c, component_shape(fname, nodes)) if np.ndim(c) == 0 else c
            coeff = (sgn * (c_arr[box[0]:box[1], box[2]:box[3], box[4]:box[5]] / np.float32(d))).astype(np.float32)
            start = soffs[axis]
            length = shape[axis]
            idx = np.arange(start, start + length, dtype=np.int64)
            if sign < 0:
                max_index = nodes[axis] - 1 if kind == 0 else nodes[axis] - 2
                idx = max_index - idx
            out.append(CompiledLinePatch(fname, box, np.ascontiguousarray(coeff), kind, axis,
                                         idx.astype(np.int32), scale))
    return aux, out


def resolve_bloch_wavevector(scene: Scene) -> tuple[float, float, float]:
    """``scene.bloch_k``, or for ``"auto"`` the wavevector of the scene's one CW
    TFSF plane wave on its Bloch axes (k_num times the direction there, 0
    elsewhere; witwin/maxwell/fdtd/boundary/bloch.py:32-78, which also requires a
    TFSF slab whose normal axis is not Bloch)."""
    if not isinstance(scene.bloch_k, str):
        return tuple(float(v) for v in scene.bloch_k)
    if scene.bloch_k != "auto":
        raise ValueError(f"bloch_k must be three numbers or 'auto', not {scene.bloch_k!r}")
    waves = [s for s in scene.sources if isinstance(s, PlaneWaveTFSF)]
    if len(scene.sources) != 1 or len(waves) != 1:
        raise ValueError("an automatic Bloch wavevector needs exactly one source, a TFSF plane wave")
    if not isinstance(waves[0].source_time, CW):
        raise ValueError("an automatic Bloch wavevector needs a CW plane wave")
    k = tfsf_bloch_wavevector(scene, waves[0])
    return tuple(k[a] if scene.boundary[2 * a] == BOUNDARY_BLOCH else 0.0 for a in range(3))


def compile_scene(scene: Scene, time_steps: int) -> CompiledScene:
    """Compile a scene into the solver tensors consumed by the FDTD step path."""
    if isinstance(scene.bloch_k, str):
        scene = replace(scene, bloch_k=resolve_bloch_wavevector(scene))
    nodes = scene.nodes
    d = float(scene.spacing)
    dt = scene.resolve_dt()
    pml_lo, pml_hi = scene.pml_lengths()
    # --- grid: uniform spacing (scene.py:1245-1281) ---
    inv_e = [np.full(n, 1.0 / d, dtype=np.float64).astype(np.float32) for n in nodes]
    inv_h = [np.full(n - 1, 1.0 / d, dtype=np.float64).astype(np.float32) for n in nodes]
    # --- materials: node rasterisation, then node -> component averaging ---
    eps_node = [np.ones(nodes, dtype=np.float64) for _ in range(3)]
    # conductivity and nonlinear channels blend like the static eps
    # (compiler/materials.py:740-756): the last structure covering a node wins
    chan_node = {k: np.zeros(nodes, dtype=np.float64) for k in ("sigma", "chi2", "chi3", "tpa")}
    offdiag_node = {k: np.zeros(nodes, dtype=np.float64) for k in ("xy", "xz", "yz")}
    pole_weights = []  # list of (pole, node weight array)
    for st in scene.structures:
        mask = st.geometry.node_mask(nodes)
        for a in range(3):
            eps_node[a][mask] = st.medium.axis_eps(a)
        med = st.medium
        for key, value in (("sigma", med.sigma), ("chi2", med.chi2), ("chi3", med.kerr_chi3), ("tpa", med.tpa_sigma)):
            chan_node[key][mask] = float(value)
        for key, value in zip(("xy", "xz", "yz"), med.eps_offdiag or (0.0, 0.0, 0.0)):
            offdiag_node[key][mask] = float(value)
        for entry in pole_weights:
            entry[1][mask] = 0.0
        for pole in st.medium.poles:
            w = np.zeros(nodes, dtype=np.float64)
            w[mask] = 1.0
            pole_weights.append((pole, w))
    design = None
    for region in scene.material_regions:
        lo, hi = region.lo, region.hi
        vals = np.asarray(region.eps_r, dtype=np.float64)
        for a in range(3):
            eps_node[a][lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = vals
        design = region
    eps = {}
    for a, name in enumerate(("Ex", "Ey", "Ez")):
        eps[name] = (EPSILON_0 * _avg_node_to_component(eps_node[a], name)).astype(np.float32)
    # --- update coefficients (materials.py:942-1008): semi-implicit lossy fold, CPML not folded ---
    # averaged channels; an all-zero channel stays zero (np.zeros: no pass over the grid)
    chan = {k: {name: (_avg_node_to_component(v, name).astype(np.float32) if np.any(v != 0)
                       else np.zeros(component_shape(name, nodes), np.float32)) for name in ("Ex", "Ey", "Ez")}
            for k, v in chan_node.items()}
    conductive = bool(np.any(chan_node["sigma"] != 0))
    is_nonlinear = any(bool(np.any(chan_node[k] != 0)) for k in ("chi2", "chi3", "tpa"))
    general = bool(np.any(chan_node["chi2"] != 0) or np.any(chan_node["tpa"] != 0))
    dt32 = np.float32(dt)
    one32 = np.float32(1.0)
    decay, curl, uniform = {}, {}, {}
    nl_channels = {}
    static_curl = {}  # the static curl coefficients, from which the source terms are built
    aniso = None
    eps_curl = eps  # the permittivity of the curl coefficients
    if any(bool(np.any(v != 0)) for v in offdiag_node.values()):
        if any(bool(np.any(chan_node[k] != 0)) for k in ("sigma", "chi2", "chi3", "tpa")) or pole_weights:
            raise ValueError("full anisotropy with conductive, nonlinear or dispersive media is not supported")
        eps_curl, aniso = _full_aniso(eps_node, offdiag_node, dt)
    for name in ("Ex", "Ey", "Ez"):
        e = eps_curl[name]
        if conductive:
            half = (np.float32(0.5) * chan["sigma"][name] * dt32) / e
            denom = one32 + half
            mdecay = ((one32 - half) / denom).astype(np.float32)
            c = ((dt32 / e) / denom).astype(np.float32)
        else:
            mdecay = None
            c = (dt32 / e).astype(np.float32)
        static_curl[name] = np.float32(c.flat[0]) if float(c.min()) == float(c.max()) else c
        if is_nonlinear:
            # the field-dependent coefficients with every nonlinear channel at
            # rest: constant on the cells without one (materials.py:1664-1770);
            # the engine rewrites the others before every step
            if general:
                ext = np.ones_like(e)
                sig = np.maximum(chan["sigma"][name], np.float32(0.0))
                half = (np.float32(0.5) * sig * dt32) / e
                inv_denom = one32 / (one32 + half)
                decay[name] = (ext * (one32 - half) * inv_denom).astype(np.float32)
                curl[name] = (ext * (dt32 / e) * inv_denom).astype(np.float32)
                dparam = ext
            else:
                static = mdecay if mdecay is not None else np.ones_like(e)
                decay[name] = mdecay
                curl[name] = ((dt32 / e) * static).astype(np.float32)
                dparam = static
            uniform[name] = (1.0 if decay[name] is None else None, None)
            nl_channels[name] = {"decay": dparam, "sigma": chan["sigma"][name], "chi2": chan["chi2"][name],
                                 "chi3": chan["chi3"][name], "tpa": chan["tpa"][name]}
            continue
        decay[name] = mdecay
        if mdecay is None and float(c.min()) == float(c.max()):
            curl[name] = None
            uniform[name] = (1.0, float(c.flat[0]))
        else:
            curl[name] = c
            uniform[name] = (1.0 if mdecay is None else None, None)
    nonlinear = CompiledNonlinear(general, EPSILON_0, nl_channels) if is_nonlinear else None
    h_curl = float(np.float32(dt) / np.float32(MU_0))
    for name in ("Hx", "Hy", "Hz"):
        decay[name] = None
        curl[name] = None
        uniform[name] = (1.0, h_curl)
    # --- CPML profiles (cpml.py:383-414) ---
    eta0 = math.sqrt(MU_0 / EPSILON_0)
    magnetic_strength = float(np.float32(MU_0 / EPSILON_0))
    cp = {k: [] for k in ("b_e", "c_e", "ik_e", "b_h", "c_h", "ik_h")}
    for a in range(3):
        nodes64 = np.arange(nodes[a], dtype=np.float64) * d
        half64 = nodes64[:-1] + 0.5 * d
        apply_low = scene.boundary[2 * a] == BOUNDARY_PML
        apply_high = scene.boundary[2 * a + 1] == BOUNDARY_PML
        ke, be, ce = cpml_profile_1d(nodes64, nodes64, scene.pml_cells, dt, EPSILON_0, 1.0, eta0,
                                     DEFAULT_CPML_CONFIG, apply_low=apply_low, apply_high=apply_high)
        kh, bh, ch = cpml_profile_1d(half64, nodes64, scene.pml_cells, dt, MU_0, magnetic_strength, eta0,
                                     DEFAULT_CPML_CONFIG, high_positions64=nodes64[1:], apply_low=apply_low,
                                     apply_high=apply_high)
        cp["b_e"].append(be)
        cp["c_e"].append(ce)
        cp["ik_e"].append((np.float32(1.0) / ke).astype(np.float32))
        cp["b_h"].append(bh)
        cp["c_h"].append(ch)
        cp["ik_h"].append((np.float32(1.0) / kh).astype(np.float32))
    # --- ADE templates (materials.py:530-589) ---
    poles = []
    for pole, w_node in pole_weights:
        if isinstance(pole, DebyePole):
            kind = 0
            decay_v = (2.0 * pole.tau - dt) / (2.0 * pole.tau + dt)
            restoring = 0.0
            base = 2.0 * EPSILON_0 * pole.delta_eps * dt / (2.0 * pole.tau + dt)
        elif isinstance(pole, DrudePole):
            kind = 1
            wp = 2.0 * math.pi * pole.plasma_frequency
            g = 2.0 * math.pi * pole.gamma
            denom = 2.0 + g * dt
            decay_v = (2.0 - g * dt) / denom
            restoring = 0.0
            base = 2.0 * EPSILON_0 * wp * wp * dt / denom
        else:
            kind = 2
            w0 = 2.0 * math.pi * pole.resonance_frequency
            g = 2.0 * math.pi * pole.gamma
            denom = 2.0 + g * dt
            decay_v = (2.0 - g * dt) / denom
            restoring = 2.0 * w0 * w0 * dt / denom
            base = 2.0 * EPSILON_0 * pole.delta_eps * w0 * w0 * dt / denom
        node_box = _node_bbox(w_node)
        if node_box is None:
            continue
        for name in ("Ex", "Ey", "Ez"):
            # the component cells whose two averaged nodes meet the pole's nodes:
            # the bounding box of the nonzero averaged weights, without a pass
            # over the whole grid
            axis = "xyz".index(name[1])
            box = []
            for a in range(3):
                lo, hi = node_box[a]
                if a == axis:
                    lo, hi = max(lo - 1, 0), min(hi, nodes[a] - 2)
                box += [lo, hi + 1]
            box = tuple(box)
            sl = (slice(box[0], box[1]), slice(box[2], box[3]), slice(box[4], box[5]))
            nsl = [slice(box[0], box[1]), slice(box[2], box[3]), slice(box[4], box[5])]
            nsl[axis] = slice(box[2 * axis], box[2 * axis + 1] + 1)
            weight = _avg_node_to_component(w_node[tuple(nsl)], name).astype(np.float32)
            drive = (weight * np.float32(base)).astype(np.float32)
            inv_eps = (np.float32(1.0) / eps[name][sl]).astype(np.float32)
            poles.append(CompiledPole(name, kind, float(decay_v), float(restoring), box,
                                      np.ascontiguousarray(drive), np.ascontiguousarray(inv_eps)))
    # --- sources ---
    patches, line_patches, aux_line, shifted = [], [], None, []
    for src in scene.sources:
        if isinstance(src, PointDipole):
            box, coeff = _dipole_patch(scene, src, eps, dt)
            patches.append(CompiledPatch(src.polarization, box, coeff, _source_signal(src.source_time, dt, time_steps)))
        elif isinstance(src, PlaneSource):
            patches.extend(_plane_source_patches(scene, src, eps, dt, time_steps))
        elif isinstance(src, GaussianBeam):
            curl_full = {name: static_curl.get(name, np.float32(uniform[name][1])) for name in COMPONENTS}
            beam_patches, beam_shifted = _beam_patches(scene, src, curl_full, dt, time_steps)
            patches.extend(beam_patches)
            shifted.extend(beam_shifted)
        elif isinstance(src, PlaneWaveTFSF) and any(b == BOUNDARY_BLOCH for b in scene.boundary):
            # CW plane wave through a TFSF slab on the complex Bloch field
            _validate_grating_slab(scene, src, eps_node)
            slab_patches, slab_shifted = _grating_slab_patches(
                scene, src, {n: static_curl.get(n, np.float32(uniform[n][1])) for n in COMPONENTS}, dt, time_steps)
            patches.extend(slab_patches)
            shifted.extend(slab_shifted)
        elif isinstance(src, PlaneWaveTFSF):
            if aux_line is not None:
                raise ValueError("one TFSF source per scene")
            curl_full = {name: static_curl.get(name, np.float32(uniform[name][1])) for name in COMPONENTS}
            aux_line, line_patches = _compile_tfsf(scene, src, curl_full, dt, time_steps)
        else:
            raise TypeError(f"unsupported source {type(src).__name__}")
    # --- monitors ---
    regions = []
    freq_list = []
    mon_freqs = {}
    for mon in scene.monitors:
        mon_freqs[mon.name] = tuple(float(f) for f in mon.frequencies)
        for f in mon.frequencies:
            if float(f) not in freq_list:
                freq_list.append(float(f))
        for comp in mon.components:
            shape = component_shape(comp, nodes)
            if isinstance(mon, PointMonitor):
                i, j, k = mon.index
                box = (i, i + 1, j, j + 1, k, k + 1)
            elif isinstance(mon, VolumeMonitor):
                lo = mon.lo if mon.lo is not None else (0, 0, 0)
                hi = mon.hi if mon.hi is not None else shape
                box = tuple(v for a in range(3) for v in (int(lo[a]), min(int(hi[a]), shape[a])))
            else:
                box = [0, shape[0], 0, shape[1], 0, shape[2]]
                box[2 * mon.axis] = mon.index
                box[2 * mon.axis + 1] = mon.index + 1
                if mon.lo is not None:
                    others = [a for a in range(3) if a != mon.axis]
                    for o, lo_v, hi_v in zip(others, mon.lo, mon.hi):
                        box[2 * o] = int(lo_v)
                        box[2 * o + 1] = min(int(hi_v) + 1, shape[o])
                box = tuple(box)
            regions.append(CompiledRegion(mon.name, comp, box))
    window = np.ones(time_steps, dtype=np.float64)  # pulses force window "none" (spectral.py:244-267)
    complex_fields = any(b == BOUNDARY_BLOCH for b in scene.boundary)
    bcos, bsin = [1.0, 1.0, 1.0], [0.0, 0.0, 0.0]
    for a in range(3):
        if scene.boundary[2 * a] == BOUNDARY_BLOCH:
            angle = float(scene.bloch_k[a]) * float(scene.cells[a]) * d
            bcos[a], bsin[a] = math.cos(angle), math.sin(angle)
    return CompiledScene(
        nodes=nodes, spacing=d, dt=dt, time_steps=time_steps, boundary=tuple(scene.boundary), pml_lo=pml_lo,
        pml_hi=pml_hi, inv_e=inv_e, inv_h=inv_h, cpml=cp, eps=eps, decay=decay, curl=curl, uniform=uniform,
        poles=poles, patches=patches, aux_line=aux_line, line_patches=line_patches, regions=regions,
        frequencies=tuple(freq_list), monitor_frequencies=mon_freqs, window=window, design=design,
        complex_fields=complex_fields, bloch_cos=tuple(bcos), bloch_sin=tuple(bsin), shifted=shifted,
        nonlinear=nonlinear, aniso=aniso,
    )


def _plane_source_patches(scene: Scene, src: PlaneSource, eps: dict, dt: float, steps: int) -> list:
    """Patches of a PlaneSource: the real part (channel 0) and, on a Bloch
    scene, the imaginary part (channel 1) of coeff * e^{i k.r} over the plane."""
    name = src.polarization
    if "xyz".index(name[1]) == src.axis:
        raise ValueError("a plane source drives a component tangential to its plane")
    d = float(scene.spacing)
    shape = component_shape(name, scene.nodes)
    box = [0, shape[0], 0, shape[1], 0, shape[2]]
    box[2 * src.axis], box[2 * src.axis + 1] = int(src.index), int(src.index) + 1
    if not 0 <= src.index < shape[src.axis]:
        raise ValueError("plane source index outside the component")
    own = "xyz".index(name[1])
    coords = []
    for a in range(3):
        c = np.arange(box[2 * a], box[2 * a + 1], dtype=np.float64) * d
        coords.append(c + (0.5 * d if a == own else 0.0))
    phase = (float(scene.bloch_k[0]) * coords[0][:, None, None] + float(scene.bloch_k[1]) * coords[1][None, :, None]
             + 0.0 * coords[2][None, None, :])
    sl = tuple(slice(box[2 * a], box[2 * a + 1]) for a in range(3))
    base = (np.float64(-dt) / eps[name][sl].astype(np.float64)) / d
    signal = _source_signal(src.source_time, dt, steps)
    out = [CompiledPatch(name, tuple(box), np.ascontiguousarray((base * np.cos(phase)).astype(np.float32)), signal, 0)]
    if any(b == BOUNDARY_BLOCH for b in scene.boundary):
        out.append(CompiledPatch(name, tuple(box), np.ascontiguousarray((base * np.sin(phase)).astype(np.float32)),
                                 signal, 1))
    return out


def _numerical_wavenumber(omega: float, dt: float, direction, d: float) -> float:
    """|k| of the discrete dispersion relation sum_a sin^2(k |u_a| d / 2) / d^2 =
    sin^2(omega dt / 2) / (c dt)^2 on a uniform grid, by 80 bisection steps over
    (0, min_a 2 pi / (|u_a| d)) (witwin/maxwell/fdtd/dispersion.py:6-48)."""
    if omega <= 0.0:
        return 0.0
    target = math.sin(0.5 * omega * dt) ** 2 / (C_0 ** 2 * dt ** 2)
    comps = [abs(float(u)) for u in direction if abs(float(u)) > 1e-12]
    if target <= 0.0 or not comps:
        return omega / C_0
    lo, hi = 0.0, min(2.0 * math.pi / max(u * d, 1e-30) for u in comps)
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if sum(math.sin(0.5 * mid * u * d) ** 2 / (d * d) for u in comps) - target >= 0.0:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


def _beam_profile(pos, direction, polarization, waist: float, focus, frequency: float, speed: float):
    """Amplitude and delay of a Gaussian beam at positions pos[..., 3] (metres):
    w(z) = w0 sqrt(1 + (z / z_R)^2), amplitude (w0 / w) exp(-(u^2 + v^2) / w^2),
    delay z / c + (u^2 + v^2) / (2 R c) - atan(z / z_R) / omega with the wavefront
    radius R = z (1 + (z_R / z)^2) (zero curvature within 1 nm of the waist plane),
    u along the polarization, v along direction x polarization
    (witwin/maxwell/fdtd/excitation/spatial.py:175-251)."""
    dvec = np.asarray(direction, dtype=np.float64)
    pvec = np.asarray(polarization, dtype=np.float64)
    bvec = np.cross(dvec, pvec)
    rel = pos - np.asarray(focus, dtype=np.float64)
    z = rel @ dvec
    u = rel @ pvec
    v = rel @ bvec
    wavelength = speed / frequency
    z_r = math.pi * waist * waist / max(wavelength, 1e-30)
    radius = waist * np.sqrt(1.0 + (z / max(z_r, 1e-30)) ** 2)
    amplitude = (waist / radius) * np.exp(-(u * u) / (radius * radius) - (v * v) / (radius * radius))
    curved = np.abs(z) > 1e-9
    with np.errstate(divide="ignore", invalid="ignore"):
        r_curv = z * (1.0 + (z_r / np.maximum(np.abs(z), 1e-30)) ** 2)
        curvature = np.where(curved, (u * u + v * v) / (2.0 * r_curv * speed), 0.0)
    gouy = np.arctan(z / max(z_r, 1e-30))
    delay = z / speed + curvature - gouy / (2.0 * math.pi * frequency)
    return amplitude, delay


def _component_positions(name: str, offsets, shape, d: float) -> np.ndarray:
    """Metres of the Yee samples of ``name`` over the box at ``offsets`` with ``shape``:
    E components sit half a cell along their own axis, H components half a cell along
    the other two (witwin/maxwell/fdtd/solver.py:406-424)."""
    own = "xyz".index(name[1])
    axes = []
    for a in range(3):
        half = (a == own) if name[0] == "E" else (a != own)
        axes.append((np.arange(offsets[a], offsets[a] + shape[a], dtype=np.float64) + (0.5 if half else 0.0)) * d)
    grid = np.meshgrid(*axes, indexing="ij")
    return np.stack(grid, axis=-1)


def _beam_launch_plane(scene: Scene, axis: int, forward: bool) -> int:
    """Node index of the soft launch plane: 5 % of the physical (CPML-free) span from
    its edge on the side the beam comes from, the nearest node, ties to the lower
    index (witwin/maxwell/fdtd/excitation/spatial.py:49-77)."""
    pml_lo, pml_hi = scene.pml_lengths()
    n = scene.nodes[axis]
    lo, hi = pml_lo[axis], n - pml_hi[axis] - 1
    if hi <= lo:
        raise ValueError("the scene has no physical interior along the injection axis")
    target = lo + 0.05 * (hi - lo) if forward else hi - 0.05 * (hi - lo)
    below = int(math.floor(target))
    return below if target - below <= (below + 1) - target else below + 1


def _discrete_plane_wave_vectors(direction, polarization, k_num: float, d: float):
    """Unit E and H vectors of the discrete plane wave (witwin/maxwell/fdtd/excitation/
    tfsf_specs.py:369-386): the polarisation made transverse to the effective
    wavevector sin(k u_a d / 2) / d, H along -(kappa x E)."""
    eff = np.array([math.sin(0.5 * k_num * float(c) * d) / d for c in direction])
    kh = eff / np.linalg.norm(eff)
    p = np.asarray(polarization, dtype=np.float64)
    e = p - float(p @ kh) * kh
    e = e / np.linalg.norm(e)
    m = -np.cross(kh, e)
    m = m / np.linalg.norm(m)
    return ({n: float(v) for n, v in zip(("Ex", "Ey", "Ez"), e)},
            {n: float(v) for n, v in zip(("Hx", "Hy", "Hz"), m)})


def tfsf_bloch_wavevector(scene: Scene, src: PlaneWaveTFSF) -> tuple[float, float, float]:
    """The Bloch wavevector (rad/m per axis) a TFSF slab's CW plane wave needs on the
    scene's grid: the numerical wavenumber of the discrete dispersion relation along
    the direction, projected on each axis (the normal axis entry is unused)."""
    dvec = np.asarray(src.direction, dtype=np.float64)
    dvec = dvec / np.linalg.norm(dvec)
    omega = 2.0 * math.pi * float(src.source_time.frequency)
    k_num = _numerical_wavenumber(omega, scene.resolve_dt(), dvec, float(scene.spacing))
    return tuple(float(k_num * c) for c in dvec)


@dataclass(frozen=True)
class GratingSlabTerm:
    """One face term of a TFSF slab on Bloch faces, as the reference's Bloch patch
    launchers receive it.  CW (witwin/maxwell/fdtd/cuda/backend.py:1817-1854): at
    step n the complex delta of the cells of ``box`` is (cos_patch s_c + sin_patch
    s_s) + i (cos_patch s_s - sin_patch s_c), (s_c, s_s) = (signal_cos[n],
    signal_sin[n]).  Pulsed (witwin/maxwell/fdtd/excitation/temporal.py:229-247,
    395-405): the real delta scale * w(n dt + t_offset - delay) per cell."""

    component: str
    box: tuple
    cos_patch: np.ndarray | None = None
    sin_patch: np.ndarray | None = None
    signal_cos: np.ndarray | None = None
    signal_sin: np.ndarray | None = None
    scale: np.ndarray | None = None
    delay: np.ndarray | None = None
    t_offset: float = 0.0
    source_time: object = None


def _validate_grating_slab(scene: Scene, src: PlaneWaveTFSF, eps_node) -> None:
    """The reference's checks of a TFSF slab (witwin/maxwell/fdtd/excitation/
    tfsf_state.py:171-199): at least two cells along the injection axis, both faces
    inside the non-CPML region, and vacuum (relative permittivity 1 within 1e-5)
    on the two face planes."""
    dvec = np.asarray(src.direction, dtype=np.float64)
    axis = int(np.argmax(np.abs(dvec)))
    lo, hi = int(src.lower[axis]), int(src.upper[axis])
    pml_lo, pml_hi = scene.pml_lengths()
    if hi <= lo + 1:
        raise ValueError(f"TFSF slab bounds must span at least two cells along {'xyz'[axis]}")
    if lo < pml_lo[axis] or hi > scene.nodes[axis] - pml_hi[axis] - 1:
        raise ValueError("TFSF slab bounds must lie strictly inside the non-PML simulation region")
    for face in (lo, hi):
        for arr in eps_node:
            plane = np.take(arr, face, axis=axis)
            if np.max(np.abs(plane - 1.0)) > 1e-5:
                raise ValueError("TFSF slab interfaces must remain in vacuum")


def grating_slab_terms(scene: Scene, src: PlaneWaveTFSF, curl: dict, dt: float, steps: int) -> list:
    """CW plane wave through a TFSF slab on a Bloch scene (the reference's grating-slab
    provider, witwin/maxwell/fdtd/excitation/tfsf_state.py:202-279): the two faces
    normal to the injection axis over the whole transverse extent (tfsf_specs.py:
    322-332), the E faces driven by the discrete magnetic vector / eta0 and the H
    faces by the electric one, each term the curl coefficient over the spacing times
    the face sign, with the CW phase omega (r - r0).u / v of the numerical phase speed
    v (tfsf_common.py:354-421); (s_c, s_s) = A (cos, sin)(omega t + phase)
    (temporal.py:71-74), E terms at (n + 1/2) dt and H terms at n dt
    (tfsf_apply.py:226-242)."""
    st = src.source_time
    cw = isinstance(st, CW)
    if not cw and not isinstance(st, GaussianPulse):
        raise ValueError("a TFSF slab on Bloch faces takes a CW or GaussianPulse source time")
    dvec = np.asarray(src.direction, dtype=np.float64)
    dvec = dvec / np.linalg.norm(dvec)
    pvec = np.asarray(src.polarization, dtype=np.float64)
    pvec = pvec / np.linalg.norm(pvec)
    axis = int(np.argmax(np.abs(dvec)))
    transverse = [a for a in range(3) if a != axis]
    for a in transverse:
        if scene.boundary[2 * a] not in (BOUNDARY_BLOCH, BOUNDARY_PERIODIC):
            raise ValueError("a TFSF slab on Bloch faces needs Bloch or periodic transverse axes")
    if scene.boundary[2 * axis] in (BOUNDARY_BLOCH, BOUNDARY_PERIODIC):
        raise ValueError("the injection axis of a TFSF slab cannot be periodic")
    d = float(scene.spacing)
    nodes = scene.nodes
    freq = float(st.frequency)
    omega = 2.0 * math.pi * freq
    k_num = _numerical_wavenumber(omega, dt, dvec, d)
    for a in transverse if cw else ():  # a pulse keeps the scene's fixed Bloch wavevector
        need = k_num * dvec[a]
        have = float(scene.bloch_k[a]) if scene.boundary[2 * a] == BOUNDARY_BLOCH else 0.0
        if abs(need - have) > 1e-6 * max(k_num, 1.0):
            raise ValueError(f"Bloch wavevector {have:.9g} on axis {'xyz'[a]} does not match the TFSF plane wave "
                             f"({need:.9g} rad/m, scene.tfsf_bloch_wavevector)")
    speed = omega / k_num if k_num > 1e-12 else C_0
    e_unit, h_unit = _discrete_plane_wave_vectors(dvec, pvec, k_num, d)
    h_vec = {n: v / ETA_0 for n, v in h_unit.items()}
    lower = [0, 0, 0]
    upper = [n - 1 for n in nodes]
    lower[axis], upper[axis] = int(src.lower[axis]), int(src.upper[axis])
    ele, mag = _tfsf_specs(lower, upper)
    ele, mag = ele[4 * axis:4 * axis + 4], mag[4 * axis:4 * axis + 4]  # the low and the high face
    ref = np.array([0.5 * (src.lower[a] + src.upper[a]) * d for a in range(3)])
    terms = []
    for specs, vector, t_off in ((ele, h_vec, 0.5 * dt), (mag, e_unit, 0.0)):
        if cw:
            times = np.arange(steps, dtype=np.float64) * dt + t_off
            ramp = np.array([st.ramp(t) for t in times])
            sc = (st.amplitude * ramp * np.cos(omega * times + st.phase)).astype(np.float32)
            ss = (st.amplitude * ramp * np.sin(omega * times + st.phase)).astype(np.float32)
        for fname, iname, offs, shape, soffs, _delta_axis, sgn in specs:
            comp_scale = float(vector[iname])
            if abs(sgn * comp_scale) <= 1e-12:
                continue
            box = (offs[0], offs[0] + shape[0], offs[1], offs[1] + shape[1], offs[2], offs[2] + shape[2])
            c = curl[fname]
            c_arr = np.broadcast_to(c, component_shape(fname, nodes)) if np.ndim(c) == 0 else c
            coeff = c_arr[box[0]:box[1], box[2]:box[3], box[4]:box[5]].astype(np.float64) / d
            delay = ((_component_positions(iname, soffs, shape, d) - ref) @ dvec) / speed
            scale = sgn * comp_scale * coeff
            if not cw:
                terms.append(GratingSlabTerm(fname, box, scale=np.ascontiguousarray(scale.astype(np.float32)),
                                             delay=np.ascontiguousarray(delay.astype(np.float32)), t_offset=t_off,
                                             source_time=st))
                continue
            terms.append(GratingSlabTerm(fname, box, np.ascontiguousarray((scale * np.cos(omega * delay)).astype(np.float32)),
                                         np.ascontiguousarray((scale * np.sin(omega * delay)).astype(np.float32)), sc, ss))
    return terms


def bloch_patch_phases(scene: Scene, component: str):
    """Per tangential axis of a field component (the two axes other than its own,
    in increasing order): whether a Bloch patch wraps there and the face phase
    (cos kL, sin kL), 1 on a periodic axis (witwin/maxwell/fdtd/excitation/
    temporal.py:126-205)."""
    own = "xyz".index(component[1])
    out = []
    for a in (x for x in range(3) if x != own):
        kind = scene.boundary[2 * a]
        if kind == BOUNDARY_BLOCH:
            ang = float(scene.bloch_k[a]) * (scene.nodes[a] - 1) * float(scene.spacing)
            out.append((a, True, math.cos(ang), math.sin(ang)))
        else:
            out.append((a, kind == BOUNDARY_PERIODIC, 1.0, 0.0))
    return out


def _fold_bloch_wrap_copies(scene: Scene, term: GratingSlabTerm):
    """Per-channel coefficients of a CW Bloch term with the reference's wrap copies
    folded in (witwin/maxwell/fdtd/cuda/kernels/sources.cu:368-440): a cell on the
    first plane of a wrapped tangential axis also adds e^{+ikL} times its delta to
    the last plane, a cell on the last plane e^{-ikL} times its delta to the first,
    and a cell on both wrapped axes' boundaries the doubly rotated delta to the
    opposite corner.  Returns (real s_c, real s_s, imag s_c, imag s_s) coefficient
    arrays over the term's box, which must span every wrapped axis whole."""
    shape = component_shape(term.component, scene.nodes)
    cp, sp = term.cos_patch.astype(np.float64), term.sin_patch.astype(np.float64)
    # delta = (Ac sc + As ss) + i (Bc sc + Bs ss)
    src = [cp, sp, -sp, cp]
    out = [x.copy() for x in src]
    wraps = []
    for a, wrap, c, s in bloch_patch_phases(scene, term.component):
        if not wrap:
            continue
        lo, hi = term.box[2 * a], term.box[2 * a + 1]
        if lo != 0 or hi != shape[a] or shape[a] < 2:
            raise ValueError("a Bloch slab term must span the wrapped axes whole")
        wraps.append((a, c, s))

    def rotate(vals, c, s):  # e^{i theta} on (Ac, As, Bc, Bs)
        ac, as_, bc, bs = vals
        return [c * ac - s * bc, c * as_ - s * bs, s * ac + c * bc, s * as_ + c * bs]

    def take(vals, a, idx):
        return [np.take(v, [idx], axis=a) for v in vals]

    def add_at(a_list, idx_list, vals):
        sl = [slice(None)] * 3
        for a, idx in zip(a_list, idx_list):
            sl[a] = slice(idx, idx + 1)
        for o, v in zip(out, vals):
            o[tuple(sl)] += v

    for a, c, s in wraps:
        n = shape[a]
        add_at([a], [n - 1], rotate(take(src, a, 0), c, s))
        add_at([a], [0], rotate(take(src, a, n - 1), c, -s))
    if len(wraps) == 2:
        (a, ca, sa), (b, cb, sb) = wraps
        na, nb = shape[a], shape[b]
        for ia, ra in ((0, 1.0), (na - 1, -1.0)):
            for ib, rb in ((0, 1.0), (nb - 1, -1.0)):
                corner = take(take(src, a, ia), b, ib)
                add_at([a, b], [na - 1 - ia, nb - 1 - ib], rotate(rotate(corner, ca, ra * sa), cb, rb * sb))
    return tuple(np.ascontiguousarray(o.astype(np.float32)) for o in out)


def _fold_shifted_wrap_copies(scene: Scene, term: GratingSlabTerm) -> list:
    """Time-shifted patches of a pulsed Bloch term with the reference kernel's wrap
    copies (sources.cu:368-440): the real delta scale * w(t - delay) on channel 0,
    and each wrapped axis' first / last plane copied to the opposite plane rotated
    by e^{+ikL} / e^{-ikL} (real part to channel 0, imaginary part to channel 1).
    A copy whose delays equal the target plane's (a wave without a phase along
    that axis) is folded into the target's scale; otherwise it is a patch of its
    own over that plane."""
    shape = component_shape(term.component, scene.nodes)
    scale = term.scale.astype(np.float64)
    main_re, main_im = scale.copy(), np.zeros_like(scale)
    extra = []
    wraps = [(a, c, s) for a, w, c, s in bloch_patch_phases(scene, term.component) if w]
    if len(wraps) > 1:
        raise ValueError("a pulsed Bloch slab term wraps on one tangential axis at most")
    for a, c, s in wraps:
        lo, hi = term.box[2 * a], term.box[2 * a + 1]
        n = shape[a]
        if lo != 0 or hi != n or n < 2:
            raise ValueError("a Bloch slab term must span the wrapped axes whole")
        for src, dst, sn in ((0, n - 1, s), (n - 1, 0, -s)):
            sl_src = [slice(None)] * 3
            sl_dst = [slice(None)] * 3
            sl_src[a], sl_dst[a] = slice(src, src + 1), slice(dst, dst + 1)
            sl_src, sl_dst = tuple(sl_src), tuple(sl_dst)
            if np.array_equal(term.delay[sl_src], term.delay[sl_dst]):
                main_re[sl_dst] += c * scale[sl_src]
                main_im[sl_dst] += sn * scale[sl_src]
                continue
            box = list(term.box)
            box[2 * a], box[2 * a + 1] = dst, dst + 1
            dly = np.ascontiguousarray(term.delay[sl_src])
            for ch, f in ((0, c), (1, sn)):
                if f != 0.0:
                    extra.append(CompiledShiftedPatch(term.component, tuple(box),
                                                      np.ascontiguousarray((f * scale[sl_src]).astype(np.float32)), dly,
                                                      term.t_offset, term.source_time, ch))
    out = [CompiledShiftedPatch(term.component, term.box, np.ascontiguousarray(main_re.astype(np.float32)), term.delay,
                                term.t_offset, term.source_time, 0)]
    if np.any(main_im != 0.0):
        out.append(CompiledShiftedPatch(term.component, term.box, np.ascontiguousarray(main_im.astype(np.float32)),
                                        term.delay, term.t_offset, term.source_time, 1))
    return out + extra


def _grating_slab_patches(scene: Scene, src: PlaneWaveTFSF, curl: dict, dt: float, steps: int):
    """The grating-slab terms on the complex field: a CW term as per-channel patches,
    real channel (A_c s_c + A_s s_s), imaginary channel (B_c s_c + B_s s_s) with the
    reference kernel's wrap copies folded into A and B; a pulsed term as
    time-shifted patches (_fold_shifted_wrap_copies).  Returns (patches, shifted)."""
    patches, shifted = [], []
    for t in grating_slab_terms(scene, src, curl, dt, steps):
        if t.cos_patch is None:
            shifted += _fold_shifted_wrap_copies(scene, t)
            continue
        ac, as_, bc, bs = _fold_bloch_wrap_copies(scene, t)
        patches += [CompiledPatch(t.component, t.box, ac, t.signal_cos, 0),
                    CompiledPatch(t.component, t.box, as_, t.signal_sin, 0),
                    CompiledPatch(t.component, t.box, bc, t.signal_cos, 1),
                    CompiledPatch(t.component, t.box, bs, t.signal_sin, 1)]
    return patches, shifted


def _beam_patches(scene: Scene, src: GaussianBeam, curl: dict, dt: float, steps: int):
    """Face terms of a soft GaussianBeam (witwin/maxwell/fdtd/excitation/injection.py:807-968):
    the E components of the launch face carry J_s from the magnetic incident vector,
    the H components M_s from the electric one, each scaled by the curl coefficient
    over the spacing, the face sign, the unit-power amplitude 1 / sqrt(pi w0^2 cos /
    (4 eta0)) / sqrt(cos(k_n d / 2)) and the beam profile evaluated with the numerical
    phase speed omega / k; the delay of the plane centre is removed (injection.py:
    907-941).  E terms sample the waveform at (n + 1/2) dt, H terms at n dt
    (runtime/stepping.py:1776, 2300-2306)."""
    if any(b in (BOUNDARY_BLOCH, BOUNDARY_PERIODIC) for b in scene.boundary):
        raise ValueError("a soft GaussianBeam supports CPML, PEC and open faces only")
    st = src.source_time
    if not isinstance(st, (CW, GaussianPulse)):
        raise TypeError("a GaussianBeam takes a CW or GaussianPulse source time")
    if src.beam_waist <= 0.0:
        raise ValueError("beam_waist must be > 0")
    dvec = np.asarray(src.direction, dtype=np.float64)
    dvec = dvec / np.linalg.norm(dvec)
    pvec = np.asarray(src.polarization, dtype=np.float64)
    pvec = pvec / np.linalg.norm(pvec)
    if abs(float(dvec @ pvec)) > 1e-6:
        raise ValueError("the polarization must be transverse to the direction")
    axis = int(np.argmax(np.abs(dvec))) if src.injection_axis is None else int(src.injection_axis)
    if abs(dvec[axis]) <= 1e-6:
        raise ValueError("the direction needs a component along the injection axis")
    forward = dvec[axis] >= 0.0
    d = float(scene.spacing)
    nodes = scene.nodes
    plane = _beam_launch_plane(scene, axis, forward)
    lower = [0, 0, 0]
    upper = [n - 1 for n in nodes]
    lower[axis], upper[axis] = (plane, plane + 1) if forward else (plane - 1, plane)
    ele, mag = _tfsf_specs(lower, upper)
    face = 4 * axis + (0 if forward else 2)  # the x-low, x-high, y-low, ... pairs of the spec table
    ele, mag = ele[face:face + 2], mag[face:face + 2]

    freq = float(st.frequency)
    omega = 2.0 * math.pi * freq
    k_num = _numerical_wavenumber(omega, dt, dvec, d)
    speed = omega / k_num if k_num > 1e-12 else C_0
    power = 1.0 / math.sqrt(math.pi * src.beam_waist ** 2 * abs(dvec[axis]) / (4.0 * ETA_0))
    factor = math.cos(0.5 * k_num * dvec[axis] * d)
    if factor <= 0.0:
        raise ValueError("the grid is too coarse for a positive discrete normal power")
    power /= math.sqrt(factor)
    e_vec = {n: power * float(pvec[i]) for i, n in enumerate(("Ex", "Ey", "Ez"))}
    h_vec = {n: power * v / ETA_0 for n, v in _magnetic_unit_vector(dvec, pvec).items()}
    pml_lo, pml_hi = scene.pml_lengths()
    centre = np.array([0.5 * (pml_lo[a] + nodes[a] - 1 - pml_hi[a]) * d for a in range(3)])
    centre[axis] = plane * d
    focus = np.asarray(src.focus, dtype=np.float64) * d
    _, ref_delay = _beam_profile(centre[None, :], dvec, pvec, src.beam_waist, focus, freq, speed)

    patches, shifted = [], []
    for specs, vector, t_off in ((ele, h_vec, 0.5 * dt), (mag, e_vec, 0.0)):
        for fname, iname, offs, shape, soffs, _delta_axis, sgn in specs:
            comp_scale = float(vector[iname])
            if abs(sgn * comp_scale) <= 1e-12:
                continue
            box = (offs[0], offs[0] + shape[0], offs[1], offs[1] + shape[1], offs[2], offs[2] + shape[2])
            c = curl[fname]
            c_arr = np.broadcast_to(c, component_shape(fname, nodes)) if np.ndim(c) == 0 else c
            coeff = c_arr[box[0]:box[1], box[2]:box[3], box[4]:box[5]].astype(np.float64) / d
            amp, delay = _beam_profile(_component_positions(iname, soffs, shape, d), dvec, pvec, src.beam_waist,
                                       focus, freq, speed)
            delay = delay - ref_delay[0]
            scale = sgn * comp_scale * amp * coeff
            if float(np.max(np.abs(scale))) <= 1e-12:
                continue
            if isinstance(st, CW):
                times = np.arange(steps, dtype=np.float64) * dt + t_off
                ramp = np.array([st.ramp(t) for t in times])
                phase = omega * times + st.phase
                for patch, sig in ((scale * np.cos(omega * delay), np.cos(phase)),
                                   (scale * np.sin(omega * delay), np.sin(phase))):
                    patches.append(CompiledPatch(fname, box, np.ascontiguousarray(patch.astype(np.float32)),
                                                 (st.amplitude * ramp * sig).astype(np.float32)))
            else:
                shifted.append(CompiledShiftedPatch(fname, box, np.ascontiguousarray(scale.astype(np.float32)),
                                                    np.ascontiguousarray(delay.astype(np.float32)), t_off, st))
    return patches, shifted


def shifted_waveform(source_time, t):
    """Waveform of a time-shifted patch at times t (array): A cos(2 pi f t + phase) for
    a CW, A exp(-(tau 2 pi fwidth)^2 / 2) cos(2 pi f tau + phase), tau = t - delay, for
    a GaussianPulse (witwin/maxwell/waveforms.py:83-107)."""
    t = np.asarray(t, dtype=np.float64)
    if isinstance(source_time, CW):
        return source_time.amplitude * np.cos(2.0 * math.pi * source_time.frequency * t + source_time.phase)
    tau = t - source_time.resolved_delay
    env = np.exp(-0.5 * (tau * 2.0 * math.pi * source_time.fwidth) ** 2)
    return source_time.amplitude * env * np.cos(2.0 * math.pi * source_time.frequency * tau + source_time.phase)
