"""Synthetic scenes of the benchmark workloads (seeded, uniform 25 nm grids).

Each builder returns a ``Scene`` with the shapes, materials, sources and
monitors of one workload; the grids are synthetic stand-ins for scenes the
reference would compile from geometry.  Cell counts include the CPML cells.
"""
from __future__ import annotations

import numpy as np

from .scene import (
    CW,
    Box,
    GaussianBeam,
    GaussianPulse,
    MaterialRegion,
    Medium,
    PlaneMonitor,
    PlaneWaveTFSF,
    PointDipole,
    PointMonitor,
    Scene,
    Sphere,
    Structure,
    closed_box_monitor,
    flux_monitor,
)

SPACING = 25e-9


def plain_small(cells: int = 64, pml: int = 10) -> Scene:
    """64^3 cells, 10-cell CPML, vacuum with a centred 24^3 eps_r=4 box, Ez dipole at
    (20,32,32) with a 300/100 THz Gaussian pulse, z=44 plane + point monitor at 250/300/350 THz."""
    sc = Scene(cells=(cells,) * 3, spacing=SPACING, pml_cells=pml)
    lo = (cells - 24) // 2
    sc.structures.append(Structure(Box((lo,) * 3, (lo + 24,) * 3), Medium(eps_r=4.0)))
    sc.sources.append(PointDipole((20, cells // 2, cells // 2), "Ez", GaussianPulse(300e12, 100e12), width=SPACING))
    freqs = (250e12, 300e12, 350e12)
    sc.monitors.append(PlaneMonitor("plane_z", 2, lo + 24, frequencies=freqs))
    sc.monitors.append(PointMonitor("point", (lo + 24, cells // 2, cells // 2), frequencies=freqs))
    return sc


def dispersive_256(cells: int = 256, pml: int = 12, n_freq: int = 16, slab_through_pml: bool = True) -> Scene:
    """256^3 cells, 12-cell CPML; radius-60 Lorentz sphere (eps_inf 2, delta_eps 3, 250 THz,
    gamma 20 THz) at the centre; 40-cell Drude slab x in [40, 80) (omega_p 2e15 rad/s,
    gamma 1e14 rad/s); x-normal Ez plane wave (300/100 THz pulse) through a TFSF box inset
    2 cells inside the CPML; 16 frequencies 200-400 THz on two z-normal flux planes and a
    closed six-face flux box.

    As specified the Drude slab spans the whole y, z extent, through the y and z
    CPML; there the CPML recursion and the Drude current feed each other and the
    field grows about threefold every 200 steps after step ~800, in FP32 and in
    the reference's arithmetic alike (the engine matches the reference's own ops
    step by step).  slab_through_pml=False stops the slab at the CPML: a stable
    copy for accuracy comparisons over the workload's 2000 steps."""
    scale = cells / 256.0
    sc = Scene(cells=(cells,) * 3, spacing=SPACING, pml_cells=pml)
    c = cells / 2.0
    sc.structures.append(Structure(Sphere((c, c, c), 60.0 * scale), Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
    x0, x1 = int(round(40 * scale)), int(round(80 * scale))
    s0, s1 = (0, cells) if slab_through_pml else (pml, cells - pml)
    sc.structures.append(Structure(Box((x0, s0, s0), (x1, s1, s1)), Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))))
    lo = pml + 2
    hi = cells - pml - 2
    sc.sources.append(PlaneWaveTFSF((1, 0, 0), (0, 0, 1), GaussianPulse(300e12, 100e12), (lo,) * 3, (hi,) * 3))
    freqs = tuple(np.linspace(200e12, 400e12, n_freq))
    sc.monitors.append(flux_monitor("flux_z_lo", 2, int(round(40 * scale)), freqs))
    sc.monitors.append(flux_monitor("flux_z_hi", 2, int(round(216 * scale)), freqs))
    b0, b1 = int(round(28 * scale)), int(round(228 * scale))
    sc.monitors.extend(closed_box_monitor("box", (b0,) * 3, (b1,) * 3, freqs))
    return sc


def adjoint_160(steps: int = 3000, seed: int = 0, scale: int = 1) -> Scene:
    """Adjoint-gradient workload: 160x160x96 cells, 10-cell CPML; eps 2.1 substrate for
    z < 40; a 64x64x16 MaterialRegion design block at x, y in [48, 112), z in [40, 56)
    with eps_r ~ U[1, 12) i.i.d. (torch.Generator().manual_seed(seed)); a soft +z Ey
    GaussianBeam (waist 1 um, focused on the design block's centre) launched from the
    substrate, 300 THz CW after a 200-step raised-cosine ramp; the objective's monitor is
    the 16x16 patch of E on the plane z = 80 at 300 THz.  ``scale`` > 1 divides every
    length but the 10-cell CPML by it (the same layout on a smaller grid, for checks
    that cannot afford the full size)."""
    import torch

    def s_(v):
        return int(v) // scale

    sc = Scene(cells=(s_(160), s_(160), s_(96)), spacing=SPACING, pml_cells=10)
    sc.structures.append(Structure(Box((0, 0, 0), (s_(160), s_(160), s_(40) - 1)), Medium(eps_r=2.1)))
    gen = torch.Generator().manual_seed(seed)
    shape = (s_(64), s_(64), s_(16))
    eps_r = (1.0 + 11.0 * torch.rand(shape, generator=gen, dtype=torch.float64)).numpy()
    sc.material_regions.append(MaterialRegion((s_(48), s_(48), s_(40)), (s_(112), s_(112), s_(56)), eps_r))
    dt = sc.resolve_dt()
    sc.sources.append(GaussianBeam((0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 1.0e-6 / scale, (s_(80), s_(80), s_(48)),
                                   CW(300e12, ramp_time=200 * dt)))
    sc.monitors.append(PlaneMonitor("patch", 2, s_(80), ("Ex", "Ey", "Ez"), (300e12,), (s_(72), s_(72)),
                                    (s_(72) + 16 // scale - 1, s_(72) + 16 // scale - 1)))
    return sc


def batched_designs(n_scenes: int = 32, seed: int = 1, size_range: tuple[int, int] = (64, 192), pml: int = 8,
                    n_freq: int = 8, design: bool = False) -> list[Scene]:
    """Batched design workload: ``n_scenes`` independent scenes whose cell counts per axis
    are drawn uniformly from ``size_range`` (numpy.random.default_rng(seed)); 8-cell CPML;
    4-8 boxes per scene (seeded positions and sizes) of diagonal anisotropic permittivity
    with eps_xx, eps_yy, eps_zz ~ U[1, 6]; an Ez point dipole (300/100 THz pulse) at the
    centre; an 8-frequency (250-350 THz) point monitor of all six components.  With
    ``design`` each scene also gets an 8x8x8-cell MaterialRegion (eps_r ~ U[1, 6) from
    numpy.random.default_rng([seed, 7]), so the scenes are the same with or without it)
    between the dipole and the probe, for per-scene adjoint gradients."""
    rng = np.random.default_rng(seed)
    design_rng = np.random.default_rng([seed, 7])
    lo_n, hi_n = size_range
    freqs = tuple(np.linspace(250e12, 350e12, n_freq))
    scenes = []
    for _ in range(n_scenes):
        cells = tuple(int(v) for v in rng.integers(lo_n, hi_n + 1, size=3))
        sc = Scene(cells=cells, spacing=SPACING, pml_cells=pml)
        for _ in range(int(rng.integers(4, 9))):
            size = [int(rng.integers(4, max(5, (c - 2 * pml) // 3))) for c in cells]
            lo = [int(rng.integers(pml + 1, max(pml + 2, c - pml - s_ - 1))) for c, s_ in zip(cells, size)]
            eps = tuple(float(v) for v in rng.uniform(1.0, 6.0, size=3))
            sc.structures.append(
                Structure(Box(tuple(lo), tuple(l + s_ for l, s_ in zip(lo, size))), Medium(eps_r=1.0, eps_diag=eps))
            )
        centre = tuple(c // 2 for c in cells)
        sc.sources.append(PointDipole(centre, "Ez", GaussianPulse(300e12, 100e12), width=SPACING))
        probe = (centre[0] + cells[0] // 4, centre[1], centre[2])
        sc.monitors.append(PointMonitor("probe", probe, frequencies=freqs))
        if design:
            lo = (centre[0] + 2, centre[1] - 4, centre[2] - 4)
            eps_r = design_rng.uniform(1.0, 6.0, size=(8, 8, 8))
            sc.material_regions.append(MaterialRegion(lo, tuple(v + 8 for v in lo), eps_r))
        scenes.append(sc)
    return scenes


def bloch_grating(cells: tuple[int, int, int] = (512, 512, 384), pml: int = 16, n_freq: int = 32,
                  kx_fraction: float = 0.1) -> Scene:
    """Large grating workload: Bloch-periodic x / y faces with k_x = kx_fraction * 2 pi / L_x
    (k_y = 0) and a 16-cell CPML on z; a Debye grating layer (eps_inf 2.5, delta_eps 3.5,
    tau 1e-14 s) 32 cells high at z in [176, 208) with a 64-cell period in x and 50 % duty
    (scaled with the grid); an Ex-polarised plane wave (300 THz, fwidth 120 THz) heading
    down z through a TFSF slab from 40 cells below the top CPML to 16 cells above the
    bottom one (the reference's grating slab, witwin/maxwell/fdtd/excitation/
    tfsf_state.py:202-279); a 32-frequency diffraction plane (Ex, Ey, Hx, Hy) at z = 320."""
    nx, ny, nz = cells
    sz = nz / 384.0
    L = nx * SPACING
    k = (kx_fraction * 2.0 * np.pi / L, 0.0, 0.0)
    sc = Scene(cells=cells, spacing=SPACING, pml_cells=pml, boundary=(3, 3, 3, 3, 1, 1), bloch_k=k)
    z0, z1 = int(round(176 * sz)), int(round(208 * sz))
    period = max(2, int(round(64 * nx / 512.0)))
    for x0 in range(0, nx, period):
        x1 = min(nx, x0 + period // 2)
        sc.structures.append(Structure(Box((x0, 0, z0), (x1, ny, z1)), Medium.debye(2.5, 3.5, 1e-14)))
    sc.sources.append(PlaneWaveTFSF((0.0, 0.0, -1.0), (1.0, 0.0, 0.0), GaussianPulse(300e12, 120e12),
                                    (0, 0, pml + int(round(16 * sz))), (nx, ny, nz - pml - int(round(40 * sz))),
                                    slab=True))
    freqs = tuple(np.linspace(250e12, 350e12, n_freq))
    sc.monitors.append(PlaneMonitor("diffraction", 2, int(round(320 * sz)) if nz >= 384 else nz - pml - 2,
                                    ("Ex", "Ey", "Hx", "Hy"), freqs))
    return sc


def algorithmic_bytes(compiled, *, kahan: bool = True, storage_bytes: int = 4) -> dict:
    """Compulsory HBM bytes per cell-update of one leapfrog step (every state array read
    once and written once), split into the fused step kernel's share and the whole step.

    fields: 6 arrays R+W; coefficients: 4 B per non-uniform decay/curl array; CPML psi:
    4 arrays per axis R+W over the slab fraction 2L/N; ADE: state arrays R+W over the
    material cells; monitors: the per-step running-DFT read-modify-write of every
    monitor point (F frequencies, re/im, x2 with Kahan compensation).  The fused kernel
    itself writes one 4-byte sample per monitor point and step; the batched DFT flush
    does the accumulator traffic.
    """
    nodes = compiled.nodes
    cells = float(np.prod([n - 1 for n in nodes]))
    s = float(storage_bytes)
    out = {"fields": 6 * 2 * s}
    nonuni = sum(1 for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz") for arr in (compiled.decay[n], compiled.curl[n]) if arr is not None)
    out["coefficients"] = 4.0 * nonuni
    psi = 0.0
    for a in range(3):
        L = compiled.pml_lo[a] + compiled.pml_hi[a]
        psi += 4 * 2 * 4.0 * L / (nodes[a] - 1)
    out["cpml_psi"] = psi
    ade = 0.0
    for p in compiled.poles:
        region = float(np.count_nonzero(p.drive))
        states = 2 if p.kind == 2 else 1
        ade += region * states * 2 * s
    out["ade"] = ade / cells
    nf = len(compiled.frequencies)
    points = sum((r.box[1] - r.box[0]) * (r.box[3] - r.box[2]) * (r.box[5] - r.box[4]) for r in compiled.regions)
    out["monitor_dft"] = points * nf * 2 * 2 * 4.0 * (2 if kahan else 1) / cells
    out["monitor_samples"] = points * 4.0 / cells
    out["step_kernel"] = out["fields"] + out["coefficients"] + out["cpml_psi"] + out["ade"] + out["monitor_samples"]
    out["total"] = out["fields"] + out["coefficients"] + out["cpml_psi"] + out["ade"] + out["monitor_dft"]
    out["cells"] = cells
    return out
