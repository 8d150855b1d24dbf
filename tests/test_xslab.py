"""x-slab decomposition (witwin-maxwell_b200/distributed.py) on CPU: world-size 2
and 3 gloo ranks, each stepping its slab with the FP64 oracle and exchanging halo
planes by torch.distributed point-to-point, reproduce the single-domain oracle
run exactly (fields and monitor spectra bit for bit): the owned cells see the
same arithmetic.  The scene puts CPML on every face, a dielectric box, a Lorentz
sphere, a Drude slab and a TFSF box across the cuts, a point dipole and plane and
point monitors."""
from __future__ import annotations

import datetime
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import load_package

ROOT = Path(__file__).resolve().parents[1]
STEPS = 40


def _scene(wm, nonlinear=False):
    sc = wm.Scene(cells=(30, 16, 14), spacing=25e-9, pml_cells=3)
    if nonlinear:
        # Kerr, chi2 and TPA channels across the cut of two ranks (node plane 16)
        sc.structures.append(wm.Structure(wm.Box((12, 3, 3), (21, 12, 11)),
                                          wm.Medium(eps_r=2.0, kerr_chi3=1e-4, chi2=0.005, tpa_beta=5e6, sigma=1e4)))
    sc.structures.append(wm.Structure(wm.Box((10, 4, 4), (20, 12, 10)), wm.Medium(eps_r=3.0)))
    sc.structures.append(wm.Structure(wm.Sphere((15, 8, 7), 3.0), wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
    sc.structures.append(wm.Structure(wm.Box((18, 3, 3), (21, 13, 11)),
                                      wm.Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))))
    sc.sources.append(wm.PointDipole((8, 8, 7), "Ez", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    sc.sources.append(wm.PlaneWaveTFSF((1, 0, 0), (0, 0, 1), wm.GaussianPulse(300e12, 100e12), (5, 5, 5),
                                       (25, 11, 9)))
    freqs = (250e12, 300e12)
    sc.monitors.append(wm.PlaneMonitor("zplane", 2, 9, ("Ex", "Ey", "Hz"), freqs))
    sc.monitors.append(wm.PlaneMonitor("yplane", 1, 7, ("Ez", "Hx", "Hy"), freqs))
    sc.monitors.append(wm.PointMonitor("probe", (22, 8, 7), frequencies=freqs))
    return sc


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out, nonlinear=False):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    from conftest import load_package as lp
    from oracle import oracle as orc

    wm = lp()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cs = wm.compile_scene(_scene(wm, nonlinear), STEPS)
        run = wm.distributed.XSlabRun(cs, rank, world, stepper=lambda local: orc.OracleSimulation(local, "f64",
                                                                                                   threads=1))
        run.run(0, STEPS)
        fields = [None] * world if rank == 0 else None
        mons = [None] * world if rank == 0 else None
        dist.gather_object(run.owned_fields(), fields, dst=0)
        dist.gather_object(run.local_monitors(), mons, dst=0)
        run.close()
        if rank == 0:
            out.put((wm.distributed.assemble_fields(cs, fields), wm.distributed.assemble_monitors(cs, mons)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nonlinear", [(2, False), (3, False), (2, True)])
def test_xslab_ranks_reproduce_single_domain(world, nonlinear):
    from oracle import oracle as orc

    wm = load_package()
    cs = wm.compile_scene(_scene(wm, nonlinear), STEPS)
    ref = orc.OracleSimulation(cs, "f64", threads=1).run(STEPS)
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, nonlinear)) for r in range(world)]
    for p in procs:
        p.start()
    fields, mons = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert max(float(np.abs(ref.fields["Ez"]).max()), 0.0) > 0
    for name, arr in ref.fields.items():
        np.testing.assert_array_equal(fields[name], arr, err_msg=name)
    refm = ref.monitor_results()
    for m, comps in refm.items():
        for c, v in comps.items():
            np.testing.assert_array_equal(mons[m][c], v, err_msg=f"{m}.{c}")
    ref.close()


def test_slab_split_and_checks():
    wm = load_package()
    d = wm.distributed
    assert d.split_planes(31, 2) == [(0, 16), (16, 31)]
    assert d.split_planes(31, 3) == [(0, 11), (11, 21), (21, 31)]
    cs = wm.compile_scene(_scene(wm), 4)
    local, placement = d.slice_scene(cs, 11, 21)
    assert local.nodes == (12, cs.nodes[1], cs.nodes[2])
    assert local.pml_lo[0] == 0 and local.pml_hi[0] == 0 and local.boundary[:2] == (0, 0)
    # every monitor cell is owned by exactly one rank
    counts = {}
    for x0, x1 in d.split_planes(cs.nodes[0], 3):
        loc, pl = d.slice_scene(cs, x0, x1)
        for reg, (g, off) in zip(loc.regions, pl):
            counts[g] = counts.get(g, 0) + (reg.box[1] - reg.box[0])
    for g, reg in enumerate(cs.regions):
        assert counts[g] == reg.box[1] - reg.box[0]
    with pytest.raises(ValueError):
        d.slice_scene(cs, 2, 16)  # the cut's ghost plane falls in the low CPML slab
    with pytest.raises(ValueError):
        d.split_planes(3, 2)


@pytest.mark.gpu
@pytest.mark.parametrize("world,nonlinear", [(2, False), (3, False), (2, True)])
def test_xslab_engines_match_single_engine(world, nonlinear):
    """The slabs as fused engines on one device (ranks of one process, halo planes
    copied device to device) against one engine over the whole grid, at the
    engine's parity bars (joint relative L2 <= 1e-5, <= 1e-4 per component)."""
    wm = load_package()
    d = wm.distributed
    steps = 200
    cs = wm.compile_scene(_scene(wm, nonlinear), steps)
    single = wm.solver.B200FDTD(cs).init_field()
    single.step_range(0, steps)
    ref_f = {n: single.field(n).cpu().numpy() for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    ref_m = {k: {c: v.cpu().numpy() for c, v in m.items()} for k, m in single.monitor_results().items()}
    single.close()
    runs = [d.XSlabRun(cs, r, world, exchange=lambda run: None) for r in range(world)]
    for n in range(steps):
        d.step_in_process(runs, n)
    for r in runs:
        r.stepper.finish()
    fields = d.assemble_fields(cs, [r.owned_fields() for r in runs])
    mons = d.assemble_monitors(cs, [r.local_monitors() for r in runs])
    for r in runs:
        r.close()
    # the engine parity bars: launch shapes differ between the slabs and the whole
    # grid, so FMA contraction and summation order differ at the rounding level
    from test_engine_parity import assert_fields_close, assert_monitors_close

    assert all(float(np.abs(a).max()) > 0 for a in ref_f.values())
    assert_fields_close(fields, ref_f)
    assert_monitors_close(mons, ref_m)
