"""fdtd_op_aux_line_history_static (incident-line history with its running
state in a fixed device array, no device allocation) against the existing
per-step entry points fdtd_op_aux_magnetic / fdtd_op_aux_electric stepped from
a zero line, through the C ABI.

Two calls in a row with different lines show that the second call does not
see the first call's state.  Tolerance rtol 1e-5, atol 1e-6 (the FP32
rounding of one op, as in the per-op parity tests).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_package

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-5, 1e-6


def _line(wm, cells, direction, steps):
    sc = wm.Scene(cells=(cells, 16, 16), spacing=25e-9, pml_cells=4)
    sc.sources.append(wm.PlaneWaveTFSF(direction, (0, 0, 1), wm.GaussianPulse(300e12, 100e12),
                                       (6, 5, 5), (cells - 6, 11, 11)))
    return wm.compile_scene(sc, steps).aux_line


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def _stepped(lib, aux):
    """History from the per-step entry points, recorded as the kernel records it."""
    ne = len(aux.e_decay)
    ed, ec, hd, hc = (_dev(a) for a in (aux.e_decay, aux.e_curl, aux.h_decay, aux.h_curl))
    e = torch.zeros(ne, device="cuda")
    h = torch.zeros(ne, device="cuda")
    e_rows, h_rows = [], []
    for n, value in enumerate(np.asarray(aux.source, dtype=np.float32)):
        e_rows.append(e.clone())
        assert lib.fdtd_op_aux_magnetic(ne, h.data_ptr(), e.data_ptr(), hd.data_ptr(), hc.data_ptr(), None) == 0
        h_rows.append(h.clone())
        assert lib.fdtd_op_aux_electric(ne, e.data_ptr(), h.data_ptr(), ed.data_ptr(), ec.data_ptr(),
                                        int(aux.source_index), float(value), None) == 0
    torch.cuda.synchronize()
    return torch.stack(e_rows).cpu().numpy(), torch.stack(h_rows).cpu().numpy()


def _static(lib, aux):
    ne = len(aux.e_decay)
    steps = len(aux.source)
    ins = [_dev(a) for a in (aux.e_decay, aux.e_curl, aux.h_decay, aux.h_curl, aux.source)]
    e_hist = torch.full((steps, ne), float("nan"), device="cuda")
    h_hist = torch.full((steps, ne), float("nan"), device="cuda")
    rc = lib.fdtd_op_aux_line_history_static(ne, ins[0].data_ptr(), ins[1].data_ptr(), ins[2].data_ptr(),
                                             ins[3].data_ptr(), int(aux.source_index), ins[4].data_ptr(), steps,
                                             e_hist.data_ptr(), h_hist.data_ptr(), None)
    assert rc == 0, lib.fdtd_last_error()
    torch.cuda.synchronize()
    return e_hist.cpu().numpy(), h_hist.cpu().numpy()


def test_static_history_matches_stepped_ops_twice_in_a_row():
    wm = load_package()
    lib = wm._lib.load()
    lines = [_line(wm, 48, (1, 0, 0), 160), _line(wm, 32, (-1, 0, 0), 120)]
    for aux in lines:
        got_e, got_h = _static(lib, aux)
        want_e, want_h = _stepped(lib, aux)
        assert np.abs(want_e).max() > 1e-3  # the pulse reached the recorded line
        np.testing.assert_allclose(got_e, want_e, rtol=RTOL, atol=ATOL)
        np.testing.assert_allclose(got_h[:, :-1], want_h[:, :-1], rtol=RTOL, atol=ATOL)
        assert np.all(got_h[:, -1] == 0.0)


def test_static_history_source_on_the_last_cell_and_no_source():
    """A source placed on the last line cell is overridden by that cell's zero
    (the reference's update_auxiliary_electric_kernel checks the last cell
    first), in the static entry point and in the per-step op alike; a negative
    source index injects nothing."""
    import dataclasses

    wm = load_package()
    lib = wm._lib.load()
    aux = _line(wm, 40, (1, 0, 0), 96)
    ne = len(aux.e_decay)
    # drive the last cell: its history stays zero and nothing propagates
    last = dataclasses.replace(aux, source_index=ne - 1)
    got_e, got_h = _static(lib, last)
    want_e, want_h = _stepped(lib, last)
    np.testing.assert_allclose(got_e, want_e, rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(got_h[:, :-1], want_h[:, :-1], rtol=RTOL, atol=ATOL)
    assert np.all(got_e == 0.0) and np.all(got_h == 0.0)
    # a source on the second-to-last cell still drives the line
    near = dataclasses.replace(aux, source_index=ne - 2)
    got_e, _ = _static(lib, near)
    want_e, _ = _stepped(lib, near)
    np.testing.assert_allclose(got_e, want_e, rtol=RTOL, atol=ATOL)
    assert np.abs(got_e).max() > 1e-3 and np.all(got_e[:, -1] == 0.0)
    none = dataclasses.replace(aux, source_index=-1)
    got_e, got_h = _static(lib, none)
    assert np.all(got_e == 0.0) and np.all(got_h == 0.0)


def test_static_history_rejects_lines_beyond_the_scratch_maximum():
    wm = load_package()
    lib = wm._lib.load()
    ne = 16384 + 1
    buf = torch.zeros(ne, device="cuda")
    rc = lib.fdtd_op_aux_line_history_static(ne, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(),
                                             1, buf.data_ptr(), 1, buf.data_ptr(), buf.data_ptr(), None)
    assert rc == -1
    assert b"exceeds the static scratch maximum of 16384" in lib.fdtd_last_error()
