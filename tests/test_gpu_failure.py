"""Failure detection: non-physical states are reported as an error status.

The reference has no such check: a bad state runs on into NaNs, and its only
failure path is an abort (ASD_ABORT, asd.h:77-79).  Here wadg_check_state
scans the conserved state, and wadg_rk_run can check it every few steps and
stop with WADG_ERR_STATE.  The bad states are made on the host (a negative
density, a NaN energy, a negative pressure); nothing faults the GPU: the
kernels compute NaNs on such states like any other arithmetic."""

import numpy as np
import pytest
import torch

from scratch_wadge_b200 import capi
from tests.helpers import Case

pytestmark = pytest.mark.gpu


def _bad(Q, Nq):
    """three non-physical nodes; returns the state and the smallest bad index"""
    Q = Q.copy()
    Q[3, 0, 5] = -1.0                      # rho < 0
    Q[7, -1, 2] = np.nan                   # E is NaN
    Q[10, -1, 0] = 0.1 * Q[10, -1, 0] - 50.0  # pressure < 0
    return Q, 3 * Nq + 5


@pytest.mark.parametrize("name", ["tg3d_affine_N3", "vortex2d_curved_N3"])
def test_check_state_kernel_entry_point(cuda, name):
    c = Case(name)
    ctx = capi.Context(c.ops, stream=torch.cuda.current_stream().cuda_stream)
    Q = c.z["in_Q"]
    K, Nq = Q.shape[0], Q.shape[2]
    work = torch.zeros(2, dtype=torch.int32, device="cuda")
    good = torch.from_numpy(np.ascontiguousarray(Q)).cuda()
    assert ctx.check_state(K, good.data_ptr(), work.data_ptr()) == (0, 0, -1)
    Qb, first = _bad(Q, Nq)
    bad = torch.from_numpy(np.ascontiguousarray(Qb)).cuda()
    r, nbad, f = ctx.check_state(K, bad.data_ptr(), work.data_ptr())
    assert (r, nbad, f) == (capi.ERR_STATE, 3, first)
    msg = capi.lib().wadg_last_error().decode()
    assert "element 3, node 5" in msg and "3 node" in msg
    # the work buffer is reset by every call: a good state after a bad one
    assert ctx.check_state(K, good.data_ptr(), work.data_ptr()) == (0, 0, -1)
    # only the first K elements are scanned
    assert ctx.check_state(3, bad.data_ptr(), work.data_ptr()) == (0, 0, -1)


def test_app_check_and_time_loop_stops_on_bad_state(cuda):
    c = Case("tg3d_affine_N3")
    st = c.state()
    app = capi.App(c.geo, c.curved)
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    assert app.check_state() == (0, 0, -1)
    # a healthy run with checks equals one without
    app.set_check_every(2)
    app.rk_run(c.dt, 4, graph=True)
    with_checks = app.get_state()["Q"]
    app.set_check_every(0)
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    app.rk_run(c.dt, 4, graph=True)
    assert np.array_equal(with_checks, app.get_state()["Q"])
    # a bad node stops the loop at the first check with WADG_ERR_STATE
    Qb, first = _bad(st["Q"], st["Q"].shape[2])
    app.set_state(Qb, st["rhsQ"], st["Qf"], st["resQ"])
    assert app.check_state()[:2] == (capi.ERR_STATE, 3)
    app.set_check_every(1)
    with pytest.raises(capi.WadgError) as ei:
        app.rk_run(c.dt, 3, graph=True)
    assert ei.value.code == capi.ERR_STATE and "after step 1" in str(ei.value)
    app.set_check_every(0)
    app.sync()  # the stream is still usable
