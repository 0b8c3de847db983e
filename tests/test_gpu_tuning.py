"""The volume kernel's CTA shapes (wadg_vol_warps_candidates /
wadg_ctx_set_vol_warps) and the autotuner that picks one (wadg_app_autotune):
every compiled shape gives the same volume RHS bit for bit (an element's
arithmetic does not depend on how many elements share a CTA), shapes that are
not compiled are rejected, and an autotuned app still matches the reference's
time step to 1e-12."""

import ctypes

import numpy as np
import pytest

from scratch_wadge_b200 import capi
from tests.helpers import RTOL, Case, golden_names, rel
from tests.test_gpu_parity import Dev

pytestmark = pytest.mark.gpu


def _candidates(ctx, curved):
    c = (ctypes.c_int * 3)()
    n = capi.lib().wadg_vol_warps_candidates(ctx.h, int(curved), c)
    assert 1 <= n <= 3
    return [c[i] for i in range(n)]


@pytest.mark.parametrize("name", golden_names())
def test_every_cta_shape_gives_the_same_volume_rhs(cuda, name):
    c = Case(name)
    d = Dev(cuda, c.geo, c.curved)
    outs = []
    for w in _candidates(d.ctx, c.curved):
        capi.check(capi.lib().wadg_ctx_set_vol_warps(d.ctx.h, int(c.curved), w), "set_vol_warps")
        assert capi.lib().wadg_ctx_get_vol_warps(d.ctx.h) == w
        s = d.put(c.state())
        d.vol(s)
        d.sync()
        outs.append(d.get(s))
    for o in outs[1:]:
        assert np.array_equal(o["rhsQ"], outs[0]["rhsQ"]) and np.array_equal(o["rhsQf"], outs[0]["rhsQf"])
    assert rel(outs[0]["rhsQ"], c.z["vol_rhsQ"]) < RTOL


def test_shapes_that_are_not_compiled_are_rejected(cuda):
    c = Case("tg3d_affine_N3")
    d = Dev(cuda, c.geo, c.curved)
    assert capi.lib().wadg_ctx_set_vol_warps(d.ctx.h, 0, 7) == 1
    assert b"not a compiled shape" in capi.lib().wadg_last_error()
    assert capi.lib().wadg_ctx_set_vol_warps(d.ctx.h, 0, 0) == 0  # back to the default


@pytest.mark.parametrize("name", ["tg3d_affine_N3", "dw3d_curved_N3", "vortex2d_curved_N4"])
def test_autotuned_app_matches_reference_step(cuda, name):
    c = Case(name)
    app = capi.App(c.geo, c.curved)
    st = c.state()
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    w, times = app.autotune(c.dt, nstages=3)
    assert w in times and all(t > 0 for t in times.values())
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    app.rk_run(c.dt, 1, graph=True)
    assert rel(app.get_state()["Q"], c.z["step_Q"]) < RTOL
