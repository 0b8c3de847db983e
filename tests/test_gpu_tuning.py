"""The volume kernel's shapes (wadg_vol_shapes / wadg_ctx_set_vol_shape:
warps per CTA and the node-to-thread map, rows per lane) and the autotuner
that picks one (wadg_app_autotune): every compiled shape gives the same volume
RHS bit for bit under one node-to-thread map (an element's arithmetic does
not depend on how many elements share a CTA), the other maps to rounding
(they split the columns over another number of warps), shapes that are not compiled
are rejected, and an autotuned app still matches the reference's time step to
1e-12."""

import numpy as np
import pytest

from scratch_wadge_b200 import capi
from tests.helpers import RTOL, Case, golden_names, rel
from tests.test_gpu_parity import Dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_names())
def test_every_cta_shape_gives_the_same_volume_rhs(cuda, name):
    c = Case(name)
    d = Dev(cuda, c.geo, c.curved)
    outs, vs = [], []
    shapes = d.ctx.vol_shapes(c.curved)
    assert 1 <= len(shapes) <= capi.MAX_VOL_SHAPES
    for w, r in shapes:
        d.ctx.set_vol_shape(c.curved, w, r)
        assert capi.lib().wadg_ctx_get_vol_warps(d.ctx.h) == w
        assert capi.lib().wadg_ctx_get_vol_rows(d.ctx.h) == r
        s = d.put(c.state())
        d.vol(s)
        d.sync()
        outs.append(d.get(s))
        s = d.put(c.state())
        d.volsurf(s)
        d.sync()
        vs.append(d.get(s))
    d.ctx.set_vol_warps(c.curved, 0)
    # the same node-to-thread map: bit for bit; another map splits an
    # element's columns over another number of warps (another summation
    # order): to rounding
    for k, (w, r) in enumerate(shapes):
        j = [i for i, (_, r0) in enumerate(shapes) if r0 == r][0]
        assert np.array_equal(outs[k]["rhsQ"], outs[j]["rhsQ"]), (w, r)
        assert np.array_equal(outs[k]["rhsQf"], outs[j]["rhsQf"]), (w, r)
        assert np.array_equal(vs[k]["rhsQ"], vs[j]["rhsQ"]), (w, r)
        assert rel(outs[k]["rhsQ"], c.z["vol_rhsQ"]) < RTOL, (w, r)
        assert rel(outs[k]["rhsQf"], c.z["vol_rhsQf"]) < RTOL, (w, r)
        assert rel(vs[k]["rhsQ"], vs[0]["rhsQ"]) < RTOL, (w, r)


def test_node_to_thread_maps_where_compiled(cuda):
    """2D N=4 (16 volume nodes: 8 lanes x 2 rows per element by default)
    also compiles 4 lanes x 4 rows; 3D N=3 (23 nodes, 8 lanes x 3 rows) has
    no other map (4 lanes x 6 rows would spill, 16 x 2 pads 9 slots)"""
    c = Case("vortex2d_curved_N4")
    d = Dev(cuda, c.geo, c.curved)
    assert (8, 4) in d.ctx.vol_shapes(c.curved)
    c3 = Case("tg3d_affine_N3")
    d3 = Dev(cuda, c3.geo, c3.curved)
    assert all(r == 0 for _, r in d3.ctx.vol_shapes(c3.curved))


def test_shapes_that_are_not_compiled_are_rejected(cuda):
    c = Case("tg3d_affine_N3")
    d = Dev(cuda, c.geo, c.curved)
    assert capi.lib().wadg_ctx_set_vol_warps(d.ctx.h, 0, 7) == 1
    assert b"not a compiled shape" in capi.lib().wadg_last_error()
    assert capi.lib().wadg_ctx_set_vol_shape(d.ctx.h, 0, 12, 3) == 1
    assert capi.lib().wadg_ctx_set_vol_warps(d.ctx.h, 0, 0) == 0  # back to the default
    assert capi.lib().wadg_ctx_get_vol_rows(d.ctx.h) == 0


@pytest.mark.parametrize("name", ["tg3d_affine_N3", "dw3d_curved_N3", "vortex2d_curved_N4"])
def test_autotuned_app_matches_reference_step(cuda, name):
    c = Case(name)
    app = capi.App(c.geo, c.curved)
    st = c.state()
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    w, times = app.autotune(c.dt, nstages=3)
    assert w in times and all(t > 0 for t in times.values())
    assert len(times) == len(capi.vol_shapes(capi.ctypes.c_void_p(capi.lib().wadg_app_ctx(app.h)), c.curved))
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    app.rk_run(c.dt, 1, graph=True)
    assert rel(app.get_state()["Q"], c.z["step_Q"]) < RTOL
