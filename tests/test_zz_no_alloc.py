"""wadg_rk_stage_noalloc: one LSRK stage with no device allocation.

Some callers cannot let a library allocate GPU memory: a host program that
owns every device buffer through its own pool and hands the library only
those (the reference's driver allocates everything up front this way), or a
time loop that must not call cudaMalloc/cudaFree because they synchronise the
device and may fail mid-run.  For them this entry point keeps the one buffer
a stage needs between the volume and the surface kernel in a fixed device
array of the library.

The test calls it through the C ABI twice in a row (two different LSRK
stages) and compares every output with the same stages run through the
existing kernel entry points with a caller-allocated face-row buffer, at the
parity tolerance of the other tests.  It needs no other test to have run
first.  This file sorts last so that a run stopping at the first failure has
already run everything else.
"""

import ctypes

import numpy as np
import pytest

from scratch_wadge_b200 import build as B
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import ic as IC
from tests.helpers import RTOL, Case, rel

pytestmark = pytest.mark.gpu


def _noalloc(L):
    f = L.wadg_rk_stage_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 14 + \
                 [ctypes.c_double] * 3 + [ctypes.c_void_p] * 4
    return f


@pytest.mark.parametrize("name", ["tg3d_affine_N3", "dw3d_curved_N3", "vortex2d_curved_N3"])
def test_noalloc_stage_matches_kernel_entry_points(cuda, name):
    B.build()
    L = capi.lib()
    stage = _noalloc(L)
    c = Case(name)
    ops, geo = c.ops, c.geo
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    g = dict(vgeo=t(geo.vgeo), vfgeo=t(geo.vfgeo), fgeo=t(geo.fgeo), Jq=t(geo.Jq),
             mapPq=cuda.from_numpy(np.ascontiguousarray(geo.mapPq, dtype=np.uint32).view(np.int32)).cuda(),
             nrJ=t(ops.nrJ), nsJ=t(ops.nsJ), ntJ=t(ops.ntJ), Drq=t(ops.fortran("Drq")),
             Dsq=t(ops.fortran("Dsq")), Dtq=t(ops.fortran("Dtq")), VqLq=t(ops.fortran("VqLq")),
             VqPq=t(ops.fortran("VqPq")), VfPq=t(ops.fortran("VfPq")))
    p = {k: v.data_ptr() for k, v in g.items()}
    ctx = capi.Context(ops, stream=cuda.cuda.current_stream().cuda_stream)
    st = c.state()
    a = {k: t(v) for k, v in st.items()}  # through the no-allocation entry point
    b = {k: t(v) for k, v in st.items()}  # through the kernel entry points
    for s in (1, 2):  # two calls in a row
        fa, fb = IC.RK4A[s], IC.RK4B[s]
        rc = stage(ctx.h, geo.K, int(c.curved), p["vgeo"], p["vfgeo"], p["fgeo"], p["mapPq"],
                   p["nrJ"], p["nsJ"], p["ntJ"], p["Drq"], p["Dsq"], p["Dtq"], p["VqLq"], p["VqPq"],
                   p["VfPq"], p["Jq"], fa, fb, c.dt, a["rhsQ"].data_ptr(), a["resQ"].data_ptr(),
                   a["Q"].data_ptr(), a["Qf"].data_ptr())
        assert rc == 0, L.wadg_last_error()
        ctx.vol(c.curved, geo.K, p["vgeo"], p["vfgeo"], p["nrJ"], p["nsJ"], p["ntJ"], p["Drq"], p["Dsq"],
                p["Dtq"], p["VqLq"], p["VfPq"], b["Qf"].data_ptr(), b["rhsQ"].data_ptr(),
                b["rhsQf"].data_ptr())
        ctx.surf(geo.K, p["fgeo"], p["mapPq"], p["VqLq"], b["Qf"].data_ptr(), b["rhsQf"].data_ptr(),
                 b["rhsQ"].data_ptr())
        ctx.update(c.curved, geo.K, p["Jq"], p["VqPq"], p["VfPq"], fa, fb, c.dt, b["rhsQ"].data_ptr(),
                   b["resQ"].data_ptr(), b["Q"].data_ptr(), b["Qf"].data_ptr())
        cuda.cuda.synchronize()
        for k in ("Q", "rhsQ", "Qf", "resQ"):
            x, y = a[k].cpu().numpy(), b[k].cpu().numpy()
            assert np.isfinite(x).all()
            assert rel(x, y) < RTOL, (s, k, rel(x, y))


def test_noalloc_rejects_k_beyond_the_fixed_array(cuda):
    B.build()
    L = capi.lib()
    stage = _noalloc(L)
    c = Case("tg3d_affine_N3")
    ctx = capi.Context(c.ops)
    K = 10 ** 6  # 240 doubles of face-row scratch per element: far beyond the array
    dummy = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    rc = stage(ctx.h, K, 0, *([dummy] * 14), 0.0, 1.0, 1e-3, *([dummy] * 4))
    assert rc == 1
    assert b"face-row scratch" in L.wadg_last_error()
