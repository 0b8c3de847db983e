"""Partitioned runs on one GPU: the halo pack kernel (wadg_halo_pack) equals
its host form bit for bit, and a mesh cut into 2-4 parts, each part stepping
its own elements with the halo exchanged between stages (all parts in one
process), gives the single-domain run's state bit for bit -- per element the
kernels do the same arithmetic in any partition."""

import numpy as np
import pytest

from scratch_wadge_b200 import build as B
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import ic as IC
from scratch_wadge_b200 import mesh as M
from scratch_wadge_b200 import partition as PT
from tests.test_partition import bounded_square

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build()


def _case(name):
    if name == "tg3d_N3":
        return M.periodic_cube(4), 3, False, "taylor_green", {}
    if name == "dw3d_curved_N2":
        return M.periodic_cube(3, warp=M.warp_cube(0.05)), 2, True, "density_wave", {}
    if name == "vortex2d_curved_N3":
        return M.periodic_square(8, 6), 3, True, "vortex", {}
    return bounded_square(6, 4), 2, False, "vortex", {}


def test_halo_pack_matches_host(cuda):
    geo = M.build_geometry(M.periodic_cube(3), 3)
    U0 = IC.initial_state(geo, "taylor_green")
    Q, rhsQ, Qf, resQ = IC.stage0(geo, U0)
    plans = PT.plan(geo, 3)
    for p in plans:
        part = PT.Part(geo, p, dict(Q=Q, rhsQ=rhsQ, Qf=Qf, resQ=resQ), False)
        rng = np.random.default_rng(p.rank)
        host = rng.standard_normal(tuple(part.Qf.shape))
        part.Qf.copy_(cuda.from_numpy(host))
        part.pack()
        cuda.cuda.synchronize()
        assert np.array_equal(part.sendbuf.cpu().numpy(), PT.pack_host(p, host))
        part.close()


@pytest.mark.parametrize("name,nparts", [("tg3d_N3", 2), ("tg3d_N3", 3), ("dw3d_curved_N2", 4),
                                         ("vortex2d_curved_N3", 3), ("bounded2d_N2", 2)])
def test_partitioned_run_equals_single_domain(cuda, name, nparts):
    mesh, N, curved, kind, kw = _case(name)
    geo = M.build_geometry(mesh, N)
    Q, rhsQ, Qf, resQ = IC.stage0(geo, IC.initial_state(geo, kind, **kw))
    dt = IC.time_step(geo, 0.5, N, nsteps=1, wave_speed=IC.max_wave_speed(Q))[0]
    app = capi.App(geo, curved)
    app.set_state(Q, rhsQ, Qf, resQ)
    app.rk_run(dt, 3, graph=False)
    ref = app.get_state()["Q"]
    app.close()
    state = dict(Q=Q, rhsQ=rhsQ, Qf=Qf, resQ=resQ)
    parts = [PT.Part(geo, p, state, curved) for p in PT.plan(geo, nparts)]
    assert sum(p.plan.ghost_pe for p in parts) > 0
    PT.run_local(parts, dt, 3)
    cuda.cuda.synchronize()
    got = PT.gather_Q(parts, geo.K)
    for p in parts:
        p.close()
    assert np.array_equal(got, ref), float(np.abs(got - ref).max() / np.abs(ref).max())
