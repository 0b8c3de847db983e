"""Per-element diagnostics on the GPU: the kinetic energy of
euler_3d_compute_aux (Euler3D.okl:3888-3934) against the reference's own
kernel compiled in oracle/_ref (and against numpy where that library is not
built, and in 2D), and the entropy integral of the reference's driver
(euler.c:4135-4156) per element against numpy and in total against
ic.entropy, at the parity tolerance."""

import math

import numpy as np
import pytest

from oracle.pyoracle import Reference, reference_available
from scratch_wadge_b200 import ic as IC
from tests.helpers import RTOL, Case, golden_names, perturbed, rel
from tests.test_gpu_parity import Dev

pytestmark = pytest.mark.gpu


def _numpy_ke(geo, Q):
    dim = geo.ops.dim
    m2 = sum(Q[:, 1 + d, :] ** 2 for d in range(dim))
    return np.sum(0.5 * m2 / Q[:, 0, :] * geo.Jq * geo.ops.wq[None, :], axis=1)


def _numpy_entropy(geo, Q, gamma=1.4):
    dim = geo.ops.dim
    rho, E = Q[:, 0, :], Q[:, dim + 1, :]
    m2 = sum(Q[:, 1 + d, :] ** 2 for d in range(dim))
    s = np.log((gamma - 1.0) * (E - 0.5 * m2 / rho) / rho ** gamma)
    return np.sum(geo.ops.wq[None, :] * geo.Jq * (-rho * s), axis=1)


@pytest.mark.parametrize("name", golden_names())
def test_element_kinetic_energy_and_entropy(cuda, name):
    c = Case(name)
    Q = perturbed(c.state(), 4, 1e-2)["Q"]
    d = Dev(cuda, c.geo, c.curved)
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    Qd, wq, Jq = t(Q), t(c.ops.wq), t(c.geo.Jq)
    ke, S = t(np.zeros(c.geo.K)), t(np.zeros(c.geo.K))
    d.ctx.compute_aux(c.geo.K, Jq.data_ptr(), wq.data_ptr(), Qd.data_ptr(), ke.data_ptr())
    d.ctx.element_entropy(c.geo.K, Jq.data_ptr(), wq.data_ptr(), Qd.data_ptr(), S.data_ptr())
    d.sync()
    ke, S = ke.cpu().numpy(), S.cpu().numpy()
    if c.dim == 3 and reference_available(3, c.N):
        ref = Reference(c.ops, curved=True).compute_aux(c.geo, Q)  # the reference's own kernel
    else:
        ref = _numpy_ke(c.geo, Q)
    assert rel(ke, ref) < RTOL
    assert rel(S, _numpy_entropy(c.geo, Q)) < RTOL
    assert abs(math.fsum(S) - IC.entropy(c.geo, Q)) <= RTOL * abs(IC.entropy(c.geo, Q))


def _entropy_balance(cuda, m, N, curved, kind, tau):
    """A stage, then vol + surf on the GPU and wadg_entropy_rhs; returns the
    device per-element balance, the host one (sum_i w V(u~_i) . rhs_i with u~
    the state the volume kernel read) and the per-element scale
    sum |w V . rhs|."""
    from scratch_wadge_b200 import mesh as M  # noqa: F401  (m is a mesh.Mesh)
    geo = M.build_geometry(m, N)
    Q, rhsQ, Qf, resQ = IC.stage0(geo, IC.initial_state(geo, kind))
    d = Dev(cuda, geo, curved, tau=tau)
    s = d.put(dict(Q=Q, rhsQ=rhsQ.copy(), Qf=Qf, resQ=resQ, rhsQf=np.zeros_like(Qf)))
    # one stage first: the stage-0 builder projects with VqPq alone, the
    # update kernel (and the diagnostic) with the weight-adjusted projection
    d.vol(s)
    d.surf(s)
    d.update(s, IC.RK4A[1], IC.RK4B[1], 1e-3)
    rhs_in = s["rhsQ"].cpu().numpy()
    d.vol(s)
    d.surf(s)
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    wq, out = t(geo.ops.wq), t(np.zeros(geo.K))
    d.ctx.entropy_rhs(curved, geo.K, wq.data_ptr(), d.g["Jq"].data_ptr(), d.g["VqPq"].data_ptr(),
                      s["Q"].data_ptr(), s["rhsQ"].data_ptr(), out.data_ptr())
    d.sync()
    r = s["rhsQ"].cpu().numpy()
    V = IC.VU(rhs_in.transpose(1, 2, 0)).transpose(2, 0, 1)  # [K][Nf][Nq]
    terms = geo.ops.wq[None, None, :] * V * r
    return out.cpu().numpy(), terms.sum(axis=(1, 2)), np.abs(terms).sum(axis=(1, 2))


@pytest.mark.parametrize("dim,N,curved,tau", [(3, 3, False, 0.0), (3, 3, True, 0.0), (3, 4, True, 1.0),
                                              (3, 2, False, 1.0), (2, 3, True, 1.0), (2, 4, False, 1.0)])
def test_entropy_rhs_matches_host(cuda, dim, N, curved, tau):
    from scratch_wadge_b200 import mesh as M
    m = (M.periodic_cube(2, warp=M.warp_cube(0.05) if curved else None) if dim == 3
         else M.periodic_square(4, 4))
    kind = ("density_wave" if curved else "taylor_green") if dim == 3 else "vortex"
    dev, host, scale = _entropy_balance(cuda, m, N, curved, kind, tau)
    assert np.all(np.abs(dev - host) <= RTOL * scale), float(np.max(np.abs(dev - host) / scale))
    if tau == 0.0:
        # entropy conservative without the penalty: the volume terms cancel
        assert abs(math.fsum(dev)) < 1e-12 * scale.sum()
    else:
        assert math.fsum(dev) > 0.0  # dissipated by the Lax-Friedrichs penalty
