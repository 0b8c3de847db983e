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
