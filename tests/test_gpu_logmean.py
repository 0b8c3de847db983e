"""The log-mean's branches, tested directly through the volume kernel.

The reference's log-mean (Euler3Daffine.okl:43-71, Euler2D.okl:36-67) takes
its series F = 1 + u/3 + u^2/5 + u^3/7 (+ u^4/9 in 2D) below
u = ((a-b)/(a+b))^2 < 1e-4 (3D) or 1e-3 (2D), and log(a/b)/(2f) above.  The
volume kernel computes it differently: a degree-8 series (of F or 1/F) below
u < 1e-2, the difference of per-node logarithms above, and, when all 32 lanes
of a warp have u < 1e-6 for both the density and beta pairs, a series cut at
u^2.  The states here put node pairs on both sides of every switch: each
element gets densities rho_i = rho0 (1 + a r_i) and pressures
p_i = p0 (1 + b s_i) with seeded r_i, s_i in [-1, 1] and amplitudes a, b
log-uniform over elements (shuffled, so the elements of one warp differ),
so that the pairs' u spans 1e-12 to 0.3: whole warps below 1e-6, warps whose
lanes disagree on that vote, and pairs just below and just above 1e-4, 1e-3
and 1e-2.  The kernel's volume RHS must equal the reference's own kernels'
(oracle/_ref; the C restatement where it is absent) to 1e-12."""

import numpy as np
import pytest

from oracle import pyoracle as O
from scratch_wadge_b200 import mesh as M
from tests.helpers import RTOL, rel
from tests.test_gpu_parity import Dev

pytestmark = pytest.mark.gpu

GAMMA = 1.4


def oracle(ops, curved):
    try:
        return O.Reference(ops, curved)
    except FileNotFoundError:
        return O.Port(ops, curved)


def branch_state(geo, seed, umax_lo=1e-12, umax_hi=0.3, rho0=1.3, p0=2.0):
    """traces (rhsQ = u~ at volume nodes, Qf = uf~ at face nodes) whose node
    pairs cover the log-mean's branches"""
    ops = geo.ops
    K, Nq, NF, dim = geo.K, ops.Nq, ops.NfqNf, ops.dim
    rng = np.random.default_rng(seed)
    n = Nq + NF
    amp = lambda: np.sqrt(np.exp(rng.uniform(np.log(umax_lo), np.log(umax_hi), K)))
    a, b = amp(), amp()
    a[rng.permutation(K)[: K // 8]] = 1e-7  # some elements entirely in the u^2 range
    r, s = rng.uniform(-1, 1, (K, n)), rng.uniform(-1, 1, (K, n))
    rho = rho0 * (1.0 + a[:, None] * r)
    p = p0 * (1.0 + b[:, None] * s)
    vel = 0.2 * rng.standard_normal((K, dim, n))
    E = p / (GAMMA - 1.0) + 0.5 * rho * (vel ** 2).sum(1)
    U = np.concatenate([rho[:, None], rho[:, None] * vel, E[:, None]], axis=1)  # [K][Nf][n]
    beta = rho / (2.0 * p)
    return np.ascontiguousarray(U[:, :, :Nq]), np.ascontiguousarray(U[:, :, Nq:]), rho, beta


def pair_u(x):
    """u of every node pair of every element, for one nodal quantity [K][n]"""
    d = x[:, :, None] - x[:, None, :]
    s = x[:, :, None] + x[:, None, :]
    return (d / s) ** 2


@pytest.mark.parametrize("dim,N,curved", [(3, 3, False), (3, 3, True), (3, 4, True), (3, 2, False),
                                          (2, 3, False), (2, 3, True), (2, 4, True)])
def test_volume_kernel_across_log_mean_branches(cuda, dim, N, curved):
    mesh = M.periodic_cube(3, warp=M.warp_cube(0.05) if curved else None) if dim == 3 \
        else M.periodic_square(6, 7)
    geo = M.build_geometry(mesh, N)
    uq, uf, rho, beta = branch_state(geo, 100 * dim + N)
    # the states cover every branch region, with pairs just either side of
    # each switch: the warp vote (1e-6), the reference's (1e-4 in 3D, 1e-3 in
    # 2D; float literals) and the kernel's series/log switch (1e-2)
    u = np.concatenate([pair_u(rho).ravel(), pair_u(beta).ravel()])
    thr_ref = float(np.float32(1e-4 if dim == 3 else 1e-3))
    for t in (1e-6, thr_ref, 1e-2):
        assert ((u >= 0.97 * t) & (u < t)).sum() >= 20, t
        assert ((u >= t) & (u < 1.03 * t)).sum() >= 20, t
    assert (u < 1e-10).sum() > 1000 and (u > 0.1).sum() >= 50

    d = Dev(cuda, geo, curved)
    st = dict(rhsQ=uq, Qf=uf, rhsQf=np.zeros_like(uf))
    s = d.put(st)
    d.vol(s)
    d.sync()
    h = d.get(s)
    ref = {k: v.copy() for k, v in st.items()}
    oracle(geo.ops, curved).vol(geo, ref["Qf"], ref["rhsQ"], ref["rhsQf"])
    assert rel(h["rhsQ"], ref["rhsQ"]) < RTOL, rel(h["rhsQ"], ref["rhsQ"])
    assert rel(h["rhsQf"], ref["rhsQf"]) < RTOL, rel(h["rhsQf"], ref["rhsQf"])


def warp_regime_state(geo, seed, targets, rho0=1.3, p0=2.0):
    """traces whose elements have a chosen largest pair u: element k's
    densities and pressures span rho0 (1 +- a_k) and p0 (1 +- b_k) (both
    extremes present), a_k^2 and about (a_k + b_k)^2 for beta set from
    targets[k % len(targets)], so whole warps fall on either side of the
    kernel's per-warp tests (u < 4e-6: the u^2 series without a vote; u <
    1e-2: the degree-8 series without the per-lane log choice)"""
    ops = geo.ops
    K, Nq, NF, dim = geo.K, ops.Nq, ops.NfqNf, ops.dim
    rng = np.random.default_rng(seed)
    n = Nq + NF
    t = np.asarray(targets, dtype=np.float64)[np.arange(K) % len(targets)]
    a = np.sqrt(t) / 2.0
    r, s = rng.uniform(-1, 1, (K, n)), rng.uniform(-1, 1, (K, n))
    r[:, 0], r[:, -1], s[:, 1], s[:, -2] = 1.0, -1.0, 1.0, -1.0
    rho = rho0 * (1.0 + a[:, None] * r)
    p = p0 * (1.0 + a[:, None] * s)
    vel = 0.2 * rng.standard_normal((K, dim, n))
    E = p / (GAMMA - 1.0) + 0.5 * rho * (vel ** 2).sum(1)
    U = np.concatenate([rho[:, None], rho[:, None] * vel, E[:, None]], axis=1)
    beta = rho / (2.0 * p)
    return np.ascontiguousarray(U[:, :, :Nq]), np.ascontiguousarray(U[:, :, Nq:]), rho, beta


def element_u(x):
    """the largest pair u of each element, for one nodal quantity [K][n]"""
    return ((x.max(1) - x.min(1)) / (x.max(1) + x.min(1))) ** 2


@pytest.mark.parametrize("dim,N,curved", [(3, 3, False), (3, 4, True), (2, 3, False), (2, 4, True)])
@pytest.mark.parametrize("targets", [[2e-6, 3.5e-6], [2e-6, 3.5e-6, 3.5e-6, 6e-6],
                                     [1e-5, 3e-3, 8e-3], [3e-3, 2e-2, 8e-3, 1e-4]])
def test_volume_kernel_per_warp_log_mean_paths(cuda, dim, N, curved, targets):
    """Warps whose elements are all nearly equal (u < 4e-6) skip the per-pair
    votes and take the u^2 series, also where a vote would have taken the
    degree-8 one (1e-6 <= u < 4e-6); warps with every pair below 1e-2 take
    the degree-8 series without the per-lane log-difference choice.  Mixed
    element lists put warps on both sides of each test.  The volume and the
    volume + surface kernels must equal the reference's kernels to 1e-12."""
    mesh = M.periodic_cube(3, warp=M.warp_cube(0.05) if curved else None) if dim == 3 \
        else M.periodic_square(6, 7)
    geo = M.build_geometry(mesh, N)
    uq, uf, rho, beta = warp_regime_state(geo, 7 * dim + N, targets)
    ue = np.maximum(element_u(rho), element_u(beta))
    assert ue.max() < 1.5 * max(targets) and ue.min() > 0.3 * min(targets)
    d = Dev(cuda, geo, curved)
    st = dict(rhsQ=uq, Qf=uf, rhsQf=np.zeros_like(uf))
    ref = {k: v.copy() for k, v in st.items()}
    oracle(geo.ops, curved).vol(geo, ref["Qf"], ref["rhsQ"], ref["rhsQf"])
    s = d.put(st)
    d.vol(s)
    d.sync()
    h = d.get(s)
    assert rel(h["rhsQ"], ref["rhsQ"]) < RTOL, rel(h["rhsQ"], ref["rhsQ"])
    assert rel(h["rhsQf"], ref["rhsQf"]) < RTOL, rel(h["rhsQf"], ref["rhsQf"])
    # the volume + surface kernel: the reference's surface kernel after its
    # volume kernel
    oracle(geo.ops, curved).surf(geo, np.ascontiguousarray(st["Qf"]).copy(), ref["rhsQf"], ref["rhsQ"])
    s = d.put(st)
    d.volsurf(s)
    d.sync()
    h = d.get(s)
    assert rel(h["rhsQ"], ref["rhsQ"]) < RTOL, rel(h["rhsQ"], ref["rhsQ"])
