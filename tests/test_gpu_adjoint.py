"""Discrete adjoint on the GPU (wadg_adjoint_*), checked three ways:

* against central finite differences of the CPU reference RHS (the
  reference's own kernels compiled in oracle/_ref when present, else the C
  restatement) on seeded random directions;
* against automatic differentiation of an independent float64 restatement of
  the same map (oracle/torch_rhs.py, pinned to the C oracle in
  tests/test_adjoint_cpu.py): the VJP
  itself and the JVP/VJP dot product <w, J d> = <J^T w, d>;
* over whole LSRK-45 runs: the checkpointed reverse sweep against autodiff
  through the restated run, against finite differences of J = int rho^2 on
  the Taylor-Green mesh of 8^3 x 6 tets (N=3, 200 steps, checkpoint every
  20), and for independence of the checkpoint interval.
"""

import math

import numpy as np
import pytest
import torch

from oracle.pyoracle import Port, Reference, reference_available
from oracle.torch_rhs import TorchRHS
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import ic as IC
from scratch_wadge_b200 import mesh as M
from scratch_wadge_b200.adjoint import Adjoint, RHSFunction, RunFunction, rho2_objective
from tests.helpers import RTOL, Case, perturbed, rel

pytestmark = pytest.mark.gpu

CASES = ["tg3d_affine_N3", "dw3d_curved_N3", "vortex2d_curved_N3", "vortex2d_affine_N2",
         "tg3d_affine_N2", "dw3d_curved_N4", "vortex2d_curved_N4"]


def _app(geo, curved):
    return capi.App(geo, curved, stream=torch.cuda.current_stream().cuda_stream)


def _cpu_reference(c):
    if reference_available(c.dim, c.N):
        return Reference(c.ops, c.curved)
    return Port(c.ops, c.curved)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _state(c, seed=1):
    return perturbed(c.state(), seed, 1e-2)["Q"]


def _directions(Q, seed):
    """seeded w (output direction) and d (input direction scaled per field by
    the state's magnitude)"""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(Q.shape)
    d = rng.standard_normal(Q.shape) * np.abs(Q).mean(axis=(0, 2), keepdims=True)
    return w, d


@pytest.mark.parametrize("name", CASES)
def test_rhs_matches_oracle(cuda, name):
    """the forward map the adjoint differentiates is the reference's stage map"""
    c = Case(name)
    Q = _state(c)
    app = _app(c.geo, c.curved)
    adj = Adjoint(app, 1, 1)
    R = adj.rhs(_dev(Q)).cpu().numpy()
    assert rel(R, Port(c.ops, c.curved).rhs(c.geo, Q)) < RTOL


@pytest.mark.parametrize("name", CASES)
def test_rhs_vjp_matches_autodiff(cuda, name):
    c = Case(name)
    Q = _state(c)
    w, d = _directions(Q, 7)
    app = _app(c.geo, c.curved)
    adj = Adjoint(app, 1, 1)
    g = adj.rhs_vjp(_dev(Q), _dev(w)).cpu().numpy()
    T = TorchRHS(c.geo, c.curved)
    Qt = torch.from_numpy(Q)
    _, vjp = torch.func.vjp(T.R, Qt)
    g_ad = vjp(torch.from_numpy(w))[0].numpy()
    assert np.isfinite(g).all()
    assert rel(g, g_ad) < 1e-10, rel(g, g_ad)
    # JVP/VJP dot product: <w, J d> (forward-mode autodiff) = <J^T w, d> (hand-written)
    _, jd = torch.func.jvp(T.R, (Qt,), (torch.from_numpy(d),))
    lhs, rhs = float(np.sum(w * jd.numpy())), float(np.sum(g * d))
    assert abs(lhs - rhs) <= 1e-11 * abs(rhs), (lhs, rhs)


@pytest.mark.parametrize("name", CASES)
def test_rhs_vjp_matches_central_fd_of_cpu_reference(cuda, name):
    """<J^T w, d> against <w, (R(Q + h d) - R(Q - h d)) / 2h> of the CPU
    reference RHS on three seeded direction pairs.

    R is smooth except where a face point's penalty max(lamM, lamP) changes
    side; on these randomly perturbed states (1% noise, thousands of face
    points) the nearest such tie lies about 1e-6 away along d, so a central
    difference with h = 1e-6 can straddle it and measure neither one-sided
    derivative.  The step is 1e-7 and the test asserts that no face point
    changes side within +-h, which makes the difference quotient a valid
    check of the derivative."""
    c = Case(name)
    Q = _state(c)
    ref = _cpu_reference(c)
    app = _app(c.geo, c.curved)
    adj = Adjoint(app, 1, 1)
    T = TorchRHS(c.geo, c.curved)
    h = 1e-7
    for seed in (11, 12, 13):
        w, d = _directions(Q, seed)
        assert torch.equal(T.lf_branch(torch.from_numpy(Q + h * d)), T.lf_branch(torch.from_numpy(Q - h * d)))
        g = adj.rhs_vjp(_dev(Q), _dev(w)).cpu().numpy()
        fd = (ref.rhs(c.geo, Q + h * d) - ref.rhs(c.geo, Q - h * d)) / (2 * h)
        a, b = float(np.sum(w * fd)), float(np.sum(g * d))
        assert abs(a - b) <= 1e-6 * abs(b), (seed, a, b)


@pytest.mark.parametrize("dim", [2, 3])
def test_gradcheck_rhs_function(cuda, dim):
    """torch.autograd.gradcheck of R(Q) with the hand-written backward, on a
    one-cell periodic mesh at N=1 (every input entry).  gradcheck's central
    differences (eps 1e-6) carry the rounding noise of R divided by eps,
    about 1e-5 absolute for Jacobian entries up to ~300 here, hence atol 1e-4
    (3e-7 of the largest entry)."""
    mesh = M.periodic_square(1, 1) if dim == 2 else M.periodic_cube(1)
    geo = M.build_geometry(mesh, 1)
    U0 = IC.initial_state(geo, "vortex" if dim == 2 else "taylor_green")
    Q0 = IC.stage0(geo, U0)[0]
    Q0 = perturbed({"Q": Q0}, 3, 1e-2)["Q"]
    app = _app(geo, False)
    adj = Adjoint(app, 1, 1)
    Q = _dev(Q0).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda q: RHSFunction.apply(q, adj), (Q,), eps=1e-6,
                                    atol=1e-4, rtol=1e-6)


def _run_case(name, nsteps):
    c = Case(name)
    Q0 = _state(c, 5)
    return c, Q0, c.dt, nsteps


@pytest.mark.parametrize("name", ["tg3d_affine_N2", "vortex2d_curved_N3", "dw3d_curved_N3"])
def test_run_adjoint_matches_autodiff_through_the_run(cuda, name):
    """gradient of J = int rho(T)^2 after 6 steps (checkpoints every 4) against
    reverse-mode autodiff through the restated run, plus the dot product with
    forward-mode autodiff"""
    c, Q0, dt, nsteps = _run_case(name, 6)
    app = _app(c.geo, c.curved)
    adj = Adjoint(app, nsteps, 4)
    QT = adj.forward(_dev(Q0), dt)
    _, gT = rho2_objective(c.geo, QT)
    g0 = adj.reverse(gT).cpu().numpy()

    T = TorchRHS(c.geo, c.curved)
    J_of = lambda q: rho2_objective(c.geo, T.run(q, dt, nsteps))[0]
    Qt = torch.from_numpy(Q0)
    QT_t = T.run(Qt, dt, nsteps)
    assert rel(QT.cpu().numpy(), QT_t.numpy()) < 1e-11
    g_ad = torch.func.grad(J_of)(Qt).numpy()
    assert rel(g0, g_ad) < 1e-9, rel(g0, g_ad)
    rng = np.random.default_rng(2)
    d = rng.standard_normal(Q0.shape)
    _, jd = torch.func.jvp(J_of, (Qt,), (torch.from_numpy(d),))
    assert abs(float(jd) - float(np.sum(g0 * d))) <= 1e-10 * abs(float(jd))


def test_checkpoint_interval_does_not_change_the_gradient(cuda):
    c, Q0, dt, nsteps = _run_case("tg3d_affine_N3", 7)
    app = _app(c.geo, c.curved)
    out = []
    for every in (1, 3, 7, 20):
        adj = Adjoint(app, nsteps, every)
        QT = adj.forward(_dev(Q0), dt)
        _, gT = rho2_objective(c.geo, QT)
        out.append(adj.reverse(gT).cpu().numpy())
        adj.close()
    for g in out[1:]:
        assert np.array_equal(g, out[0])


@pytest.mark.parametrize("every", [1, 4, 7])
def test_repeated_reverse_sweeps_give_the_same_gradient(cuda, every):
    """The first reverse sweep after a forward run reads the last segment
    from the forward run's tape; later sweeps recompute it when another
    segment has refilled that tape (7 steps: 7, 2 and 1 segments)"""
    c, Q0, dt, nsteps = _run_case("tg3d_affine_N3", 7)
    app = _app(c.geo, c.curved)
    adj = Adjoint(app, nsteps, every)
    QT = adj.forward(_dev(Q0), dt)
    _, gT = rho2_objective(c.geo, QT)
    g = [adj.reverse(gT).cpu().numpy() for _ in range(3)]
    adj.close()
    assert np.array_equal(g[1], g[0]) and np.array_equal(g[2], g[0])


def test_run_function_autograd(cuda):
    """RunFunction: torch.autograd through the checkpointed run"""
    c, Q0, dt, nsteps = _run_case("vortex2d_curved_N3", 3)
    app = _app(c.geo, c.curved)
    adj = Adjoint(app, nsteps, 2)
    Q = _dev(Q0).requires_grad_(True)
    J, _ = rho2_objective(c.geo, RunFunction.apply(Q, adj, dt))
    J.backward()
    QT = adj.forward(_dev(Q0), dt)
    _, gT = rho2_objective(c.geo, QT)
    assert torch.equal(Q.grad, adj.reverse(gT))


def test_adjoint_rejects_unpaired_faces(cuda):
    c = Case("tg3d_affine_N2")
    geo = c.geo
    bad = geo.mapPq.copy()
    bad[0] = bad[1]  # two face points share one neighbour
    g2 = M.Geometry(geo.ops, geo.K, geo.vgeo, geo.vfgeo, geo.fgeo, geo.Jq, bad, None, None)
    app = _app(g2, False)
    with pytest.raises(capi.WadgError, match="face pairing"):
        Adjoint(app, 1, 1)


def _fsum_J(geo, Q):
    w = (np.asarray(geo.ops.wq)[None, :] * np.asarray(geo.Jq))
    rho = Q[:, 0, :]
    return math.fsum((w * rho * rho).ravel())


def test_taylor_green_adjoint_against_finite_differences(cuda):
    """Taylor-Green on 8^3 x 6 = 3072 affine tets, N=3, 200 LSRK-45 steps,
    checkpoint every 20: dJ/dQ0 . d for 8 seeded unit-norm Gaussian directions
    d against central differences of J with step 1e-6 relative to |Q0|
    (J summed exactly), agreement 1e-6 relative"""
    mesh = M.periodic_cube(8)
    geo = M.build_geometry(mesh, 3)
    U0 = IC.initial_state(geo, "taylor_green")
    Q0 = IC.stage0(geo, U0)[0]
    dt = IC.time_step(geo, 0.5, 3, nsteps=200, wave_speed=IC.max_wave_speed(Q0))[0]
    app = _app(geo, False)
    adj = Adjoint(app, 200, 20)
    QT = adj.forward(_dev(Q0), dt)
    _, gT = rho2_objective(geo, QT)
    g0 = adj.reverse(gT).cpu().numpy()
    assert np.isfinite(g0).all()
    eps = 1e-6 * float(np.linalg.norm(Q0))
    rng = np.random.default_rng(20261203)
    worst = 0.0
    for _ in range(8):
        z = rng.standard_normal(Q0.shape)
        d = z / np.linalg.norm(z)
        Jp = _fsum_J(geo, adj.forward(_dev(Q0 + eps * d), dt).cpu().numpy())
        Jm = _fsum_J(geo, adj.forward(_dev(Q0 - eps * d), dt).cpu().numpy())
        fd = (Jp - Jm) / (2 * eps)
        an = float(np.sum(g0 * d))
        worst = max(worst, abs(fd - an) / abs(an))
    assert worst < 1e-6, worst
