"""CPU checks of the discrete adjoint's building blocks (no GPU needed):

* the node-level derivative formulas the adjoint kernels use
  (wadg_adjoint_math.cuh, built for the host through tests/adjoint_math/
  shim.cpp) against central differences: the two-point flux VJP in both
  log-mean branches, the wave speed, V(U) and U(V);
* the float64 PyTorch restatement of the stage map (oracle/torch_rhs.py),
  which the GPU tests differentiate by autodiff, against the C oracle, and its
  autodiff VJP against central differences of the oracle RHS.
"""

import ctypes
import os
import subprocess

import numpy as np
import pytest
import torch

from oracle.pyoracle import Port
from oracle.torch_rhs import TorchRHS
from tests.helpers import RTOL, Case, perturbed, rel

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "adjoint_math", "shim.cpp")
SO = os.path.join(HERE, "adjoint_math", "_build", "libadjoint_math.so")
HDR = os.path.join(os.path.dirname(HERE), "scratch_wadge_b200", "csrc", "wadg_adjoint_math.cuh")

_P = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def am():
    if not os.path.exists(SO) or os.path.getmtime(SO) < max(os.path.getmtime(SHIM), os.path.getmtime(HDR)):
        os.makedirs(os.path.dirname(SO), exist_ok=True)
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off",
                               SHIM, "-o", SO])
    L = ctypes.CDLL(SO)
    L.am_lambda.restype = ctypes.c_double
    for f in ("am_flux", "am_flux_vjp", "am_lambda", "am_VU", "am_UV", "am_VU_vjp", "am_UV_vjp",
              "am_UV_vjp_U"):
        getattr(L, f).argtypes = None
    return L


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_P)


def _state(rng, dim, amp=1.0):
    rho = 1.0 + 0.3 * amp * rng.uniform(-1, 1)
    m = rho * 0.5 * amp * rng.uniform(-1, 1, dim)
    E = (2.0 + 0.5 * amp * rng.uniform(-1, 1)) / 0.4 + 0.5 * (m @ m) / rho
    return np.concatenate([[rho], m, [E]])


def _call(f, dim, *arrs_and_scalars, nout=1, size=None):
    outs = [np.zeros(size or dim + 2) for _ in range(nout)]
    args = [ctypes.c_int(dim)]
    for a in arrs_and_scalars:
        args.append(ctypes.c_double(a) if np.isscalar(a) else _p(a))
    f(*args, *[o.ctypes.data_as(_P) for o in outs])
    return outs


G = 1.4


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("near", [False, True])
def test_flux_vjp_against_central_differences(am, dim, near):
    """both log-mean branches: general states, and states 1e-3 apart (series)"""
    rng = np.random.default_rng(10 * dim + near)
    for _ in range(5):
        A = _state(rng, dim)
        B = A * (1 + 1e-3 * rng.uniform(-1, 1, dim + 2)) if near else _state(rng, dim)
        n, c = rng.uniform(-1, 1, dim), rng.uniform(-1, 1, dim + 2)
        gA, gB = _call(am.am_flux_vjp, dim, A, B, n, c, G, nout=2)
        F = lambda a, b: _call(am.am_flux, dim, a, b, n, G)[0]
        for side, X, g in ((0, A, gA), (1, B, gB)):
            fd = np.zeros(dim + 2)
            for i in range(dim + 2):
                h = 1e-6 * abs(X[i]) + 1e-9
                e = np.zeros(dim + 2)
                e[i] = h
                if side == 0:
                    fd[i] = c @ (F(A + e, B) - F(A - e, B)) / (2 * h)
                else:
                    fd[i] = c @ (F(A, B + e) - F(A, B - e)) / (2 * h)
            assert np.abs(fd - g).max() <= 1e-6 * np.abs(g).max(), (side, fd, g)


@pytest.mark.parametrize("dim", [2, 3])
def test_node_map_vjps_against_central_differences(am, dim):
    rng = np.random.default_rng(dim)
    for _ in range(5):
        U = _state(rng, dim)
        # wave speed |u| + sqrt(gamma p / rho)
        dl = np.zeros(dim + 2)
        am.am_lambda(ctypes.c_int(dim), _p(U), ctypes.c_double(G), dl.ctypes.data_as(_P))
        lam = lambda u: am.am_lambda(ctypes.c_int(dim), _p(u), ctypes.c_double(G), _p(np.zeros(dim + 2)))
        # V(U) and U(V)
        Vb, Ub = rng.standard_normal(dim + 2), rng.standard_normal(dim + 2)
        gU = _call(am.am_VU_vjp, dim, U, Vb, G)[0]
        V = _call(am.am_VU, dim, U, G)[0]
        gV = _call(am.am_UV_vjp, dim, V, Ub, G)[0]
        assert rel(_call(am.am_UV, dim, V, G)[0], U) < 1e-13
        # the kernels' form of the U(V) adjoint, written in terms of U = U(V)
        assert rel(_call(am.am_UV_vjp_U, dim, U, Ub, G)[0], gV) < 1e-13
        for i in range(dim + 2):
            h = 1e-6 * abs(U[i]) + 1e-9
            e = np.zeros(dim + 2)
            e[i] = h
            assert abs((lam(U + e) - lam(U - e)) / (2 * h) - dl[i]) <= 1e-6 * np.abs(dl).max()
            fd = Vb @ (_call(am.am_VU, dim, U + e, G)[0] - _call(am.am_VU, dim, U - e, G)[0]) / (2 * h)
            assert abs(fd - gU[i]) <= 1e-6 * np.abs(gU).max()
            hv = 1e-6 * abs(V[i]) + 1e-9
            ev = np.zeros(dim + 2)
            ev[i] = hv
            fd = Ub @ (_call(am.am_UV, dim, V + ev, G)[0] - _call(am.am_UV, dim, V - ev, G)[0]) / (2 * hv)
            assert abs(fd - gV[i]) <= 1e-6 * np.abs(gV).max()


@pytest.mark.parametrize("name", ["tg3d_affine_N3", "dw3d_curved_N3", "vortex2d_curved_N3",
                                  "vortex2d_affine_N2"])
def test_torch_restatement_matches_oracle(name):
    c = Case(name)
    Q = perturbed(c.state(), 1, 1e-2)["Q"]
    R = TorchRHS(c.geo, c.curved).R(torch.from_numpy(Q)).numpy()
    assert rel(R, Port(c.ops, c.curved).rhs(c.geo, Q)) < RTOL


@pytest.mark.parametrize("name", ["tg3d_affine_N3", "dw3d_curved_N3", "vortex2d_curved_N3"])
def test_torch_autodiff_against_central_differences_of_oracle(name):
    c = Case(name)
    Q = perturbed(c.state(), 1, 1e-2)["Q"]
    rng = np.random.default_rng(0)
    w = rng.standard_normal(Q.shape)
    d = rng.standard_normal(Q.shape) * np.abs(Q).mean(axis=(0, 2), keepdims=True)
    T = TorchRHS(c.geo, c.curved)
    _, vjp = torch.func.vjp(T.R, torch.from_numpy(Q))
    g = vjp(torch.from_numpy(w))[0].numpy()
    P = Port(c.ops, c.curved)
    # step small enough that no face point's penalty max changes side within +-h
    h = 1e-7
    assert torch.equal(T.lf_branch(torch.from_numpy(Q + h * d)), T.lf_branch(torch.from_numpy(Q - h * d)))
    fd = (P.rhs(c.geo, Q + h * d) - P.rhs(c.geo, Q - h * d)) / (2 * h)
    a, b = float(np.sum(w * fd)), float(np.sum(g * d))
    assert abs(a - b) <= 1e-6 * abs(b)
