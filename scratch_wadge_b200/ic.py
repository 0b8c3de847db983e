"""Initial states, the stage-0 solver state and host-side diagnostics.

Follows the reference's host code in euler.c:
  * isentropic vortex (2D)           euler.c:3280-3306 (strength, centre as parameters)
  * Taylor-Green vortex (3D)         euler.c:3381-3411
  * density wave (3D, curved tests)  rho = 2 + 0.5 sin(x+y+z), u=v=w=1, p=1
  * stage-0 state                    euler.c:3958-4133: L2 projection of the
    initial state at quadrature points (VqPq), then the entropy projection
    rhsQ = u(VqPq v(Q)), Qf = u(VfPq v(Q)), resQ = 0
  * time step                        euler.c:3177-3213 (hmin), 4180-4193 (dt)
  * entropy  int -rho s              euler.c:4135-4156, 4276-4315
  * L2 error                         euler.c:4227-4274
  * LSRK-45 coefficients             euler.c:2779-2796
"""

from __future__ import annotations

import math

import numpy as np

# Carpenter-Kennedy low-storage RK, euler.c:2779-2796
RK4A = np.array([0.0,
                 -567301805773.0 / 1357537059087.0,
                 -2404267990393.0 / 2016746695238.0,
                 -3550918686646.0 / 2091501179385.0,
                 -1275806237668.0 / 842570457699.0])
RK4B = np.array([1432997174477.0 / 9575080441755.0,
                 5161836677717.0 / 13612068292357.0,
                 1720146321549.0 / 2090206949498.0,
                 3134564353537.0 / 4481467310338.0,
                 2277821191437.0 / 14882151754819.0])
RK4C = np.array([0.0,
                 1432997174477.0 / 9575080441755.0,
                 2526269341429.0 / 6820363962896.0,
                 2006345519317.0 / 3224310063776.0,
                 2802321613138.0 / 2924317926251.0,
                 1.0])


def vortex_2d(x, y, t=0.0, gamma=1.4, beta=5.0, x0=5.0, y0=0.0):
    """Isentropic vortex, euler.c:3289-3305 (without the constant-state
    override of :3307-3312)."""
    gm1 = gamma - 1.0
    r2 = (x - x0 - t) ** 2 + (y - y0) ** 2
    u = 1.0 - beta * np.exp(1.0 - r2) * (y - y0) / (2.0 * math.pi)
    v = beta * np.exp(1.0 - r2) * (x - x0 - t) / (2.0 * math.pi)
    rho0 = 1.0 - .5 * gm1 * (1.0 / (8.0 * gamma * math.pi * math.pi)) * (beta * np.exp(1.0 - r2)) ** 2
    rho = rho0 ** (1.0 / gm1)
    p = rho ** gamma
    E = p / gm1 + .5 * rho * (u * u + v * v)
    return np.stack([rho, rho * u, rho * v, E], axis=0)


def taylor_green(x, y, z, gamma=1.4):
    """euler.c:3381-3411."""
    gm1 = gamma - 1.0
    rho = np.ones_like(x)
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(x)
    p = 100.0 / gamma + (1.0 / 16.0) * (np.cos(2.0 * x) + np.cos(2.0 * y)) * (2.0 + np.cos(2.0 * z))
    return np.stack([rho, rho * u, rho * v, rho * w, p / gm1 + .5 * rho * (u * u + v * v + w * w)], axis=0)


def density_wave(x, y, z, t=0.0, gamma=1.4):
    """rho = 2 + 0.5 sin(x+y+z - 3t), u = v = w = 1, p = 1 (exact advection)."""
    rho = 2.0 + 0.5 * np.sin(x + y + z - 3.0 * t)
    one = np.ones_like(x)
    E = 1.0 / (gamma - 1.0) + .5 * rho * 3.0
    return np.stack([rho, rho * one, rho * one, rho * one, E], axis=0)


def constant_state(shape, dim, gamma=1.4):
    """The free-stream state the reference uses for testing (euler.c:3307-3312,
    3351-3357)."""
    if dim == 2:
        rho, ru, rv = 1.0, 2.0, 5.0
        E = 1.0 + .5 * (ru * ru + rv * rv) / rho
        return np.stack([np.full(shape, rho), np.full(shape, ru), np.full(shape, rv), np.full(shape, E)])
    rho, ru, rv, rw = 1.0, 2.0, 3.0, 4.0
    E = 1.0 + .5 * (ru * ru + rv * rv + rw * rw) / rho
    return np.stack([np.full(shape, v) for v in (rho, ru, rv, rw, E)])


# ------------------------------------------------- entropy variables (numpy)
def VU(U, gamma=1.4):
    """conservative -> entropy variables; euler.c:3216-3246 / Euler3Daffine.okl:73-93."""
    dim = U.shape[0] - 2
    rho, E = U[0], U[-1]
    m2 = sum(U[1 + d] ** 2 for d in range(dim))
    rhoe = E - .5 * m2 / rho
    s = np.log((gamma - 1.0) * rhoe / rho ** gamma)
    V = [(-E + rhoe * (gamma + 1.0 - s)) / rhoe]
    V += [U[1 + d] / rhoe for d in range(dim)]
    V += [(-rho) / rhoe]
    return np.stack(V, axis=0)


def UV(V, gamma=1.4):
    """entropy -> conservative variables; euler.c:3249-3278 / Euler3Daffine.okl:95-105."""
    dim = V.shape[0] - 2
    Vl = V[-1]
    vv = sum(V[1 + d] ** 2 for d in range(dim))
    sV = gamma - V[0] + vv / (2.0 * Vl)
    rhoe = ((gamma - 1.0) / (-Vl) ** gamma) ** (1.0 / (gamma - 1.0)) * np.exp(-sV / (gamma - 1.0))
    U = [rhoe * (-Vl)] + [rhoe * V[1 + d] for d in range(dim)] + [rhoe * (1.0 - vv / (2.0 * Vl))]
    return np.stack(U, axis=0)


# ------------------------------------------------------------- stage 0
def stage0(geo, Uq, gamma=1.4):
    """Uq: (Nfields, Nq, K) initial state at quadrature points.
    Returns Q, rhsQ, Qf, resQ in the kernel layouts [K][Nfields][Nq|NfqNf]
    (euler.c:3958-4133)."""
    ops = geo.ops
    Q = np.einsum("ij,fjk->fik", ops.VqPq, Uq)          # L2 projection
    V = VU(Q, gamma)
    Vq = np.einsum("ij,fjk->fik", ops.VqPq, V)
    Vf = np.einsum("ij,fjk->fik", ops.VfPq, V)
    rhsQ = UV(Vq, gamma)
    Qf = UV(Vf, gamma)
    lay = lambda a: np.ascontiguousarray(a.transpose(2, 0, 1))
    return lay(Q), lay(rhsQ), lay(Qf), np.zeros_like(lay(Q))


def initial_state(geo, kind, gamma=1.4, **kw):
    """Initial state at quadrature points, (Nfields, Nq, K)."""
    x = geo.xyzq.transpose(1, 2, 0)  # (3, Nq, K)
    if kind == "vortex":
        return vortex_2d(x[0], x[1], 0.0, gamma, **kw)
    if kind == "taylor_green":
        return taylor_green(x[0], x[1], x[2], gamma)
    if kind == "density_wave":
        return density_wave(x[0], x[1], x[2], 0.0, gamma)
    if kind == "constant":
        return constant_state(x[0].shape, geo.ops.dim, gamma)
    raise ValueError(kind)


def exact_state(geo, kind, t, gamma=1.4, **kw):
    x = geo.xyzq.transpose(1, 2, 0)
    if kind == "vortex":
        return vortex_2d(x[0], x[1], t, gamma, **kw)
    if kind == "density_wave":
        return density_wave(x[0], x[1], x[2], t, gamma)
    if kind == "constant":
        return constant_state(x[0].shape, geo.ops.dim, gamma)
    raise ValueError(f"no exact solution for {kind}")


def hmin(geo):
    """euler.c:3177-3213: min over elements of min(Jq) / max(sJ)."""
    sJ = geo.fgeo[:, -1, :]
    return float(np.min(geo.Jq.min(axis=1) / sJ.max(axis=1)))


def max_wave_speed(Q, gamma=1.4):
    """max over nodes of |u| + sqrt(gamma p / rho); Q in kernel layout."""
    dim = Q.shape[1] - 2
    rho, E = Q[:, 0], Q[:, -1]
    u2 = sum((Q[:, 1 + d] / rho) ** 2 for d in range(dim))
    p = (gamma - 1.0) * (E - 0.5 * rho * u2)
    return float(np.max(np.sqrt(u2) + np.sqrt(gamma * p / rho)))


def time_step(geo, CFL, N, FinalTime=None, nsteps=None, wave_speed=None):
    """dt = CFL*hmin/C_N (euler.c:4180-4193); with FinalTime, Nsteps =
    ceil(T/dt) and dt = T/Nsteps (euler.c:3680-3688).

    The reference's formula carries no wave speed (it assumes one of order 1).
    With ``wave_speed`` the step is divided by it: the Taylor-Green state
    (p0 = 100/gamma, sound speed ~10) runs the reference's own kernels into
    NaN within two steps at CFL 0.5 otherwise."""
    dim = geo.ops.dim
    CN = (N + 1) * (N + 2) / 2 if dim == 2 else (N + 1) * (N + 3) / 3
    dt = CFL * hmin(geo) / CN
    if wave_speed is not None:
        dt /= wave_speed
    if FinalTime is not None:
        n = int(math.ceil(FinalTime / dt))
        return FinalTime / n, n
    return dt, nsteps


def entropy(geo, Q, gamma=1.4):
    """int -rho*s dx (euler.c:4276-4315); Q in kernel layout [K][Nf][Nq]."""
    ops = geo.ops
    dim = ops.dim
    rho, E = Q[:, 0, :], Q[:, -1, :]
    m2 = sum(Q[:, 1 + d, :] ** 2 for d in range(dim))
    rhoe = E - .5 * m2 / rho
    s = np.log((gamma - 1.0) * rhoe / rho ** gamma)
    return float(np.sum(ops.wq[None, :] * geo.Jq * (-rho * s)))


def l2_error(geo, Q, Uex):
    """euler.c:4227-4274; Uex (Nfields, Nq, K)."""
    ops = geo.ops
    err = (Q.transpose(1, 2, 0) - Uex) ** 2
    return float(np.sqrt(np.sum(err.sum(axis=0) * ops.wq[:, None] * geo.Jq.T)))
