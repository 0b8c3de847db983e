"""Discrete adjoint: Python side of the C ABI wadg_adjoint_* (include/wadg.h).

* ``Adjoint``        — the checkpointed LSRK-45 adjoint of an ``App`` and the
                       RHS vector-Jacobian product, on device tensors.
* ``RHSFunction``    — R(Q) as a torch.autograd.Function whose backward is the
                       hand-written VJP (for torch.autograd.gradcheck).
* ``RunFunction``    — Q0 -> Q(T) over the whole run, backward = reverse sweep.
* ``rho2_objective`` — J = integral of rho(x, T)^2 over the mesh and its
                       gradient with respect to Q(T).

The reference has no adjoint; the forward pieces it differentiates are the
kernels of Euler3Daffine.okl / Euler3D.okl / Euler2D.okl driven by rk_run
(euler.c:3672-3738).  Device work runs on the app's stream; every call here
synchronises with torch's current stream on entry and with the app's stream
on return.
"""

from __future__ import annotations

import ctypes
import weakref

import torch

from . import capi


def _ptr(t: torch.Tensor) -> int:
    assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous(), "float64 contiguous CUDA tensor"
    return t.data_ptr()


class Adjoint:
    def __init__(self, app: capi.App, nsteps: int, every: int = 20):
        self.app, self.nsteps, self.every = app, int(nsteps), int(every)
        h = ctypes.c_void_p()
        self._destroy = capi.lib().wadg_adjoint_destroy  # kept for close() at interpreter exit
        capi.check(capi.lib().wadg_adjoint_create(app.h, self.nsteps, self.every, ctypes.byref(h)),
                   "wadg_adjoint_create")
        self.h = h
        self.shape = app.vshape
        if not hasattr(app, "_dependents"):
            app._dependents = weakref.WeakSet()
        app._dependents.add(self)

    def close(self):
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    __del__ = close

    def _enter(self):
        torch.cuda.current_stream().synchronize()

    def _leave(self):
        self.app.sync()

    def forward(self, Q0: torch.Tensor, dt: float) -> torch.Tensor:
        """Run nsteps from Q0 with checkpoints; returns Q(T)."""
        QT = torch.empty_like(Q0)
        self._enter()
        capi.check(capi.lib().wadg_adjoint_forward(self.h, _ptr(Q0), float(dt), _ptr(QT)),
                   "wadg_adjoint_forward")
        self._leave()
        return QT

    def reverse(self, QbarT: torch.Tensor) -> torch.Tensor:
        """dJ/dQ0 given dJ/dQ(T) for the last forward run."""
        out = torch.empty_like(QbarT)
        self._enter()
        capi.check(capi.lib().wadg_adjoint_reverse(self.h, _ptr(QbarT), _ptr(out)), "wadg_adjoint_reverse")
        self._leave()
        return out

    def rhs(self, Q: torch.Tensor) -> torch.Tensor:
        out = torch.empty_like(Q)
        self._enter()
        capi.check(capi.lib().wadg_adjoint_rhs(self.h, _ptr(Q), _ptr(out)), "wadg_adjoint_rhs")
        self._leave()
        return out

    def rhs_vjp(self, Q: torch.Tensor, w: torch.Tensor) -> torch.Tensor:
        out = torch.empty_like(Q)
        self._enter()
        capi.check(capi.lib().wadg_adjoint_rhs_vjp(self.h, _ptr(Q), _ptr(w), _ptr(out)),
                   "wadg_adjoint_rhs_vjp")
        self._leave()
        return out


class RHSFunction(torch.autograd.Function):
    """R(Q) with the hand-written VJP as its backward (gradcheck only)."""

    @staticmethod
    def forward(ctx, Q, adj: Adjoint):
        ctx.adj = adj
        ctx.save_for_backward(Q)
        return adj.rhs(Q.contiguous())

    @staticmethod
    def backward(ctx, g):
        (Q,) = ctx.saved_tensors
        return ctx.adj.rhs_vjp(Q.contiguous(), g.contiguous()), None


class RunFunction(torch.autograd.Function):
    """Q0 -> Q(T) over the adjoint's nsteps; backward is the checkpointed reverse sweep."""

    @staticmethod
    def forward(ctx, Q0, adj: Adjoint, dt: float):
        ctx.adj = adj
        return adj.forward(Q0.contiguous(), dt)

    @staticmethod
    def backward(ctx, g):
        return ctx.adj.reverse(g.contiguous()), None, None


def rho2_objective(geo, Q: torch.Tensor):
    """J = sum_k sum_i wq_i Jq_ik rho_ik^2 (the integral of rho^2 by the
    volume cubature) and dJ/dQ; Q is [K][Nfields][Nq]."""
    w = torch.as_tensor(geo.ops.wq, dtype=torch.float64, device=Q.device)[None, :] * \
        torch.as_tensor(geo.Jq, dtype=torch.float64, device=Q.device)
    rho = Q[:, 0, :]
    J = (w * rho * rho).sum()
    g = torch.zeros_like(Q)
    g[:, 0, :] = 2.0 * w * rho
    return J, g


def main(argv=None):
    """Gradient of J = int rho(T)^2 for a periodic Taylor-Green cube, N=3:
    forward run with checkpoints, then the reverse sweep, `repeat` times
    (a small case for profilers).

        python -m scratch_wadge_b200.adjoint --cube 8 --steps 2 --every 2
    """
    import argparse

    from . import ic as IC
    from . import mesh as M

    ap = argparse.ArgumentParser(description=main.__doc__.split("\n")[0])
    ap.add_argument("--cube", type=int, default=8, help="hexes per direction (6 tets each)")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--every", type=int, default=2, help="checkpoint every this many steps")
    ap.add_argument("--repeat", type=int, default=2)
    a = ap.parse_args(argv)
    geo = M.build_geometry(M.periodic_cube(a.cube), 3)
    Q0 = IC.stage0(geo, IC.initial_state(geo, "taylor_green"))[0]
    dt = IC.time_step(geo, 0.5, 3, nsteps=200, wave_speed=IC.max_wave_speed(Q0))[0]
    app = capi.App(geo, False)
    adj = Adjoint(app, a.steps, a.every)
    Qd = torch.from_numpy(Q0).cuda()
    for _ in range(a.repeat):
        QT = adj.forward(Qd, dt)
        J, gT = rho2_objective(geo, QT)
        g = adj.reverse(gT)
    torch.cuda.synchronize()
    print(f"K={geo.K} steps={a.steps} J={float(J):.15g} max|dJ/dQ0|={float(g.abs().max()):.6e}")
    adj.close()
    app.close()


if __name__ == "__main__":
    main()
