"""Test infrastructure only: the stage map of the entropy-stable RHS restated
in float64 PyTorch tensor algebra, so that automatic differentiation gives an
independent Jacobian to check the hand-written discrete adjoint against
(a JVP/VJP dot-product test).  Nothing in the product imports this.

It restates oracle/wadg_ref.c (itself the reference kernels
Euler3Daffine.okl:22-773, Euler3D.okl:2123-3473, Euler2D.okl:19-2282) for a
whole mesh at once:

    R(Q) = Minv rhs(u~(Q), uf~(Q))

with the projected traces u~ = U(VqPq v~), uf~ = U(VfPq v~), v~ = V(Q)
(affine) or VqPq((VqPq(V(Q) J))/J) (WADG, curved), the volume flux
differencing with the log-mean (series branch below the reference's
thresholds 1e-4 / 1e-3, Euler3Daffine.okl:43-71, Euler2D.okl:36-67), the
surface flux with the Lax-Friedrichs penalty tau/4 max(lamM, lamP) sJ
(Euler3Daffine.okl:421-552; tau = 1 in 2D, Euler2D.okl:1423-1425), and the
affine or weight-adjusted inverse mass.  Its values agree with the C oracle
to rounding (tests/test_adjoint.py pins it); branches are written so that
derivatives of the branch not taken are never NaN.
"""

from __future__ import annotations

import numpy as np
import torch


class TorchRHS:
    def __init__(self, geo, curved, gamma=1.4, tau=1.0, device=None):
        """device: where the restated map's tensors live (CPU by default; a
        CUDA device runs the check at large K through torch's own kernels)"""
        ops = geo.ops
        self.dim, self.curved, self.gamma = ops.dim, bool(curved), gamma
        self.tau = tau if ops.dim == 3 else 1.0
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=device)
        self.K, self.Nq, self.NF, self.Nfq = geo.K, ops.Nq, ops.NfqNf, ops.Nfq
        self.Nf = ops.dim + 2
        self.D = [t(ops.Drq), t(ops.Dsq)] + ([t(ops.Dtq)] if ops.dim == 3 else [])
        self.VqLq, self.VqPq, self.VfPq = t(ops.VqLq), t(ops.VqPq), t(ops.VfPq)
        d = ops.dim
        nr = [np.asarray(ops.nrJ), np.asarray(ops.nsJ)] + ([np.asarray(ops.ntJ)] if d == 3 else [])
        # reference normal of each face point's face, read at the face's first point
        fidx = (np.arange(self.NF) // self.Nfq) * self.Nfq
        self.nref = t(np.stack([n[fidx] for n in nr], axis=1))            # [NF, d]
        self.vgeo = t(geo.vgeo).reshape(self.K, d, d, self.Nq)             # [K, a, x, Nq]
        self.vfgeo = t(geo.vfgeo).reshape(self.K, d, d, self.NF) if curved else None
        self.fgeo = t(geo.fgeo)                                            # [K, d+1, NF]
        self.Jq = t(geo.Jq)                                                # [K, Nq]
        mp = np.asarray(geo.mapPq, dtype=np.int64).reshape(self.K, self.NF)
        blk = self.NF * self.Nf
        self.mapK = torch.as_tensor(mp // blk, device=device)
        self.mapJ = torch.as_tensor(mp % blk, device=device)
        # the reference's float thresholds 1.fe-4 / 1.fe-3, as doubles
        self.thr = float(np.float32(1e-4)) if d == 3 else float(np.float32(1e-3))

    # ---- node maps
    def VU(self, U):
        g, d = self.gamma, self.dim
        rho, m, E = U[:, 0], U[:, 1:d + 1], U[:, d + 1]
        rhoe = E - 0.5 * (m * m).sum(1) / rho
        s = torch.log((g - 1.0) * rhoe / rho ** g)
        V0 = (-E + rhoe * (g + 1.0 - s)) / rhoe
        return torch.cat([V0[:, None], m / rhoe[:, None], (-rho / rhoe)[:, None]], 1)

    def UV(self, V):
        g, d = self.gamma, self.dim
        V1, Vm, Vl = V[:, 0], V[:, 1:d + 1], V[:, d + 1]
        vv = (Vm * Vm).sum(1)
        sV = g - V1 + vv / (2.0 * Vl)
        rhoe = ((g - 1.0) / (-Vl) ** g) ** (1.0 / (g - 1.0)) * torch.exp(-sV / (g - 1.0))
        return torch.cat([(-rhoe * Vl)[:, None], rhoe[:, None] * Vm,
                          (rhoe * (1.0 - vv / (2.0 * Vl)))[:, None]], 1)

    def prim(self, U):
        """rho, velocity [.., d], beta from U [K, Nf, n] -> tensors over [K, n]"""
        d = self.dim
        rho = U[:, 0]
        u = U[:, 1:d + 1] / rho[:, None]
        p = (self.gamma - 1.0) * (U[:, d + 1] - 0.5 * rho * (u * u).sum(1))
        return rho, u, rho / (2.0 * p)

    def logmean(self, a, b):
        xi = a / b
        f = (xi - 1.0) / (xi + 1.0)
        u = f * f
        small = u < self.thr
        xs = torch.where(small, torch.full_like(xi, 2.0), xi)
        fs = (xs - 1.0) / (xs + 1.0)
        Flog = torch.log(xs) / 2.0 / fs
        u2 = u * u
        Fser = 1.0 + u / 3.0 + u2 / 5.0 + u2 * u / 7.0
        if self.dim == 2:
            Fser = Fser + u2 * u2 / 9.0
        return (a + b) / (2.0 * torch.where(small, Fser, Flog))

    def flux_n(self, A, B, n):
        """contracted EC flux sum_x F_x(A, B) n_x; A, B broadcastable primitive
        tuples, n [..., d]; returns [..., Nf]"""
        ra, ua, ba = A
        rb, ub, bb = B
        d = self.dim
        rl = self.logmean(ra, rb)
        pa = 0.5 * (ra + rb) / (2.0 * 0.5 * (ba + bb))
        uavg = 0.5 * (ua + ub)
        vnavg = 2.0 * (uavg * uavg).sum(-1) - 0.5 * ((ua * ua).sum(-1) + (ub * ub).sum(-1))
        f4 = rl / (2.0 * (self.gamma - 1.0) * self.logmean(ba, bb)) + pa + 0.5 * rl * vnavg
        un = (uavg * n).sum(-1)
        F0 = rl * un
        Fm = F0[..., None] * uavg + pa[..., None] * n
        return torch.cat([F0[..., None], Fm, (f4 * un)[..., None]], -1)

    # ---- the stage map
    def project(self, Q):
        """u~ [K, Nf, Nq], uf~ [K, Nf, NF]"""
        V = self.VU(Q)
        if self.curved:
            J = self.Jq[:, None, :]
            sV = torch.einsum("ij,kfj->kfi", self.VqPq, V * J) / J
            V = torch.einsum("ij,kfj->kfi", self.VqPq, sV)
        uq = self.UV(torch.einsum("ij,kfj->kfi", self.VqPq, V))
        uf = self.UV(torch.einsum("ij,kfj->kfi", self.VfPq, V))
        return uq, uf

    def rhs(self, uq, uf):
        d, Nq, NF = self.dim, self.Nq, self.NF
        rq, vq, bq = self.prim(uq)     # [K, Nq], [K, d, Nq], [K, Nq]
        rf, vf, bf = self.prim(uf)
        vq, vf = vq.transpose(1, 2), vf.transpose(1, 2)  # [K, n, d]
        G = self.vgeo  # [K, a, x, Nq]
        # volume-volume: direction sum_a D^a_ij G_a(x) (node 0, or the pair average)
        Dst = torch.stack(self.D, 0)  # [a, i, j]
        if self.curved:
            Gp = 0.5 * (G[:, :, :, :, None] + G[:, :, :, None, :])   # [K, a, x, i, j]
            nvv = torch.einsum("aij,kaxij->kijx", Dst, Gp)
        else:
            nvv = torch.einsum("aij,kax->kijx", Dst, G[..., 0])
        Fvv = self.flux_n((rq[:, :, None], vq[:, :, None, :], bq[:, :, None]),
                          (rq[:, None, :], vq[:, None, :, :], bq[:, None, :]), nvv)  # [K, i, j, Nf]
        rhs_v = Fvv.sum(2)
        # volume-face pairs: direction nJ of the face point (G of node 0, or the pair average)
        if self.curved:
            Gp = 0.5 * (G[:, :, :, :, None] + self.vfgeo[:, :, :, None, :])  # [K, a, x, i, f]
            nvf = torch.einsum("fa,kaxif->kifx", self.nref, Gp)
        else:
            nvf = torch.einsum("fa,kax->kfx", self.nref, G[..., 0])[:, None, :, :].expand(-1, Nq, -1, -1)
        Fvf = self.flux_n((rq[:, :, None], vq[:, :, None, :], bq[:, :, None]),
                          (rf[:, None, :], vf[:, None, :, :], bf[:, None, :]), nvf)  # [K, i, f, Nf]
        rhs_v = rhs_v + torch.einsum("if,kifq->kiq", 0.5 * self.VqLq, Fvf)
        rhs_f = torch.einsum("fi,kifq->kfq", -0.5 * self.VfPq, Fvf)
        # surface: 1/2 F(M, P).nJ + rhsQf - tau/4 max(lamM, lamP) sJ (uP - uM)
        UM = uf
        UP = uf[self.mapK, :, self.mapJ]            # [K, NF, Nf]
        UP = UP.transpose(1, 2)                      # [K, Nf, NF]
        rP, vP, bP = self.prim(UP)
        vP = vP.transpose(1, 2)
        nJ = self.fgeo[:, :d, :].transpose(1, 2)     # [K, NF, d]
        sJ = self.fgeo[:, d, :]
        Fs = 0.5 * self.flux_n((rf, vf, bf), (rP, vP, bP), nJ)  # [K, NF, Nf]

        def lam(r, v, b):
            p = r / (2.0 * b)
            return torch.sqrt((v * v).sum(-1)) + torch.sqrt(self.gamma * p / r)

        lM, lP = lam(rf, vf, bf), lam(rP, vP, bP)
        Lfc = self.tau * 0.25 * torch.where(lM > lP, lM, lP) * sJ
        sf = Fs + rhs_f - Lfc[..., None] * (UP - UM).transpose(1, 2)
        rhs_v = rhs_v + torch.einsum("if,kfq->kiq", self.VqLq, sf)
        return rhs_v.transpose(1, 2)  # [K, Nf, Nq]

    def lf_branch(self, Q):
        """which side's wave speed the penalty's max takes at every face point
        (lamM > lamP), for the projected traces of Q"""
        _, uf = self.project(Q)
        d = self.dim
        UP = uf[self.mapK, :, self.mapJ].transpose(1, 2)
        rf, vf, bf = self.prim(uf)
        rP, vP, bP = self.prim(UP)

        def lam(r, v, b):
            return torch.sqrt((v * v).sum(1)) + torch.sqrt(self.gamma * (r / (2.0 * b)) / r)

        return lam(rf, vf, bf) > lam(rP, vP, bP)

    def minv(self, rhs):
        J = self.Jq[:, None, :]
        r = torch.einsum("ij,kfj->kfi", -2.0 * self.VqPq, rhs) / J
        if self.curved:
            r = torch.einsum("ij,kfj->kfi", self.VqPq, r)
        return r

    def R(self, Q):
        uq, uf = self.project(Q)
        return self.minv(self.rhs(uq, uf))

    def run(self, Q0, dt, nsteps):
        """nsteps LSRK-45 steps from Q0 (traces projected from Q0)."""
        from scratch_wadge_b200.ic import RK4A as A, RK4B as B
        Q, res = Q0, torch.zeros_like(Q0)
        for _ in range(nsteps):
            for s in range(5):
                res = A[s] * res + dt * self.R(Q)
                Q = Q + B[s] * res
        return Q
