"""Reference-element operators built from the node and cubature point sets.

The reference builds its operators on the host (build_ref_ops_2D/3D,
operators.cpp:104-341, and the hybridised operators of
host_operators_new_2D/3D, operators_c.cpp:46-69, 212-241) from three point
sets tabulated in its node_data.h: the interpolation nodes of degree N, the
volume cubature of degree M = 2N and, in 3D, the triangle cubature of degree
M for the faces (in 2D the face rule is Gauss-Legendre, computed).  This
module takes those point sets (data/points_<dim>d_N<N>.npz, the tables as the
reference's builder reads them) and builds every operator from them:

  V, Dr, Ds, Dt       orthonormal simplex basis at the nodes and its gradient,
                      D = Vr V^-1 (Hesthaven & Warburton, "Nodal Discontinuous
                      Galerkin Methods", 2008, App. A: Simplex2DP/3DP and
                      GradSimplex2DP/3DP)
  Vq, Pq              interpolation to the volume cubature and the L2
                      projection back, Pq = M^-1 Vq^T W, M = Vq^T W Vq
  rfq, sfq, tfq, wfq  the face cubature mapped to every face (face-major)
  nrJ, nsJ, ntJ       reference normals scaled by the face Jacobian
  Vfq, Lq             interpolation to the face points and the lift
                      Lq = M^-1 Vfq^T Wf
  VqLq, VqPq, VfPq    the products the kernels take
  Drq, Dsq, Dtq       hybridised derivatives Vq D Pq - 1/2 Vq Lq diag(n) Vfq Pq

The same formulas as the reference (they are the method), computed with numpy
in float64; basis-independent, so they agree with the reference's tables to
rounding (tests/test_refbuild.py pins every table).
"""

from __future__ import annotations

import math
import os

import numpy as np

from . import refops as R

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def grad_jacobi_p(x, alpha, beta, n):
    """d/dx of the orthonormal Jacobi polynomial P_n^(alpha,beta)(x)."""
    x = np.asarray(x, dtype=np.float64)
    if n == 0:
        return np.zeros_like(x)
    return math.sqrt(n * (n + alpha + beta + 1)) * R.jacobi_p(x, alpha + 1, beta + 1, n - 1)


def grad_vandermonde(dim, N, r, s, t=None):
    """Gradient of the orthonormal P_N basis at points: (Vr, Vs[, Vt]),
    each (npts, Np), in the mode order of refops.vandermonde."""
    r = np.asarray(r, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    if dim == 2:
        a, b = R._collapse2(r, s)
        Vr, Vs = [], []
        hb = 0.5 * (1 - b)
        for i in range(N + 1):
            for j in range(N - i + 1):
                fa, dfa = R.jacobi_p(a, 0, 0, i), grad_jacobi_p(a, 0, 0, i)
                gb, dgb = R.jacobi_p(b, 2 * i + 1, 0, j), grad_jacobi_p(b, 2 * i + 1, 0, j)
                dr = dfa * gb
                ds = dfa * gb * (0.5 * (1 + a))
                if i > 0:
                    dr = dr * hb ** (i - 1)
                    ds = ds * hb ** (i - 1)
                tmp = dgb * hb ** i
                if i > 0:
                    tmp = tmp - 0.5 * i * gb * hb ** (i - 1)
                ds = ds + fa * tmp
                c = 2.0 ** (i + 0.5)
                Vr.append(c * dr)
                Vs.append(c * ds)
        return np.stack(Vr, axis=1), np.stack(Vs, axis=1)
    t = np.asarray(t, dtype=np.float64)
    a, b, c3 = R._collapse3(r, s, t)
    hb, hc = 0.5 * (1 - b), 0.5 * (1 - c3)
    Vr, Vs, Vt = [], [], []
    for i in range(N + 1):
        for j in range(N - i + 1):
            for k in range(N - i - j + 1):
                fa, dfa = R.jacobi_p(a, 0, 0, i), grad_jacobi_p(a, 0, 0, i)
                gb, dgb = R.jacobi_p(b, 2 * i + 1, 0, j), grad_jacobi_p(b, 2 * i + 1, 0, j)
                hcp = R.jacobi_p(c3, 2 * (i + j) + 2, 0, k)
                dhc = grad_jacobi_p(c3, 2 * (i + j) + 2, 0, k)
                dr = dfa * (gb * hcp)
                if i > 0:
                    dr = dr * hb ** (i - 1)
                if i + j > 0:
                    dr = dr * hc ** (i + j - 1)
                ds = 0.5 * (1 + a) * dr
                tmp = dgb * hb ** i
                if i > 0:
                    tmp = tmp - 0.5 * i * gb * hb ** (i - 1)
                if i + j > 0:
                    tmp = tmp * hc ** (i + j - 1)
                tmp = fa * (tmp * hcp)
                ds = ds + tmp
                dt = 0.5 * (1 + a) * dr + 0.5 * (1 + b) * tmp
                tmp = dhc * hc ** (i + j)
                if i + j > 0:
                    tmp = tmp - 0.5 * (i + j) * hcp * hc ** (i + j - 1)
                tmp = fa * (gb * tmp) * hb ** i
                dt = dt + tmp
                cn = 2.0 ** (2 * i + j + 1.5)
                Vr.append(cn * dr)
                Vs.append(cn * ds)
                Vt.append(cn * dt)
    return np.stack(Vr, axis=1), np.stack(Vs, axis=1), np.stack(Vt, axis=1)


def gauss_legendre(n):
    """n+1 Gauss-Legendre points and weights on [-1, 1], ascending, from the
    eigenvalues of the symmetric Jacobi matrix (Golub & Welsch, 1969) -- the
    reference's JacobiGQ(n, 0, 0)."""
    if n == 0:
        return np.zeros(1), np.full(1, 2.0)
    i = np.arange(n, dtype=np.float64)
    off = 2.0 / (2 * i + 2) * np.sqrt((i + 1) ** 4 / ((2 * i + 1) * (2 * i + 3)))
    J = np.diag(off, 1) + np.diag(off, -1)
    x, V = np.linalg.eigh(J)
    return x, 2.0 * V[0, :] ** 2


def _rdiv(A, V):
    """A V^-1"""
    return np.linalg.solve(V.T, A.T).T


def points(dim, N):
    """The tabulated point sets of degree N: nodes, volume cubature and (3D)
    the triangle cubature of the faces."""
    path = os.path.join(DATA, f"points_{dim}d_N{N}.npz")
    if not os.path.exists(path):
        raise ValueError(f"no point sets for dim={dim} N={N} ({path})")
    with np.load(path) as z:
        return {k: np.asarray(z[k], dtype=np.float64) for k in z.files}


def build(dim, N, pts=None) -> dict:
    """Every table of the reference element (the RefOps attributes) from the
    point sets."""
    p = points(dim, N) if pts is None else pts
    M = 2 * N
    r, s = p["r"], p["s"]
    t = p["t"] if dim == 3 else np.zeros_like(r)
    rq, sq, wq = p["rq"], p["sq"], p["wq"]
    tq = p["tq"] if dim == 3 else np.zeros_like(rq)
    if dim == 2:
        rq1, wq1 = gauss_legendre(int(math.ceil(M / 2.0)))
        one = np.ones_like(rq1)
        rf = np.concatenate([rq1, -rq1, -one])                   # faces s=-1, r+s=0, r=-1
        sf = np.concatenate([-one, rq1, -rq1])
        tf = np.zeros_like(rf)
        nr = np.concatenate([0 * one, one, -one])
        ns = np.concatenate([-one, one, 0 * one])
        nt = np.zeros_like(nr)
        wfq = np.tile(wq1, 3)
        ref_rfq, ref_sfq, nfaces = rq1, np.zeros_like(rq1), 3
    else:
        rt, st, wt = p["ref_rfq"], p["ref_sfq"], p["wtri"]
        one = np.ones_like(rt)
        rf = np.concatenate([rt, rt, -(one + rt + st), -one])    # faces t=-1, s=-1, r+s+t=-1, r=-1
        sf = np.concatenate([st, -one, rt, rt])
        tf = np.concatenate([-one, st, st, st])
        nr = np.concatenate([0 * one, 0 * one, one, -one])
        ns = np.concatenate([0 * one, -one, one, 0 * one])
        nt = np.concatenate([-one, 0 * one, one, 0 * one])
        wfq = np.tile(wt, 4)
        ref_rfq, ref_sfq, nfaces = rt, st, 4
    Np, Nq, NfqNf = r.size, rq.size, rf.size
    Nfq = NfqNf // nfaces
    args = (r, s, t) if dim == 3 else (r, s)
    V = R.vandermonde(dim, N, *args)
    G = grad_vandermonde(dim, N, *args)
    D = [_rdiv(g, V) for g in G]
    if dim == 2:
        D.append(np.zeros((Np, Np)))
    qargs = (rq, sq, tq) if dim == 3 else (rq, sq)
    fargs = (rf, sf, tf) if dim == 3 else (rf, sf)
    Vq = _rdiv(R.vandermonde(dim, N, *qargs), V)
    Mm = Vq.T @ (wq[:, None] * Vq)
    Pq = np.linalg.solve(Mm, Vq.T * wq[None, :])
    Vfq = _rdiv(R.vandermonde(dim, N, *fargs), V)
    Lq = np.linalg.solve(Mm, Vfq.T * wfq[None, :])
    VqLq, VqPq, VfPq = Vq @ Lq, Vq @ Pq, Vfq @ Pq
    hyb = lambda Dx, nx: Vq @ Dx @ Pq - 0.5 * (VqLq * nx[None, :]) @ VfPq
    out = dict(r=r, s=s, t=t, rq=rq, sq=sq, tq=tq, wq=wq, rfq=rf, sfq=sf, tfq=tf, wfq=wfq,
               nrJ=nr, nsJ=ns, ntJ=nt, V=V, Dr=D[0], Ds=D[1], Dt=D[2], Vq=Vq, Pq=Pq, Vfq=Vfq,
               ref_rfq=ref_rfq, ref_sfq=ref_sfq if dim == 3 else np.zeros(Nfq),
               VqLq=VqLq, VqPq=VqPq, VfPq=VfPq, Drq=hyb(D[0], nr), Dsq=hyb(D[1], ns),
               Dtq=hyb(D[2], nt) if dim == 3 else np.zeros((Nq, Nq)))
    out["sizes"] = np.array([dim, N, M, Np, Nq, Nfq, nfaces, NfqNf], dtype=np.int64)
    return out
