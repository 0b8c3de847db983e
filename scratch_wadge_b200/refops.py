"""Reference-element operators for the entropy-stable DG right-hand side.

``load(dim, N)`` returns the operator tables of the reference element of degree
N (cubature degree 2N), as the reference's host builder produces them
(build_ref_ops_2D/3D in operators.cpp:104-341 and the hybridized operators of
host_operators_new_2D/3D, operators_c.cpp:46-69, 212-241), built by
refbuild.py from the node and cubature point sets in
data/points_<dim>d_N<N>.npz:

  nodes r,s,t (Np); volume cubature rq,sq,tq,wq (Nq); face cubature
  rfq,sfq,tfq,wfq and reference normals nrJ,nsJ,ntJ (Nfq*Nfaces, face-major);
  V, Dr, Ds, Dt (Np x Np); Vq (Nq x Np); Pq (Np x Nq); Vfq (NfqNf x Np);
  VqLq (Nq x NfqNf); VqPq (Nq x Nq); VfPq (NfqNf x Nq);
  Drq, Dsq, Dtq (Nq x Nq) = Vq D Pq - 1/2 Vq Lq diag(n) Vfq Pq.

The reference builder's own tables (tests/golden/refops/, made by
tests/golden/gen_refops.py) pin the built ones in tests/test_refbuild.py.
This module also holds the orthonormal simplex basis (Hesthaven & Warburton,
"Nodal Discontinuous Galerkin Methods", 2008, App. A; the same construction
as operators.cpp's Vandermonde2D/3D), which the builder and the interpolation
between node sets of different degree (curved geometry) use.
"""

from __future__ import annotations

import functools
import math
import os

import numpy as np

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


class RefOps:
    """Operator tables of one reference element (attributes as listed above)."""

    def __init__(self, d: dict):
        sizes = [int(x) for x in d["sizes"]]
        self.dim, self.N, self.M, self.Np, self.Nq, self.Nfq, self.Nfaces, self.NfqNf = sizes
        for k, v in d.items():
            if k != "sizes":
                setattr(self, k, np.ascontiguousarray(v, dtype=np.float64))
        self.Nfields = self.dim + 2
        self.Nvgeo = 4 if self.dim == 2 else 9
        self.Nfgeo = 3 if self.dim == 2 else 4

    def fortran(self, name: str) -> np.ndarray:
        """Column-major flat copy (the layout the kernels index as A[i + j*rows])."""
        return np.asfortranarray(getattr(self, name)).ravel(order="F")


@functools.lru_cache(maxsize=None)
def load(dim: int, N: int) -> RefOps:
    from . import refbuild
    return RefOps(refbuild.build(dim, N))


# ----------------------------------------------------------- simplex basis
def jacobi_p(x, alpha, beta, n):
    """Orthonormal Jacobi polynomial P_n^(alpha,beta)(x) (H&W JacobiP)."""
    x = np.asarray(x, dtype=np.float64)
    pl = np.zeros((n + 1,) + x.shape)
    g0 = 2 ** (alpha + beta + 1) / (alpha + beta + 1) * math.gamma(alpha + 1) * \
        math.gamma(beta + 1) / math.gamma(alpha + beta + 1)
    pl[0] = 1.0 / math.sqrt(g0)
    if n == 0:
        return pl[0]
    g1 = (alpha + 1) * (beta + 1) / (alpha + beta + 3) * g0
    pl[1] = ((alpha + beta + 2) * x / 2 + (alpha - beta) / 2) / math.sqrt(g1)
    aold = 2 / (2 + alpha + beta) * math.sqrt((alpha + 1) * (beta + 1) / (alpha + beta + 3))
    for i in range(1, n):
        h1 = 2 * i + alpha + beta
        anew = 2 / (h1 + 2) * math.sqrt((i + 1) * (i + 1 + alpha + beta) * (i + 1 + alpha) *
                                        (i + 1 + beta) / (h1 + 1) / (h1 + 3))
        bnew = -(alpha ** 2 - beta ** 2) / h1 / (h1 + 2)
        pl[i + 1] = 1 / anew * (-aold * pl[i - 1] + (x - bnew) * pl[i])
        aold = anew
    return pl[n]


def _collapse2(r, s):
    a = np.where(np.abs(s - 1) > 1e-14, 2 * (1 + r) / np.where(np.abs(s - 1) > 1e-14, 1 - s, 1) - 1, -1.0)
    return a, s


def _collapse3(r, s, t):
    den = -s - t
    a = np.where(np.abs(den) > 1e-14, 2 * (1 + r) / np.where(np.abs(den) > 1e-14, den, 1) - 1, -1.0)
    b = np.where(np.abs(t - 1) > 1e-14, 2 * (1 + s) / np.where(np.abs(t - 1) > 1e-14, 1 - t, 1) - 1, -1.0)
    return a, b, t


def vandermonde(dim, N, r, s, t=None):
    """Orthonormal P_N basis evaluated at points (rows) -> (npts, Np)."""
    r = np.asarray(r, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    cols = []
    if dim == 2:
        a, b = _collapse2(r, s)
        for i in range(N + 1):
            for j in range(N - i + 1):
                cols.append(math.sqrt(2.0) * jacobi_p(a, 0, 0, i) *
                            jacobi_p(b, 2 * i + 1, 0, j) * (1 - b) ** i)
    else:
        a, b, c = _collapse3(r, s, np.asarray(t, dtype=np.float64))
        for i in range(N + 1):
            for j in range(N - i + 1):
                for k in range(N - i - j + 1):
                    cols.append(2 * math.sqrt(2.0) * jacobi_p(a, 0, 0, i) *
                                jacobi_p(b, 2 * i + 1, 0, j) * (1 - b) ** i *
                                jacobi_p(c, 2 * (i + j) + 2, 0, k) * (1 - c) ** (i + j))
    return np.stack(cols, axis=1)


def interp_matrix(ops_from: RefOps, pts) -> np.ndarray:
    """Matrix evaluating the degree-N nodal interpolant of ops_from at pts."""
    V = vandermonde(ops_from.dim, ops_from.N, ops_from.r, ops_from.s,
                    ops_from.t if ops_from.dim == 3 else None)
    Vp = vandermonde(ops_from.dim, ops_from.N, *pts)
    return np.linalg.solve(V.T, Vp.T).T
