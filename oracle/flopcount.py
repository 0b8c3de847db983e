"""Test infrastructure only: a counting-scalar evaluation of the reference's
per-pair arithmetic, to fix the algorithmic flop count the volume kernel's
roofline uses (frozen in scratch_wadge_b200/roofline.py and checked against
this file by tests/test_roofline.py).

Counted: each +, -, *, / and each log/exp/pow/sqrt as one floating-point
operation, exactly as the reference source writes them (no fusion credit).
Per-node work (primitive variables and beta of the row node) is excluded; the
reference recomputes the column node's primitives for every pair
(Euler3Daffine.okl:296-303), and that recomputation is excluded too, so the
count is the pair work proper:

  flux       euler3d_flux (Euler3Daffine.okl:107-148) / euler2d_flux
             (Euler2D.okl:139-161) with both log-means (:43-71 / :36-67)
  contract   the geometric contraction and the accumulation into divF of
             the three loops of euler_vol_3d (:296-324, :327-362, :387-406)
             and their 2D / curved counterparts.
"""

from __future__ import annotations

import math


class C:
    """A float that counts the operations applied to it."""

    n = 0

    def __init__(self, v):
        self.v = float(v.v if isinstance(v, C) else v)

    @staticmethod
    def _v(x):
        return x.v if isinstance(x, C) else float(x)

    def _op(self, o, f):
        C.n += 1
        return C(f(self.v, C._v(o)))

    def __add__(self, o): return self._op(o, lambda a, b: a + b)
    def __radd__(self, o): return self._op(o, lambda a, b: b + a)
    def __sub__(self, o): return self._op(o, lambda a, b: a - b)
    def __rsub__(self, o): return self._op(o, lambda a, b: b - a)
    def __mul__(self, o): return self._op(o, lambda a, b: a * b)
    def __rmul__(self, o): return self._op(o, lambda a, b: b * a)
    def __truediv__(self, o): return self._op(o, lambda a, b: a / b)
    def __rtruediv__(self, o): return self._op(o, lambda a, b: b / a)
    def __neg__(self): return C(-self.v)
    def __lt__(self, o): return self.v < C._v(o)
    def __abs__(self): return C(abs(self.v))


def clog(x):
    C.n += 1
    return C(math.log(C._v(x)))


def logmean(aL, aR, thr, order):
    # Euler3Daffine.okl:43-71 / Euler2D.okl:36-67 (TESTING off)
    xi = aL / aR
    f = (xi - 1.0) / (xi + 1.0)
    u = f * f
    u2 = u * u
    if abs(u) < thr:
        F = 1.0 + u / 3.0 + u2 / 5.0 + u2 * u / 7.0
        if order == 2:
            F = F + u2 * u2 / 9.0
    else:
        F = clog(xi) / 2.0 / f
    return (aL + aR) / (2.0 * F)


def avg(a, b):
    return 0.5 * (a + b)


def flux(dim, g, a, b):
    """two-point flux; a, b = (rho, u, v[, w], beta) counting scalars"""
    thr = 1e-4 if dim == 3 else 1e-3
    rho_i, rho_j = a[0], b[0]
    vel_i, vel_j = a[1:1 + dim], b[1:1 + dim]
    beta_i, beta_j = a[-1], b[-1]
    rholog = logmean(rho_i, rho_j, thr, dim)
    rhoavg = avg(rho_i, rho_j)
    ua = [avg(x, y) for x, y in zip(vel_i, vel_j)]
    s1 = ua[0] * ua[0]
    for q in ua[1:]:
        s1 = s1 + q * q
    s2 = avg(vel_i[0] * vel_i[0], vel_j[0] * vel_j[0])
    for x, y in zip(vel_i[1:], vel_j[1:]):
        s2 = s2 + avg(x * x, y * y)
    vnavg = 2.0 * s1 - s2
    beta_avg = avg(beta_i, beta_j)
    pa = rhoavg / (2.0 * beta_avg)
    f4aux = rholog / (2.0 * (g - 1.0) * logmean(beta_i, beta_j, thr, dim)) + pa + 0.5 * rholog * vnavg
    # components (FxS etc.): mass dim, momentum dim*dim (+pa on the diagonal), energy dim
    F0 = [rholog * q for q in ua]
    mom = [[F0[d] * ua[c] + (pa if c == d else 0.0) for d in range(dim)] for c in range(dim)]
    if dim == 2:
        mom[1][0] = mom[0][1]  # FxS3 = FyS2 (Euler2D.okl:158)
    FE = [f4aux * q for q in ua]
    return F0, mom, FE


def _state(dim, series):
    if series:
        a = [C(1.0), C(0.1), C(0.2), C(0.3), C(0.007)][: dim + 1] + [C(0.007)]
        b = [C(1.0001), C(0.11), C(0.19), C(0.29), C(0.00701)][: dim + 1] + [C(0.00701)]
    else:
        a = [C(1.0), C(0.1), C(0.2), C(0.3), C(0.5)][: dim + 1] + [C(0.5)]
        b = [C(2.0), C(0.11), C(0.19), C(0.29), C(0.9)][: dim + 1] + [C(0.9)]
    return a, b


def pair_flops(dim, kind, curved, series=True, g=1.4):
    """Operations of one ordered pair of the volume kernel.
    kind: 'vv' (volume row x volume column), 'vf' (volume row x face column),
    'fv' (face row x volume column)."""
    a, b = _state(dim, series)
    G = [C(0.3 + 0.1 * i) for i in range(dim * dim)]
    Gj = [C(0.31 + 0.1 * i) for i in range(dim * dim)]
    C.n = 0
    F0, mom, FE = flux(dim, g, a, b)
    fields = [[F0[d] for d in range(dim)]] + [mom[c] for c in range(dim)] + [FE]
    if curved:
        G = [0.5 * (x + y) for x, y in zip(G, Gj)]
    if kind == "vv":
        r = [C(0.2), C(-0.1), C(0.05)][:dim]
        acc = C(0.0)
        if dim == 3:
            # Dx = Drq*rxJ + Dsq*sxJ + Dtq*txJ, ...; divF += Dx*FxS + Dy*FyS + Dz*FzS
            D = [r[0] * G[d] + r[1] * G[3 + d] + r[2] * G[6 + d] for d in range(3)]
            for comp in fields:
                acc = acc + (D[0] * comp[0] + D[1] * comp[1] + D[2] * comp[2])
        else:
            # divF += Drq*(Fx*rxJ + Fy*ryJ) + Dsq*(Fx*sxJ + Fy*syJ)
            for comp in fields:
                acc = acc + (r[0] * (comp[0] * G[0] + comp[1] * G[1]) +
                             r[1] * (comp[0] * G[2] + comp[1] * G[3]))
    else:
        nref = [C(0.0), C(0.0), C(-1.0)][:dim]
        w = 0.5 * C(0.3) if kind == "vf" else -0.5 * C(0.3)
        acc = C(0.0)
        if dim == 3:
            n = [G[d] * nref[0] + G[3 + d] * nref[1] + G[6 + d] * nref[2] for d in range(3)]
            for comp in fields:
                acc = acc + w * (comp[0] * n[0] + comp[1] * n[1] + comp[2] * n[2])
        else:
            for comp in fields:
                acc = acc + w * ((comp[0] * G[0] + comp[1] * G[1]) * nref[0] +
                                 (comp[0] * G[2] + comp[1] * G[3]) * nref[1])
    return C.n


def element_flops(dim, Nq, NfqNf, curved, series=True):
    """Algorithmic flops of one element of the volume kernel (reference
    algorithm: Nq^2 volume pairs, Nq*NfqNf volume-face and NfqNf*Nq
    face-volume pairs)."""
    return (Nq * Nq * pair_flops(dim, "vv", curved, series) +
            Nq * NfqNf * pair_flops(dim, "vf", curved, series) +
            NfqNf * Nq * pair_flops(dim, "fv", curved, series))


if __name__ == "__main__":
    for dim in (2, 3):
        for curved in (False, True):
            for series in (True, False):
                print(dim, curved, series,
                      [pair_flops(dim, k, curved, series) for k in ("vv", "vf", "fv")])
