"""Structured periodic simplex meshes and the geometric data the kernels read.

The reference reads unstructured gmsh meshes and builds its geometric factors
with Eigen (operators.cpp:343-719) and its neighbour maps by face-node matching
plus an O(n^2) periodic fix-up (operators.cpp:765-1025, euler.c:3004-3175).
The workloads here are seeded, structured periodic meshes, so this module
generates them directly and produces the same arrays with the same layouts:

  vgeo  [K][Nvgeo][Nq]        rxJ ryJ (rzJ) sxJ syJ (szJ) (txJ tyJ tzJ)
  vfgeo [K][Nvgeo][NfqNf]     the same factors at face quadrature points
  fgeo  [K][Nfgeo][NfqNf]     nxJ nyJ (nzJ) sJ
  Jq    [K][Nq]               VqPq * J  (operators.cpp:455, 758)
  mapPq [K][NfqNf] (uint32)   neighbour face point, field-strided:
                              j + e*NfqNf*Nfields  (euler.c:3156-3174)
  xyzq  [K][3][Nq], xyzf [K][3][NfqNf]

Geometric factors follow the reference's construction: the 2D cross-product
form (operators.cpp:387-428) and, in 3D, the Kopriva conservative curl form
interpolated from degree N+1 (operators.cpp:617-719), so that curved meshes
satisfy the discrete GCL exactly as in the reference.
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np

from . import refops as R


@dataclass
class Mesh:
    dim: int
    VX: np.ndarray            # (Nv, dim) vertex coordinates
    EToV: np.ndarray          # (K, dim+1) vertex ids, positive orientation
    lo: np.ndarray            # domain lower corner (dim,)
    hi: np.ndarray            # domain upper corner (dim,)
    warp: object = None       # optional callable (x,y[,z]) -> displaced coords
    boundary_self: bool = False  # unpaired face points are boundary points (mapPq(j) = j)

    @property
    def K(self):
        return self.EToV.shape[0]


def periodic_square(nx, ny, lo=(0.0, -5.0), hi=(20.0, 5.0)) -> Mesh:
    """nx x ny quads, each split into two counter-clockwise triangles."""
    xs = np.linspace(lo[0], hi[0], nx + 1)
    ys = np.linspace(lo[1], hi[1], ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    VX = np.stack([X.ravel(), Y.ravel()], axis=1)
    vid = lambda i, j: i * (ny + 1) + j
    tris = []
    for i in range(nx):
        for j in range(ny):
            a, b, c, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            tris.append((a, b, c))
            tris.append((a, c, d))
    return Mesh(2, VX, np.array(tris, dtype=np.int64), np.array(lo, float), np.array(hi, float))


def periodic_cube(n, lo=(-np.pi,) * 3, hi=(np.pi,) * 3, warp=None) -> Mesh:
    """n^3 hexes, each split into 6 tetrahedra along its main diagonal
    (Kuhn/Freudenthal split, conforming across neighbouring hexes)."""
    ls = [np.linspace(lo[d], hi[d], n + 1) for d in range(3)]
    X, Y, Z = np.meshgrid(*ls, indexing="ij")
    VX = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    vid = lambda i, j, k: (i * (n + 1) + j) * (n + 1) + k
    tets = []
    eye = np.eye(3, dtype=np.int64)
    for i in range(n):
        for j in range(n):
            for k in range(n):
                base = np.array([i, j, k])
                for perm in itertools.permutations(range(3)):
                    p0 = base
                    p1 = p0 + eye[perm[0]]
                    p2 = p1 + eye[perm[1]]
                    p3 = p2 + eye[perm[2]]
                    tets.append([vid(*p) for p in (p0, p1, p2, p3)])
    EToV = np.array(tets, dtype=np.int64)
    # positive orientation: det[vb-va, vc-va, vd-va] > 0
    v = VX[EToV]
    det = np.linalg.det(np.stack([v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]], axis=2))
    flip = det < 0
    EToV[flip] = EToV[flip][:, [0, 2, 1, 3]]
    return Mesh(3, VX, EToV, np.array(lo, float), np.array(hi, float), warp)


def warp_cube(amp=0.05):
    """x_i += amp * prod_k cos(x_k / 2): smooth, fixes the faces of [-pi,pi]^3."""
    def f(x, y, z):
        w = amp * np.cos(x / 2) * np.cos(y / 2) * np.cos(z / 2)
        return x + w, y + w, z + w
    return f


@dataclass
class Geometry:
    ops: R.RefOps
    K: int
    vgeo: np.ndarray
    vfgeo: np.ndarray
    fgeo: np.ndarray
    Jq: np.ndarray
    mapPq: np.ndarray
    xyzq: np.ndarray
    xyzf: np.ndarray
    extra: dict = field(default_factory=dict)


def _nodal_coords(mesh: Mesh, ops: R.RefOps):
    """Vertex map at the reference nodes (operators.cpp:365-367, 488-493)."""
    v = mesh.VX[mesh.EToV]  # (K, nv, dim)
    r, s = ops.r, ops.s
    if mesh.dim == 2:
        lam = np.stack([-(r + s), 1 + r, 1 + s], axis=0) * 0.5  # (3, Np)
    else:
        t = ops.t
        lam = np.stack([-(1 + r + s + t), 1 + r, 1 + s, 1 + t], axis=0) * 0.5
    x = np.einsum("vn,kvd->dnk", lam, v)  # (dim, Np, K)
    return x


def build_geometry(mesh: Mesh, N: int) -> Geometry:
    ops = R.load(mesh.dim, N)
    x = _nodal_coords(mesh, ops)
    xa = x.copy()                      # affine (unwarped) coordinates: topology
    if mesh.warp is not None:
        x = np.stack(mesh.warp(*x), axis=0)
    K = mesh.K
    Nq, NfqNf = ops.Nq, ops.NfqNf
    if mesh.dim == 2:
        g = _geofacs_2d(ops, x)
    else:
        g = _geofacs_3d(ops, x)
    vgeo = np.ascontiguousarray(np.stack(g["vq"], axis=0).transpose(2, 0, 1))   # (K,Nvgeo,Nq)
    vfgeo = np.ascontiguousarray(np.stack(g["vf"], axis=0).transpose(2, 0, 1))  # (K,Nvgeo,NfqNf)
    fgeo = np.ascontiguousarray(np.stack(g["fg"], axis=0).transpose(2, 0, 1))   # (K,Nfgeo,NfqNf)
    Jq = np.ascontiguousarray((ops.VqPq @ g["J"]).T)                            # (K,Nq)
    xq = np.stack([ops.Vq @ x[d] for d in range(mesh.dim)], axis=0)             # (dim,Nq,K)
    xf = np.stack([ops.Vfq @ x[d] for d in range(mesh.dim)], axis=0)
    xfa = np.stack([ops.Vfq @ xa[d] for d in range(mesh.dim)], axis=0)
    mapPq = _match_faces(mesh, ops, xfa, mesh.boundary_self)
    pad = lambda a: np.concatenate([a, np.zeros((3 - mesh.dim,) + a.shape[1:])], 0)
    xyzq = np.ascontiguousarray(pad(xq).transpose(2, 0, 1))
    xyzf = np.ascontiguousarray(pad(xf).transpose(2, 0, 1))
    if np.any(Jq <= 0):
        raise ValueError("mesh has elements with non-positive Jacobian")
    return Geometry(ops, K, vgeo, vfgeo, fgeo, Jq, mapPq, xyzq, xyzf,
                    {"J": g["J"], "x": x})


def _geofacs_2d(ops, x):
    """operators.cpp:385-440 (cross-product form)."""
    Drq, Dsq = ops.Vq @ ops.Dr, ops.Vq @ ops.Ds
    X, Y = x
    xr, yr, xs, ys = Drq @ X, Drq @ Y, Dsq @ X, Dsq @ Y
    rxJ, sxJ, ryJ, syJ = ys, -yr, -xs, xr
    J = xr * ys - yr * xs
    Drf, Dsf = ops.Vfq @ ops.Dr, ops.Vfq @ ops.Ds
    xr, yr, xs, ys = Drf @ X, Drf @ Y, Dsf @ X, Dsf @ Y
    rxJf, sxJf, ryJf, syJf = ys, -yr, -xs, xr
    Jf = xr * ys - yr * xs
    nrJ, nsJ = ops.nrJ[:, None], ops.nsJ[:, None]
    nxJ = rxJf * nrJ + sxJf * nsJ
    nyJ = ryJf * nrJ + syJf * nsJ
    sJ = np.sqrt((nxJ / Jf) ** 2 + (nyJ / Jf) ** 2) * Jf
    return {"vq": [rxJ, ryJ, sxJ, syJ], "vf": [rxJf, ryJf, sxJf, syJf],
            "fg": [nxJ, nyJ, sJ], "J": J}


def _cross_factors(xr, yr, zr, xs, ys, zs, xt, yt, zt):
    rxJ = ys * zt - zs * yt
    sxJ = yt * zr - zt * yr
    txJ = yr * zs - zr * ys
    ryJ = xt * zs - xs * zt
    syJ = xr * zt - xt * zr
    tyJ = xs * zr - zs * xr
    rzJ = xs * yt - xt * ys
    szJ = xt * yr - xr * yt
    tzJ = xr * ys - xs * yr
    J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt)
    return (rxJ, ryJ, rzJ, sxJ, syJ, szJ, txJ, tyJ, tzJ), J


def _geofacs_3d(ops, x):
    """operators.cpp:542-719: J and sJ from the cross-product form, the
    metric terms from Kopriva's conservative curl form at degree N+1."""
    X, Y, Z = x
    Drq, Dsq, Dtq = ops.Vq @ ops.Dr, ops.Vq @ ops.Ds, ops.Vq @ ops.Dt
    _, J = _cross_factors(Drq @ X, Drq @ Y, Drq @ Z, Dsq @ X, Dsq @ Y, Dsq @ Z,
                          Dtq @ X, Dtq @ Y, Dtq @ Z)
    Drf, Dsf, Dtf = ops.Vfq @ ops.Dr, ops.Vfq @ ops.Ds, ops.Vfq @ ops.Dt
    gf, Jf = _cross_factors(Drf @ X, Drf @ Y, Drf @ Z, Dsf @ X, Dsf @ Y, Dsf @ Z,
                            Dtf @ X, Dtf @ Y, Dtf @ Z)
    nrJ, nsJ, ntJ = ops.nrJ[:, None], ops.nsJ[:, None], ops.ntJ[:, None]
    rxJf, ryJf, rzJf, sxJf, syJf, szJf, txJf, tyJf, tzJf = gf
    nx = (rxJf * nrJ + sxJf * nsJ + txJf * ntJ) / Jf
    ny = (ryJf * nrJ + syJf * nsJ + tyJf * ntJ) / Jf
    nz = (rzJf * nrJ + szJf * nsJ + tzJf * ntJ) / Jf
    sJ = np.sqrt(nx ** 2 + ny ** 2 + nz ** 2) * Jf

    # Kopriva curl form at degree N+1, interpolated back to degree N
    o2 = R.load(3, ops.N + 1)
    V12 = R.interp_matrix(ops, (o2.r, o2.s, o2.t))
    V21 = R.interp_matrix(o2, (ops.r, ops.s, ops.t))
    Dr, Ds, Dt = o2.Dr, o2.Ds, o2.Dt
    x2, y2, z2 = V12 @ X, V12 @ Y, V12 @ Z
    xr, yr, zr = Dr @ x2, Dr @ y2, Dr @ z2
    xs, ys, zs = Ds @ x2, Ds @ y2, Ds @ z2
    xt, yt, zt = Dt @ x2, Dt @ y2, Dt @ z2
    rxJ = Dt @ (ys * z2) - Ds @ (yt * z2)
    sxJ = Dr @ (yt * z2) - Dt @ (yr * z2)
    txJ = Ds @ (yr * z2) - Dr @ (ys * z2)
    ryJ = -(Dt @ (xs * z2) - Ds @ (xt * z2))
    syJ = -(Dr @ (xt * z2) - Dt @ (xr * z2))
    tyJ = -(Ds @ (xr * z2) - Dr @ (xs * z2))
    rzJ = -(Dt @ (ys * x2) - Ds @ (yt * x2))
    szJ = -(Dr @ (yt * x2) - Dt @ (yr * x2))
    tzJ = -(Ds @ (yr * x2) - Dr @ (ys * x2))
    G = [V21 @ a for a in (rxJ, ryJ, rzJ, sxJ, syJ, szJ, txJ, tyJ, tzJ)]
    Gf = [ops.Vfq @ a for a in G]
    Gq = [ops.Vq @ a for a in G]
    rxJf, ryJf, rzJf, sxJf, syJf, szJf, txJf, tyJf, tzJf = Gf
    nxJ = rxJf * nrJ + sxJf * nsJ + txJf * ntJ
    nyJ = ryJf * nrJ + syJf * nsJ + tyJf * ntJ
    nzJ = rzJf * nrJ + szJf * nsJ + tzJf * ntJ
    return {"vq": Gq, "vf": Gf, "fg": [nxJ, nyJ, nzJ, sJ], "J": J}


def _match_faces(mesh: Mesh, ops, xf, unpaired_self=False) -> np.ndarray:
    """Neighbour of every face quadrature point, periodic in every direction,
    by matching physical coordinates (the result the reference reaches with
    build_maps_2D/3D plus modify_mapP).  With unpaired_self, a point with no
    partner is a boundary point and its own neighbour (the reference's
    idM == idP); otherwise it is an error.  Returns field-strided mapPq."""
    dim, K, NfqNf = mesh.dim, mesh.K, ops.NfqNf
    L = mesh.hi - mesh.lo
    n = K * NfqNf
    pts = xf.transpose(2, 1, 0).reshape(n, dim)  # point id = j + e*NfqNf
    t = (pts - mesh.lo) / L
    t = t - np.floor(t)
    t[t > 1 - 1e-9] = 0.0
    h = 1e-7
    key = np.round(t / h).astype(np.int64)
    order = np.lexsort(key.T[::-1])
    ks = key[order]
    start = np.ones(n, dtype=bool)
    start[1:] = np.any(ks[1:] != ks[:-1], axis=1)
    first = np.flatnonzero(start)
    size = np.diff(np.append(first, n))
    if np.any(size > 2) or (not unpaired_self and np.any(size == 1)):
        raise ValueError("face points do not pair up: mesh is not a closed periodic mesh")
    partner = np.arange(n, dtype=np.int64)
    two = first[size == 2]
    a, b = order[two], order[two + 1]
    partner[a] = b
    partner[b] = a
    e = partner // NfqNf
    j = partner % NfqNf
    own = np.arange(n) // NfqNf
    if np.any((e == own) & (partner != np.arange(n))):
        raise ValueError("face point matched inside its own element")
    mapPq = (j + e * NfqNf * ops.Nfields).astype(np.uint32)
    return mapPq.reshape(K, NfqNf)
