"""Mesh files through the library's C ABI (include/wadg.h, mesh I/O):
gmsh 2.2 in (the reference's host_mesh_read_msh, euler.c:556-833), gmsh 2.2
and MFEM out (host_mesh_write_mfem, euler.c:1771-1857).

A mesh read from gmsh carries the reference's boundary semantics: faces on the
bounding box are matched periodically (modify_mapP, euler.c:3004-3175) and a
face point with no partner is a boundary point, its own neighbour
(``Mesh.boundary_self``)."""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import capi
from . import mesh as M


def read_gmsh(path: str, dim: int) -> M.Mesh:
    """ASCII gmsh 2.x -> Mesh (periodic box = the vertices' bounding box)."""
    L = capi.lib()
    h = ctypes.c_void_p()
    capi.check(L.wadg_mesh_read_gmsh(os.fsencode(path), dim, ctypes.byref(h)), "read_gmsh")
    try:
        d, nv, K, flipped = ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        capi.check(L.wadg_mesh_sizes(h, ctypes.byref(d), ctypes.byref(nv), ctypes.byref(K),
                                     ctypes.byref(flipped)), "mesh_sizes")
        VX = np.empty((nv.value, dim))
        EToV = np.empty((K.value, dim + 1), dtype=np.int64)
        lo, hi = np.empty(dim), np.empty(dim)
        capi.check(L.wadg_mesh_get(h, VX.ctypes.data, EToV.ctypes.data, lo.ctypes.data,
                                   hi.ctypes.data), "mesh_get")
    finally:
        L.wadg_mesh_destroy(h)
    m = M.Mesh(dim, VX, EToV, lo, hi, boundary_self=True)
    m.flipped = int(flipped.value)
    return m


def write_gmsh(mesh: M.Mesh, path: str) -> None:
    VX = np.ascontiguousarray(mesh.VX, dtype=np.float64)
    EToV = np.ascontiguousarray(mesh.EToV, dtype=np.int64)
    capi.check(capi.lib().wadg_mesh_write_gmsh(os.fsencode(path), mesh.dim, VX.shape[0],
                                               VX.ctypes.data, EToV.shape[0], EToV.ctypes.data),
               "write_gmsh")


def boundary_faces(geo: M.Geometry) -> np.ndarray:
    """uint8 [K][Nfaces]: 1 where every face point of the face is its own
    neighbour (mapPq(j) = j), the reference's boundary faces."""
    ops = geo.ops
    K, NF, Nfq, Nf = geo.K, ops.NfqNf, ops.Nfq, ops.Nfields
    own = (np.arange(NF)[None, :] + np.arange(K)[:, None] * NF * Nf).astype(np.uint32)
    selfp = (geo.mapPq == own).reshape(K, ops.Nfaces, Nfq)
    return np.ascontiguousarray(selfp.all(axis=2).astype(np.uint8))


def write_mfem(mesh: M.Mesh, geo: M.Geometry, path: str) -> None:
    """MFEM mesh v1.0 of the mesh, the boundary faces taken from geo."""
    EToVX = np.ascontiguousarray(mesh.VX[mesh.EToV], dtype=np.float64)  # [K][nv][dim]
    bface = boundary_faces(geo)
    capi.check(capi.lib().wadg_mesh_write_mfem(os.fsencode(path), mesh.dim, mesh.K,
                                               EToVX.ctypes.data, bface.ctypes.data),
               "write_mfem")
