"""Geometry built on the GPU: the arrays of mesh.build_geometry, made by the
library's geometry builder (wadg_geofacs, wadg_match_faces in
include/wadg.h) instead of numpy.

The reference builds its geometric factors on the host, element by element
with Eigen (host_operators_new_2D / _3D, operators_c.cpp:39, 205;
build_geofacs_2D / _3D, operators.cpp:343-719), and its periodic neighbour
maps with an O(n^2) fix-up (euler.c:3004-3175).  Here the host computes the
nodal coordinates (the vertex map, operators.cpp:365-367, 488-493, and a
curved mesh's displacement), and the device builds everything else.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import capi
from . import mesh as M
from . import refops as R


class GeoOps(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("N", ctypes.c_int), ("Np", ctypes.c_int),
                ("Nq", ctypes.c_int), ("NfqNf", ctypes.c_int), ("Np2", ctypes.c_int)] + \
               [(n, ctypes.c_void_p) for n in ("Vq", "Vfq", "VqDr", "VqDs", "VqDt", "VfDr", "VfDs",
                                              "VfDt", "VqPq", "nrJ", "nsJ", "ntJ", "V12", "Dr2",
                                              "Ds2", "Dt2", "V21")]


class DeviceOps:
    """The reference-element operators of one (dim, N) on the device, and the
    wadg_geo_ops struct pointing at them (the tensors stay alive with it)."""

    def __init__(self, dim: int, N: int, device="cuda"):
        import torch

        ops = R.load(dim, N)
        self.ops = ops
        col = lambda a: torch.from_numpy(np.asfortranarray(a, dtype=np.float64).ravel(order="F")).to(device)
        vec = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(device)
        t = {"Vq": col(ops.Vq), "Vfq": col(ops.Vfq), "VqDr": col(ops.Vq @ ops.Dr),
             "VqDs": col(ops.Vq @ ops.Ds), "VfDr": col(ops.Vfq @ ops.Dr),
             "VfDs": col(ops.Vfq @ ops.Ds), "VqPq": col(ops.VqPq), "nrJ": vec(ops.nrJ),
             "nsJ": vec(ops.nsJ)}
        Np2 = 0
        if dim == 3:
            o2 = R.load(3, N + 1)
            Np2 = o2.Np
            t.update({"VqDt": col(ops.Vq @ ops.Dt), "VfDt": col(ops.Vfq @ ops.Dt),
                      "ntJ": vec(ops.ntJ),
                      "V12": col(R.interp_matrix(ops, (o2.r, o2.s, o2.t))),
                      "Dr2": col(o2.Dr), "Ds2": col(o2.Ds), "Dt2": col(o2.Dt),
                      "V21": col(R.interp_matrix(o2, (ops.r, ops.s, ops.t)))})
        self.tensors = t
        self.struct = GeoOps(dim, N, ops.Np, ops.Nq, ops.NfqNf, Np2,
                             *[(t[n].data_ptr() if n in t else None) for n, _ in GeoOps._fields_[6:]])


_CACHE: dict = {}


def device_ops(dim: int, N: int) -> DeviceOps:
    key = (dim, N)
    if key not in _CACHE:
        _CACHE[key] = DeviceOps(dim, N)
    return _CACHE[key]


def build_geometry_gpu(mesh: M.Mesh, N: int) -> M.Geometry:
    """mesh.build_geometry on the device (same arrays, same layouts); the
    result is copied back to host arrays."""
    import torch

    L = capi.lib()
    dops = device_ops(mesh.dim, N)
    ops = dops.ops
    dim, K, Nq, NF = mesh.dim, mesh.K, ops.Nq, ops.NfqNf
    x = M._nodal_coords(mesh, ops)                 # (dim, Np, K)
    xa = x
    if mesh.warp is not None:
        x = np.stack(mesh.warp(*x), axis=0)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a.transpose(2, 0, 1))).cuda()
    xd, xad = dev(x), (dev(xa) if mesh.warp is not None else None)
    f64 = dict(dtype=torch.float64, device="cuda")
    Nvgeo, Nfgeo = dim * dim, dim + 1
    out = {"vgeo": torch.empty((K, Nvgeo, Nq), **f64), "vfgeo": torch.empty((K, Nvgeo, NF), **f64),
           "fgeo": torch.empty((K, Nfgeo, NF), **f64), "Jq": torch.empty((K, Nq), **f64),
           "xyzq": torch.empty((K, 3, Nq), **f64), "xyzf": torch.empty((K, 3, NF), **f64)}
    mapPq = torch.empty((K, NF), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    capi.check(L.wadg_geofacs(ctypes.byref(dops.struct), K, xd.data_ptr(),
                              *(out[k].data_ptr() for k in ("vgeo", "vfgeo", "fgeo", "Jq", "xyzq", "xyzf")),
                              stream), "geofacs")
    nbytes = L.wadg_match_faces_workspace(K, NF)
    work = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")
    lo = (ctypes.c_double * dim)(*mesh.lo)
    hi = (ctypes.c_double * dim)(*mesh.hi)
    capi.check(L.wadg_match_faces(ctypes.byref(dops.struct), K,
                                  (xad if xad is not None else xd).data_ptr(), lo, hi,
                                  int(mesh.boundary_self), work.data_ptr(), nbytes,
                                  mapPq.data_ptr(), stream), "match_faces")
    h = {k: v.cpu().numpy() for k, v in out.items()}
    if np.any(h["Jq"] <= 0):
        raise ValueError("mesh has elements with non-positive Jacobian")
    return M.Geometry(ops, K, h["vgeo"], h["vfgeo"], h["fgeo"], h["Jq"],
                      mapPq.cpu().numpy().view(np.uint32), h["xyzq"], h["xyzf"], {"x": x})
