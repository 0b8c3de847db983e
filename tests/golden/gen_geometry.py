"""Generate geometry fixtures from the reference's own geometry builder.

host_operators_new_2D / _3D (operators_c.cpp:39, 205) with build_geofacs_2D /
_3D (operators.cpp:343-719), compiled from the reference sources by
oracle/build.py into oracle/_ref/libwadgref_ops.so, are run on small affine
periodic meshes (the stock builder has no curved map).  Each fixture holds the
mesh (vertex coordinates, element-to-vertex table, the periodic box) and the
builder's outputs in the kernels' layouts: vgeo, vfgeo, fgeo, Jq, xyzq, xyzf.
The host and GPU geometry builders are tested against these where the
reference tree is absent.

    python tests/golden/gen_geometry.py
"""

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import build  # noqa: E402
from scratch_wadge_b200 import mesh as M  # noqa: E402
from scratch_wadge_b200 import refops as R  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# name: (dim, N, mesh builder)
CASES = {
    "geo3d_N2": (3, 2, lambda: M.periodic_cube(2)),
    "geo3d_N3": (3, 3, lambda: M.periodic_cube(2)),
    "geo3d_N4": (3, 4, lambda: M.periodic_cube(2)),
    "geo2d_N2": (2, 2, lambda: M.periodic_square(3, 2)),
    "geo2d_N3": (2, 3, lambda: M.periodic_square(3, 3)),
    "geo2d_N4": (2, 4, lambda: M.periodic_square(2, 3)),
}


def reference_geometry(mesh, N):
    lib = ctypes.CDLL(os.path.join(build.OUT_REF, "libwadgref_ops.so"))
    ops = R.load(mesh.dim, N)
    K, dim = mesh.K, mesh.dim
    Nvgeo, Nfgeo = dim * dim, dim + 1
    EToVX = np.ascontiguousarray(mesh.VX[mesh.EToV].reshape(K, -1))  # vertex-major per element
    out = dict(vgeo=np.zeros((K, Nvgeo, ops.Nq)), vfgeo=np.zeros((K, Nvgeo, ops.NfqNf)),
               fgeo=np.zeros((K, Nfgeo, ops.NfqNf)), Jq=np.zeros((K, ops.Nq)),
               xyzq=np.zeros((K, 3, ops.Nq)), xyzf=np.zeros((K, 3, ops.NfqNf)))
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    lib.wadgref_geofacs.argtypes = [ctypes.c_int] * 3 + [ctypes.c_uint32] + [ctypes.c_void_p] * 7
    rc = lib.wadgref_geofacs(dim, N, 2 * N, K, p(EToVX), *(p(out[k]) for k in
                             ("vgeo", "vfgeo", "fgeo", "Jq", "xyzq", "xyzf")))
    if rc:
        raise RuntimeError("reference geometry builder failed")
    return out


def main():
    if not build.reference_present():
        raise SystemExit("reference tree not found")
    build.build_ref_ops()
    for name, (dim, N, mk) in CASES.items():
        mesh = mk()
        out = reference_geometry(mesh, N)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), dim=np.array(dim), N=np.array(N),
                            VX=mesh.VX, EToV=mesh.EToV, lo=mesh.lo, hi=mesh.hi, **out)
        print(name, "K =", mesh.K)


if __name__ == "__main__":
    main()
