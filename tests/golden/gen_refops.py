"""Generate, from the reference's own operator builder
(build_ref_ops_2D/3D, operators.cpp:104-341, and the hybridized operators of
host_operators_new_2D/3D, operators_c.cpp:46-69, 212-241, compiled from the
reference sources by oracle/build.py):

* tests/golden/refops/refops_<dim>d_N<N>.npz -- every table of the reference
  element (the inputs the reference's kernels receive: Drq, Dsq, Dtq, VqLq,
  VqPq, VfPq, nrJ, ...; and V, Dr, Vq, Pq, Vfq, ...), the check that
  tests/test_refbuild.py pins scratch_wadge_b200/refbuild.py against;
* scratch_wadge_b200/data/points_<dim>d_N<N>.npz -- the point sets those
  tables are built from: the interpolation nodes, the volume cubature and,
  in 3D, the triangle cubature of the faces, as tabulated in the
  reference's node_data.h and read by its builder.  refbuild.py builds the
  product's operators from these.

Run once in a checkout where the reference tree exists:
    python tests/golden/gen_refops.py
"""

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import build  # noqa: E402

NAMES = ["r", "s", "t", "rq", "sq", "tq", "wq", "rfq", "sfq", "tfq", "wfq",
         "nrJ", "nsJ", "ntJ", "V", "Dr", "Ds", "Dt", "Vq", "Pq", "Vfq",
         "ref_rfq", "ref_sfq", "VqLq", "VqPq", "VfPq", "Drq", "Dsq", "Dtq"]


def shapes(dim, sz):
    Np, Nq, Nfq, Nfaces, NfqNf = sz
    return {
        "r": (Np,), "s": (Np,), "t": (Np,), "rq": (Nq,), "sq": (Nq,), "tq": (Nq,),
        "wq": (Nq,), "rfq": (NfqNf,), "sfq": (NfqNf,), "tfq": (NfqNf,), "wfq": (NfqNf,),
        "nrJ": (NfqNf,), "nsJ": (NfqNf,), "ntJ": (NfqNf,), "V": (Np, Np), "Dr": (Np, Np),
        "Ds": (Np, Np), "Dt": (Np, Np), "Vq": (Nq, Np), "Pq": (Np, Nq), "Vfq": (NfqNf, Np),
        "ref_rfq": (Nfq,), "ref_sfq": (Nfq,), "VqLq": (Nq, NfqNf), "VqPq": (Nq, Nq),
        "VfPq": (NfqNf, Nq), "Drq": (Nq, Nq), "Dsq": (Nq, Nq), "Dtq": (Nq, Nq),
    }


def refelem(dim, N, M=None):
    """All arrays of the reference element of degree N (cubature degree M=2N)
    as produced by the reference builder."""
    M = 2 * N if M is None else M
    lib = ctypes.CDLL(build.build_ref_ops())
    sz = (ctypes.c_int * 5)()
    lib.wadgref_refelem_sizes(dim, N, M, sz)
    sz = list(sz)
    shp = shapes(dim, sz)
    # Fortran-ordered buffers receive Eigen's column-major data as-is
    arrs = {k: np.zeros(shp[k], dtype=np.float64, order="F") for k in NAMES}
    ptrs = (ctypes.POINTER(ctypes.c_double) * len(NAMES))(
        *[arrs[k].ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for k in NAMES])
    lib.wadgref_refelem_fill(dim, N, M, ptrs)
    if dim == 2:
        for k in ("t", "tq", "tfq", "ntJ", "Dt", "Dtq", "ref_sfq"):
            arrs[k] = np.zeros(shp[k])
    out = {k: np.ascontiguousarray(v) for k, v in arrs.items()}
    out["sizes"] = np.array([dim, N, M] + sz, dtype=np.int64)
    return out


def main():
    if not build.reference_present():
        raise SystemExit("reference tree not found")
    checkdir = os.path.join(ROOT, "tests", "golden", "refops")
    ptsdir = os.path.join(ROOT, "scratch_wadge_b200", "data")
    os.makedirs(checkdir, exist_ok=True)
    os.makedirs(ptsdir, exist_ok=True)
    for dim, degs in ((2, (1, 2, 3, 4, 5)), (3, (1, 2, 3, 4, 5))):
        for N in degs:
            d = refelem(dim, N)
            path = os.path.join(checkdir, f"refops_{dim}d_N{N}.npz")
            np.savez_compressed(path, **d)
            Nfq = int(d["sizes"][5])
            pts = dict(r=d["r"], s=d["s"], rq=d["rq"], sq=d["sq"], wq=d["wq"])
            if dim == 3:
                pts.update(t=d["t"], tq=d["tq"], ref_rfq=d["ref_rfq"], ref_sfq=d["ref_sfq"],
                           wtri=d["wfq"][:Nfq])
            np.savez_compressed(os.path.join(ptsdir, f"points_{dim}d_N{N}.npz"), **pts)
            print(path, d["sizes"].tolist())


if __name__ == "__main__":
    main()
