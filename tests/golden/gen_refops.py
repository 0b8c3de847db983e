"""Generate the reference-element operator tables shipped in
scratch_wadge_b200/data/refops_<dim>d_N<N>.npz.

The tables are outputs of the reference's own operator builder
(build_ref_ops_2D/3D, operators.cpp:104-341, and the hybridized operators of
host_operators_new_2D/3D, operators_c.cpp:46-69, 212-241), compiled from the
reference sources by oracle/build.py.  They are the inputs the reference's
kernels receive (Drq, Dsq, Dtq, VqLq, VqPq, VfPq, nrJ, ...) together with the
node, cubature and interpolation data the host geometry builder needs.  They
hold the quadrature rules tabulated in the reference's node_data.h as the
reference's builder consumes them, so the GPU path sees exactly the
reference's operators.

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
    outdir = os.path.join(ROOT, "scratch_wadge_b200", "data")
    os.makedirs(outdir, exist_ok=True)
    for dim, degs in ((2, (1, 2, 3, 4, 5)), (3, (1, 2, 3, 4, 5))):
        for N in degs:
            d = refelem(dim, N)
            path = os.path.join(outdir, f"refops_{dim}d_N{N}.npz")
            np.savez_compressed(path, **d)
            print(path, d["sizes"].tolist())


if __name__ == "__main__":
    main()
