"""Generate golden vectors from the reference's own kernels.

The reference has no tests and no stored outputs, so the golden vectors are
made here: the OKL kernels of okl/Euler3Daffine.okl, okl/Euler3D.okl and
okl/Euler2D.okl, compiled from their sources by oracle/build.py (only the
listed minimal patches, see oracle/okl_to_cpp.py), are run on small seeded
cases.  Each fixture holds the inputs (geometry, maps, stage-0 state) and the
reference outputs after the volume kernel, the surface kernel, one update, and
one full LSRK-45 time step.  The GPU tests compare against these on machines
where the reference tree is absent.

    python tests/golden/gen_golden.py
"""

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import build, pyoracle  # noqa: E402
from scratch_wadge_b200 import ic as IC  # noqa: E402
from scratch_wadge_b200 import mesh as M  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# name: (dim, N, curved, mesh builder, initial state, ic args)
CASES = {
    "tg3d_affine_N3": (3, 3, False, lambda: M.periodic_cube(2), "taylor_green", {}),
    "dw3d_curved_N3": (3, 3, True, lambda: M.periodic_cube(2, warp=M.warp_cube(0.05)), "density_wave", {}),
    "tg3d_affine_N2": (3, 2, False, lambda: M.periodic_cube(2), "taylor_green", {}),
    "dw3d_curved_N4": (3, 4, True, lambda: M.periodic_cube(2, warp=M.warp_cube(0.05)), "density_wave", {}),
    "vortex2d_curved_N3": (2, 3, True, lambda: M.periodic_square(4, 4), "vortex", {"beta": 5.0, "x0": 5.0, "y0": 0.0}),
    "vortex2d_affine_N2": (2, 2, False, lambda: M.periodic_square(4, 3), "vortex", {"beta": 4.0, "x0": 8.0, "y0": 1.0}),
    "vortex2d_curved_N4": (2, 4, True, lambda: M.periodic_square(3, 3), "vortex", {"beta": 6.0, "x0": 10.0, "y0": -1.0}),
}


def make_case(name):
    dim, N, curved, mk, kind, args = CASES[name]
    geo = M.build_geometry(mk(), N)
    U0 = IC.initial_state(geo, kind, **args)
    Q, rhsQ, Qf, resQ = IC.stage0(geo, U0)
    return geo, dict(Q=Q, rhsQ=rhsQ, Qf=Qf, resQ=resQ), curved


def main():
    if not build.reference_present():
        raise SystemExit("reference tree not found")
    build.build_ref()
    for name in CASES:
        geo, st0, curved = make_case(name)
        ref = pyoracle.Reference(geo.ops, curved)
        dt = 1e-3
        out = {}
        s = {k: v.copy() for k, v in st0.items()}
        s["rhsQf"] = np.zeros_like(s["Qf"])
        ref.vol(geo, s["Qf"], s["rhsQ"], s["rhsQf"])
        out["vol_rhsQ"], out["vol_rhsQf"] = s["rhsQ"].copy(), s["rhsQf"].copy()
        ref.surf(geo, s["Qf"], s["rhsQf"], s["rhsQ"])
        out["surf_rhsQ"] = s["rhsQ"].copy()
        ref.update(geo, IC.RK4A[1], IC.RK4B[1], dt, s["rhsQ"], s["resQ"], s["Q"], s["Qf"])
        for k in ("Q", "rhsQ", "Qf", "resQ"):
            out["upd_" + k] = s[k].copy()
        s = {k: v.copy() for k, v in st0.items()}
        s["rhsQf"] = np.zeros_like(s["Qf"])
        ref.step(geo, dt, s)
        out["step_Q"] = s["Q"].copy()
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"),
                            vgeo=geo.vgeo, vfgeo=geo.vfgeo, fgeo=geo.fgeo, Jq=geo.Jq, mapPq=geo.mapPq,
                            dt=np.array(dt), dim=np.array(geo.ops.dim), N=np.array(geo.ops.N),
                            curved=np.array(int(curved)),
                            **{"in_" + k: v for k, v in st0.items()}, **out)
        print(name, "K =", geo.K)


if __name__ == "__main__":
    main()
