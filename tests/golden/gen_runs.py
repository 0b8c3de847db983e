"""Generate the long-run golden numbers of the workload configurations from
the reference's own kernels.

The reference's kernels (okl/Euler2D.okl, okl/Euler3D.okl, compiled from
their sources by oracle/build.py) are run over whole solves, starting from
the host stage-0 state the reference's driver builds (euler.c:3958-4133,
ic.stage0 here), with the time step of euler.c:4180-4193 and the L2 error of
euler.c:4227-4274 against the exact solution:

  * vortex2d_N3_K2048: the isentropic vortex on [0,20]x[-5,5], 32x32 quads
    split into 2048 triangles, N = 3, CFL 0.5, the reference's dt (no wave
    speed), T = 1: the L2 error of the whole run.
  * density_wave_N4: rho = 2 + 0.5 sin(x+y+z-3t), u = v = w = 1, p = 1 on
    the warped periodic cube (x_i += 0.05 prod cos(x_k/2)), curved (WADG)
    kernels, N = 4, CFL 0.25 with the wave speed, T = 0.1, on n^3 x 6
    tetrahedra for n = 4, 6, 8, 12: the L2 error at T of each refinement.

Written to tests/golden/runs.json; the GPU tests repeat the runs through the
library and compare.

    python tests/golden/gen_runs.py
"""

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import build, pyoracle  # noqa: E402
from scratch_wadge_b200 import ic as IC  # noqa: E402
from scratch_wadge_b200 import mesh as M  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "runs.json")

DW_LEVELS = (4, 6, 8, 12)
DW_T, DW_CFL, DW_N = 0.1, 0.25, 4
VX_T, VX_CFL, VX_N = 1.0, 0.5, 3


def run_reference(geo, curved, kind, dt, nsteps, T, ic_args=None):
    U0 = IC.initial_state(geo, kind, **(ic_args or {}))
    st = dict(zip(("Q", "rhsQ", "Qf", "resQ"), IC.stage0(geo, U0)))
    st["rhsQf"] = np.zeros_like(st["Qf"])
    ref = pyoracle.Reference(geo.ops, curved)
    for _ in range(nsteps):
        ref.step(geo, dt, st)
    return IC.l2_error(geo, st["Q"], IC.exact_state(geo, kind, T, **(ic_args or {}))), st["Q"]


def dw_mesh(n):
    return M.periodic_cube(n, warp=M.warp_cube(0.05))


def dw_step(geo):
    U0 = IC.initial_state(geo, "density_wave")
    Q0 = IC.stage0(geo, U0)[0]
    return IC.time_step(geo, DW_CFL, DW_N, FinalTime=DW_T, wave_speed=IC.max_wave_speed(Q0))


def vortex_mesh():
    return M.periodic_square(32, 32)


def main():
    if not build.reference_present():
        raise SystemExit("reference tree not found")
    build.build_ref()
    out = {}
    geo = M.build_geometry(vortex_mesh(), VX_N)
    dt, ns = IC.time_step(geo, VX_CFL, VX_N, FinalTime=VX_T)
    err, Q = run_reference(geo, False, "vortex", dt, ns, VX_T)
    out["vortex2d_N3_K2048"] = dict(K=geo.K, N=VX_N, T=VX_T, dt=dt, nsteps=ns, l2=err,
                                    rho_sum=float(Q[:, 0].sum()))
    print("vortex", geo.K, ns, err, flush=True)
    levels = {}
    for n in DW_LEVELS:
        geo = M.build_geometry(dw_mesh(n), DW_N)
        dt, ns = dw_step(geo)
        err, Q = run_reference(geo, True, "density_wave", dt, ns, DW_T)
        levels[str(n)] = dict(K=geo.K, dt=dt, nsteps=ns, l2=err, rho_sum=float(Q[:, 0].sum()))
        print("density wave", n, geo.K, ns, err, flush=True)
    out["density_wave_N4"] = dict(N=DW_N, T=DW_T, CFL=DW_CFL, levels=levels)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
