"""Command-line solver: the reference's main program on the CUDA path.

The reference's `main` (euler.c:3833-4215) reads a Lua preferences file
(prefs/euler_default.lua: app.mesh.filename, app.mesh.N, app.physical.gamma,
FinalTime, CFL, tau, app.output.datadir), builds the mesh, operators and
geometric factors, sets the initial condition and its entropy projection,
runs LSRK-45 to FinalTime through rk_run and reports the L2 error and the
entropy.  This driver takes the same preferences as options, with the mesh
either read from a gmsh 2.2 file or generated (the periodic square and cube
of the synthetic workloads):

    python -m scratch_wadge_b200.solve --case tg3d --N 3 --n 16 --steps 100
    python -m scratch_wadge_b200.solve --mesh-filename m.msh --dim 2 --ic vortex --final-time 1

It prints one JSON line: sizes, dt and steps, device time per step (CUDA
events around the graph-launched run), per-kernel times with --time-kernels,
the entropy before and after, and the L2 error where the initial condition
has an exact solution (vortex, density wave).  --datadir writes the mesh in
MFEM format (euler.c:1771-1857)."""

from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

from . import capi
from . import ic as IC
from . import mesh as M
from . import meshio

CASES = {
    # the synthetic workloads: mesh, dimension, curved, initial condition
    "vortex2d": dict(dim=2, curved=False, ic="vortex", n=32),
    "tg3d": dict(dim=3, curved=False, ic="taylor_green", n=16),
    "curved3d": dict(dim=3, curved=True, ic="density_wave", n=12),
}


def build_mesh(args):
    if args.mesh_filename:
        return meshio.read_gmsh(args.mesh_filename, args.dim)
    if args.case == "vortex2d":
        return M.periodic_square(args.n, args.n)
    if args.case == "curved3d":
        return M.periodic_cube(args.n, warp=M.warp_cube(args.warp))
    return M.periodic_cube(args.n)


def main(argv=None):
    """Run an Euler solve on the GPU and print a JSON summary."""
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--case", choices=sorted(CASES), default="tg3d",
                    help="generated mesh + initial condition (ignored for the mesh with --mesh-filename)")
    ap.add_argument("--mesh-filename", default=None, help="gmsh 2.2 mesh (app.mesh.filename)")
    ap.add_argument("--dim", type=int, choices=[2, 3], default=None, help="dimension of --mesh-filename")
    ap.add_argument("--curved", action="store_true", help="weight-adjusted (curved) kernels for --mesh-filename")
    ap.add_argument("--ic", default=None, help="vortex | taylor_green | density_wave | constant")
    ap.add_argument("--N", type=int, default=3, help="polynomial degree (app.mesh.N)")
    ap.add_argument("--n", type=int, default=None,
                    help="generated mesh: quads / hexes per direction (defaults: vortex2d 32, tg3d 16, "
                         "curved3d 12); each quad is split into 2 triangles, each hex into 6 tets")
    ap.add_argument("--warp", type=float, default=0.05, help="curved3d: node warping amplitude")
    ap.add_argument("--gamma", type=float, default=1.4, help="app.physical.gamma")
    ap.add_argument("--tau", type=float, default=1.0, help="app.physical.tau (3D penalty scale)")
    ap.add_argument("--cfl", type=float, default=0.5, help="app.physical.CFL")
    ap.add_argument("--final-time", type=float, default=None, help="app.physical.FinalTime")
    ap.add_argument("--steps", type=int, default=None, help="a fixed number of steps instead of FinalTime")
    ap.add_argument("--no-wave-speed", action="store_true",
                    help="dt = CFL hmin / C_N exactly as the reference (by default dt is also divided by "
                         "the initial maximum wave speed, which the Taylor-Green state needs)")
    ap.add_argument("--fused", action="store_true", help="the fused one-launch stage kernel")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default CTA shape of the volume kernel (by default a few stages "
                         "are timed per candidate shape and the fastest is kept)")
    ap.add_argument("--time-kernels", type=int, default=0, metavar="STAGES",
                    help="also time the volume, surface and update kernels over this many stages")
    ap.add_argument("--datadir", default=None, help="write the mesh as MFEM here (app.output.datadir)")
    args = ap.parse_args(argv)

    case = CASES[args.case]
    if args.n is None:
        args.n = case["n"]
    if args.mesh_filename:
        if args.dim is None:
            ap.error("--dim is required with --mesh-filename")
        curved = args.curved
    else:
        args.dim, curved = case["dim"], case["curved"]
    kind = args.ic or case["ic"]
    if args.steps is None and args.final_time is None:
        args.steps = 10

    mesh = build_mesh(args)
    solver = capi.Solver(mesh, args.N, curved, ic=kind, gamma=args.gamma, tau=args.tau)
    geo, app = solver.geo, solver.app
    wave = None if args.no_wave_speed else IC.max_wave_speed(solver.Q0, args.gamma)
    dt, nsteps = IC.time_step(geo, args.cfl, args.N, args.final_time, args.steps, wave_speed=wave)
    app.set_fused(args.fused)
    S0 = IC.entropy(geo, solver.Q0, args.gamma)
    warps = None
    if not args.no_autotune:
        warps, _ = app.autotune(dt, 5)
        solver.reset()

    kernels = None
    if args.time_kernels:
        app.time_kernels(dt, 1)  # warm-up: module loading, kernel attributes
        ms = app.time_kernels(dt, args.time_kernels)
        kernels = {k: v / args.time_kernels for k, v in zip(("vol", "surf", "update"), ms)}
        solver.reset()
    ms = app.time_run(dt, nsteps, graph=True)
    Q = app.get_state()["Q"]
    out = dict(dim=args.dim, N=args.N, K=int(geo.K), curved=curved, ic=kind, dt=dt, steps=nsteps,
               t=dt * nsteps, ms_per_step=ms / max(nsteps, 1),
               dof_stages_per_s=5 * geo.K * geo.ops.Np * nsteps / (ms * 1e-3) if ms > 0 else None,
               entropy0=S0, entropy=IC.entropy(geo, Q, args.gamma),
               finite=bool(np.isfinite(Q).all()))
    if kernels:
        out["kernel_ms"] = kernels
    if warps is not None:
        out["vol_shape"] = warps
    if kind in ("vortex", "density_wave", "constant"):
        out["l2_error"] = IC.l2_error(geo, Q, IC.exact_state(geo, kind, dt * nsteps, args.gamma))
    if args.datadir:
        os.makedirs(args.datadir, exist_ok=True)
        meshio.write_mfem(mesh, geo, os.path.join(args.datadir, "mesh.mfem"))
    print(json.dumps(out))
    return 0 if out["finite"] else 1


if __name__ == "__main__":
    sys.exit(main())
