"""Throughput of the entropy-stable flux-differencing RHS on B200.

Workload (one "step" = one LSRK-45 time step = 5 stages x {vol, surf, update}):
  3D Taylor-Green vortex on affine tetrahedra (Euler3Daffine kernels), FP64,
  periodic [-pi,pi]^3, 16^3 hexes x 6 tets = 24576 elements, N = 3,
  gamma = 1.4, CFL 0.5 (dt = CFL hmin / (C_N max(|u|+c)); the reference's
  formula without the wave speed is unstable on this state).  Synthetic: the
  mesh and the initial state are generated here (no external data).
Metric: FP64 DOF*stages/s, DOF = K * Np per field (Np = 20, Nfields = 5).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A time step runs either the three reference-facing kernels per stage or the
fused stage kernel (wadg_euler_stage_3d: vol + surf + update in one launch per
stage), whichever is faster on this GPU (both are timed, `stage_variant`),
replayed as a CUDA graph; the line also reports the three kernels timed one by
one (`roofline`, `hbm_kernels`).  Two more workloads are reported beside the
headline: `ensemble` (256 independent 2D vortex solves to a final time, each
with its own step, batched against one solver per instance) and `adjoint` (the checkpointed discrete adjoint of a
200-step Taylor-Green run on 3072 tets: reverse-sweep cost over the forward
run, and a finite-difference check of the gradient).  `setup` compares the
geometry builders on the workload mesh (GPU: wadg_geofacs + wadg_match_faces;
host: numpy).

Multi-GPU runs are replicas: the headline path is single-rank (the
reference's rk_step exchanges nothing).  Partitioned solves with a halo
exchange are scratch_wadge_b200/partition.py (not benchmarked here).

--impl ours       the CUDA library through its C ABI; `value` is timed with
                  CUDA events around K graph-replayed time steps with the state
                  resident in HBM (working set ~0.3 GB > L2); `e2e` is the
                  user-level host-buffer solve (wadg_app_solve_host_q: H2D of
                  Q0 from pinned memory, the stage-0 projection on the device,
                  the config's 100 time steps, D2H of Q).  Multi-GPU: independent replicas (the path
                  has no data exchange), max time over ranks.
--impl reference  the reference's own kernels compiled from its OKL sources
                  (oracle/_ref, OpenMP over all host cores; the C restatement
                  when oracle/_ref is absent) on the same workload; rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 DOF*stages/s at N=3 (3D affine-tet Taylor-Green, Euler3Daffine RHS)"
UNIT = "DOF*stages/s"
WORKLOAD = "taylor_green_3d_affine_N3_K24576"
NHEX, N, CFL, E2E_STEPS = 16, 3, 0.5, 100
# stage implementations the time step can run, and kernel launches per step
VARIANTS = ["three_kernels", "fused", "volsurf"]
LAUNCHES = {"three_kernels": 15, "fused": 5, "volsurf": 10}


def dist_env():
    from scratch_wadge_b200 import replicas as RP
    return RP.env()


def build_workload(builder=None):
    """Geometry (host builder by default; the reference arm keeps it), stage-0
    state and time step of the workload."""
    from scratch_wadge_b200 import ic as IC
    from scratch_wadge_b200 import mesh as M
    geo = (builder or M.build_geometry)(M.periodic_cube(NHEX), N)
    Q, rhsQ, Qf, resQ = IC.stage0(geo, IC.initial_state(geo, "taylor_green"))
    dt, _ = IC.time_step(geo, CFL, N, nsteps=E2E_STEPS, wave_speed=IC.max_wave_speed(Q))
    return geo, dict(Q=Q, rhsQ=rhsQ, Qf=Qf, resQ=resQ), dt


def config_dict(geo, n_gpus):
    return {"workload": WORKLOAD, "mesh": f"periodic [-pi,pi]^3, {NHEX}^3 hexes x 6 tets",
            "K": geo.K, "N": N, "Np": geo.ops.Np, "Nq": geo.ops.Nq, "NfqNf": geo.ops.NfqNf,
            "Nfields": 5, "dofs_per_field": geo.K * geo.ops.Np,
            "step": "one LSRK-45 time step (5 stages x vol+surf+update)",
            "l2": "inputs larger than L2 (state + geometry ~0.3 GB per replica)",
            "parallelism": f"replicas x{n_gpus}" if n_gpus > 1 else "single GPU"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def ncu_traffic():
    """DRAM bytes per launch from the committed ncu summary, if present."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def cpu_impl():
    """The CPU implementation of the path: the reference's kernels compiled
    from its sources when available, else the oracle's C restatement."""
    from oracle import pyoracle as O
    if O.reference_available(3, N):
        return O.Reference, "reference"
    return O.Port, "port"


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def time_cpu(geo, st0, dt, steps):
    """Wall time of `steps` full time steps of the CPU implementation."""
    cls, kind = cpu_impl()
    impl = cls(geo.ops, False)
    st = {k: v.copy() for k, v in st0.items()}
    st["rhsQf"] = np.zeros_like(st["Qf"])
    t0 = time.perf_counter()
    for _ in range(steps):
        impl.step(geo, dt, st)
    return time.perf_counter() - t0, kind


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(cpu_threads()))
    geo, st0, dt = build_workload()
    dofs = geo.K * geo.ops.Np
    _, kind = cpu_impl()
    # each step: one full time step of the whole workload (5 stages)
    if args.warmup > 0:
        time_cpu(geo, st0, dt, min(args.warmup, 1))
    sec, _ = time_cpu(geo, st0, dt, args.steps)
    v = dofs * 5 * args.steps / sec
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_dict(geo, 1),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]),
                             "kind": kind,
                             "sample": f"{args.steps} full LSRK-45 time steps of the whole workload "
                                       f"(K={geo.K}), OpenMP over elements"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    from scratch_wadge_b200 import replicas as RP
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = RP.init("nccl", 120.0)

    from scratch_wadge_b200 import build as B
    from scratch_wadge_b200 import capi
    from scratch_wadge_b200 import roofline as RF
    B.build()

    # geometry on the GPU (wadg_geofacs / wadg_match_faces); the host builder
    # is timed beside it for the setup comparison
    from scratch_wadge_b200 import geometry_gpu as GG
    from scratch_wadge_b200 import mesh as M
    GG.build_geometry_gpu(M.periodic_cube(2), N)  # module and operator upload, outside the timing
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    geo, st0, dt = build_workload(GG.build_geometry_gpu)
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    GG.build_geometry_gpu(M.periodic_cube(NHEX), N)
    t_gpu = time.perf_counter() - t0
    t0 = time.perf_counter()
    M.build_geometry(M.periodic_cube(NHEX), N)
    t_host = time.perf_counter() - t0
    setup = {"geometry_gpu_s": t_gpu, "geometry_host_s": t_host, "workload_setup_s": t_setup,
             "note": "geometric factors + neighbour maps of the workload mesh: the GPU builder "
                     "(wadg_geofacs + wadg_match_faces, with the host nodal coordinates and the "
                     "copies) against the numpy host builder; workload_setup_s adds the stage-0 "
                     "state and time step"}
    ops = geo.ops
    K, Nq, NfqNf, Np = geo.K, ops.Nq, ops.NfqNf, ops.Np
    dofs = K * Np
    stream = torch.cuda.Stream()
    app = capi.App(geo, curved=False, stream=stream.cuda_stream)
    app.set_state(st0["Q"], st0["rhsQ"], st0["Qf"], st0["resQ"])

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    if args.profile:
        # a short run for profilers: warm-up and a few time steps (in the
        # stage variant --stage-variant names; three kernels for auto),
        # nothing else
        if args.stage_variant != "auto":
            app.set_stage_variant(args.stage_variant)
        app.rk_run(dt, args.warmup + args.steps, graph=False)
        barrier()
        app.close()
        RP.finish(pg)
        return
    # warm-up (also captures the time-step graphs) and the choice between the
    # stage implementations: three reference kernels, the fused kernel, or
    # the volume + surface kernel and the update kernel; the first and the
    # last with their volume kernel's CTA shape autotuned on this workload
    variants, tuned = {}, {}
    for name in VARIANTS:
        app.set_stage_variant(name)
        if name != "fused":
            app.set_state(st0["Q"], st0["rhsQ"], st0["Qf"], st0["resQ"])
            label, times = app.autotune(dt)
            tuned[name] = (label, times, app.vol_shape())
        app.set_state(st0["Q"], st0["rhsQ"], st0["Qf"], st0["resQ"])
        app.rk_run(dt, max(args.warmup, 1), graph=True)
        variants[name] = app.time_run(dt, 10, graph=True) / 10
    pick = min(VARIANTS, key=lambda n: variants[n])
    if args.stage_variant != "auto":  # pinned (profiling: timings under a profiler mislead the choice)
        pick = args.stage_variant
    # every rank takes the same variant (rank 0's choice)
    pick = VARIANTS[int(RP.all_max(pg, VARIANTS.index(pick) if rank == 0 else 0))]
    app.set_stage_variant(pick)
    if pick in tuned:
        app.set_vol_shape(*tuned[pick][2])
    app.set_state(st0["Q"], st0["rhsQ"], st0["Qf"], st0["resQ"])
    app.rk_run(dt, max(args.warmup, 1), graph=True)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        time.sleep(0.5)  # let the sampler start
        barrier()
        ev0.record(stream)
        app.rk_run(dt, args.steps, graph=True)
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    clocks = clk.summary()
    ms = RP.all_max(pg, ms)
    value = RP.job_throughput(ws, dofs * 5 * args.steps, ms * 1e-3)

    # per-kernel device times (CUDA events on the app stream): the fused stage
    # kernel the time step runs, and the three reference kernels one by one
    nst = 20
    stage_ms = app.time_stage(dt, nst) / nst
    kms = app.time_kernels(dt, nst)
    vol_ms, surf_ms, upd_ms = (x / nst for x in kms)
    vs_ms, vs_upd_ms = (x / nst for x in app.time_volsurf(dt, nst))
    fl_stage = RF.stage_flops_per_element(3, Nq, NfqNf, False) * K
    fl_vs = RF.volsurf_flops_per_element(3, Nq, NfqNf, False) * K
    fl = RF.vol_flops_per_element(3, Nq, NfqNf, False) * K
    probe = fp64_peak(stream)
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    prof = ncu_traffic()
    # the roofline line describes the dominant kernel of the variant the time
    # step ran: the fused stage kernel, the volume + surface kernel, or the
    # volume kernel of the three
    if pick == "fused":
        roof = {"kernel": "stage_kernel (fused vol + surf + update, one launch per LSRK stage)",
                "algorithmic_flops_per_launch": fl_stage, "launch_ms": stage_ms,
                "flops_per_element": RF.stage_flops_per_element(3, Nq, NfqNf, False),
                "ncu": prof.get("stage_3d_affine_N3_K24576")}
    elif pick == "volsurf":
        roof = {"kernel": "vol_pairs_kernel<SURF> (wadg_euler_volsurf_3d: volume pairs, surface "
                          "flux and lift in one launch)",
                "algorithmic_flops_per_launch": fl_vs, "launch_ms": vs_ms,
                "flops_per_element": RF.volsurf_flops_per_element(3, Nq, NfqNf, False),
                "ncu": prof.get("volsurf_3d_affine_N3_K24576")}
    else:
        roof = {"kernel": "vol_pairs_kernel (euler_vol_3d, the pair-scheduled volume kernel)",
                "algorithmic_flops_per_launch": fl, "launch_ms": vol_ms,
                "flops_per_element": RF.vol_flops_per_element(3, Nq, NfqNf, False),
                "ncu": prof.get("vol_3d_affine_N3_K24576")}
    achieved = roof["algorithmic_flops_per_launch"] / (roof["launch_ms"] * 1e-3) / 1e12
    ncu = roof.pop("ncu") or {}
    roof.update({"bound": "fp64", "achieved": achieved, "peak": probe, "unit": "TFLOP/s",
                 "frac": achieved / probe,
                 "peak_source": "measured in-run: FP64 FMA probe (wadg_probe_fp64_fma)",
                 "traffic": ncu.get("dram_bytes"),
                 "ncu_fp64_pipe_active": ncu.get("fp64_pipe_active"),
                 "ncu_source": ncu.get("source"),
                 "pairs_per_element": RF.pairs_per_element(Nq, NfqNf),
                 "stage_ms": {"three_kernels": vol_ms + surf_ms + upd_ms, "fused": stage_ms,
                              "volsurf": vs_ms + vs_upd_ms}})
    sb = RF.surf_bytes_per_element(3, Nq, NfqNf) * K
    ub = RF.update_bytes_per_element(3, Nq, NfqNf) * K
    hbm_kernels = {
        "euler_vol_3d": {"launch_ms": vol_ms, "achieved_tflops": fl / (vol_ms * 1e-3) / 1e12,
                         "frac_of_fp64_peak": fl / (vol_ms * 1e-3) / 1e12 / probe,
                         "flops_per_element": RF.vol_flops_per_element(3, Nq, NfqNf, False)},
        "euler_surf_3d": {"launch_ms": surf_ms, "achieved_gbs": sb / (surf_ms * 1e-3) / 1e9,
                          "frac": (sb / (surf_ms * 1e-3) / 1e9) / hbm if hbm else None},
        "euler_update_3d": {"launch_ms": upd_ms, "achieved_gbs": ub / (upd_ms * 1e-3) / 1e9,
                            "frac": (ub / (upd_ms * 1e-3) / 1e9) / hbm if hbm else None},
        "peak_gbs": hbm, "peak_source": "MEASURED_PEAKS.json hbm_gbs (copy bandwidth)" if hbm else None,
        "note": "the reference-facing kernels one by one, CUDA events around each launch"}

    # end to end through the user-level host-buffer call
    pin = {"Q": torch.from_numpy(st0["Q"]).pin_memory()}
    Qout = torch.empty(pin["Q"].shape, dtype=torch.float64).pin_memory()
    host = {k: v.numpy() for k, v in pin.items()}
    qo = Qout.numpy()
    app.solve_host_q(host["Q"], dt, 2, out=qo)  # warm
    barrier()
    e2e_calls = max(1, args.e2e_calls)
    t0 = time.perf_counter()
    for _ in range(e2e_calls):
        app.solve_host_q(host["Q"], dt, E2E_STEPS, out=qo)
    barrier()
    e2e_s = time.perf_counter() - t0
    e2e_s = RP.all_max(pg, e2e_s)
    e2e_v = RP.job_throughput(ws, dofs * 5 * E2E_STEPS * e2e_calls, e2e_s)
    h2d = host["Q"].nbytes
    d2h = qo.nbytes

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(geo, ws),
            "e2e": {"value": e2e_v, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "step": f"one wadg_app_solve_host_q call: H2D of Q0, the stage-0 projection "
                            f"on the device, {E2E_STEPS} time steps, D2H of Q (pinned host "
                            f"buffers, wall clock)",
                    "calls": e2e_calls},
            "gpu_launches": LAUNCHES[pick] * args.steps,
            "autotune": {v: {"vol_shape": w, "ms_per_shape": c} for v, (w, c, _) in tuned.items()},
            "stage_variant": {"used": pick, "ms_per_step": variants},
            "roofline": roof, "hbm_kernels": hbm_kernels, "clocks": clocks, "setup": setup}
    if not args.no_ensemble:
        line["ensemble"] = run_ensemble_measurement()
    if not args.no_adjoint:
        line["adjoint"] = run_adjoint_measurement()
        # the bench workload's own size: 40 steps, checkpoint every 20
        line["adjoint_K24576"] = run_adjoint_measurement(nhex=NHEX, nsteps=40, every=20, reps=2,
                                                         fd_dirs=1)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(cpu_threads()))
        sec, kind = time_cpu(geo, st0, dt, 2)
        line["cpu_baseline"] = {"value": dofs * 10 / sec, "unit": UNIT,
                                "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": kind,
                                "sample": f"2 full LSRK-45 time steps (10 stages) of the whole "
                                          f"workload (K={K}), OpenMP over elements"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    app.close()
    RP.finish(pg)


def run_adjoint_measurement(nhex=8, nsteps=200, every=20, reps=3, fd_dirs=2):
    """Discrete adjoint of the Taylor-Green run: gradient of J = int rho(T)^2
    with respect to the initial state on nhex^3 x 6 affine tets (3072 by
    default), N = 3, nsteps LSRK-45 steps (200), checkpoint every `every`
    steps (20); the time steps run the volume + surface stage variant.  Times (CUDA events on the
    app's stream, best of `reps`): the plain forward run (graph-replayed), the
    checkpointed forward run and the reverse sweep (segment recompute + stage
    adjoints).  `fd_check`: relative difference of dJ/dQ0 . d from central
    differences of J (step 1e-6 relative to |Q0|, J summed exactly) on
    `fd_dirs` seeded unit-norm Gaussian directions."""
    import torch

    from scratch_wadge_b200 import capi
    from scratch_wadge_b200 import ic as IC
    from scratch_wadge_b200 import mesh as M
    from scratch_wadge_b200.adjoint import Adjoint, rho2_objective

    geo = M.build_geometry(M.periodic_cube(nhex), N)
    Q0 = IC.stage0(geo, IC.initial_state(geo, "taylor_green"))[0]
    dt = IC.time_step(geo, CFL, N, nsteps=nsteps, wave_speed=IC.max_wave_speed(Q0))[0]
    app = capi.App(geo, False)
    app.set_stage_variant("volsurf")  # the forward run and the recompute alike
    adj = Adjoint(app, nsteps, every)
    Qd = torch.from_numpy(Q0).cuda()
    stream = torch.cuda.ExternalStream(capi.lib().wadg_app_stream(app.h))

    def timed(fn):
        best, out = None, None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            out = fn()
            e1.record(stream)
            e1.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        return best, out

    QT = adj.forward(Qd, dt)
    J, gT = rho2_objective(geo, QT)
    adj.reverse(gT)  # warm-up
    fwd_ckpt_ms, QT = timed(lambda: adj.forward(Qd, dt))
    J, gT = rho2_objective(geo, QT)
    rev_ms, g0 = timed(lambda: adj.reverse(gT))
    adj.forward(Qd, dt)
    plain_ms = min(app.time_run(dt, nsteps, True) for _ in range(reps))

    def Jexact(Q):
        w = np.asarray(geo.ops.wq)[None, :] * np.asarray(geo.Jq)
        return math.fsum((w * Q[:, 0, :] ** 2).ravel())

    g0n = g0.cpu().numpy()
    eps = 1e-6 * float(np.linalg.norm(Q0))
    rng = np.random.default_rng(20261203)
    worst = 0.0
    for _ in range(fd_dirs):
        z = rng.standard_normal(Q0.shape)
        d = z / np.linalg.norm(z)
        Jp = Jexact(adj.forward(torch.from_numpy(Q0 + eps * d).cuda(), dt).cpu().numpy())
        Jm = Jexact(adj.forward(torch.from_numpy(Q0 - eps * d).cuda(), dt).cpu().numpy())
        an = float(np.sum(g0n * d))
        worst = max(worst, abs((Jp - Jm) / (2 * eps) - an) / abs(an))
    adj.close()
    app.close()
    return {"workload": f"taylor_green_3d_affine_N3_K{geo.K}_{nsteps}steps_checkpoint{every}",
            "objective": "J = integral of rho(x,T)^2 (volume cubature)", "J": float(J),
            "forward_ms": plain_ms, "forward_checkpointed_ms": fwd_ckpt_ms, "reverse_ms": rev_ms,
            "adjoint_over_forward": rev_ms / plain_ms,
            "gradient_over_forward": (fwd_ckpt_ms + rev_ms) / plain_ms,
            "fd_check": {"directions": fd_dirs, "worst_rel_diff": worst,
                         "step": "1e-6 relative to |Q0|"},
            "note": "adjoint_over_forward = reverse sweep (segment recompute from checkpoints + "
                    "stage adjoint kernels) / plain forward run; gradient_over_forward adds "
                    "the checkpointed forward run"}


def run_ensemble_measurement(T=0.05, reps=2):
    """The batched-ensemble workload: 256 independent 2D vortex solves (K log-uniform in
    [200, 8192], N uniform in {2,3,4}, seeded), each run to the final time T with its
    own step (the reference's dt per instance), batched (degree bins, work lists of
    the instances still running, one CUDA graph per time step) against the plain
    one-instance-per-launch path; throughput in DOF*stages/s over the whole run,
    timed with CUDA events."""
    from scratch_wadge_b200 import ensemble as EN
    from scratch_wadge_b200 import geometry_gpu as GG
    t0 = time.perf_counter()
    inst = EN.draw_instances(n=256, kmin=200, kmax=8192, degrees=(2, 3, 4), seed=0)
    parts = [EN.build_instance(i, builder=GG.build_geometry_gpu) for i in inst]
    setup_s = time.perf_counter() - t0
    ens = EN.Ensemble(inst, parts, T=T, autotune=True)
    nsteps = [n for _, n in ens.steps]
    work = ens.stage_dofs
    ens.run()  # warm-up (and the graph), then timed runs from the start
    best = float("inf")
    for _ in range(reps):
        ens.restart()
        best = min(best, ens.time_run())
    ens_tuning = ens.tuning
    ens.close()
    single = EN.SingleInstances(inst, parts, T=T)
    ms_single = single.time_run()
    single.close()
    return {"instances": len(inst), "K_total": sum(i.K for i in inst),
            "degrees": {str(N): sum(1 for i in inst if i.N == N) for N in (2, 3, 4)},
            "final_time": T, "steps_per_instance": {"min": min(nsteps), "max": max(nsteps),
                                                    "mean": sum(nsteps) / len(nsteps)},
            "setup_s": setup_s, "dof_stages": work,
            "batched_ms": best, "batched_value": work / (best * 1e-3),
            "single_ms": ms_single, "single_value": work / (ms_single * 1e-3),
            "speedup": ms_single / best, "unit": UNIT,
            "autotune": {str(N): {"vol_shape": w, "ms_per_shape": c} for N, (w, c) in ens_tuning.items()},
            "single_path": "one wadg_app per instance, 3 kernels x 5 stages launched per instance "
                           "and step, each instance its own steps",
            "batched_path": "one bin per degree (concatenated instances), volume + surface and "
                            "update kernels over work lists of the batches still running, per-element "
                            "steps, one CUDA graph per time step, bins on concurrent streams"}


def fp64_peak(stream):
    import ctypes

    from scratch_wadge_b200 import capi
    L = capi.lib()
    tf = ctypes.c_double()
    ms = ctypes.c_float()
    best = 0.0
    for _ in range(3):
        capi.check(L.wadg_probe_fp64_fma(ctypes.c_void_p(stream.cuda_stream), 20000,
                                         ctypes.byref(tf), ctypes.byref(ms)), "fp64 probe")
        best = max(best, tf.value)
    return best


def launch_ranks(n, argv):
    """Re-run this script as n ranks on this node (torch.distributed.run on
    127.0.0.1, a free port); returns the launcher's exit status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + argv
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-calls", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--stage-variant", choices=["auto"] + VARIANTS, default="auto",
                    help="stage implementation of the time step (auto: the faster one, timed)")
    ap.add_argument("--profile", action="store_true",
                    help="only warm-up + steps of the device path (for ncu), no JSON line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if args.gpus > 1 and ws == 1 and "RANK" not in os.environ:
        # not under a launcher: start one rank per GPU here
        sys.exit(launch_ranks(args.gpus, sys.argv[1:]))
    if ws != args.gpus:
        sys.exit(f"bench.py: --gpus {args.gpus} but the launcher started {ws} rank(s) "
                 f"(WORLD_SIZE={ws}); run it under torchrun with --nproc-per-node {args.gpus}")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
