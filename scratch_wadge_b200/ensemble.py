"""Batched ensemble of independent 2D vortex solves.

Each instance is a periodic triangle mesh of [0,20]x[-5,5] (quads split in
two, as the single-solve 2D workload), with its own element count, degree,
vortex strength and centre.  Instances of one degree form a *bin*: their
geometry and state arrays are concatenated and their neighbour maps offset,
so the bin is one element list that the persistent kernels walk without
knowing instance boundaries (every kernel is element-local apart from the
mapPq gather, which stays inside its instance).  All instances advance with
one common dt (the smallest stable one), so a bin is exactly one solver.

``Ensemble``          the batched path: one wadg_app per bin, one CUDA graph
                      per time step covering all bins (wadg_ensemble_run).
``SingleInstances``   the plain path: one wadg_app per instance, each time
                      step launched instance by instance (3 kernels x 5
                      stages x instances).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import capi
from . import ic as IC
from . import mesh as M


@dataclass
class Instance:
    K: int
    N: int
    beta: float
    x0: float
    y0: float
    nx: int
    ny: int


def draw_instances(n=256, kmin=200, kmax=8192, degrees=(2, 3, 4), seed=0):
    """Element counts log-uniform in [kmin, kmax], N uniform in `degrees`,
    vortex strength beta ~ U[3, 6], centre uniform in the domain (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        target = math.exp(rng.uniform(math.log(kmin), math.log(kmax)))
        # K = 2 nx ny with nx = 2 ny (domain aspect 2:1)
        ny = max(2, int(round(math.sqrt(target / 4.0))))
        nx = 2 * ny
        N = int(rng.choice(degrees))
        beta = float(rng.uniform(3.0, 6.0))
        x0 = float(rng.uniform(0.0, 20.0))
        y0 = float(rng.uniform(-5.0, 5.0))
        out.append(Instance(2 * nx * ny, N, beta, x0, y0, nx, ny))
    return out


def build_instance(inst: Instance, gamma=1.4, builder=None):
    """Geometry (builder(mesh, N): mesh.build_geometry by default, or
    geometry_gpu.build_geometry_gpu) and stage-0 state of one instance."""
    geo = (builder or M.build_geometry)(M.periodic_square(inst.nx, inst.ny), inst.N)
    U0 = IC.initial_state(geo, "vortex", gamma, beta=inst.beta, x0=inst.x0, y0=inst.y0)
    Q, rhsQ, Qf, resQ = IC.stage0(geo, U0, gamma)
    return geo, dict(Q=Q, rhsQ=rhsQ, Qf=Qf, resQ=resQ)


def concat(parts):
    """Concatenate (geometry, state) of instances of one degree into a bin;
    returns the bin geometry, state and each instance's element offset."""
    geos = [p[0] for p in parts]
    ops = geos[0].ops
    offs = np.cumsum([0] + [g.K for g in geos])
    per = ops.NfqNf * ops.Nfields
    mapPq = np.concatenate([g.mapPq.astype(np.int64) + o * per for g, o in zip(geos, offs[:-1])])
    if int(offs[-1]) * per > 2 ** 32:
        raise ValueError(f"bin of {int(offs[-1])} elements: neighbour indices exceed the 32-bit mapPq")
    cat = lambda name: np.concatenate([getattr(g, name) for g in geos])
    geo = M.Geometry(ops, int(offs[-1]), cat("vgeo"), cat("vfgeo"), cat("fgeo"), cat("Jq"),
                     mapPq.astype(np.uint32), cat("xyzq"), cat("xyzf"))
    st = {k: np.concatenate([p[1][k] for p in parts]) for k in ("Q", "rhsQ", "Qf", "resQ")}
    return geo, st, offs


def common_dt(parts, CFL=0.5):
    """Smallest stable step over the instances (wave-speed scaled)."""
    dts = []
    for geo, st in parts:
        dt, _ = IC.time_step(geo, CFL, geo.ops.N, nsteps=1, wave_speed=IC.max_wave_speed(st["Q"]))
        dts.append(dt)
    return min(dts)


class Ensemble:
    """The batched path."""

    def __init__(self, instances, parts=None, fused=False, gamma=1.4, autotune_dt=None):
        self.instances = instances
        self.parts = parts if parts is not None else [build_instance(i, gamma) for i in instances]
        self.degrees = sorted({i.N for i in instances})
        self.bins = {}
        for N in self.degrees:
            idx = [j for j, i in enumerate(instances) if i.N == N]
            geo, st, offs = concat([self.parts[j] for j in idx])
            app = capi.App(geo, curved=True, gamma=gamma)
            app.set_fused(fused)
            tuning = None
            if autotune_dt is not None:  # the volume kernel's CTA shape for this bin
                app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
                tuning = app.autotune(autotune_dt)
            app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
            self.bins[N] = dict(idx=idx, geo=geo, state=st, offs=offs, app=app, tuning=tuning)
        self.h = None
        self.joint_tuning = None
        if autotune_dt is not None:
            self._tune_jointly(autotune_dt)
        self.h = self._create()
        self.K = sum(g.K for g, _ in self.parts)
        self.dofs = sum(g.K * g.ops.Np for g, _ in self.parts)

    def _create(self):
        apps = (ctypes.c_void_p * len(self.bins))(*[b["app"].h.value for b in self.bins.values()])
        h = ctypes.c_void_p()
        L = capi.lib()
        L.wadg_ensemble_create.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        capi.check(L.wadg_ensemble_create(len(self.bins), apps, ctypes.byref(h)), "ensemble_create")
        return h

    def _set_shapes(self, shapes):
        L = capi.lib()
        for N, b in self.bins.items():
            ctx = ctypes.c_void_p(L.wadg_app_ctx(b["app"].h))
            capi.check(L.wadg_ctx_set_vol_warps(ctx, 1, shapes[N]), "set_vol_warps")

    def _tune_jointly(self, dt, steps=3):
        """Each bin's shape was tuned alone, but the bins run concurrently:
        keep the per-bin choices only if the whole batched step is faster
        with them than with every bin at its default shape."""
        tuned = {N: b["tuning"][0] for N, b in self.bins.items()}
        default = {N: 0 for N in self.bins}
        if all(tuned[N] == self._default_shape(N) for N in self.bins):
            return
        times = {}
        L = capi.lib()
        for name, shapes in (("tuned", tuned), ("default", default)):
            self._set_shapes(shapes)
            h = self._create()
            self.h = h
            try:
                self.run(dt, 1)
                times[name] = self.time_run(dt, steps) / steps
            finally:
                L.wadg_ensemble_destroy(h)
                self.h = None
        best = "tuned" if times["tuned"] <= times["default"] else "default"
        self._set_shapes(tuned if best == "tuned" else default)
        self.joint_tuning = dict(ms_per_step=times, kept=best)
        self.reset()

    def _default_shape(self, N):
        L = capi.lib()
        ctx = ctypes.c_void_p(L.wadg_app_ctx(self.bins[N]["app"].h))
        cand = (ctypes.c_int * 3)()
        L.wadg_vol_warps_candidates(ctx, 1, cand)
        return int(cand[0])

    def close(self):
        if getattr(self, "h", None):
            capi.lib().wadg_ensemble_destroy(self.h)
            self.h = None
        for b in self.bins.values():
            b["app"].close()

    __del__ = close

    def reset(self):
        for b in self.bins.values():
            st = b["state"]
            b["app"].set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])

    def run(self, dt, nsteps):
        L = capi.lib()
        L.wadg_ensemble_run.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        capi.check(L.wadg_ensemble_run(self.h, dt, nsteps), "ensemble_run")
        capi.check(L.wadg_ensemble_sync(self.h), "ensemble_sync")

    def time_run(self, dt, nsteps):
        L = capi.lib()
        L.wadg_ensemble_time_run.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_float)]
        ms = ctypes.c_float()
        capi.check(L.wadg_ensemble_time_run(self.h, dt, nsteps, ctypes.byref(ms)), "ensemble_time_run")
        return ms.value

    def instance_state(self, j):
        """State arrays of instance j (host copies)."""
        N = self.instances[j].N
        b = self.bins[N]
        pos = b["idx"].index(j)
        a, z = b["offs"][pos], b["offs"][pos + 1]
        s = b["app"].get_state()
        return {k: v[a:z] for k, v in s.items()}


class SingleInstances:
    """The plain path: one solver per instance, launched one after another."""

    def __init__(self, instances, parts=None, gamma=1.4):
        import torch
        self.instances = instances
        self.parts = parts if parts is not None else [build_instance(i, gamma) for i in instances]
        self.stream = torch.cuda.Stream()  # one stream for all instances, in order
        self.apps = []
        for geo, st in self.parts:
            app = capi.App(geo, curved=True, gamma=gamma, stream=self.stream.cuda_stream)
            app.set_fused(False)
            app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
            self.apps.append(app)
        self.K = sum(g.K for g, _ in self.parts)
        self.dofs = sum(g.K * g.ops.Np for g, _ in self.parts)

    def close(self):
        for a in self.apps:
            a.close()

    def run(self, dt, nsteps):
        for _ in range(nsteps):
            for a in self.apps:
                a.rk_run(dt, 1, graph=False)
        self.apps[0].sync()

    def time_run(self, dt, nsteps):
        """Device time of nsteps on the shared stream (CUDA events)."""
        import torch
        s = self.stream
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(nsteps):
            for a in self.apps:
                a.rk_run(dt, 1, graph=False)
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1)
