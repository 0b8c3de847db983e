"""Batched ensemble of independent 2D vortex solves.

Each instance is a periodic triangle mesh of [0,20]x[-5,5] (quads split in
two, as the single-solve 2D workload), with its own element count, degree,
vortex strength and centre.  Instances of one degree form a *bin*: their
geometry and state arrays are concatenated and their neighbour maps offset,
so the bin is one element list that the persistent kernels walk without
knowing instance boundaries (every kernel is element-local apart from the
mapPq gather, which stays inside its instance).  Every instance runs to the
common final time T with its own step (the reference's dt with the
instance's wave speed); the
kernels take the step per element and walk work lists of the batches of
instances still running.

``Ensemble``          the batched path: one wadg_app per bin, one CUDA graph
                      per time step covering all bins (wadg_ensemble_run).
``SingleInstances``   the plain path: one wadg_app per instance, each time
                      step launched instance by instance (3 kernels x 5
                      stages x instances), each instance its own steps.
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


def instance_steps(parts, T, CFL=0.5):
    """Each instance's own step and step count to the final time T: the
    reference's dt = CFL hmin / C_N (euler.c:4180-4193) divided by the
    instance's largest wave speed |u| + c, then n = ceil(T / dt) and
    dt = T / n (euler.c:3680-3688).  Without the wave speed the coarsest
    instances (a few dozen triangles, |u| + c up to 2.5) blow up within one
    step."""
    return [IC.time_step(geo, CFL, geo.ops.N, FinalTime=T, wave_speed=IC.max_wave_speed(st["Q"]))
            for geo, st in parts]


class Ensemble:
    """The batched path: one wadg_app per degree bin, every instance with its
    own step to the final time T (wadg_ensemble_*)."""

    def __init__(self, instances, parts=None, T=0.1, CFL=0.5, gamma=1.4, autotune=False):
        """autotune: pick each bin's CTA shape of the volume + surface kernel
        by timing it on the bin (wadg_app_autotune)"""
        self.instances = instances
        self.parts = parts if parts is not None else [build_instance(i, gamma) for i in instances]
        self.steps = instance_steps(self.parts, T, CFL)
        self.T = T
        self.degrees = sorted({i.N for i in instances})
        self.bins = {}
        self.tuning = {}
        for N in self.degrees:
            idx = [j for j, i in enumerate(instances) if i.N == N]
            geo, st, offs = concat([self.parts[j] for j in idx])
            app = capi.App(geo, curved=True, gamma=gamma)
            app.set_stage_variant("volsurf")
            if autotune:
                app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
                self.tuning[N] = app.autotune(min(self.steps[j][0] for j in idx))
            app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
            self.bins[N] = dict(idx=idx, geo=geo, state=st, offs=offs, app=app,
                                dt=np.array([self.steps[j][0] for j in idx], dtype=np.float64),
                                nsteps=np.array([self.steps[j][1] for j in idx], dtype=np.int32),
                                offs32=np.ascontiguousarray(offs, dtype=np.int32))
        self.h = self._create()
        self.K = sum(g.K for g, _ in self.parts)
        self.dofs = sum(g.K * g.ops.Np for g, _ in self.parts)

    @property
    def stage_dofs(self):
        """DOF x stages of the whole run to T (each instance its own steps)."""
        return sum(g.K * g.ops.Np * 5 * n for (g, _), (_, n) in zip(self.parts, self.steps))

    def _create(self):
        L = capi.lib()
        descs = (EnsembleBin * len(self.bins))()
        for d, b in zip(descs, self.bins.values()):
            d.app = b["app"].h.value
            d.ninst = len(b["idx"])
            d.offsets = b["offs32"].ctypes.data_as(ctypes.POINTER(ctypes.c_int))
            d.dt = b["dt"].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            d.nsteps = b["nsteps"].ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        h = ctypes.c_void_p()
        capi.check(L.wadg_ensemble_create(len(self.bins), ctypes.cast(descs, ctypes.c_void_p),
                                          ctypes.byref(h)), "ensemble_create")
        return h

    def close(self):
        if getattr(self, "h", None):
            capi.lib().wadg_ensemble_destroy(self.h)
            self.h = None
        for b in self.bins.values():
            b["app"].close()

    __del__ = close

    def restart(self):
        """Back to the initial states and step 0."""
        for b in self.bins.values():
            st = b["state"]
            b["app"].set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
        capi.check(capi.lib().wadg_ensemble_restart(self.h), "ensemble_restart")

    def progress(self):
        """(time steps done, the longest instance's step count)"""
        done, mx = ctypes.c_int(), ctypes.c_int()
        capi.check(capi.lib().wadg_ensemble_steps(self.h, ctypes.byref(done), ctypes.byref(mx)),
                   "ensemble_steps")
        return done.value, mx.value

    def run(self, nsteps=None):
        """Advance nsteps time steps (None: to the end of every instance)."""
        L = capi.lib()
        n = self.progress()[1] if nsteps is None else nsteps
        capi.check(L.wadg_ensemble_run(self.h, n), "ensemble_run")
        capi.check(L.wadg_ensemble_sync(self.h), "ensemble_sync")

    def time_run(self, nsteps=None):
        """Device time (ms) of nsteps time steps (None: to the end)."""
        ms = ctypes.c_float()
        n = self.progress()[1] if nsteps is None else nsteps
        capi.check(capi.lib().wadg_ensemble_time_run(self.h, n, ctypes.byref(ms)), "ensemble_time_run")
        return ms.value

    def instance_state(self, j):
        """State arrays of instance j (host copies)."""
        N = self.instances[j].N
        b = self.bins[N]
        pos = b["idx"].index(j)
        a, z = b["offs"][pos], b["offs"][pos + 1]
        s = b["app"].get_state()
        return {k: v[a:z] for k, v in s.items()}


class EnsembleBin(ctypes.Structure):
    _fields_ = [("app", ctypes.c_void_p), ("ninst", ctypes.c_int),
                ("offsets", ctypes.POINTER(ctypes.c_int)), ("dt", ctypes.POINTER(ctypes.c_double)),
                ("nsteps", ctypes.POINTER(ctypes.c_int))]


class SingleInstances:
    """The plain path: one solver per instance, launched one after another,
    each with its own step to the final time T."""

    def __init__(self, instances, parts=None, T=0.1, CFL=0.5, gamma=1.4):
        import torch
        self.instances = instances
        self.parts = parts if parts is not None else [build_instance(i, gamma) for i in instances]
        self.steps = instance_steps(self.parts, T, CFL)
        self.done = [0] * len(self.parts)
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

    def _advance(self, nsteps):
        for j, a in enumerate(self.apps):
            dt, n = self.steps[j]
            m = n - self.done[j] if nsteps is None else min(nsteps, n - self.done[j])
            if m > 0:
                a.rk_run(dt, m, graph=False)
                self.done[j] += m

    def run(self, nsteps=None):
        """Advance every instance by nsteps of its own steps, at most to its
        end (None: to the end)."""
        self._advance(nsteps)
        self.apps[0].sync()

    def time_run(self):
        """Device time (ms) of the whole run to T on the shared stream."""
        import torch
        s = self.stream
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        self._advance(None)
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1)
