"""ctypes binding of the C ABI (include/wadg.h) and the host-side solver.

The product path is the CUDA library libwadg_b200.so built in-tree by
scratch_wadge_b200/build.py.  Loading fails loudly when it is missing: there is
no CPU fallback.

* ``Context``   kernel-level entry points with the OKL argument lists
                (device pointers as ints, e.g. torch ``tensor.data_ptr()``).
* ``App``       the reference's app_t / rk_step / rk_run over library-owned
                device buffers (euler.c:2607-2796, 3610-3738).
* ``Solver``    mesh + operators + geometry + stage-0 state + App, the
                user-level object (the reference's main(), euler.c:3833-4350).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import ic as IC
from . import mesh as M
from . import refops as R

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwadg_b200.so")

_D = ctypes.POINTER(ctypes.c_double)
_U32 = ctypes.POINTER(ctypes.c_uint32)
_V = ctypes.c_void_p
_lib = None


# status codes (include/wadg.h)
OK, ERR_INVALID, ERR_UNSUPPORTED, ERR_CUDA, ERR_STATE = 0, 1, 2, 3, 4


class WadgError(RuntimeError):
    def __init__(self, msg, code=None):
        super().__init__(msg)
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("N", ctypes.c_int), ("Nq", ctypes.c_int),
                ("Nfq", ctypes.c_int), ("Nfaces", ctypes.c_int), ("gamma", ctypes.c_double),
                ("tau", ctypes.c_double), ("stream", ctypes.c_void_p)]


class HostData(ctypes.Structure):
    _fields_ = [(n, _D) for n in ("vgeo", "vfgeo", "fgeo", "Jq")] + [("mapPq", _U32)] + \
               [(n, _D) for n in ("nrJ", "nsJ", "ntJ", "Drq", "Dsq", "Dtq", "VqLq", "VqPq", "VfPq")]


def lib():
    """The CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise WadgError(f"{LIB_PATH} missing: run scratch_wadge_b200/build.py (no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.wadg_last_error.restype = ctypes.c_char_p
        i, d, v = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
        for name in ("wadg_euler_vol_3d", "wadg_euler_vol_3d_curved"):
            getattr(L, name).argtypes = [v, i] + [v] * 15
        for name in ("wadg_euler_vol_2d", "wadg_euler_vol_2d_curved"):
            getattr(L, name).argtypes = [v, i] + [v] * 12
        for name in ("wadg_euler_surf_3d", "wadg_euler_surf_2d"):
            getattr(L, name).argtypes = [v, i] + [v] * 6
        for name in ("wadg_euler_update_3d", "wadg_euler_update_3d_curved",
                     "wadg_euler_update_2d", "wadg_euler_update_2d_curved"):
            getattr(L, name).argtypes = [v, i, v, v, v, d, d, d, v, v, v, v]
        L.wadg_rk_step.argtypes = [v, d, d, d]
        L.wadg_rk_run.argtypes = [v, d, i, i]
        L.wadg_app_time_run.argtypes = [v, d, i, i, ctypes.POINTER(ctypes.c_float)]
        L.wadg_app_time_kernels.argtypes = [v, d, i, ctypes.POINTER(ctypes.c_float)]
        L.wadg_app_solve_host.argtypes = [v, v, v, v, v, d, i, v, v, v, v]
        L.wadg_app_solve_host_q.argtypes = [v, v, d, i, v]
        L.wadg_app_project.argtypes = [v]
        L.wadg_app_set_state.argtypes = [v, v, v, v, v]
        L.wadg_app_get_state.argtypes = [v, v, v, v, v]
        L.wadg_app_state_ptrs.argtypes = [v] + [ctypes.POINTER(ctypes.c_void_p)] * 5
        L.wadg_euler_stage_3d.argtypes = [v, i, i] + [v] * 14 + [d, d, d] + [v] * 6
        L.wadg_euler_stage_2d.argtypes = [v, i, i] + [v] * 12 + [d, d, d] + [v] * 6
        L.wadg_app_set_fused.argtypes = [v, i]
        L.wadg_app_time_stage.argtypes = [v, d, i, ctypes.POINTER(ctypes.c_float)]
        L.wadg_app_time_volsurf.argtypes = [v, d, i, ctypes.POINTER(ctypes.c_float)]
        L.wadg_euler_volsurf_3d.argtypes = [v, i, i] + [v] * 14
        L.wadg_euler_volsurf_2d.argtypes = [v, i, i] + [v] * 12
        L.wadg_probe_fp64_fma.argtypes = [v, i, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_float)]
        L.wadg_app_ctx.restype = ctypes.c_void_p
        L.wadg_app_ctx.argtypes = [v]
        L.wadg_app_stream.restype = ctypes.c_void_p
        L.wadg_app_stream.argtypes = [v]
        L.wadg_app_set_parity.argtypes = [v, i]
        L.wadg_app_get_fused.argtypes = [v]
        L.wadg_ensemble_create.argtypes = [i, v, ctypes.POINTER(ctypes.c_void_p)]
        L.wadg_ensemble_destroy.argtypes = [v]
        L.wadg_ensemble_sync.argtypes = [v]
        L.wadg_ensemble_run.argtypes = [v, i]
        L.wadg_ensemble_restart.argtypes = [v]
        L.wadg_ensemble_steps.argtypes = [v, ctypes.POINTER(i), ctypes.POINTER(i)]
        L.wadg_ensemble_time_run.argtypes = [v, i, ctypes.POINTER(ctypes.c_float)]
        L.wadg_app_create.argtypes = [ctypes.POINTER(Params), i, i, ctypes.POINTER(HostData),
                                      ctypes.POINTER(ctypes.c_void_p)]
        L.wadg_ctx_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_void_p)]
        L.wadg_ctx_destroy.argtypes = [v]
        L.wadg_app_destroy.argtypes = [v]
        L.wadg_app_sync.argtypes = [v]
        L.wadg_ctx_set_stream.argtypes = [v, v]
        L.wadg_euler_3d_compute_aux.argtypes = [v, i, v, v, v, v]
        L.wadg_element_entropy.argtypes = [v, i, v, v, v, v]
        L.wadg_entropy_rhs.argtypes = [v, i, i] + [v] * 6
        L.wadg_halo_pack.argtypes = [v, i, v, v, ctypes.c_size_t, v]
        L.wadg_vol_warps_candidates.argtypes = [v, i, ctypes.POINTER(ctypes.c_int)]
        L.wadg_ctx_set_vol_warps.argtypes = [v, i, i]
        L.wadg_ctx_get_vol_warps.argtypes = [v]
        L.wadg_vol_shapes.argtypes = [v, i, ctypes.POINTER(i), ctypes.POINTER(i)]
        L.wadg_ctx_set_vol_shape.argtypes = [v, i, i, i]
        L.wadg_ctx_get_vol_rows.argtypes = [v]
        L.wadg_check_state.argtypes = [v, i, v, v, ctypes.POINTER(i), ctypes.POINTER(i)]
        L.wadg_app_check_state.argtypes = [v, ctypes.POINTER(i), ctypes.POINTER(i)]
        L.wadg_app_set_check_every.argtypes = [v, i]
        L.wadg_kernel_shape.argtypes = [v, i, i, i, ctypes.POINTER(i), ctypes.POINTER(i)]
        L.wadg_app_autotune.argtypes = [v, d, i, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_float)]
        L.wadg_adjoint_create.argtypes = [v, i, i, ctypes.POINTER(ctypes.c_void_p)]
        L.wadg_adjoint_destroy.argtypes = [v]
        L.wadg_adjoint_forward.argtypes = [v, v, d, v]
        L.wadg_adjoint_reverse.argtypes = [v, v, v]
        L.wadg_adjoint_rhs.argtypes = [v, v, v]
        L.wadg_adjoint_rhs_vjp.argtypes = [v, v, v, v]
        L.wadg_geofacs.argtypes = [v, i] + [v] * 8
        L.wadg_match_faces_workspace.argtypes = [i, i]
        L.wadg_match_faces_workspace.restype = ctypes.c_size_t
        L.wadg_match_faces.argtypes = [v, i, v, v, v, i, v, ctypes.c_size_t, v, v]
        i64 = ctypes.c_int64
        L.wadg_mesh_read_gmsh.argtypes = [ctypes.c_char_p, i, ctypes.POINTER(ctypes.c_void_p)]
        L.wadg_mesh_sizes.argtypes = [v, ctypes.POINTER(i), ctypes.POINTER(i64), ctypes.POINTER(i64),
                                      ctypes.POINTER(i64)]
        L.wadg_mesh_get.argtypes = [v] * 5
        L.wadg_mesh_destroy.argtypes = [v]
        L.wadg_mesh_destroy.restype = None
        L.wadg_mesh_write_gmsh.argtypes = [ctypes.c_char_p, i, i64, v, i64, v]
        L.wadg_mesh_write_mfem.argtypes = [ctypes.c_char_p, i, i64, v, v]
        _lib = L
    return _lib


def check(code: int, what: str = ""):
    if code != 0:
        msg = lib().wadg_last_error().decode()
        raise WadgError(f"{what} failed ({code}): {msg}", code)


def params_for(ops: R.RefOps, gamma=1.4, tau=1.0, stream=None) -> Params:
    return Params(ops.dim, ops.N, ops.Nq, ops.Nfq, ops.Nfaces, gamma, tau, stream)


class Context:
    """Kernel-level API: each method is one OKL kernel launch on device
    pointers (ints)."""

    def __init__(self, ops: R.RefOps, gamma=1.4, tau=1.0, stream=None):
        self.ops = ops
        self.p = params_for(ops, gamma, tau, stream)
        h = ctypes.c_void_p()
        check(lib().wadg_ctx_create(ctypes.byref(self.p), ctypes.byref(h)), "wadg_ctx_create")
        self.h = h

    def close(self):
        if self.h:
            lib().wadg_ctx_destroy(self.h)
            self.h = None

    __del__ = close

    def set_stream(self, stream):
        check(lib().wadg_ctx_set_stream(self.h, stream), "set_stream")

    def vol(self, curved, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ, rhsQf):
        L = lib()
        if self.ops.dim == 3:
            fn = L.wadg_euler_vol_3d_curved if curved else L.wadg_euler_vol_3d
            check(fn(self.h, K, vgeo, vfgeo, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, None, VqLq, VfPq, None,
                     Qf, rhsQ, rhsQf), "vol")
        else:
            fn = L.wadg_euler_vol_2d_curved if curved else L.wadg_euler_vol_2d
            check(fn(self.h, K, vgeo, vfgeo, nrJ, nsJ, Drq, Dsq, VqLq, VfPq, None, Qf, rhsQ, rhsQf), "vol")

    def surf(self, K, fgeo, mapPq, VqLq, Qf, rhsQf, rhsQ):
        L = lib()
        fn = L.wadg_euler_surf_3d if self.ops.dim == 3 else L.wadg_euler_surf_2d
        check(fn(self.h, K, fgeo, mapPq, VqLq, Qf, rhsQf, rhsQ), "surf")

    def stage(self, curved, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq,
              VqPq, Jq, fa, fb, fdt, rhsQ_in, Qf_in, Q, resQ, rhsQ_out, Qf_out):
        """The fused stage (wadg_euler_stage_3d/_2d): vol + surf + update."""
        L = lib()
        if self.ops.dim == 3:
            check(L.wadg_euler_stage_3d(self.h, K, int(curved), vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ, ntJ,
                                        Drq, Dsq, Dtq, VqLq, VfPq, VqPq, Jq, fa, fb, fdt, rhsQ_in,
                                        Qf_in, Q, resQ, rhsQ_out, Qf_out), "stage")
        else:
            check(L.wadg_euler_stage_2d(self.h, K, int(curved), vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ,
                                        Drq, Dsq, VqLq, VfPq, VqPq, Jq, fa, fb, fdt, rhsQ_in, Qf_in,
                                        Q, resQ, rhsQ_out, Qf_out), "stage")

    def volsurf(self, curved, K, vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ, ntJ, Drq, Dsq, Dtq, VqLq, VfPq,
                Qf, rhsQ):
        """The volume + surface kernel (wadg_euler_volsurf_3d/_2d)."""
        L = lib()
        if self.ops.dim == 3:
            check(L.wadg_euler_volsurf_3d(self.h, K, int(curved), vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ, ntJ,
                                          Drq, Dsq, Dtq, VqLq, VfPq, Qf, rhsQ), "volsurf")
        else:
            check(L.wadg_euler_volsurf_2d(self.h, K, int(curved), vgeo, vfgeo, fgeo, mapPq, nrJ, nsJ,
                                          Drq, Dsq, VqLq, VfPq, Qf, rhsQ), "volsurf")

    def compute_aux(self, K, Jq, wq, Q, aux):
        """per-element kinetic energy (euler_3d_compute_aux)"""
        check(lib().wadg_euler_3d_compute_aux(self.h, K, Jq, wq, Q, aux), "compute_aux")

    def halo_pack(self, n, src, Qf, nQf, buf):
        """wadg_halo_pack: n send slots gathered from Qf (device pointers)"""
        check(lib().wadg_halo_pack(self.h, n, src, Qf, nQf, buf), "halo_pack")

    def entropy_rhs(self, curved, K, wq, Jq, VqPq, Q, rhs, out):
        """per-element entropy balance sum_i w v~ . rhs (wadg_entropy_rhs)"""
        check(lib().wadg_entropy_rhs(self.h, K, int(curved), wq, Jq, VqPq, Q, rhs, out),
              "entropy_rhs")

    def element_entropy(self, K, Jq, wq, Q, S):
        """per-element entropy integral sum_i w J (-rho s)"""
        check(lib().wadg_element_entropy(self.h, K, Jq, wq, Q, S), "element_entropy")

    def check_state(self, K, Q, work):
        """Failure detection (wadg_check_state): (status, bad nodes, first bad
        node index k*Nq + i or -1); status 0 or WADG_ERR_STATE (4)"""
        nbad, first = ctypes.c_int(), ctypes.c_int()
        r = lib().wadg_check_state(self.h, K, Q, work, ctypes.byref(nbad), ctypes.byref(first))
        if r not in (0, ERR_STATE):
            check(r, "check_state")
        return r, nbad.value, first.value

    KERNELS = {"vol": 0, "surf": 1, "update": 2, "stage": 3, "adj_pairs": 4, "volsurf": 5}

    def shape(self, kernel, curved, K):
        """(elements per batch, CTAs launched) of `kernel` for K elements
        (wadg_kernel_shape); persistent CTAs run several batches when
        K > elements * CTAs"""
        E, g = ctypes.c_int(), ctypes.c_int()
        check(lib().wadg_kernel_shape(self.h, self.KERNELS[kernel], int(curved), K, ctypes.byref(E),
                                      ctypes.byref(g)), "kernel_shape")
        return E.value, g.value

    def set_vol_warps(self, curved, warps):
        check(lib().wadg_ctx_set_vol_warps(self.h, int(curved), warps), "set_vol_warps")

    def set_vol_shape(self, curved, warps, rows):
        check(lib().wadg_ctx_set_vol_shape(self.h, int(curved), warps, rows), "set_vol_shape")

    def vol_shapes(self, curved):
        return vol_shapes(self.h, curved)

    def vol_warps_candidates(self, curved):
        c = (ctypes.c_int * 3)()
        n = lib().wadg_vol_warps_candidates(self.h, int(curved), c)
        if n < 1:
            raise WadgError(lib().wadg_last_error().decode())
        return [c[k] for k in range(n)]

    def update(self, curved, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ, resQ, Q, Qf):
        L = lib()
        d = self.ops.dim
        fn = getattr(L, f"wadg_euler_update_{d}d" + ("_curved" if curved else ""))
        check(fn(self.h, K, Jq, VqPq, VfPq, fa, fb, fdt, rhsQ, resQ, Q, Qf), "update")


MAX_VOL_SHAPES = 5  # WADG_MAX_VOL_SHAPES


def shape_label(warps, rows):
    return str(warps) if rows == 0 else f"{warps}w{rows}r"


def vol_shapes(ctx_handle, curved):
    """[(warps, rows per lane)] of every compiled shape of the volume kernel
    (wadg_vol_shapes; rows 0 = the default node-to-thread map)"""
    w = (ctypes.c_int * MAX_VOL_SHAPES)()
    r = (ctypes.c_int * MAX_VOL_SHAPES)()
    n = lib().wadg_vol_shapes(ctx_handle, int(curved), w, r)
    if n < 1:
        raise WadgError(lib().wadg_last_error().decode())
    return [(w[k], r[k]) for k in range(n)]


def _dp(a):
    return a.ctypes.data_as(_D) if a is not None else None


class App:
    """Library-owned device state and the LSRK driver."""

    def __init__(self, geo: M.Geometry, curved: bool, gamma=1.4, tau=1.0, stream=None):
        ops = geo.ops
        self.geo, self.ops, self.curved = geo, ops, bool(curved)
        self.K = geo.K
        self.p = params_for(ops, gamma, tau, stream)
        c = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        self._keep = dict(
            vgeo=c(geo.vgeo), vfgeo=c(geo.vfgeo), fgeo=c(geo.fgeo), Jq=c(geo.Jq),
            mapPq=np.ascontiguousarray(geo.mapPq, dtype=np.uint32),
            nrJ=c(ops.nrJ), nsJ=c(ops.nsJ), ntJ=c(ops.ntJ), Drq=c(ops.fortran("Drq")),
            Dsq=c(ops.fortran("Dsq")), Dtq=c(ops.fortran("Dtq")), VqLq=c(ops.fortran("VqLq")),
            VqPq=c(ops.fortran("VqPq")), VfPq=c(ops.fortran("VfPq")))
        k = self._keep
        hd = HostData(*([_dp(k[n]) for n in ("vgeo", "vfgeo", "fgeo", "Jq")] +
                        [k["mapPq"].ctypes.data_as(_U32)] +
                        [_dp(k[n]) for n in ("nrJ", "nsJ", "ntJ", "Drq", "Dsq", "Dtq", "VqLq", "VqPq", "VfPq")]))
        h = ctypes.c_void_p()
        self._destroy = lib().wadg_app_destroy  # kept for close() at interpreter exit
        check(lib().wadg_app_create(ctypes.byref(self.p), self.K, int(self.curved), ctypes.byref(hd),
                                    ctypes.byref(h)), "wadg_app_create")
        self.h = h
        Nf, Nq, NfqNf = ops.Nfields, ops.Nq, ops.NfqNf
        self.vshape, self.fshape = (self.K, Nf, Nq), (self.K, Nf, NfqNf)

    def close(self):
        # adjoints borrow the app's buffers: release them first
        for adj in list(getattr(self, "_dependents", ())):
            adj.close()
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    __del__ = close

    def set_state(self, Q=None, rhsQ=None, Qf=None, resQ=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (Q, rhsQ, Qf, resQ)]
        check(lib().wadg_app_set_state(self.h, *[None if a is None else a.ctypes.data for a in arrs]), "set_state")
        check(lib().wadg_app_sync(self.h), "sync")

    def get_state(self):
        Q, rhsQ, resQ = (np.empty(self.vshape) for _ in range(3))
        Qf = np.empty(self.fshape)
        check(lib().wadg_app_get_state(self.h, Q.ctypes.data, rhsQ.ctypes.data, Qf.ctypes.data,
                                       resQ.ctypes.data), "get_state")
        return dict(Q=Q, rhsQ=rhsQ, Qf=Qf, resQ=resQ)

    def state_ptrs(self):
        ps = [ctypes.c_void_p() for _ in range(5)]
        check(lib().wadg_app_state_ptrs(self.h, *[ctypes.byref(p) for p in ps]), "state_ptrs")
        return dict(zip(("Q", "rhsQ", "Qf", "resQ", "rhsQf"), [p.value for p in ps]))

    def rk_step(self, rka, rkb, dt):
        check(lib().wadg_rk_step(self.h, rka, rkb, dt), "rk_step")

    def rk_run(self, dt, nsteps, graph=True):
        check(lib().wadg_rk_run(self.h, dt, nsteps, int(graph)), "rk_run")

    def sync(self):
        check(lib().wadg_app_sync(self.h), "sync")

    def check_state(self):
        """(status, bad nodes, first bad node) of the app's Q (wadg_app_check_state)"""
        nbad, first = ctypes.c_int(), ctypes.c_int()
        r = lib().wadg_app_check_state(self.h, ctypes.byref(nbad), ctypes.byref(first))
        if r not in (0, ERR_STATE):
            check(r, "check_state")
        return r, nbad.value, first.value

    def set_check_every(self, nsteps):
        """wadg_rk_run checks the state every nsteps steps (0 = never) and
        raises WadgError (code WADG_ERR_STATE) at the first bad one"""
        check(lib().wadg_app_set_check_every(self.h, nsteps), "set_check_every")

    def solve_host(self, Q0, rhsQ0, Qf0, dt, nsteps, resQ0=None, out=None):
        """User-level solve with host buffers (H2D, nsteps, D2H of Q)."""
        Q = out if out is not None else np.empty(self.vshape)
        c = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64).ctypes.data
        check(lib().wadg_app_solve_host(self.h, c(Q0), c(rhsQ0), c(Qf0), c(resQ0), dt, nsteps,
                                        Q.ctypes.data, None, None, None), "solve_host")
        return Q

    def solve_host_q(self, Q0, dt, nsteps, out=None):
        """User-level solve from the conserved state alone (H2D of Q0, the
        stage-0 projection on the device, nsteps, D2H of Q)."""
        Q = out if out is not None else np.empty(self.vshape)
        Q0 = np.ascontiguousarray(Q0, dtype=np.float64)
        check(lib().wadg_app_solve_host_q(self.h, Q0.ctypes.data, dt, nsteps, Q.ctypes.data),
              "solve_host_q")
        return Q

    def project(self):
        """stage-0 traces and resQ = 0 from the app's Q, on the device"""
        check(lib().wadg_app_project(self.h), "project")

    def time_run(self, dt, nsteps, graph=True):
        ms = ctypes.c_float()
        check(lib().wadg_app_time_run(self.h, dt, nsteps, int(graph), ctypes.byref(ms)), "time_run")
        return ms.value

    STAGE_VARIANTS = {"three_kernels": 0, "fused": 1, "volsurf": 2}

    def set_fused(self, fused: bool):
        """fused stage kernel (one launch per stage) or, the default, the three
        reference kernels per stage"""
        check(lib().wadg_app_set_fused(self.h, int(bool(fused))), "set_fused")

    def set_stage_variant(self, name: str):
        """the stage the time loop launches: "three_kernels" (vol, surf,
        update), "fused" (one launch) or "volsurf" (volume + surface, then
        update)"""
        check(lib().wadg_app_set_fused(self.h, self.STAGE_VARIANTS[name]), "set_stage_variant")

    def time_volsurf(self, dt, nstages):
        """(volume + surface ms, update ms) summed over nstages stages"""
        ms = (ctypes.c_float * 2)()
        check(lib().wadg_app_time_volsurf(self.h, dt, nstages, ms), "time_volsurf")
        return ms[0], ms[1]

    def time_stage(self, dt, nstages):
        ms = ctypes.c_float()
        check(lib().wadg_app_time_stage(self.h, dt, nstages, ctypes.byref(ms)), "time_stage")
        return ms.value

    def time_kernels(self, dt, nstages):
        ms = (ctypes.c_float * 3)()
        check(lib().wadg_app_time_kernels(self.h, dt, nstages, ms), "time_kernels")
        return list(ms)

    def autotune(self, dt, nstages=10):
        """Pick the volume kernel's shape (warps per CTA and node-to-thread
        map) by timing each compiled one on this app (advances the state: set
        it afterwards).  Returns (the chosen shape, {shape: ms per launch});
        a shape is its warps per CTA ("12") or, for another map than the
        default, warps and rows per lane ("16w2r")."""
        w = ctypes.c_int()
        t = (ctypes.c_float * MAX_VOL_SHAPES)()
        check(lib().wadg_app_autotune(self.h, dt, nstages, ctypes.byref(w), t), "autotune")
        ctx = ctypes.c_void_p(lib().wadg_app_ctx(self.h))
        shapes = vol_shapes(ctx, self.curved)
        rows = lib().wadg_ctx_get_vol_rows(ctx)
        return shape_label(w.value, rows), {shape_label(a, b): float(t[k]) for k, (a, b) in enumerate(shapes)}

    def vol_shape(self):
        """(warps, rows) of the volume kernel shape the app's kernels use"""
        ctx = ctypes.c_void_p(lib().wadg_app_ctx(self.h))
        return lib().wadg_ctx_get_vol_warps(ctx), lib().wadg_ctx_get_vol_rows(ctx)

    def set_vol_shape(self, warps, rows):
        ctx = ctypes.c_void_p(lib().wadg_app_ctx(self.h))
        check(lib().wadg_ctx_set_vol_shape(ctx, int(self.curved), warps, rows), "set_vol_shape")


class Solver:
    """Mesh, operators, geometry, stage-0 state and the device driver: what
    the reference's main() sets up before rk_run (euler.c:3833-4215)."""

    def __init__(self, mesh: M.Mesh, N: int, curved: bool, ic="taylor_green", gamma=1.4, tau=1.0,
                 ic_args=None, stream=None):
        from .geometry_gpu import build_geometry_gpu  # (imports this module)

        self.mesh, self.N, self.curved, self.gamma = mesh, N, curved, gamma
        self.geo = build_geometry_gpu(mesh, N)  # geometric factors and maps on the device
        self.ic, self.ic_args = ic, dict(ic_args or {})
        U0 = IC.initial_state(self.geo, ic, gamma, **self.ic_args)
        self.Q0, self.rhsQ0, self.Qf0, self.resQ0 = IC.stage0(self.geo, U0, gamma)
        self.app = App(self.geo, curved, gamma, tau, stream)
        self.reset()

    @property
    def ops(self):
        return self.geo.ops

    @property
    def dofs(self):
        """DOF per field = K * Np (the throughput unit)."""
        return self.geo.K * self.ops.Np

    def reset(self):
        self.app.set_state(self.Q0, self.rhsQ0, self.Qf0, self.resQ0)

    def time_step(self, CFL, FinalTime=None, nsteps=None):
        return IC.time_step(self.geo, CFL, self.N, FinalTime, nsteps)
