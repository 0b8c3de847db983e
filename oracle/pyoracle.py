"""Test infrastructure only: ctypes bindings to the two CPU checkers.

* ``Port``      — the C restatement oracle/wadg_ref.c (always available).
* ``Reference`` — the reference's own OKL kernels compiled from their sources
                  into oracle/_ref/ (available where oracle/_ref was built).

Both expose the same three calls with the reference's argument meaning:
    vol(geo, Qf, rhsQ, rhsQf)      rhsQ in: u(VqPq v), out: volume RHS
    surf(geo, Qf, rhsQf, rhsQ)     rhsQ += lift of the surface flux (over the
                                   elements of rhsQ; Qf may hold more)
    update(geo, fa, fb, dt, rhsQ, resQ, Q, Qf)
All arrays are float64 numpy arrays in the kernel layouts; they are updated in
place.  ``stage`` / ``step`` chain them like rk_step / rk_run (euler.c:3610-3699).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_P = ctypes.POINTER(ctypes.c_double)
_U = ctypes.POINTER(ctypes.c_uint32)


def _p(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_P)


def _u(a):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_U)


class _Dims(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("Nq", ctypes.c_int), ("Nfq", ctypes.c_int),
                ("Nfaces", ctypes.c_int), ("gamma", ctypes.c_double), ("tau", ctypes.c_double)]


class _Base:
    def __init__(self, ops, curved, gamma=1.4, tau=1.0):
        self.ops, self.curved, self.gamma, self.tau = ops, bool(curved), gamma, tau
        f = lambda n: np.ascontiguousarray(ops.fortran(n))
        self.Drq, self.Dsq, self.Dtq = f("Drq"), f("Dsq"), f("Dtq")
        self.VqLq, self.VfPq, self.VqPq = f("VqLq"), f("VfPq"), f("VqPq")
        self.nrJ, self.nsJ, self.ntJ = (np.ascontiguousarray(getattr(ops, n)) for n in ("nrJ", "nsJ", "ntJ"))
        self.Drstq = np.concatenate([self.Drq, self.Dsq, self.Dtq])

    def stage(self, geo, a, b, dt, st):
        """One LSRK stage: vol, surf, update (euler.c:3610-3625)."""
        Q, rhsQ, Qf, resQ, rhsQf = st["Q"], st["rhsQ"], st["Qf"], st["resQ"], st["rhsQf"]
        self.vol(geo, Qf, rhsQ, rhsQf)
        self.surf(geo, Qf, rhsQf, rhsQ)
        self.update(geo, a, b, dt, rhsQ, resQ, Q, Qf)

    def step(self, geo, dt, st):
        from scratch_wadge_b200.ic import RK4A, RK4B
        for s in range(5):
            self.stage(geo, RK4A[s], RK4B[s], dt, st)

    def project(self, geo, Q):
        """The projected traces (u~, uf~) of Q: the update kernel with a zero
        RHS and zero coefficients leaves Q and writes U(VqPq v~), U(VfPq v~)."""
        K, Nf, NF = Q.shape[0], Q.shape[1], self.ops.NfqNf
        rhsQ, resQ = np.zeros_like(Q), np.zeros_like(Q)
        Qc, Qf = np.ascontiguousarray(Q, dtype=np.float64).copy(), np.zeros((K, Nf, NF))
        self.update(geo, 0.0, 0.0, 0.0, rhsQ, resQ, Qc, Qf)
        return rhsQ, Qf

    def rhs(self, geo, Q):
        """R(Q) = Minv rhs(u~(Q), uf~(Q)): the update's r for the state Q
        (res = 0 * res + 1 * r)."""
        rhsQ, Qf = self.project(geo, Q)
        rhsQf = np.zeros_like(Qf)
        self.vol(geo, Qf, rhsQ, rhsQf)
        self.surf(geo, Qf, rhsQf, rhsQ)
        resQ, Qc = np.zeros_like(Q), np.ascontiguousarray(Q, dtype=np.float64).copy()
        self.update(geo, 0.0, 0.0, 1.0, rhsQ, resQ, Qc, Qf)
        return resQ

    def run(self, geo, Q0, dt, nsteps):
        """nsteps LSRK-45 steps from Q0, the traces projected from Q0."""
        rhsQ, Qf = self.project(geo, Q0)
        st = dict(Q=np.ascontiguousarray(Q0, dtype=np.float64).copy(), rhsQ=rhsQ, Qf=Qf,
                  resQ=np.zeros_like(rhsQ), rhsQf=np.zeros_like(Qf))
        for _ in range(nsteps):
            self.step(geo, dt, st)
        return st["Q"]


class Port(_Base):
    """oracle/wadg_ref.c (restatement)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            from . import build
            cls._lib = ctypes.CDLL(build.build_port())
        return cls._lib

    def __init__(self, ops, curved, gamma=1.4, tau=1.0):
        super().__init__(ops, curved, gamma, tau)
        self.d = _Dims(ops.dim, ops.Nq, ops.Nfq, ops.Nfaces, gamma, tau)
        self.L = self.lib()
        self.L.wadg_ref_logmean.restype = ctypes.c_double
        self.L.wadg_ref_logmean.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]

    def vol(self, geo, Qf, rhsQ, rhsQf):
        K = Qf.shape[0]
        if self.ops.dim == 3:
            self.L.wadg_ref_vol_3d(ctypes.byref(self.d), int(self.curved), K, _p(geo.vgeo), _p(geo.vfgeo),
                                   _p(self.nrJ), _p(self.nsJ), _p(self.ntJ), _p(self.Drq), _p(self.Dsq),
                                   _p(self.Dtq), _p(self.VqLq), _p(self.VfPq), _p(Qf), _p(rhsQ), _p(rhsQf))
        else:
            self.L.wadg_ref_vol_2d(ctypes.byref(self.d), int(self.curved), K, _p(geo.vgeo), _p(geo.vfgeo),
                                   _p(self.nrJ), _p(self.nsJ), _p(self.Drq), _p(self.Dsq),
                                   _p(self.VqLq), _p(self.VfPq), _p(Qf), _p(rhsQ), _p(rhsQf))

    def surf(self, geo, Qf, rhsQf, rhsQ):
        K = rhsQ.shape[0]  # Qf may be longer: neighbour traces are gathered from all of it
        fn = self.L.wadg_ref_surf_3d if self.ops.dim == 3 else self.L.wadg_ref_surf_2d
        fn(ctypes.byref(self.d), K, _p(geo.fgeo), _u(geo.mapPq), _p(self.VqLq), _p(Qf), _p(rhsQf), _p(rhsQ))

    def update(self, geo, fa, fb, fdt, rhsQ, resQ, Q, Qf):
        K = Q.shape[0]
        fn = self.L.wadg_ref_update_3d if self.ops.dim == 3 else self.L.wadg_ref_update_2d
        fn(ctypes.byref(self.d), int(self.curved), K, _p(geo.Jq), _p(self.VqPq), _p(self.VfPq),
           ctypes.c_double(fa), ctypes.c_double(fb), ctypes.c_double(fdt),
           _p(rhsQ), _p(resQ), _p(Q), _p(Qf))

    def logmean(self, dim, a, b):
        return self.L.wadg_ref_logmean(dim, a, b)


def reference_available(dim=3, N=3):
    return os.path.exists(_ref_path("Euler3Daffine" if dim == 3 else "Euler2D", N))


def _ref_path(stem, N):
    return os.path.join(HERE, "_ref", f"libokl_{stem}_N{N}.so")


class Reference(_Base):
    """The reference's OKL kernels compiled from their own sources.

    3D affine -> okl/Euler3Daffine.okl (euler_vol_3d, euler_surf_3d,
    euler_update_3d); 3D curved -> okl/Euler3D.okl (euler_vol_3d_curved,
    euler_surf_3d, euler_update_3d_curved); 2D -> okl/Euler2D.okl
    (euler_vol_2d[_curved], euler_surf_2d, euler_update_2d[_curved])."""

    def __init__(self, ops, curved, gamma=1.4, tau=1.0):
        super().__init__(ops, curved, gamma, tau)
        if abs(gamma - 1.4) > 0 or abs(tau - 1.0) > 0:
            raise ValueError("oracle/_ref is compiled for gamma=1.4, tau=1")
        stem = ("Euler3D" if curved else "Euler3Daffine") if ops.dim == 3 else "Euler2D"
        path = _ref_path(stem, ops.N)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.L = ctypes.CDLL(path)
        d = ops.dim
        self._vol = getattr(self.L, f"euler_vol_{d}d" + ("_curved" if curved else ""))
        self._surf = getattr(self.L, f"euler_surf_{d}d")
        self._upd = getattr(self.L, f"euler_update_{d}d" + ("_curved" if curved else ""))
        self._upd.argtypes = [ctypes.c_int, _P, _P, _P, ctypes.c_double, ctypes.c_double,
                              ctypes.c_double, _P, _P, _P, _P]

    def vol(self, geo, Qf, rhsQ, rhsQf):
        K = Qf.shape[0]
        Qdummy = rhsQ  # the Q argument is unused by every volume kernel
        if self.ops.dim == 3:
            self._vol(K, _p(geo.vgeo), _p(geo.vfgeo), _p(self.nrJ), _p(self.nsJ), _p(self.ntJ),
                      _p(self.Drq), _p(self.Dsq), _p(self.Dtq), _p(self.Drstq), _p(self.VqLq),
                      _p(self.VfPq), _p(Qdummy), _p(Qf), _p(rhsQ), _p(rhsQf))
        else:
            self._vol(K, _p(geo.vgeo), _p(geo.vfgeo), _p(self.nrJ), _p(self.nsJ),
                      _p(self.Drq), _p(self.Dsq), _p(self.VqLq), _p(self.VfPq),
                      _p(Qdummy), _p(Qf), _p(rhsQ), _p(rhsQf))

    def surf(self, geo, Qf, rhsQf, rhsQ):
        K = rhsQ.shape[0]  # Qf may be longer: neighbour traces are gathered from all of it
        self._surf(K, _p(geo.fgeo), _u(geo.mapPq), _p(self.VqLq), _p(Qf), _p(rhsQf), _p(rhsQ))

    def update(self, geo, fa, fb, fdt, rhsQ, resQ, Q, Qf):
        K = Q.shape[0]
        self._upd(K, _p(geo.Jq), _p(self.VqPq), _p(self.VfPq), fa, fb, fdt,
                  _p(rhsQ), _p(resQ), _p(Q), _p(Qf))

    def compute_aux(self, geo, Q):
        """euler_3d_compute_aux (Euler3D.okl:3888): per-element kinetic
        energy; only the Euler3D library (3D, curved) has it."""
        if not hasattr(self.L, "euler_3d_compute_aux"):
            raise AttributeError("euler_3d_compute_aux is in the Euler3D (curved 3D) library")
        K = Q.shape[0]
        aux = np.zeros(K)
        wq = np.ascontiguousarray(self.ops.wq, dtype=np.float64)
        self.L.euler_3d_compute_aux(K, _p(geo.Jq), _p(wq), _p(np.ascontiguousarray(Q)), _p(aux))
        return aux
