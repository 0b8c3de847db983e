"""Parity of the CUDA path (through the C ABI) with the reference.

Kernel by kernel and over full LSRK-45 steps, against
  * the golden vectors made by the reference's own kernels (tests/golden/), and
  * the oracle (oracle/wadg_ref.c) on seeded perturbed states,
at 1e-12 relative in the max norm (FP64).  Also: free-stream preservation,
discrete entropy conservation with tau = 0 (3D), entropy dissipation (2D, whose
surface kernel fixes tau = 1), and the host-buffer solve."""

import ctypes

import numpy as np
import pytest

from oracle import pyoracle as O
from scratch_wadge_b200 import build as B
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import ic as IC
from scratch_wadge_b200 import mesh as M
from tests.helpers import RTOL, Case, golden_names, perturbed, rel

pytestmark = pytest.mark.gpu


class Dev:
    """Device copies (torch) of a golden case's inputs + a kernel context."""

    def __init__(self, torch, geo, curved, gamma=1.4, tau=1.0):
        self.torch = torch
        self.geo, self.curved, self.ops = geo, curved, geo.ops
        ops = geo.ops
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
        self.g = dict(vgeo=t(geo.vgeo), vfgeo=t(geo.vfgeo), fgeo=t(geo.fgeo), Jq=t(geo.Jq),
                      mapPq=torch.from_numpy(np.ascontiguousarray(geo.mapPq, dtype=np.uint32).view(np.int32)).cuda(),
                      nrJ=t(ops.nrJ), nsJ=t(ops.nsJ), ntJ=t(ops.ntJ), Drq=t(ops.fortran("Drq")),
                      Dsq=t(ops.fortran("Dsq")), Dtq=t(ops.fortran("Dtq")), VqLq=t(ops.fortran("VqLq")),
                      VqPq=t(ops.fortran("VqPq")), VfPq=t(ops.fortran("VfPq")))
        self.ctx = capi.Context(ops, gamma, tau, torch.cuda.current_stream().cuda_stream)

    def put(self, st):
        t = self.torch
        return {k: t.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in st.items()}

    @staticmethod
    def get(d):
        return {k: v.cpu().numpy() for k, v in d.items()}

    def vol(self, s):
        g = self.g
        self.ctx.vol(self.curved, self.geo.K, g["vgeo"].data_ptr(), g["vfgeo"].data_ptr(),
                     g["nrJ"].data_ptr(), g["nsJ"].data_ptr(), g["ntJ"].data_ptr(), g["Drq"].data_ptr(),
                     g["Dsq"].data_ptr(), g["Dtq"].data_ptr(), g["VqLq"].data_ptr(), g["VfPq"].data_ptr(),
                     s["Qf"].data_ptr(), s["rhsQ"].data_ptr(), s["rhsQf"].data_ptr())

    def surf(self, s):
        g = self.g
        self.ctx.surf(self.geo.K, g["fgeo"].data_ptr(), g["mapPq"].data_ptr(), g["VqLq"].data_ptr(),
                      s["Qf"].data_ptr(), s["rhsQf"].data_ptr(), s["rhsQ"].data_ptr())

    def update(self, s, a, b, dt):
        g = self.g
        self.ctx.update(self.curved, self.geo.K, g["Jq"].data_ptr(), g["VqPq"].data_ptr(),
                        g["VfPq"].data_ptr(), a, b, dt, s["rhsQ"].data_ptr(), s["resQ"].data_ptr(),
                        s["Q"].data_ptr(), s["Qf"].data_ptr())

    def stage(self, s, out, a, b, dt):
        g = self.g
        self.ctx.stage(self.curved, self.geo.K, g["vgeo"].data_ptr(), g["vfgeo"].data_ptr(),
                       g["fgeo"].data_ptr(), g["mapPq"].data_ptr(), g["nrJ"].data_ptr(),
                       g["nsJ"].data_ptr(), g["ntJ"].data_ptr(), g["Drq"].data_ptr(), g["Dsq"].data_ptr(),
                       g["Dtq"].data_ptr(), g["VqLq"].data_ptr(), g["VfPq"].data_ptr(),
                       g["VqPq"].data_ptr(), g["Jq"].data_ptr(), a, b, dt, s["rhsQ"].data_ptr(),
                       s["Qf"].data_ptr(), s["Q"].data_ptr(), s["resQ"].data_ptr(),
                       out["rhsQ"].data_ptr(), out["Qf"].data_ptr())

    def volsurf(self, s):
        g = self.g
        self.ctx.volsurf(self.curved, self.geo.K, g["vgeo"].data_ptr(), g["vfgeo"].data_ptr(),
                         g["fgeo"].data_ptr(), g["mapPq"].data_ptr(), g["nrJ"].data_ptr(),
                         g["nsJ"].data_ptr(), g["ntJ"].data_ptr(), g["Drq"].data_ptr(), g["Dsq"].data_ptr(),
                         g["Dtq"].data_ptr(), g["VqLq"].data_ptr(), g["VfPq"].data_ptr(),
                         s["Qf"].data_ptr(), s["rhsQ"].data_ptr())

    def sync(self):
        self.torch.cuda.synchronize()


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build()


@pytest.mark.parametrize("name", golden_names())
def test_kernels_match_reference_golden(cuda, name):
    c = Case(name)
    d = Dev(cuda, c.geo, c.curved)
    s = d.put(c.state())
    d.vol(s)
    d.sync()
    h = d.get(s)
    assert rel(h["rhsQ"], c.z["vol_rhsQ"]) < RTOL
    assert rel(h["rhsQf"], c.z["vol_rhsQf"]) < RTOL
    d.surf(s)
    d.sync()
    assert rel(s["rhsQ"].cpu().numpy(), c.z["surf_rhsQ"]) < RTOL
    d.update(s, IC.RK4A[1], IC.RK4B[1], c.dt)
    d.sync()
    h = d.get(s)
    for k in ("Q", "rhsQ", "Qf", "resQ"):
        assert rel(h[k], c.z["upd_" + k]) < RTOL, (k, rel(h[k], c.z["upd_" + k]))


@pytest.mark.parametrize("name", golden_names())
def test_stage_matches_oracle_perturbed(cuda, name):
    c = Case(name)
    d = Dev(cuda, c.geo, c.curved)
    P = O.Port(c.ops, c.curved)
    for seed in (11, 12):
        s0 = perturbed(c.state(), seed)
        s0["resQ"] = 1e-3 * perturbed({"x": c.z["in_Q"]}, seed + 100)["x"]
        a = {k: v.copy() for k, v in s0.items()}
        P.stage(c.geo, IC.RK4A[3], IC.RK4B[3], 3e-3, a)
        s = d.put(s0)
        d.vol(s)
        d.surf(s)
        d.update(s, IC.RK4A[3], IC.RK4B[3], 3e-3)
        d.sync()
        h = d.get(s)
        for k in ("Q", "rhsQ", "Qf", "resQ"):
            assert rel(h[k], a[k]) < RTOL, (k, rel(h[k], a[k]))


@pytest.mark.parametrize("name", golden_names())
def test_fused_stage_matches_reference_golden(cuda, name):
    """wadg_euler_stage_*: one launch = vol + surf + update of the reference."""
    c = Case(name)
    d = Dev(cuda, c.geo, c.curved)
    s = d.put(c.state())
    out = {"rhsQ": cuda.empty_like(s["rhsQ"]), "Qf": cuda.empty_like(s["Qf"])}
    d.stage(s, out, IC.RK4A[1], IC.RK4B[1], c.dt)
    d.sync()
    got = dict(Q=s["Q"].cpu().numpy(), resQ=s["resQ"].cpu().numpy(),
               rhsQ=out["rhsQ"].cpu().numpy(), Qf=out["Qf"].cpu().numpy())
    for k in ("Q", "rhsQ", "Qf", "resQ"):
        assert rel(got[k], c.z["upd_" + k]) < RTOL, (k, rel(got[k], c.z["upd_" + k]))
    # the inputs are untouched
    assert np.array_equal(s["rhsQ"].cpu().numpy(), c.z["in_rhsQ"])


@pytest.mark.parametrize("name", golden_names())
def test_volsurf_matches_reference_golden(cuda, name):
    """wadg_euler_volsurf_*: the volume and surface kernels in one launch
    leave the reference's right-hand side after its surface kernel"""
    c = Case(name)
    d = Dev(cuda, c.geo, c.curved)
    s = d.put(c.state())
    d.volsurf(s)
    d.sync()
    assert rel(s["rhsQ"].cpu().numpy(), c.z["surf_rhsQ"]) < RTOL
    assert np.array_equal(s["Qf"].cpu().numpy(), c.z["in_Qf"])  # traces only read


@pytest.mark.parametrize("name", golden_names())
def test_app_volsurf_variant_matches_reference_step(cuda, name):
    c = Case(name)
    app = capi.App(c.geo, c.curved)
    app.set_stage_variant("volsurf")
    st = c.state()
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    app.rk_run(c.dt, 1, graph=True)
    assert rel(app.get_state()["Q"], c.z["step_Q"]) < RTOL


def test_fused_stage_rejects_aliasing(cuda):
    c = Case("tg3d_affine_N3")
    d = Dev(cuda, c.geo, c.curved)
    s = d.put(c.state())
    with pytest.raises(capi.WadgError):
        d.stage(s, {"rhsQ": s["rhsQ"], "Qf": s["Qf"]}, IC.RK4A[1], IC.RK4B[1], c.dt)


@pytest.mark.parametrize("name", ["tg3d_affine_N3", "dw3d_curved_N4", "vortex2d_curved_N3"])
def test_fused_stage_state_in_place(cuda, name):
    """the stage's state buffer may be both input and output (each element's
    own state is read before its RHS and next state are written); only the
    traces need a second buffer"""
    c = Case(name)
    d = Dev(cuda, c.geo, c.curved)
    s = d.put(c.state())
    out = {"rhsQ": s["rhsQ"], "Qf": cuda.empty_like(s["Qf"])}
    d.stage(s, out, IC.RK4A[1], IC.RK4B[1], c.dt)
    d.sync()
    assert rel(s["rhsQ"].cpu().numpy(), c.z["upd_rhsQ"]) < RTOL
    assert rel(out["Qf"].cpu().numpy(), c.z["upd_Qf"]) < RTOL
    assert rel(s["Q"].cpu().numpy(), c.z["upd_Q"]) < RTOL


@pytest.mark.parametrize("name", golden_names())
def test_fused_and_three_kernel_paths_agree(cuda, name):
    c = Case(name)
    outs = []
    for fused in (True, False):
        app = capi.App(c.geo, c.curved)
        app.set_fused(fused)
        st = c.state()
        app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
        app.rk_run(c.dt, 3, graph=True)
        outs.append(app.get_state())
    for k in ("Q", "rhsQ", "Qf"):
        assert rel(outs[0][k], outs[1][k]) < RTOL, k


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("graph", [True, False])
def test_app_time_step_matches_reference(cuda, name, graph):
    c = Case(name)
    app = capi.App(c.geo, c.curved)
    st = c.state()
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    app.rk_run(c.dt, 1, graph=graph)
    out = app.get_state()
    assert rel(out["Q"], c.z["step_Q"]) < RTOL


@pytest.mark.parametrize("name", ["tg3d_affine_N3", "dw3d_curved_N4", "vortex2d_curved_N3"])
def test_many_steps_match_oracle(cuda, name):
    c = Case(name)
    app = capi.App(c.geo, c.curved)
    st = c.state()
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    app.rk_run(c.dt, 10, graph=True)
    out = app.get_state()
    P = O.Port(c.ops, c.curved)
    for _ in range(10):
        P.step(c.geo, c.dt, st)
    for k in ("Q", "rhsQ", "Qf"):
        assert rel(out[k], st[k]) < RTOL, (k, rel(out[k], st[k]))
    # resQ is the LSRK register (a dt-scaled RHS, ~1e-5 of the state here): its
    # differences are rounding of the RHS, measured on the scale of the state
    # it is added to
    assert np.abs(out["resQ"] - st["resQ"]).max() < RTOL * np.abs(st["Q"]).max()
    assert np.isfinite(out["Q"]).all()


@pytest.mark.parametrize("dim,N,curved", [(3, 3, False), (3, 4, True), (2, 3, True), (2, 2, False)])
def test_free_stream(cuda, dim, N, curved):
    m = M.periodic_cube(2, warp=M.warp_cube(0.05) if curved else None) if dim == 3 else M.periodic_square(4, 4)
    sol = capi.Solver(m, N, curved, ic="constant")
    sol.app.rk_run(1e-3, 3)
    out = sol.app.get_state()
    assert rel(out["Q"], sol.Q0) < 1e-12


def _entropy_rhs(cuda, m, N, curved, kind, tau):
    geo = M.build_geometry(m, N)
    Q, rhsQ, Qf, resQ = IC.stage0(geo, IC.initial_state(geo, kind))
    d = Dev(cuda, geo, curved, tau=tau)
    s = d.put(dict(Q=Q, rhsQ=rhsQ.copy(), Qf=Qf, resQ=resQ, rhsQf=np.zeros_like(Qf)))
    d.vol(s)
    d.surf(s)
    d.sync()
    r = s["rhsQ"].cpu().numpy().transpose(1, 2, 0)
    V = IC.VU(rhsQ.transpose(1, 2, 0))
    w = geo.ops.wq[None, :, None]
    return float(np.sum(w * V * r)), float(np.sum(np.abs(w * V * r)))


@pytest.mark.parametrize("N,curved", [(3, False), (3, True), (4, True)])
def test_entropy_conservation_3d(cuda, N, curved):
    """tau = 0: the flux-differencing RHS conserves entropy to round-off
    (sum_i w_i v~_i . rhs_i = 0 on a periodic mesh)."""
    m = M.periodic_cube(2, warp=M.warp_cube(0.05) if curved else None)
    S, A = _entropy_rhs(cuda, m, N, curved, "taylor_green" if not curved else "density_wave", 0.0)
    assert abs(S) < 1e-12 * A


def test_entropy_dissipation_2d(cuda):
    """2D: the reference's surface kernel fixes tau = 1, so entropy decays:
    dS/dt = -2 sum w v~.rhs <= 0."""
    S, A = _entropy_rhs(cuda, M.periodic_square(4, 4), 3, True, "vortex", 1.0)
    assert S > 0


@pytest.mark.parametrize("name", ["tg3d_affine_N3", "tg3d_affine_N2", "vortex2d_affine_N2",
                                  "dw3d_curved_N3", "dw3d_curved_N4", "vortex2d_curved_N3"])
def test_device_projection_matches_stage0(cuda, name):
    """wadg_app_project = the reference's stage-0 builder, which projects with
    VqPq alone on curved meshes too (euler.c:3958-4133)."""
    c = Case(name)
    app = capi.App(c.geo, c.curved)
    st = c.state()
    app.set_state(st["Q"], st["rhsQ"] * 0 + 1.0, st["Qf"] * 0 + 1.0, st["resQ"] + 1.0)
    app.project()
    out = app.get_state()
    assert rel(out["rhsQ"], st["rhsQ"]) < RTOL and rel(out["Qf"], st["Qf"]) < RTOL
    assert np.array_equal(out["Q"], st["Q"]) and not out["resQ"].any()


@pytest.mark.parametrize("name", ["tg3d_affine_N3", "vortex2d_affine_N2", "dw3d_curved_N4",
                                  "vortex2d_curved_N3"])
def test_solve_from_q_equals_solve_from_stage0_state(cuda, name):
    c = Case(name)
    app = capi.App(c.geo, c.curved)
    st = c.state()
    a = app.solve_host(st["Q"], st["rhsQ"], st["Qf"], c.dt, 4)
    b = app.solve_host_q(st["Q"], c.dt, 4)
    assert rel(b, a) < RTOL


def test_solve_host_equals_device_run(cuda):
    c = Case("tg3d_affine_N3")
    app = capi.App(c.geo, c.curved)
    st = c.state()
    Q = app.solve_host(st["Q"], st["rhsQ"], st["Qf"], c.dt, 4, resQ0=st["resQ"])
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    app.rk_run(c.dt, 4, graph=False)
    assert np.array_equal(Q, app.get_state()["Q"])
