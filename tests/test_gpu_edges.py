"""Edge cases of the CUDA path against the oracle, at the parity tolerance:
ragged element counts (K not a multiple of any batch size), every compiled
degree N=1..4 in 2D and 3D on affine and warped meshes, and boundary points
(mapPq(j) = j, the reference's idM == idP faces) in the forward step and in
the adjoint's RHS vector-Jacobian product."""

import numpy as np
import pytest
import torch

from oracle.pyoracle import Port
from oracle.torch_rhs import TorchRHS
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import ic as IC
from scratch_wadge_b200 import mesh as M
from scratch_wadge_b200.adjoint import Adjoint
from tests.helpers import RTOL, perturbed, rel

pytestmark = pytest.mark.gpu


def _setup(dim, N, curved, n):
    if dim == 2:
        mesh = M.periodic_square(n, n + 2)
        kind = "vortex"
    else:
        mesh = M.periodic_cube(n, warp=M.warp_cube(0.05) if curved else None)
        kind = "density_wave" if curved else "taylor_green"
    geo = M.build_geometry(mesh, N)
    st = dict(zip(("Q", "rhsQ", "Qf", "resQ"), IC.stage0(geo, IC.initial_state(geo, kind))))
    dt = IC.time_step(geo, 0.5, N, nsteps=1, wave_speed=IC.max_wave_speed(st["Q"]))[0]
    return geo, st, dt


def _step_both(geo, st, dt, curved):
    app = capi.App(geo, curved)
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    app.rk_run(dt, 1, graph=False)
    out = app.get_state()
    ref = {k: np.ascontiguousarray(v).copy() for k, v in st.items()}
    ref["rhsQf"] = np.zeros_like(ref["Qf"])
    Port(geo.ops, curved).step(geo, dt, ref)
    return out, ref


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("N", [1, 2, 3, 4])
@pytest.mark.parametrize("curved", [False, True])
def test_ragged_meshes_all_degrees(cuda, dim, N, curved):
    n = 3 if dim == 3 else 5  # K = 162 (3D) or 70 (2D): no batch size divides it
    geo, st, dt = _setup(dim, N, curved, n)
    out, ref = _step_both(geo, st, dt, curved)
    for k in ("Q", "rhsQ", "Qf"):
        assert np.isfinite(out[k]).all()
        assert rel(out[k], ref[k]) < RTOL, (k, rel(out[k], ref[k]))


def _with_boundary(geo):
    """the periodic wrap in x replaced by boundary points: face points whose
    neighbour lies across the period map to themselves (both sides)"""
    NF, Nf = geo.ops.NfqNf, geo.ops.dim + 2
    m = np.asarray(geo.mapPq, dtype=np.int64).reshape(geo.K, NF).copy()
    blk = NF * Nf
    k_idx = np.repeat(np.arange(geo.K), NF).reshape(geo.K, NF)
    eP, jP = m // blk, m % blk
    xs = np.asarray(geo.xyzf)[:, 0, :]  # x of the face points, [K][NF]
    wrap = np.abs(xs - xs[eP, jP]) > 1.0  # partners across the period
    own = np.arange(NF)[None, :] + k_idx * blk
    m[wrap] = own[wrap]
    assert wrap.any()
    return M.Geometry(geo.ops, geo.K, geo.vgeo, geo.vfgeo, geo.fgeo, geo.Jq,
                      m.reshape(-1).astype(np.uint32), geo.xyzq, geo.xyzf)


@pytest.mark.parametrize("dim,N,curved", [(3, 3, False), (3, 2, True), (2, 3, False)])
def test_boundary_points_forward_and_adjoint(cuda, dim, N, curved):
    geo, st, dt = _setup(dim, N, curved, 2 if dim == 3 else 4)
    geo = _with_boundary(geo)
    out, ref = _step_both(geo, st, dt, curved)
    for k in ("Q", "rhsQ", "Qf"):
        assert rel(out[k], ref[k]) < RTOL, k
    # the adjoint accepts self-paired faces (mapPq(mapPq(j)) = j holds)
    Q = perturbed({"Q": st["Q"]}, 9, 1e-2)["Q"]
    w = np.random.default_rng(1).standard_normal(Q.shape)
    app = capi.App(geo, curved)
    adj = Adjoint(app, 1, 1)
    g = adj.rhs_vjp(torch.from_numpy(Q).cuda(), torch.from_numpy(w).cuda()).cpu().numpy()
    T = TorchRHS(geo, curved)
    _, vjp = torch.func.vjp(T.R, torch.from_numpy(Q))
    assert rel(g, vjp(torch.from_numpy(w))[0].numpy()) < 1e-10


@pytest.mark.parametrize("dim,n", [(2, 1), (3, 1), (2, 2)])
@pytest.mark.parametrize("variant", ["three_kernels", "volsurf", "fused"])
def test_meshes_smaller_than_one_group(cuda, dim, n, variant):
    """K below one element group (2D: 2 or 8 triangles against 8 elements a
    group; 3D: 6 tets against 4): the groups past the end leave at once, the
    partial group computes on the clamped last element, and every stage
    variant still takes the reference's step"""
    if dim == 2:
        mesh, kind, curved = M.periodic_square(n, n), "vortex", False
    else:
        mesh, kind, curved = M.periodic_cube(n), "taylor_green", False
    geo = M.build_geometry(mesh, 3)
    st = dict(zip(("Q", "rhsQ", "Qf", "resQ"), IC.stage0(geo, IC.initial_state(geo, kind))))
    st = perturbed(st, 11)
    dt = IC.time_step(geo, 0.1, 3, nsteps=1, wave_speed=IC.max_wave_speed(st["Q"]))[0]
    app = capi.App(geo, curved)
    app.set_stage_variant(variant)
    app.set_state(st["Q"], st["rhsQ"], st["Qf"], st["resQ"])
    app.rk_run(dt, 1, graph=False)
    out = app.get_state()
    ref = {k: np.ascontiguousarray(v).copy() for k, v in st.items()}
    ref["rhsQf"] = np.zeros_like(ref["Qf"])
    Port(geo.ops, curved).step(geo, dt, ref)
    for k in ("Q", "rhsQ", "Qf"):
        assert np.isfinite(out[k]).all()
        assert rel(out[k], ref[k]) < RTOL, (k, rel(out[k], ref[k]))
