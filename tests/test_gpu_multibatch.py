"""The persistent kernels over several batches per CTA, against the oracle.

The volume, volume + surface, update and fused stage kernels (and the
adjoint's pair VJP kernel) launch at most as many CTAs as are resident at once; CTA b then takes
batches b, b + grid, b + 2 grid, ...  Small meshes never leave the first
batch, so each case here takes the kernel's own launch shape
(wadg_kernel_shape) and runs it on K = 2 * grid * E + r elements with
0 < r < E: CTA 0 runs three batches, the last one partial (its elements past
the end replicate element K-1 and are not stored).  That exercises the
prefetch of the next batch's traces, the per-group barriers across batches and
the partial-batch clamp.  Every compiled degree, affine and curved, 2D and 3D,
and every compiled CTA shape of the volume kernel, compared with the
reference's own kernels (oracle/_ref; the C restatement where it is absent)
at 1e-12.  The kernels run over the first K elements of larger arrays, so the
elements past K must come back untouched."""

import math

import numpy as np
import pytest
import torch

from oracle import pyoracle as O
from oracle.torch_rhs import TorchRHS
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import ic as IC
from scratch_wadge_b200 import mesh as M
from scratch_wadge_b200 import refops as R
from scratch_wadge_b200.adjoint import Adjoint
from scratch_wadge_b200.geometry_gpu import build_geometry_gpu
from tests.helpers import RTOL, perturbed, rel
from tests.test_gpu_parity import Dev

pytestmark = pytest.mark.gpu

CASES = [(d, N, c) for d in (2, 3) for N in (1, 2, 3, 4) for c in (False, True)]
SENTINEL = 12345.0


def oracle(ops, curved):
    """the reference's kernels where oracle/_ref was built, else the restatement"""
    try:
        return O.Reference(ops, curved)
    except FileNotFoundError:
        return O.Port(ops, curved)


def multibatch_K(E, grid):
    """2 * grid batches plus a partial one: CTA 0 runs three batches"""
    return 2 * grid * E + max(1, E // 3)


def mesh_with_at_least(dim, curved, K):
    if dim == 3:
        n = max(2, math.ceil((K / 6.0) ** (1.0 / 3.0)))
        return M.periodic_cube(n, warp=M.warp_cube(0.05) if curved else None)
    n = max(2, math.ceil(math.sqrt(K / 2.0)))
    return M.periodic_square(n, n)


def state(geo, curved, seed):
    """the stage-0 state of the case's flow, perturbed by 1% so that the
    log-mean's node pairs fall on both sides of its series switch"""
    dim = geo.ops.dim
    kind = "vortex" if dim == 2 else ("density_wave" if curved else "taylor_green")
    st = dict(zip(("Q", "rhsQ", "Qf", "resQ"), IC.stage0(geo, IC.initial_state(geo, kind))))
    st = perturbed(st, seed)
    st["resQ"] = 1e-3 * st["Q"]
    st["rhsQf"] = np.full_like(st["Qf"], SENTINEL)
    return st


def shapes(ctx, curved, K):
    """per volume kernel shape: ((warps, rows), E, grid at K)"""
    out = []
    for w, r in ctx.vol_shapes(curved):
        ctx.set_vol_shape(curved, w, r)
        out.append(((w, r),) + ctx.shape("vol", curved, K))
    ctx.set_vol_warps(curved, 0)
    return out


def _first(st, K):
    return {k: np.ascontiguousarray(v[:K]).copy() for k, v in st.items()}


@pytest.mark.parametrize("dim,N,curved", CASES)
def test_kernels_over_several_batches_per_cta(cuda, dim, N, curved):
    ops = R.load(dim, N)
    ctx = capi.Context(ops)
    big = 1 << 22  # the grid no longer grows with K beyond this
    sh = shapes(ctx, curved, big)
    Ku_E, Ku_g = ctx.shape("update", curved, big)
    Ks_E, Ks_g = ctx.shape("stage", curved, big)
    Kvs_E, Kvs_g = ctx.shape("volsurf", curved, big)
    Kvol = {w: multibatch_K(E, g) for w, E, g in sh}
    Kupd, Kst, Kvs = multibatch_K(Ku_E, Ku_g), multibatch_K(Ks_E, Ks_g), multibatch_K(Kvs_E, Kvs_g)
    mesh = mesh_with_at_least(dim, curved, max(max(Kvol.values()), Kupd, Kst, Kvs))
    geo = build_geometry_gpu(mesh, N)
    d = Dev(cuda, geo, curved)
    ref = oracle(ops, curved)
    st = state(geo, curved, 5)
    # a stable step for the mesh (the finer the mesh, the smaller), so that
    # the update of these rough states stays physical
    dt = IC.time_step(geo, 0.1, N, nsteps=1, wave_speed=IC.max_wave_speed(st["Q"]))[0]

    # volume kernel, every compiled shape
    for w, E, g in sh:
        K = Kvol[w]
        assert (K + E - 1) // E > 2 * g and K % E, (w, E, g, K)
        d.ctx.set_vol_shape(curved, *w)
        s = d.put(st)
        d.ctx.vol(curved, K, *[d.g[n].data_ptr() for n in ("vgeo", "vfgeo", "nrJ", "nsJ", "ntJ", "Drq",
                                                           "Dsq", "Dtq", "VqLq", "VfPq")],
                  s["Qf"].data_ptr(), s["rhsQ"].data_ptr(), s["rhsQf"].data_ptr())
        d.sync()
        h = d.get(s)
        a = _first(st, K)
        ref.vol(geo, a["Qf"], a["rhsQ"], a["rhsQf"])
        assert rel(h["rhsQ"][:K], a["rhsQ"]) < RTOL, (w, rel(h["rhsQ"][:K], a["rhsQ"]))
        assert rel(h["rhsQf"][:K], a["rhsQf"]) < RTOL, (w, rel(h["rhsQf"][:K], a["rhsQf"]))
        assert np.array_equal(h["rhsQ"][K:], st["rhsQ"][K:]), w
        assert (h["rhsQf"][K:] == SENTINEL).all(), w
    d.ctx.set_vol_warps(curved, 0)

    # surface (one CTA per group, not persistent) and update over Kupd elements
    K = Kupd
    s = d.put(st)
    rhsQf = st["Qf"] * 0.01  # stands in for the volume kernel's face rows
    s["rhsQf"] = torch.from_numpy(rhsQf).cuda()
    d.ctx.surf(K, d.g["fgeo"].data_ptr(), d.g["mapPq"].data_ptr(), d.g["VqLq"].data_ptr(),
               s["Qf"].data_ptr(), s["rhsQf"].data_ptr(), s["rhsQ"].data_ptr())
    d.ctx.update(curved, K, d.g["Jq"].data_ptr(), d.g["VqPq"].data_ptr(), d.g["VfPq"].data_ptr(),
                 IC.RK4A[2], IC.RK4B[2], dt, s["rhsQ"].data_ptr(), s["resQ"].data_ptr(),
                 s["Q"].data_ptr(), s["Qf"].data_ptr())
    d.sync()
    h = d.get(s)
    a = _first(dict(st, rhsQf=rhsQf), K)
    # the surface kernel gathers neighbour traces past K: give the oracle the
    # whole trace array, updating only the first K elements
    Qf_all = np.ascontiguousarray(st["Qf"]).copy()
    ref.surf(geo, Qf_all, a["rhsQf"], a["rhsQ"])
    ref.update(geo, IC.RK4A[2], IC.RK4B[2], dt, a["rhsQ"], a["resQ"], a["Q"], a["Qf"])
    for k in ("Q", "rhsQ", "Qf", "resQ"):
        assert np.isfinite(a[k]).all(), k
        assert rel(h[k][:K], a[k]) < RTOL, (k, rel(h[k][:K], a[k]))
        assert np.array_equal(h[k][K:], st[k][K:]), k

    # volume + surface kernel over Kvs elements (gathers traces past K)
    K = Kvs
    s = d.put(st)
    d.ctx.volsurf(curved, K, *[d.g[n].data_ptr() for n in ("vgeo", "vfgeo", "fgeo", "mapPq", "nrJ", "nsJ",
                                                           "ntJ", "Drq", "Dsq", "Dtq", "VqLq", "VfPq")],
                  s["Qf"].data_ptr(), s["rhsQ"].data_ptr())
    d.sync()
    h = d.get(s)
    a = _first(st, K)
    a["rhsQf"][:] = 0.0
    ref.vol(geo, a["Qf"], a["rhsQ"], a["rhsQf"])
    ref.surf(geo, np.ascontiguousarray(st["Qf"]).copy(), a["rhsQf"], a["rhsQ"])
    assert np.isfinite(a["rhsQ"]).all()
    assert rel(h["rhsQ"][:K], a["rhsQ"]) < RTOL, rel(h["rhsQ"][:K], a["rhsQ"])
    assert np.array_equal(h["rhsQ"][K:], st["rhsQ"][K:])
    assert np.array_equal(h["Qf"], st["Qf"])

    # fused stage kernel over Kst elements (reads the state, writes new buffers)
    K = Kst
    s = d.put(st)
    out = {"rhsQ": torch.full_like(s["rhsQ"], SENTINEL), "Qf": torch.full_like(s["Qf"], SENTINEL)}
    g = d.g
    fn = capi.lib().wadg_euler_stage_3d if dim == 3 else capi.lib().wadg_euler_stage_2d
    args = [g[n].data_ptr() for n in ("vgeo", "vfgeo", "fgeo", "mapPq", "nrJ", "nsJ")]
    args += [g["ntJ"].data_ptr()] if dim == 3 else []
    args += [g["Drq"].data_ptr(), g["Dsq"].data_ptr()] + ([g["Dtq"].data_ptr()] if dim == 3 else [])
    args += [g[n].data_ptr() for n in ("VqLq", "VfPq", "VqPq", "Jq")]
    capi.check(fn(d.ctx.h, K, int(curved), *args, IC.RK4A[3], IC.RK4B[3], dt, s["rhsQ"].data_ptr(),
                  s["Qf"].data_ptr(), s["Q"].data_ptr(), s["resQ"].data_ptr(), out["rhsQ"].data_ptr(),
                  out["Qf"].data_ptr()), "stage")
    d.sync()
    a = _first(st, K)
    a["rhsQf"][:] = 0.0
    Qf_all = np.ascontiguousarray(st["Qf"]).copy()
    ref.vol(geo, a["Qf"], a["rhsQ"], a["rhsQf"])
    ref.surf(geo, Qf_all, a["rhsQf"], a["rhsQ"])
    ref.update(geo, IC.RK4A[3], IC.RK4B[3], dt, a["rhsQ"], a["resQ"], a["Q"], a["Qf"])
    got = dict(Q=s["Q"].cpu().numpy(), resQ=s["resQ"].cpu().numpy(), rhsQ=out["rhsQ"].cpu().numpy(),
               Qf=out["Qf"].cpu().numpy())
    for k in ("Q", "rhsQ", "Qf", "resQ"):
        assert np.isfinite(a[k]).all(), k
        assert rel(got[k][:K], a[k]) < RTOL, (k, rel(got[k][:K], a[k]))
    assert np.array_equal(got["Q"][K:], st["Q"][K:])
    assert (got["rhsQ"][K:] == SENTINEL).all() and (got["Qf"][K:] == SENTINEL).all()


@pytest.mark.parametrize("dim,N,curved", [(3, 3, False), (3, 4, True), (2, 3, True)])
def test_adjoint_pair_kernel_over_several_batches(cuda, dim, N, curved):
    """the RHS VJP (pair kernel over several batches per CTA, a partial last
    batch) against reverse-mode autodiff of the restated stage map, run on the
    GPU through torch at this size"""
    ops = R.load(dim, N)
    ctx = capi.Context(ops)
    E, g = ctx.shape("adj_pairs", curved, 1 << 22)
    # smallest structured mesh with more than 2 grid batches and a partial one
    n = 2
    while True:
        mesh = M.periodic_cube(n, warp=M.warp_cube(0.05) if curved else None) if dim == 3 \
            else M.periodic_square(n, n)
        if (mesh.K + E - 1) // E > 2 * g and mesh.K % E:
            break
        n += 1
    geo = build_geometry_gpu(mesh, N)
    kind = "vortex" if dim == 2 else ("density_wave" if curved else "taylor_green")
    Q = perturbed({"Q": IC.stage0(geo, IC.initial_state(geo, kind))[0]}, 3, 1e-2)["Q"]
    w = np.random.default_rng(2).standard_normal(Q.shape)
    app = capi.App(geo, curved)
    adj = Adjoint(app, 1, 1)
    dev = torch.device("cuda")
    gq = adj.rhs_vjp(torch.from_numpy(Q).to(dev), torch.from_numpy(w).to(dev)).cpu().numpy()
    T = TorchRHS(geo, curved, device=dev)
    _, vjp = torch.func.vjp(T.R, torch.from_numpy(Q).to(dev))
    want = vjp(torch.from_numpy(w).to(dev))[0].cpu().numpy()
    assert rel(gq, want) < 1e-10, rel(gq, want)
