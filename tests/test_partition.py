"""Element partitioning with a face-trace halo (scratch_wadge_b200/partition.py),
without a GPU: the plan routes every face point's neighbour trace through the
part's own elements or its ghost pseudo-elements, the send and receive
counts agree between parts, and the exchange works across two gloo ranks
(packing done by pack_host, the host form of wadg_halo_pack)."""

import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from scratch_wadge_b200 import mesh as M
from scratch_wadge_b200 import partition as PT

def bounded_square(nx=5, ny=3):
    """A square mesh inside a larger box: its outer face points are boundary
    points (their own neighbours)."""
    m = M.periodic_square(nx, ny)
    return M.Mesh(2, m.VX, m.EToV, m.lo - 1.0, m.hi + 1.0, boundary_self=True)


MESHES = {
    "cube3_N2": (lambda: M.periodic_cube(3), 2),
    "warped2_N3": (lambda: M.periodic_cube(2, warp=M.warp_cube(0.05)), 3),
    "square_N3": (lambda: M.periodic_square(6, 4), 3),
    "bounded_N2": (bounded_square, 2),
}


def _traces(geo, seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((geo.K, geo.ops.Nfields, geo.ops.NfqNf))


def _local_arrays(parts, Qf):
    return [np.concatenate([Qf[p.elems], np.zeros((p.ghost_pe,) + Qf.shape[1:])]) for p in parts]


def _exchange_host(parts, Ql):
    bufs = [PT.pack_host(p, Ql[i]) for i, p in enumerate(parts)]
    for r, pr in enumerate(parts):
        rc = np.concatenate([[0], np.cumsum(pr.recv_counts())])
        flat = Ql[r].reshape(-1)
        g0 = pr.K * pr.NF * pr.Nf
        for s, ps in enumerate(parts):
            sc = np.concatenate([[0], np.cumsum(ps.send_counts())])
            flat[g0 + rc[s]:g0 + rc[s + 1]] = bufs[s][sc[r]:sc[r + 1]]


def _check_reads(geo, parts, Ql, Qf):
    """Every face point reads, through its part's mapPq, the trace the
    global map points at (all fields)."""
    NF, Nf = geo.ops.NfqNf, geo.ops.Nfields
    gflat = Qf.reshape(-1)
    for r, p in enumerate(parts):
        flat = Ql[r].reshape(-1)
        want = geo.mapPq[p.elems].astype(np.int64)
        got = p.mapPq.astype(np.int64)
        assert got.max() < len(flat)
        for f in range(Nf):
            assert np.array_equal(flat[got + f * NF], gflat[want + f * NF])


@pytest.mark.parametrize("name", sorted(MESHES))
@pytest.mark.parametrize("nparts", [1, 2, 3, 5])
def test_plan_routes_every_face_point(name, nparts):
    mk, N = MESHES[name]
    geo = M.build_geometry(mk(), N)
    parts = PT.plan(geo, nparts)
    assert np.array_equal(np.sort(np.concatenate([p.elems for p in parts])), np.arange(geo.K))
    for s, ps in enumerate(parts):
        assert ps.recv_pe[s] == 0 and ps.send_pe[s] == 0
        for r, pr in enumerate(parts):
            assert ps.send_pe[r] == pr.recv_pe[s]
        assert len(ps.send_src) == sum(ps.send_pe) * ps.NF
    if nparts == 1:
        assert parts[0].ghost_pe == 0
    Qf = _traces(geo)
    Ql = _local_arrays(parts, Qf)
    _exchange_host(parts, Ql)
    _check_reads(geo, parts, Ql, Qf)


def test_morton_parts_have_smaller_halos_than_slabs():
    geo = M.build_geometry(M.periodic_cube(6), 1)
    ghosts = lambda order: sum(p.ghost_pe for p in PT.plan(geo, 8, order))
    assert ghosts("morton") < ghosts("natural")


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    import os
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    import torch
    import torch.distributed as dist
    from scratch_wadge_b200 import mesh as MM
    from scratch_wadge_b200 import partition as P
    from scratch_wadge_b200 import replicas as R
    pg = R.init("gloo", 30.0)
    geo = MM.build_geometry(MM.periodic_cube(3), 2)
    parts = P.plan(geo, ws)
    p = parts[rank]
    Qf = _traces(geo, seed=7)
    Ql = np.concatenate([Qf[p.elems], np.zeros((p.ghost_pe,) + Qf.shape[1:])])
    send = torch.from_numpy(P.pack_host(p, Ql))
    ghost = torch.zeros(p.ghost_pe * p.NF * p.Nf, dtype=torch.float64)
    dist.all_to_all_single(ghost, send, p.recv_counts(), p.send_counts())
    Ql.reshape(-1)[p.K * p.NF * p.Nf:] = ghost.numpy()
    flat, gflat = Ql.reshape(-1), Qf.reshape(-1)
    want = geo.mapPq[p.elems].astype(np.int64)
    got = p.mapPq.astype(np.int64)
    ok = all(np.array_equal(flat[got + f * p.NF], gflat[want + f * p.NF]) for f in range(p.Nf))
    R.finish(pg)
    q.put((rank, bool(ok), p.ghost_pe))


def test_two_gloo_ranks_exchange_the_halo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ws = 2
    ps = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(ws))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] for o in out) and all(o[2] > 0 for o in out)
