"""Element partitioning with a face-trace halo exchange.

The reference partitions its mesh along a Hilbert curve and leaves the halo
exchange of the face traces unwritten (euler.c:2015-2605).  Here a mesh is cut
into parts along a Morton curve of the element centroids.  Each part keeps
the traces its faces need from other parts as ghost pseudo-elements appended
to its Qf array. The ghosts received from part s are one contiguous run of
whole pseudo-elements, so the surface kernel reads them through the part's
mapPq unchanged, and an all-to-all of packed send buffers (wadg_halo_pack)
lands each block directly in place.  Per LSRK stage: exchange, then the
volume, surface and update kernels on the part's own elements.

Only the surface kernel reads a neighbour's trace, so the exchange of stage s
only has to finish before the surface kernel of stage s.  Per element the
kernels do the same arithmetic in any partition, except for the volume
kernel's per-warp choice of log-mean evaluation (which elements share a warp
differs between a part and the whole mesh), so a partitioned run equals the
single-domain run to rounding.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import capi
from . import ic as IC
from . import mesh as M

NONE = 0xFFFFFFFF


@dataclass
class PartPlan:
    """One part: its elements (global ids, in local order), its neighbour map
    in local numbering (ghosts as pseudo-elements K_r, K_r + 1, ...), and the
    halo: pseudo-elements received from / sent to every part, and the
    field-strided local Qf index of every send slot (blocks in part order,
    NONE in padding slots)."""
    rank: int
    nparts: int
    NF: int
    Nf: int
    elems: np.ndarray
    mapPq: np.ndarray
    recv_pe: list
    send_pe: list
    send_src: np.ndarray = field(repr=False)

    @property
    def K(self):
        return len(self.elems)

    @property
    def ghost_pe(self):
        return int(sum(self.recv_pe))

    def recv_counts(self):
        return [p * self.NF * self.Nf for p in self.recv_pe]

    def send_counts(self):
        return [p * self.NF * self.Nf for p in self.send_pe]


def morton_order(geo: M.Geometry) -> np.ndarray:
    """Elements sorted along a Morton (Z-order) curve of their centroids."""
    dim = geo.ops.dim
    c = geo.xyzq[:, :dim, :].mean(axis=2)
    lo, hi = c.min(axis=0), c.max(axis=0)
    q = np.floor((c - lo) / np.maximum(hi - lo, 1e-300) * ((1 << 20) - 1)).astype(np.uint64)
    code = np.zeros(geo.K, dtype=np.uint64)
    for b in range(20):
        for d in range(dim):
            code |= ((q[:, d] >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * dim + d)
    return np.argsort(code, kind="stable")


def plan(geo: M.Geometry, nparts: int, order: str = "morton") -> list:
    """Cut the mesh into nparts contiguous pieces of the element order."""
    ops = geo.ops
    K, NF, Nf = geo.K, ops.NfqNf, ops.Nfields
    if not 1 <= nparts <= K:
        raise ValueError("need 1 <= nparts <= K")
    blk = NF * Nf
    perm = morton_order(geo) if order == "morton" else np.arange(K)
    bounds = [(r * K) // nparts for r in range(nparts + 1)]
    owner = np.empty(K, dtype=np.int64)
    local = np.empty(K, dtype=np.int64)
    for r in range(nparts):
        ids = perm[bounds[r]:bounds[r + 1]]
        owner[ids] = r
        local[ids] = np.arange(len(ids))
    mp = geo.mapPq.astype(np.int64)
    pe, pj = mp // blk, mp % blk
    mapPqs, recv_pe, requests = [], [], []
    for r in range(nparts):
        ids = perm[bounds[r]:bounds[r + 1]]
        Kr = len(ids)
        e2, j2 = pe[ids], pj[ids]
        own = owner[e2]
        out = np.empty((Kr, NF), dtype=np.int64)
        here = own == r
        out[here] = j2[here] + local[e2[here]] * blk
        gm = ~here
        key = (own[gm] * K + e2[gm]) * NF + j2[gm]
        ukey, inv = np.unique(key, return_inverse=True)   # sorted: grouped by owner
        u_own, u_e, u_j = ukey // (K * NF), (ukey // NF) % K, ukey % NF
        counts = np.bincount(u_own, minlength=nparts)
        pes = (counts + NF - 1) // NF
        off_pe = np.concatenate([[0], np.cumsum(pes)[:-1]])
        first = np.concatenate([[0], np.cumsum(counts)[:-1]])
        slot = np.arange(len(ukey)) - first[u_own] + off_pe[u_own] * NF
        g = slot[inv]
        out[gm] = (g % NF) + (Kr + g // NF) * blk
        mapPqs.append(out.astype(np.uint32))
        recv_pe.append([int(x) for x in pes])
        req = []
        for s in range(nparts):
            sel = u_own == s
            src = np.full(pes[s] * NF, NONE, dtype=np.uint32)
            src[:sel.sum()] = (u_j[sel] + local[u_e[sel]] * blk).astype(np.uint32)
            req.append(src)
        requests.append(req)
    parts = []
    for s in range(nparts):
        send = [requests[r][s] for r in range(nparts)]
        parts.append(PartPlan(s, nparts, NF, Nf, perm[bounds[s]:bounds[s + 1]].copy(), mapPqs[s],
                              recv_pe[s], [recv_pe[r][s] for r in range(nparts)],
                              np.concatenate(send) if send else np.zeros(0, np.uint32)))
    return parts


def pack_host(p: PartPlan, Qf_local: np.ndarray) -> np.ndarray:
    """The send buffer wadg_halo_pack builds, on the host (Qf_local: the part's
    Qf array, ghosts included, [K_r + ghost_pe][Nf][NF])."""
    NF, Nf = p.NF, p.Nf
    flat = Qf_local.reshape(-1)
    n = len(p.send_src)
    buf = np.zeros(n * Nf)
    g = np.arange(n)
    ok = p.send_src != NONE
    base = (g // NF) * NF * Nf + g % NF
    for f in range(Nf):
        buf[base[ok] + f * NF] = flat[p.send_src[ok].astype(np.int64) + f * NF]
    return buf


class Part:
    """One part on the device: its geometry, state and halo buffers (torch),
    and the kernels of a stage on its K_r elements through the C ABI."""

    def __init__(self, geo: M.Geometry, p: PartPlan, state: dict, curved: bool, gamma=1.4, tau=1.0,
                 device="cuda"):
        import torch

        self.torch, self.plan, self.curved = torch, p, curved
        ops = geo.ops
        self.ops = ops
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(device)
        idx = p.elems
        self.g = dict(vgeo=t(geo.vgeo[idx]), vfgeo=t(geo.vfgeo[idx]), fgeo=t(geo.fgeo[idx]),
                      Jq=t(geo.Jq[idx]),
                      mapPq=torch.from_numpy(p.mapPq.view(np.int32)).to(device),
                      nrJ=t(ops.nrJ), nsJ=t(ops.nsJ), ntJ=t(ops.ntJ), Drq=t(ops.fortran("Drq")),
                      Dsq=t(ops.fortran("Dsq")), Dtq=t(ops.fortran("Dtq")),
                      VqLq=t(ops.fortran("VqLq")), VqPq=t(ops.fortran("VqPq")),
                      VfPq=t(ops.fortran("VfPq")))
        self.Q, self.rhsQ, self.resQ = (t(state[k][idx]) for k in ("Q", "rhsQ", "resQ"))
        Qf = np.zeros((p.K + p.ghost_pe, ops.Nfields, ops.NfqNf))
        Qf[:p.K] = state["Qf"][idx]
        self.Qf = t(Qf)
        self.rhsQf = torch.zeros((p.K, ops.Nfields, ops.NfqNf), dtype=torch.float64, device=device)
        self.ghost = self.Qf[p.K:].view(-1)
        self.send_src = torch.from_numpy(p.send_src.view(np.int32)).to(device)
        self.sendbuf = torch.zeros(len(p.send_src) * ops.Nfields, dtype=torch.float64, device=device)
        self.ctx = capi.Context(ops, gamma, tau, torch.cuda.current_stream().cuda_stream)

    def pack(self):
        n = len(self.plan.send_src)
        if n:
            self.ctx.halo_pack(n, self.send_src.data_ptr(), self.Qf.data_ptr(), self.Qf.numel(),
                               self.sendbuf.data_ptr())

    def vol(self):
        """the volume kernel (reads the part's own traces only)"""
        g, K = self.g, self.plan.K
        self.ctx.vol(self.curved, K, g["vgeo"].data_ptr(), g["vfgeo"].data_ptr(), g["nrJ"].data_ptr(),
                     g["nsJ"].data_ptr(), g["ntJ"].data_ptr(), g["Drq"].data_ptr(), g["Dsq"].data_ptr(),
                     g["Dtq"].data_ptr(), g["VqLq"].data_ptr(), g["VfPq"].data_ptr(),
                     self.Qf.data_ptr(), self.rhsQ.data_ptr(), self.rhsQf.data_ptr())

    def surf_update(self, a, b, dt):
        """the surface kernel (reads the ghosts) and the update"""
        g, K = self.g, self.plan.K
        self.ctx.surf(K, g["fgeo"].data_ptr(), g["mapPq"].data_ptr(), g["VqLq"].data_ptr(),
                      self.Qf.data_ptr(), self.rhsQf.data_ptr(), self.rhsQ.data_ptr())
        self.ctx.update(self.curved, K, g["Jq"].data_ptr(), g["VqPq"].data_ptr(), g["VfPq"].data_ptr(),
                        a, b, dt, self.rhsQ.data_ptr(), self.resQ.data_ptr(), self.Q.data_ptr(),
                        self.Qf.data_ptr())

    def stage(self, a, b, dt):
        self.vol()
        self.surf_update(a, b, dt)

    def close(self):
        self.ctx.close()


def _blocks(counts):
    off = np.concatenate([[0], np.cumsum(counts)])
    return [(int(off[i]), int(off[i + 1])) for i in range(len(counts))]


def exchange_local(parts: list) -> None:
    """The all-to-all of the halo within one process (all parts on one
    device): pack every part, then copy each block into its receiver's
    ghost region."""
    for p in parts:
        p.pack()
    for r, pr in enumerate(parts):
        rb = _blocks(pr.plan.recv_counts())
        for s, ps in enumerate(parts):
            if s == r:
                continue
            sb = _blocks(ps.plan.send_counts())[r]
            if sb[1] > sb[0]:
                pr.ghost[rb[s][0]:rb[s][1]].copy_(ps.sendbuf[sb[0]:sb[1]])


def exchange_dist(part: Part, group=None, async_op=False):
    """The all-to-all of the halo across ranks (one part per rank), between
    stages: every rank takes it in the same order.  With async_op the
    collective is queued behind the pack and the caller waits on the returned
    work before the surface kernel."""
    import torch.distributed as dist
    part.pack()
    return dist.all_to_all_single(part.ghost, part.sendbuf, part.plan.recv_counts(),
                                  part.plan.send_counts(), group=group, async_op=async_op)


def run_local(parts: list, dt: float, nsteps: int) -> None:
    """nsteps LSRK-45 time steps of all parts in one process."""
    for _ in range(nsteps):
        for st in range(5):
            exchange_local(parts)
            for p in parts:
                p.stage(IC.RK4A[st], IC.RK4B[st], dt)


def run_dist(part: Part, dt: float, nsteps: int, group=None) -> None:
    """nsteps LSRK-45 time steps of this rank's part.  The halo exchange of a
    stage runs while its volume kernel does (only the surface kernel reads
    the ghosts).  The part's kernels run on torch's current stream, the
    stream the collective is ordered on."""
    import torch
    part.ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    for _ in range(nsteps):
        for st in range(5):
            work = exchange_dist(part, group, async_op=True)
            part.vol()
            work.wait()
            part.surf_update(IC.RK4A[st], IC.RK4B[st], dt)


def gather_Q(parts: list, K: int) -> np.ndarray:
    """The parts' Q in global element order."""
    first = parts[0]
    out = np.empty((K, first.ops.Nfields, first.ops.Nq))
    for p in parts:
        out[p.plan.elems] = p.Q.cpu().numpy()
    return out
