"""Partitioned runs on one GPU: the halo pack kernel (wadg_halo_pack) equals
its host form bit for bit, and a mesh cut into 2-4 parts, each part stepping
its own elements with the halo exchanged between stages (all parts in one
process), gives the single-domain run's state to rounding (the volume
kernel's per-warp choice of log-mean evaluation depends on which elements
share a warp)."""

import numpy as np
import pytest

from scratch_wadge_b200 import build as B
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import ic as IC
from scratch_wadge_b200 import mesh as M
from scratch_wadge_b200 import partition as PT
from tests.test_partition import bounded_square

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build()


def _case(name):
    if name == "tg3d_N3":
        return M.periodic_cube(4), 3, False, "taylor_green", {}
    if name == "dw3d_curved_N2":
        return M.periodic_cube(3, warp=M.warp_cube(0.05)), 2, True, "density_wave", {}
    if name == "vortex2d_curved_N3":
        return M.periodic_square(8, 6), 3, True, "vortex", {}
    return bounded_square(6, 4), 2, False, "vortex", {}


def test_halo_pack_matches_host(cuda):
    geo = M.build_geometry(M.periodic_cube(3), 3)
    U0 = IC.initial_state(geo, "taylor_green")
    Q, rhsQ, Qf, resQ = IC.stage0(geo, U0)
    plans = PT.plan(geo, 3)
    for p in plans:
        part = PT.Part(geo, p, dict(Q=Q, rhsQ=rhsQ, Qf=Qf, resQ=resQ), False)
        rng = np.random.default_rng(p.rank)
        host = rng.standard_normal(tuple(part.Qf.shape))
        part.Qf.copy_(cuda.from_numpy(host))
        part.pack()
        cuda.cuda.synchronize()
        assert np.array_equal(part.sendbuf.cpu().numpy(), PT.pack_host(p, host))
        part.close()


@pytest.mark.parametrize("name,nparts", [("tg3d_N3", 2), ("tg3d_N3", 3), ("dw3d_curved_N2", 4),
                                         ("vortex2d_curved_N3", 3), ("bounded2d_N2", 2)])
def test_partitioned_run_equals_single_domain(cuda, name, nparts):
    mesh, N, curved, kind, kw = _case(name)
    geo = M.build_geometry(mesh, N)
    Q, rhsQ, Qf, resQ = IC.stage0(geo, IC.initial_state(geo, kind, **kw))
    dt = IC.time_step(geo, 0.5, N, nsteps=1, wave_speed=IC.max_wave_speed(Q))[0]
    app = capi.App(geo, curved)
    app.set_state(Q, rhsQ, Qf, resQ)
    app.rk_run(dt, 3, graph=False)
    ref = app.get_state()["Q"]
    app.close()
    state = dict(Q=Q, rhsQ=rhsQ, Qf=Qf, resQ=resQ)
    parts = [PT.Part(geo, p, state, curved) for p in PT.plan(geo, nparts)]
    assert sum(p.plan.ghost_pe for p in parts) > 0
    PT.run_local(parts, dt, 3)
    cuda.cuda.synchronize()
    got = PT.gather_Q(parts, geo.K)
    for p in parts:
        p.close()
    assert _agree(got, ref), float(np.abs(got - ref).max() / np.abs(ref).max())


def _agree(got, ref):
    """The partitioned run equals the single-domain run to rounding (1e-12
    relative, max norm): a part's elements share warps with other elements
    than in the whole mesh, and the volume kernel picks its log-mean
    evaluation per warp (the u^2 series without a vote where every pair of
    the warp's elements is nearly equal), so a value can differ in its last
    bit."""
    return float(np.abs(got - ref).max() / np.abs(ref).max()) < 1e-12


class _FakeAllToAll:
    """dist.all_to_all_single for ranks that are threads of one process, each
    on its own CUDA stream: a rank's call records an event on its current
    stream (after its pack), all ranks meet on the host, then one side stream
    waits for every rank's event and copies every block into its receiver's
    ghost region; the returned work's wait() makes the caller's current
    stream wait for those copies (so a rank's send buffer is free again and
    its ghosts are filled, as when an NCCL all-to-all completes)."""

    def __init__(self, torch, nranks):
        import threading
        self.torch, self.n = torch, nranks
        self.bar = threading.Barrier(nranks)
        self.side = torch.cuda.Stream()
        self.slots = [None] * nranks
        self.done = None

    def __call__(self, rank):
        torch = self.torch

        def a2a(output, input, output_split_sizes, input_split_sizes, group=None, async_op=False):
            ev = torch.cuda.Event()
            ev.record(torch.cuda.current_stream())
            self.slots[rank] = (output, input, list(output_split_sizes), list(input_split_sizes), ev)
            self.bar.wait()
            if rank == 0:
                with torch.cuda.stream(self.side):
                    for *_, e in self.slots:
                        self.side.wait_event(e)
                    for r, (out, _, osz, _, _) in enumerate(self.slots):
                        ro = np.concatenate([[0], np.cumsum(osz)])
                        for s_, (_, inp, _, isz, _) in enumerate(self.slots):
                            io = np.concatenate([[0], np.cumsum(isz)])
                            n = int(io[r + 1] - io[r])
                            assert n == int(ro[s_ + 1] - ro[s_])
                            if n:
                                out[int(ro[s_]):int(ro[s_ + 1])].copy_(inp[int(io[r]):int(io[r + 1])])
                    self.done = torch.cuda.Event()
                    self.done.record(self.side)
            self.bar.wait()
            done = self.done

            class Work:
                def wait(self_):
                    torch.cuda.current_stream().wait_event(done)

            self.bar.wait()  # every rank holds this exchange's event before the next one
            return Work()

        return a2a


def test_run_dist_stream_ordering_with_a_fake_collective(cuda, monkeypatch):
    """run_dist (the overlapped exchange of partitioned multi-GPU runs) with
    two ranks as threads, each on its own stream, and the collective replaced
    by device copies on a third stream: the result equals the single-domain
    run to rounding, so pack -> exchange -> surface are ordered right."""
    import threading

    import torch.distributed as dist
    mesh, N, curved, kind, kw = _case("tg3d_N3")
    geo = M.build_geometry(mesh, N)
    Q, rhsQ, Qf, resQ = IC.stage0(geo, IC.initial_state(geo, kind, **kw))
    dt = IC.time_step(geo, 0.5, N, nsteps=1, wave_speed=IC.max_wave_speed(Q))[0]
    app = capi.App(geo, curved)
    app.set_state(Q, rhsQ, Qf, resQ)
    app.rk_run(dt, 3, graph=False)
    ref = app.get_state()["Q"]
    app.close()
    state = dict(Q=Q, rhsQ=rhsQ, Qf=Qf, resQ=resQ)
    fake = _FakeAllToAll(cuda, 2)
    streams = [cuda.cuda.Stream() for _ in range(2)]
    parts = []
    for r, p in enumerate(PT.plan(geo, 2)):
        with cuda.cuda.stream(streams[r]):
            parts.append(PT.Part(geo, p, state, curved))
    cuda.cuda.synchronize()
    local = threading.local()
    monkeypatch.setattr(dist, "all_to_all_single",
                        lambda *a, **k: fake(local.rank)(*a, **k))
    errors = []

    def rank_main(r):
        local.rank = r
        try:
            with cuda.cuda.stream(streams[r]):
                PT.run_dist(parts[r], dt, 3)
        except Exception as e:  # surfaced by the main thread
            errors.append(e)
            fake.bar.abort()

    th = [threading.Thread(target=rank_main, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(120)
    assert not errors, errors
    cuda.cuda.synchronize()
    got = PT.gather_Q(parts, geo.K)
    for p in parts:
        p.close()
    assert _agree(got, ref), float(np.abs(got - ref).max() / np.abs(ref).max())
