"""Replica coordination of multi-GPU runs (scratch_wadge_b200/replicas.py),
exercised with two gloo ranks on CPU: the slowest rank's time is the job's
time, all ranks take the same stage variant, and the throughput counts the
units of every rank."""

import socket

import torch.multiprocessing as mp

from scratch_wadge_b200 import replicas as RP


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    import os
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    from scratch_wadge_b200 import replicas as R
    pg = R.init("gloo", 30.0)
    t = R.all_max(pg, 1.0 + rank)          # rank r took 1 + r seconds
    f = R.agree(pg, rank == ws - 1)        # only the last rank prefers the other variant
    g = R.agree(pg, False)
    v = R.job_throughput(ws, 100.0, t)
    R.finish(pg)
    q.put((rank, t, f, g, v))


def test_two_gloo_ranks_agree_and_take_the_slowest_time():
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
    for _, t, f, g, v in out:
        assert t == 2.0 and f is True and g is False
        assert v == ws * 100.0 / 2.0


def test_single_process_needs_no_group(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    assert RP.env()[0] == 1
    pg = RP.init("gloo")
    assert pg is None
    assert RP.all_max(pg, 3.5) == 3.5 and RP.agree(pg, True) is True
    RP.finish(pg)


def test_bench_refuses_a_rank_count_other_than_gpus():
    """bench.py --gpus N under a launcher that started a different number of
    ranks exits non-zero before any GPU work (it would otherwise report one
    GPU's throughput as N GPUs')."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, WORLD_SIZE="3", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2"], env=env,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "WORLD_SIZE=3" in r.stderr
