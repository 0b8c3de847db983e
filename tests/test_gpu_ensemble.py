"""The batched ensemble (bins of concatenated instances, one CUDA graph per
time step) against the plain one-instance-per-launch path and the oracle."""

import numpy as np
import pytest

from oracle import pyoracle as O
from scratch_wadge_b200 import build as B
from scratch_wadge_b200 import ensemble as EN
from scratch_wadge_b200 import ic as IC
from tests.helpers import RTOL, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    B.build()
    inst = EN.draw_instances(n=7, kmin=40, kmax=300, seed=3)
    parts = [EN.build_instance(i) for i in inst]
    return inst, parts, EN.common_dt(parts)


@pytest.mark.parametrize("fused", [False, True])
def test_batched_equals_single(cuda, small, fused):
    inst, parts, dt = small
    ens = EN.Ensemble(inst, parts, fused=fused)
    single = EN.SingleInstances(inst, parts)
    ens.run(dt, 3)
    single.run(dt, 3)
    for j in range(len(inst)):
        a = ens.instance_state(j)
        b = single.apps[j].get_state()
        for k in ("Q", "rhsQ", "Qf"):
            assert rel(a[k], b[k]) < RTOL, (j, k)
    ens.close()
    single.close()


def test_autotuned_ensemble(cuda, small):
    """Per-bin shape tuning, then the joint check of the batched step: the
    shapes kept are compiled candidates, the tuned ensemble starts from the
    initial state, and its results equal the plain path's."""
    import ctypes
    from scratch_wadge_b200 import capi
    inst, parts, dt = small
    ens = EN.Ensemble(inst, parts, autotune_dt=dt)
    L = capi.lib()
    for N, b in ens.bins.items():
        ctx = ctypes.c_void_p(L.wadg_app_ctx(b["app"].h))
        cand = (ctypes.c_int * 3)()
        n = L.wadg_vol_warps_candidates(ctx, 1, cand)
        w = L.wadg_ctx_get_vol_warps(ctx)
        assert w == 0 or w in list(cand[:n]), (N, w)
        assert b["tuning"][0] in list(cand[:n])
    if ens.joint_tuning is not None:
        assert ens.joint_tuning["kept"] in ("tuned", "default")
    single = EN.SingleInstances(inst, parts)
    ens.run(dt, 2)
    single.run(dt, 2)
    for j in range(len(inst)):
        a = ens.instance_state(j)
        b = single.apps[j].get_state()
        assert rel(a["Q"], b["Q"]) < RTOL, j
    ens.close()
    single.close()


def test_batched_matches_oracle(cuda, small):
    inst, parts, dt = small
    ens = EN.Ensemble(inst, parts)
    ens.run(dt, 2)
    for j in (0, len(inst) - 1):
        geo, st0 = parts[j]
        st = {k: v.copy() for k, v in st0.items()}
        st["rhsQf"] = np.zeros_like(st["Qf"])
        P = O.Port(geo.ops, True)
        for _ in range(2):
            P.step(geo, dt, st)
        got = ens.instance_state(j)
        assert rel(got["Q"], st["Q"]) < RTOL
    ens.close()


@pytest.mark.parametrize("x", [0])
def test_instance_draw_is_seeded(x):
    a = EN.draw_instances(n=20, seed=5)
    b = EN.draw_instances(n=20, seed=5)
    assert a == b
    ks = [i.K for i in EN.draw_instances(n=256, seed=0)]
    assert min(ks) >= 150 and max(ks) <= 9000
    assert {i.N for i in EN.draw_instances(n=256, seed=0)} == {2, 3, 4}
