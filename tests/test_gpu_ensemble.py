"""The batched ensemble (degree bins of concatenated instances, one CUDA graph
per time step, work lists of the batches still running) against the plain
one-instance-per-launch path and the oracle.  Every instance runs to the
common final time with its own step, so instances finish after different
step counts."""

import ctypes

import numpy as np
import pytest

from oracle import pyoracle as O
from scratch_wadge_b200 import build as B
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import ensemble as EN
from tests.helpers import RTOL, rel

pytestmark = pytest.mark.gpu

T = 0.05


@pytest.fixture(scope="module")
def small():
    B.build()
    inst = EN.draw_instances(n=7, kmin=40, kmax=300, seed=3)
    parts = [EN.build_instance(i) for i in inst]
    steps = EN.instance_steps(parts, T)
    assert len({n for _, n in steps}) > 2  # instances finish at different steps
    return inst, parts


def _compare(ens, single, inst):
    for j in range(len(inst)):
        a = ens.instance_state(j)
        b = single.apps[j].get_state()
        for k in ("Q", "rhsQ", "Qf"):
            assert np.isfinite(a[k]).all()
            assert rel(a[k], b[k]) < RTOL, (j, k, rel(a[k], b[k]))


def test_batched_equals_single_to_final_time(cuda, small):
    inst, parts = small
    ens = EN.Ensemble(inst, parts, T=T)
    single = EN.SingleInstances(inst, parts, T=T)
    ens.run()
    single.run()
    assert ens.progress() == (max(n for _, n in ens.steps),) * 2
    _compare(ens, single, inst)
    ens.close()
    single.close()


def test_batched_equals_single_mid_run(cuda, small):
    """After s steps, each instance has made min(s, n_i) of its own steps,
    the ones done frozen exactly."""
    inst, parts = small
    ns = sorted({n for _, n in EN.instance_steps(parts, T)})
    s = ns[len(ns) // 2]  # some instances done, others running
    ens = EN.Ensemble(inst, parts, T=T)
    single = EN.SingleInstances(inst, parts, T=T)
    ens.run(s)
    single.run(s)
    assert ens.progress()[0] == s
    _compare(ens, single, inst)
    # a frozen instance stays bit for bit while the others go on
    done = [j for j, (_, n) in enumerate(ens.steps) if n <= s]
    assert done
    before = {j: ens.instance_state(j)["Q"].copy() for j in done}
    ens.run(2)
    for j in done:
        assert np.array_equal(ens.instance_state(j)["Q"], before[j]), j
    ens.close()
    single.close()


def test_autotuned_bins_equal_single(cuda, small):
    """Per-bin CTA shapes of the volume + surface kernel, picked by timing
    (every shape computes the same RHS), then the run to the final time."""
    inst, parts = small
    ens = EN.Ensemble(inst, parts, T=T, autotune=True)
    for N, (w, times) in ens.tuning.items():
        assert w in times and all(t > 0 for t in times.values()), N
    single = EN.SingleInstances(inst, parts, T=T)
    ens.run()
    single.run()
    _compare(ens, single, inst)
    ens.close()
    single.close()


def test_batched_matches_oracle(cuda, small):
    inst, parts = small
    ens = EN.Ensemble(inst, parts, T=T)
    ens.run()
    for j in (0, len(inst) - 1):
        geo, st0 = parts[j]
        dt, n = ens.steps[j]
        st = {k: v.copy() for k, v in st0.items()}
        st["rhsQf"] = np.zeros_like(st["Qf"])
        P = O.Port(geo.ops, True)
        for _ in range(n):
            P.step(geo, dt, st)
        got = ens.instance_state(j)
        assert rel(got["Q"], st["Q"]) < RTOL
    ens.close()


def test_restart_repeats_the_run(cuda, small):
    inst, parts = small
    ens = EN.Ensemble(inst, parts, T=T)
    ens.run()
    first = [ens.instance_state(j)["Q"].copy() for j in range(len(inst))]
    ens.restart()
    assert ens.progress()[0] == 0
    ens.run()
    for j in range(len(inst)):
        assert np.array_equal(ens.instance_state(j)["Q"], first[j])
    ens.close()


def test_ensemble_rejects_bad_descriptors(cuda, small):
    inst, parts = small
    geo, st = parts[0]
    app = capi.App(geo, curved=True)
    off = np.array([0, geo.K], dtype=np.int32)
    dt = np.array([1e-3])
    for n, o, d in ((np.array([-1], dtype=np.int32), off, dt),
                    (np.array([3], dtype=np.int32), np.array([0, geo.K - 1], dtype=np.int32), dt),
                    (np.array([3], dtype=np.int32), off, np.array([0.0]))):
        b = EN.EnsembleBin(app.h.value, 1, o.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                           d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                           n.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        h = ctypes.c_void_p()
        r = capi.lib().wadg_ensemble_create(1, ctypes.cast(ctypes.pointer(b), ctypes.c_void_p),
                                            ctypes.byref(h))
        assert r == capi.ERR_INVALID and not h.value
    app.set_fused(True)
    b = EN.EnsembleBin(app.h.value, 1, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                       dt.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                       np.array([3], dtype=np.int32).ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    h = ctypes.c_void_p()
    assert capi.lib().wadg_ensemble_create(1, ctypes.cast(ctypes.pointer(b), ctypes.c_void_p),
                                           ctypes.byref(h)) == capi.ERR_INVALID
    app.close()


@pytest.mark.parametrize("x", [0])
def test_instance_draw_is_seeded(x):
    a = EN.draw_instances(n=20, seed=5)
    b = EN.draw_instances(n=20, seed=5)
    assert a == b
    ks = [i.K for i in EN.draw_instances(n=256, seed=0)]
    assert min(ks) >= 150 and max(ks) <= 9000
    assert {i.N for i in EN.draw_instances(n=256, seed=0)} == {2, 3, 4}
