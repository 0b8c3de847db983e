"""The oracle (C restatement, oracle/wadg_ref.c) pinned against the reference:
the golden vectors made by the reference's own kernels, and -- where the
reference was compiled here (oracle/_ref) -- the reference kernels on fresh
seeded inputs.  CPU only."""

import math

import numpy as np
import pytest

from oracle import pyoracle as O
from scratch_wadge_b200 import ic as IC
from scratch_wadge_b200 import mesh as M
from tests.helpers import RTOL, Case, golden_names, perturbed, rel


@pytest.mark.parametrize("name", golden_names())
def test_port_matches_golden(name):
    c = Case(name)
    P = O.Port(c.ops, c.curved)
    s = c.state()
    P.vol(c.geo, s["Qf"], s["rhsQ"], s["rhsQf"])
    assert rel(s["rhsQ"], c.z["vol_rhsQ"]) < RTOL
    assert rel(s["rhsQf"], c.z["vol_rhsQf"]) < RTOL
    P.surf(c.geo, s["Qf"], s["rhsQf"], s["rhsQ"])
    assert rel(s["rhsQ"], c.z["surf_rhsQ"]) < RTOL
    P.update(c.geo, IC.RK4A[1], IC.RK4B[1], c.dt, s["rhsQ"], s["resQ"], s["Q"], s["Qf"])
    for k in ("Q", "rhsQ", "Qf", "resQ"):
        assert rel(s[k], c.z["upd_" + k]) < RTOL, k
    s = c.state()
    P.step(c.geo, c.dt, s)
    assert rel(s["Q"], c.z["step_Q"]) < RTOL


@pytest.mark.skipif(not O.reference_available(), reason="reference not compiled here (oracle/_ref)")
@pytest.mark.parametrize("name", golden_names())
def test_port_matches_reference_perturbed(name):
    c = Case(name)
    P, Rf = O.Port(c.ops, c.curved), O.Reference(c.ops, c.curved)
    for seed in (1, 2):
        s0 = perturbed(c.state(), seed)
        a = {k: v.copy() for k, v in s0.items()}
        b = {k: v.copy() for k, v in s0.items()}
        P.stage(c.geo, IC.RK4A[2], IC.RK4B[2], 2e-3, a)
        Rf.stage(c.geo, IC.RK4A[2], IC.RK4B[2], 2e-3, b)
        for k in ("Q", "rhsQ", "Qf", "resQ"):
            assert rel(a[k], b[k]) < RTOL, (k, rel(a[k], b[k]))


def test_logmean_branches():
    P = O.Port.lib()
    P.wadg_ref_logmean.restype = __import__("ctypes").c_double
    P.wadg_ref_logmean.argtypes = [__import__("ctypes").c_int, __import__("ctypes").c_double,
                                   __import__("ctypes").c_double]
    for dim in (2, 3):
        for a, b in [(1.0, 1.0), (1.0, 1.001), (2.0, 1.0), (0.3, 5.0), (1.0, 1.0 + 1e-9)]:
            exact = a if a == b else (a - b) / (math.log(a) - math.log(b))
            got = P.wadg_ref_logmean(dim, a, b)
            assert abs(got - exact) <= 1e-13 * exact
            assert P.wadg_ref_logmean(dim, b, a) == pytest.approx(got, rel=1e-15)


@pytest.mark.parametrize("dim,N,curved", [(3, 3, False), (3, 3, True), (2, 3, True), (3, 2, True)])
def test_free_stream_preservation(dim, N, curved):
    """A constant state is a steady solution: the RHS vanishes to round-off,
    on affine and warped meshes (needs the discrete GCL of the geometric
    factors, operators.cpp:617-687)."""
    m = M.periodic_cube(2, warp=M.warp_cube(0.05) if curved else None) if dim == 3 else M.periodic_square(3, 3)
    geo = M.build_geometry(m, N)
    Q, rhsQ, Qf, resQ = IC.stage0(geo, IC.initial_state(geo, "constant"))
    P = O.Port(geo.ops, curved)
    rhsQf = np.zeros_like(Qf)
    P.vol(geo, Qf, rhsQ, rhsQf)
    P.surf(geo, Qf, rhsQf, rhsQ)
    # round-off of the discrete identities behind it (SBP, GCL), amplified by
    # the operators' norms: 1e-12 to 2e-11 of |Q| for these cases, with the
    # reference's own tables as with the built ones
    assert np.abs(rhsQ).max() < 5e-11 * np.abs(Q).max()
