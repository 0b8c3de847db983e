"""Geometry against the reference's own geometry builder.

tests/golden/geo*.npz hold the outputs of host_operators_new_2D / _3D
(operators_c.cpp:39, 205; build_geofacs_2D / _3D, operators.cpp:343-719),
compiled from the reference sources, on small affine periodic meshes
(tests/golden/gen_geometry.py).  The host builder (mesh.build_geometry) must
reproduce them to RTOL relative in the max norm; the GPU builder is held to
the same fixtures in tests/test_gpu_geometry.py.  Argument validation of the
GPU builder's C ABI needs no GPU."""

import ctypes
import glob
import os

import numpy as np
import pytest

from scratch_wadge_b200 import build as B
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import geometry_gpu as GG
from scratch_wadge_b200 import mesh as M

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# Both sides evaluate the same formulas in float64, each from its own
# reference-element tables (the reference's; here refbuild.py's, equal to
# them to 2e-14).  The 3D metric terms take second derivatives of degree
# N+1 coordinate products (Kopriva's curl form), which amplify the tables'
# rounding: the largest difference is 7e-14 at N = 2, 2e-13 at N = 3 and
# 1.0e-12 at N = 4 (2D: below 4e-14).
RTOL = 3e-12
FIELDS = ("vgeo", "vfgeo", "fgeo", "Jq")


def geo_cases():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "geo*.npz")))


def load_case(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    dim, N = int(z["dim"]), int(z["N"])
    return M.Mesh(dim, z["VX"], z["EToV"], z["lo"], z["hi"]), N, z


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_geometry_fixtures_present():
    assert len(geo_cases()) == 6


@pytest.mark.parametrize("name", geo_cases())
def test_host_builder_matches_reference_builder(name):
    mesh, N, z = load_case(name)
    g = M.build_geometry(mesh, N)
    for k in FIELDS:
        assert rel(getattr(g, k), z[k]) < RTOL, (k, rel(getattr(g, k), z[k]))
    d = mesh.dim
    assert np.abs(g.xyzq[:, :d] - z["xyzq"][:, :d]).max() < 1e-13
    assert np.abs(g.xyzf[:, :d] - z["xyzf"][:, :d]).max() < 1e-13


def test_geometry_abi_validation():
    B.build()
    L = capi.lib()
    empty = GG.GeoOps()
    # incomplete operator set, K < 0, K = 0: rejected or no-ops before any CUDA call
    assert L.wadg_geofacs(ctypes.byref(empty), 1, *([None] * 7), None) != 0
    ops = GG.GeoOps(2, 3, 10, 12, 12, 0, *([1] * 11), *([None] * 6))  # a complete 2D set
    assert L.wadg_geofacs(ctypes.byref(ops), -1, *([None] * 7), None) != 0
    assert L.wadg_geofacs(ctypes.byref(ops), 0, *([None] * 7), None) == 0
    assert L.wadg_geofacs(ctypes.byref(ops), 4, *([None] * 7), None) != 0  # null outputs
    assert L.wadg_match_faces_workspace(0, 12) == 0
    assert L.wadg_match_faces_workspace(100, 12) >= 100 * 12 * 8
    lo = (ctypes.c_double * 2)(0.0, 0.0)
    hi = (ctypes.c_double * 2)(1.0, 1.0)
    assert L.wadg_match_faces(ctypes.byref(ops), 0, None, lo, hi, 0, None, 0, None, None) == 0
    assert L.wadg_match_faces(ctypes.byref(ops), 4, None, lo, hi, 0, None, 0, None, None) != 0
