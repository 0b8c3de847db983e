"""The GPU geometry builder (wadg_geofacs, wadg_match_faces) against the
reference's own builder (fixtures from host_operators_new_2D / _3D,
tests/golden/gen_geometry.py) and against the host builder on larger and
curved meshes: geometric factors to 1e-12 relative (max norm), neighbour maps
bit for bit."""

import numpy as np
import pytest

from scratch_wadge_b200 import build as B
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import geometry_gpu as GG
from scratch_wadge_b200 import mesh as M
from tests.test_geometry import FIELDS, RTOL, geo_cases, load_case, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build()


@pytest.mark.parametrize("name", geo_cases())
def test_gpu_builder_matches_reference_builder(cuda, name):
    mesh, N, z = load_case(name)
    g = GG.build_geometry_gpu(mesh, N)
    for k in FIELDS:
        assert rel(getattr(g, k), z[k]) < RTOL, (k, rel(getattr(g, k), z[k]))
    d = mesh.dim
    assert np.abs(g.xyzq[:, :d] - z["xyzq"][:, :d]).max() < 1e-13
    assert np.abs(g.xyzf[:, :d] - z["xyzf"][:, :d]).max() < 1e-13


MESHES = {
    "cube4_N3": (lambda: M.periodic_cube(4), 3),
    "cube3_N2": (lambda: M.periodic_cube(3), 2),
    "warped3_N4": (lambda: M.periodic_cube(3, warp=M.warp_cube(0.05)), 4),
    "warped4_N3": (lambda: M.periodic_cube(4, warp=M.warp_cube(0.05)), 3),
    "square_N3": (lambda: M.periodic_square(16, 8), 3),
    "square_N4": (lambda: M.periodic_square(5, 7, lo=(-1.0, 2.0), hi=(3.0, 9.0)), 4),
    "square_N1": (lambda: M.periodic_square(6, 6), 1),
}


@pytest.mark.parametrize("name", sorted(MESHES))
def test_gpu_builder_matches_host_builder(cuda, name):
    mk, N = MESHES[name]
    mesh = mk()
    h = M.build_geometry(mesh, N)
    g = GG.build_geometry_gpu(mesh, N)
    for k in FIELDS:
        assert rel(getattr(g, k), getattr(h, k)) < RTOL, (k, rel(getattr(g, k), getattr(h, k)))
    assert np.array_equal(g.mapPq, h.mapPq)
    assert np.abs(g.xyzq - h.xyzq).max() < 1e-13 and np.abs(g.xyzf - h.xyzf).max() < 1e-13
    # the map is an involution between different elements
    K, NF = g.mapPq.shape
    Nf = mesh.dim + 2
    m = g.mapPq.astype(np.int64)
    e, j = m // (NF * Nf), m % (NF * Nf)
    back = g.mapPq.reshape(-1)[j + e * NF].ravel()
    assert np.array_equal(back, (np.arange(NF)[None, :] + np.arange(K)[:, None] * NF * Nf).ravel())
    assert not np.any(e == np.arange(K)[:, None])


def test_gpu_builder_bench_size(cuda):
    """3D affine N=3 at K=24576 (the bench workload)."""
    mesh = M.periodic_cube(16)
    h = M.build_geometry(mesh, 3)
    g = GG.build_geometry_gpu(mesh, 3)
    for k in FIELDS:
        assert rel(getattr(g, k), getattr(h, k)) < RTOL, k
    assert np.array_equal(g.mapPq, h.mapPq)


def test_match_faces_rejects_a_non_periodic_box(cuda):
    """A box twice as long as the mesh in x: the points on x = hi no longer
    wrap onto x = lo, so they do not pair up."""
    mesh = M.periodic_square(4, 4)
    bad = M.Mesh(2, mesh.VX, mesh.EToV, mesh.lo, mesh.hi + np.array([20.0, 0.0]))
    with pytest.raises(capi.WadgError):
        GG.build_geometry_gpu(bad, 3)


def test_gpu_builder_on_gmsh_meshes(cuda, tmp_path):
    """Meshes through the gmsh reader: an unstructured-looking periodic mesh,
    and a mesh inside a larger box whose outer face points become their own
    neighbours (the reference's boundary semantics)."""
    from scratch_wadge_b200 import meshio as IO
    from tests.test_meshio import jittered_square
    p = str(tmp_path / "j.msh")
    IO.write_gmsh(jittered_square(8), p)
    m = IO.read_gmsh(p, 2)
    for mesh in (m, M.Mesh(2, m.VX, m.EToV, m.lo - 1.0, m.hi + 1.0, boundary_self=True)):
        for N in (2, 4):
            h = M.build_geometry(mesh, N)
            g = GG.build_geometry_gpu(mesh, N)
            assert np.array_equal(g.mapPq, h.mapPq)
            for k in FIELDS:
                assert rel(getattr(g, k), getattr(h, k)) < RTOL, k
    assert IO.boundary_faces(g).sum() > 0
