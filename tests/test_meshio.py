"""Mesh files (no GPU): the gmsh 2.2 reader against meshes written here, the
reference's own meshes where its tree is present, orientation repair, the
reference's boundary semantics (unpaired face points are their own
neighbours), the MFEM writer's layout, and the readers' errors."""

import os

import numpy as np
import pytest

from oracle.build import REF_DIR
from scratch_wadge_b200 import build as B
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import mesh as M
from scratch_wadge_b200 import meshio as IO

REF_MESHES = os.path.join(REF_DIR, "meshes")


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build()


def jittered_square(n=6, amp=0.15, seed=1):
    """periodic_square with interior vertices displaced (an unstructured-looking
    but still periodic mesh)."""
    m = M.periodic_square(n, n)
    rng = np.random.default_rng(seed)
    VX = m.VX.copy()
    h = (m.hi - m.lo) / n
    inner = np.all((VX > m.lo + 1e-9) & (VX < m.hi - 1e-9), axis=1)
    VX[inner] += amp * h * rng.uniform(-1, 1, size=(inner.sum(), 2))
    return M.Mesh(2, VX, m.EToV, m.lo, m.hi)


@pytest.mark.parametrize("dim", [2, 3])
def test_gmsh_round_trip(tmp_path, dim):
    m = M.periodic_cube(2) if dim == 3 else jittered_square()
    p = str(tmp_path / "m.msh")
    IO.write_gmsh(m, p)
    r = IO.read_gmsh(p, dim)
    assert np.array_equal(r.VX, m.VX) and np.array_equal(r.EToV, m.EToV)
    assert np.allclose(r.lo, m.VX.min(axis=0)) and np.allclose(r.hi, m.VX.max(axis=0))
    assert r.flipped == 0 and r.boundary_self
    N = 3
    g0, g1 = M.build_geometry(m, N), M.build_geometry(r, N)
    for k in ("vgeo", "vfgeo", "fgeo", "Jq", "mapPq"):
        assert np.array_equal(getattr(g0, k), getattr(g1, k)), k


def test_gmsh_orientation_repair(tmp_path):
    m = M.periodic_cube(2)
    bad = m.EToV.copy()
    bad[::3] = bad[::3][:, [0, 2, 1, 3]]  # every third element negatively oriented
    p = str(tmp_path / "neg.msh")
    IO.write_gmsh(M.Mesh(3, m.VX, bad, m.lo, m.hi), p)
    r = IO.read_gmsh(p, 3)
    assert r.flipped == len(bad[::3])
    g = M.build_geometry(r, 2)
    assert np.all(g.Jq > 0)


def test_unpaired_points_are_boundary_points(tmp_path):
    """A box larger than the mesh: the mesh's outer faces no longer wrap onto
    each other.  Strict matching rejects the mesh; the reference's semantics
    make those face points their own neighbours."""
    m = M.periodic_square(4, 4)
    big = M.Mesh(2, m.VX, m.EToV, m.lo - 1.0, m.hi + 1.0)
    with pytest.raises(ValueError):
        M.build_geometry(big, 2)
    big.boundary_self = True
    g = M.build_geometry(big, 2)
    bf = IO.boundary_faces(g)
    assert bf.sum() == 2 * (4 + 4)  # the outer edges of the 4 x 4 quad grid
    # interior faces still pair between two elements
    assert bf.sum() < bf.size


def test_mfem_writer(tmp_path):
    m = M.periodic_square(3, 2)
    g = M.build_geometry(m, 2)
    p = str(tmp_path / "mesh.000000")
    IO.write_mfem(m, g, p)
    lines = open(p).read().splitlines()
    assert lines[0] == "MFEM mesh v1.0"
    i = lines.index("elements")
    assert int(lines[i + 1]) == m.K
    assert lines[i + 2].split() == ["1", "2", "0", "1", "2"]
    b = lines.index("boundary")
    assert int(lines[b + 1]) == 0  # fully periodic: no boundary faces
    v = lines.index("vertices")
    assert int(lines[v + 1]) == 3 * m.K and int(lines[v + 2]) == 2
    first = np.array([float(x) for x in lines[v + 3].split()])
    assert np.allclose(first, m.VX[m.EToV[0, 0]])
    # with boundaries: one boundary element per self-mapped face
    big = M.Mesh(2, m.VX, m.EToV, m.lo - 1.0, m.hi + 1.0, boundary_self=True)
    gb = M.build_geometry(big, 2)
    IO.write_mfem(big, gb, p)
    lines = open(p).read().splitlines()
    b = lines.index("boundary")
    nb = int(lines[b + 1])
    assert nb == int(IO.boundary_faces(gb).sum()) == 2 * (3 + 2)
    assert all(len(lines[b + 2 + k].split()) == 4 for k in range(nb))


def test_gmsh_reader_errors(tmp_path):
    with pytest.raises(capi.WadgError):
        IO.read_gmsh(str(tmp_path / "missing.msh"), 3)
    p = tmp_path / "bin.msh"
    p.write_text("$MeshFormat\n2.2 1 8\n$EndMeshFormat\n")
    with pytest.raises(capi.WadgError):
        IO.read_gmsh(str(p), 3)
    p.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n1\n1 0 0 0\n$EndNodes\n"
                 "$Elements\n1\n1 15 2 0 1 1\n$EndElements\n")
    with pytest.raises(capi.WadgError):  # no tetrahedra
        IO.read_gmsh(str(p), 3)


@pytest.mark.skipif(not os.path.isdir(REF_MESHES), reason="reference meshes not present")
@pytest.mark.parametrize("name,dim", [("periodicSquare1.msh", 2), ("periodicSquare2.msh", 2),
                                      ("periodicCubeTG1.msh", 3), ("periodicCube1.msh", 3),
                                      ("hole_tri.msh", 2)])
def test_reference_meshes(name, dim):
    """The reference's shipped meshes read, build positive Jacobians, and
    match their faces (periodic on the bounding box, boundaries self-mapped)."""
    m = IO.read_gmsh(os.path.join(REF_MESHES, name), dim)
    assert m.K > 0
    g = M.build_geometry(m, 2)
    assert np.all(g.Jq > 0)
    K, NF = g.mapPq.shape
    Nf = dim + 2
    mp = g.mapPq.astype(np.int64)
    e, j = mp // (NF * Nf), mp % (NF * Nf)
    back = g.mapPq.reshape(-1)[(j + e * NF).ravel()]
    assert np.array_equal(back, (np.arange(NF)[None, :] + np.arange(K)[:, None] * NF * Nf).ravel())
    if name.startswith("periodic"):
        assert IO.boundary_faces(g).sum() == 0
    else:
        assert IO.boundary_faces(g).sum() > 0
