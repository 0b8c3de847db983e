"""The reference-element operators the product builds from the node and
cubature point sets (scratch_wadge_b200/refbuild.py) equal the tables of the
reference's own builder (build_ref_ops_2D/3D, operators.cpp:104-341;
host_operators_new_2D/3D, operators_c.cpp:46-69, 212-241), compiled from its
sources by tests/golden/gen_refops.py into tests/golden/refops/, for every
degree 1..5 in 2D and 3D."""

import os

import numpy as np
import pytest

from scratch_wadge_b200 import refbuild as B
from scratch_wadge_b200 import refops as R
from tests.helpers import GOLDEN

# both sides are float64 linear algebra on the same point sets; the largest
# difference over all tables and degrees is 1.9e-14 (N = 5)
TOL = 5e-14


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
def test_built_tables_equal_the_reference_builder(dim, N):
    with np.load(os.path.join(GOLDEN, "refops", f"refops_{dim}d_N{N}.npz")) as z:
        ref = {k: z[k] for k in z.files}
    out = B.build(dim, N)
    assert out["sizes"].tolist() == ref["sizes"].tolist()
    assert set(out) == set(ref)
    for k, v in out.items():
        if k == "sizes":
            continue
        w = ref[k]
        assert v.shape == w.shape, k
        den = np.abs(w).max() if w.size and np.abs(w).max() > 0 else 1.0
        assert np.abs(v - w).max() / den < TOL, (k, np.abs(v - w).max() / den)


def test_load_builds_from_the_point_sets():
    ops = R.load(3, 3)
    assert (ops.Np, ops.Nq, ops.Nfq, ops.Nfaces, ops.NfqNf) == (20, 23, 12, 4, 48)
    # exactness of the cubature the builder assumed: M = Vq^T W Vq = I for the
    # orthonormal basis, so Pq Vq = I
    assert np.abs(ops.Pq @ ops.Vq - np.eye(ops.Np)).max() < 1e-13
    # Gauss-Legendre: 2D faces integrate x^(2n+1) exactly
    x, w = B.gauss_legendre(4)
    assert abs(w.sum() - 2.0) < 1e-14 and abs((w * x ** 8).sum() - 2.0 / 9.0) < 1e-14
