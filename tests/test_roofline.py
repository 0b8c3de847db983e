"""The frozen per-pair flop counts of the roofline equal a fresh
counting-scalar evaluation of the reference formulas (oracle/flopcount.py)."""

import pytest

from oracle import flopcount
from scratch_wadge_b200 import roofline


@pytest.mark.parametrize("key", sorted(roofline.PAIR_FLOPS))
def test_pair_flops_frozen(key):
    dim, curved, series = key
    got = tuple(flopcount.pair_flops(dim, k, curved, series) for k in ("vv", "vf", "fv"))
    assert got == roofline.PAIR_FLOPS[key]


def test_element_flops_tg3d():
    # 3D N=3 affine (Nq=23, NfqNf=48): 529*140 + 2*1104*146
    assert roofline.vol_flops_per_element(3, 23, 48, False) == 529 * 140 + 2 * 1104 * 146
    assert roofline.pairs_per_element(23, 48) == 2737
