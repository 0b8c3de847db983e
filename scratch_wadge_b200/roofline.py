"""Algorithmic work of each kernel, per element and per launch.

Volume kernel (FP64-pipe bound): flops of the reference algorithm per element,
Nq^2 volume pairs + Nq*NfqNf volume-face pairs + NfqNf*Nq face-volume pairs,
each pair at the per-pair count of the reference's arithmetic
(euler3d_flux with both log-means, the geometric contraction and the
accumulation; +,-,*,/,log each one flop, no fusion credit).  The per-pair
counts below come from a counting-scalar evaluation of the reference formulas
(oracle/flopcount.py; tests/test_roofline.py checks these frozen values
against it).  The series branch of the log-mean is the one the Taylor-Green
workload takes (density constant, inverse temperature varying by ~0.3%).

Surface and update kernels (HBM bound): algorithmic bytes per element, each
array read or written once per launch (FP64, 4-byte mapPq):
  surf   = 8*Nf*NfqNf [Qf; the plus-side gather re-reads a neighbour's
           trace, counted once] + 8*Nf*NfqNf [rhsQf]
           + 8*Nfgeo*NfqNf [fgeo] + 4*NfqNf [mapPq] + 16*Nf*Nq [rhsQ r/w]
  update = 8*Nf*Nq*(rhsQ r/w 2 + resQ r/w 2 + Q r/w 2) + 8*Nq [Jq]
           + 8*Nf*NfqNf [Qf write]
  vol    = 8*Nf*(Nq+NfqNf) in + 8*Nf*(Nq+NfqNf) out + geometric factors
           (8*Nvgeo*1 affine; 8*Nvgeo*(Nq+NfqNf) curved)
"""

# per ordered pair: {(dim, curved, series): (vv, vf, fv)}
PAIR_FLOPS = {
    (2, False, True): (120, 125, 125), (2, False, False): (106, 111, 111),
    (2, True, True): (128, 133, 133), (2, True, False): (114, 119, 119),
    (3, False, True): (140, 146, 146), (3, False, False): (132, 138, 138),
    (3, True, True): (158, 164, 164), (3, True, False): (150, 156, 156),
}


def vol_flops_per_element(dim, Nq, NfqNf, curved, series=True):
    vv, vf, fv = PAIR_FLOPS[(dim, bool(curved), bool(series))]
    return Nq * Nq * vv + Nq * NfqNf * vf + NfqNf * Nq * fv


def pairs_per_element(Nq, NfqNf):
    return Nq * Nq + 2 * Nq * NfqNf


def vol_bytes_per_element(dim, Nq, NfqNf, curved):
    Nf = dim + 2
    g = dim * dim * ((Nq + NfqNf) if curved else 1)
    return 8 * (2 * Nf * (Nq + NfqNf) + g)


def surf_bytes_per_element(dim, Nq, NfqNf):
    Nf = dim + 2
    return 8 * Nf * NfqNf + 8 * Nf * NfqNf + 8 * (dim + 1) * NfqNf + 4 * NfqNf + 16 * Nf * Nq


def update_bytes_per_element(dim, Nq, NfqNf):
    Nf = dim + 2
    return 8 * Nf * Nq * 6 + 8 * Nq + 8 * Nf * NfqNf


def stage_flops_per_element(dim, Nq, NfqNf, curved, series=True):
    """Algorithmic flops of the fused stage kernel per element: the volume
    pairs, the surface flux (one face-volume pair's count per face node), the
    lift VqLq*sfS and the update's matrix-vector products (2 flops per
    multiply-add; affine: -2 VqPq rhs, VfPq v, VqPq v; WADG adds two more
    Nq x Nq products).  VU/UV transcendentals are not counted."""
    Nf = dim + 2
    vf = PAIR_FLOPS[(dim, bool(curved), bool(series))][1]
    mm = 2 * Nf * (Nq * NfqNf + (Nq * Nq * (4 if curved else 2)) + NfqNf * Nq)
    return vol_flops_per_element(dim, Nq, NfqNf, curved, series) + NfqNf * vf + mm


def volsurf_flops_per_element(dim, Nq, NfqNf, curved, series=True):
    """Algorithmic flops of the volume + surface kernel per element: the
    volume pairs, the surface flux (one face-volume pair's count per face
    node) and the lift VqLq*sf (2 flops per multiply-add)."""
    Nf = dim + 2
    vf = PAIR_FLOPS[(dim, bool(curved), bool(series))][1]
    return vol_flops_per_element(dim, Nq, NfqNf, curved, series) + NfqNf * vf + 2 * Nf * Nq * NfqNf
