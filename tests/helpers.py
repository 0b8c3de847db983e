"""Shared test helpers: golden fixtures, tolerances, state perturbations."""

import glob
import os

import numpy as np

from scratch_wadge_b200 import mesh as M
from scratch_wadge_b200 import refops as R

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Parity bar of the hot path: FP64, 1e-12 relative in the max norm.
RTOL = 1e-12


def rel(a, b):
    """max|a-b| / max|b| (max-norm relative difference)."""
    a, b = np.asarray(a), np.asarray(b)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def golden_names():
    """The stage fixtures (gen_golden.py); the geometry fixtures geo*.npz
    (gen_geometry.py) are read by tests/test_geometry.py."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith("geo"))


class Case:
    """A golden fixture: geometry, stage-0 state and reference outputs."""

    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.name = name
        self.z = {k: z[k] for k in z.files}
        self.dim, self.N = int(self.z["dim"]), int(self.z["N"])
        self.curved = bool(int(self.z["curved"]))
        self.dt = float(self.z["dt"])
        ops = R.load(self.dim, self.N)
        K = self.z["Jq"].shape[0]
        self.geo = M.Geometry(ops, K, self.z["vgeo"], self.z["vfgeo"], self.z["fgeo"],
                              self.z["Jq"], self.z["mapPq"].astype(np.uint32), None, None)

    @property
    def ops(self):
        return self.geo.ops

    def state(self):
        s = {k: self.z["in_" + k].copy() for k in ("Q", "rhsQ", "Qf", "resQ")}
        s["rhsQf"] = np.zeros_like(s["Qf"])
        return s


def perturbed(state, seed, amp=1e-2):
    """Seeded smooth-ish perturbation of a stage-0 state that keeps it
    physical (density and internal energy stay positive)."""
    rng = np.random.default_rng(seed)
    out = {}
    for k, v in state.items():
        if k == "rhsQf":
            out[k] = v.copy()
            continue
        f = 1.0 + amp * rng.standard_normal(v.shape)
        w = v * f
        out[k] = w
    return out
