"""The C-ABI library loads and exports every entry point include/wadg.h
declares; argument validation works without a GPU (no CUDA call is reached
for invalid arguments or K = 0)."""

import ctypes
import os
import re

import pytest

from scratch_wadge_b200 import build as B
from scratch_wadge_b200 import capi
from scratch_wadge_b200 import refops as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "wadg.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wadg_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def L():
    B.build()
    return capi.lib()


def test_exports_every_declared_symbol(L):
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n


def test_ctx_validation(L):
    ops = R.load(3, 3)
    h = ctypes.c_void_p()
    p = capi.params_for(ops)
    assert L.wadg_ctx_create(ctypes.byref(p), ctypes.byref(h)) == 0
    # K = 0 is a no-op; a null pointer is rejected before any launch
    assert L.wadg_euler_vol_3d(h, 0, *([None] * 15)) == 0
    assert L.wadg_euler_vol_3d(h, 10, *([None] * 15)) == 1
    assert b"null" in L.wadg_last_error()
    assert L.wadg_euler_update_3d(h, -1, None, None, None, 0.0, 0.0, 0.0, None, None, None, None) == 1
    # a 3D context refuses 2D kernels
    assert L.wadg_euler_surf_2d(h, 1, *([None] * 6)) == 1
    L.wadg_ctx_destroy(h)

    bad = capi.params_for(ops)
    bad.Nq = 22
    assert L.wadg_ctx_create(ctypes.byref(bad), ctypes.byref(h)) == 2
    bad = capi.params_for(ops)
    bad.N = 9
    assert L.wadg_ctx_create(ctypes.byref(bad), ctypes.byref(h)) == 2
    bad = capi.params_for(ops)
    bad.dim = 4
    assert L.wadg_ctx_create(ctypes.byref(bad), ctypes.byref(h)) == 1


def test_supported_degrees(L):
    for dim in (2, 3):
        mask = L.wadg_supported_degrees(dim)
        for N in (1, 2, 3, 4):
            assert mask & (1 << N)
            ops = R.load(dim, N)
            h = ctypes.c_void_p()
            p = capi.params_for(ops)
            assert L.wadg_ctx_create(ctypes.byref(p), ctypes.byref(h)) == 0
            L.wadg_ctx_destroy(h)


def test_diagnostic_and_halo_validation(L):
    """wadg_entropy_rhs and wadg_halo_pack reject bad arguments before any
    CUDA call; empty work is a no-op."""
    ops = R.load(3, 3)
    h = ctypes.c_void_p()
    p = capi.params_for(ops)
    assert L.wadg_ctx_create(ctypes.byref(p), ctypes.byref(h)) == 0
    # entropy balance: K < 0, K = 0, null arrays, curved without Jq
    assert L.wadg_entropy_rhs(h, -1, 0, *([None] * 6)) == 1
    assert L.wadg_entropy_rhs(h, 0, 0, *([None] * 6)) == 0
    assert L.wadg_entropy_rhs(h, 4, 0, *([None] * 6)) == 1
    assert L.wadg_entropy_rhs(h, 4, 1, 8, None, 8, 8, 8, 8) == 1  # curved reads Jq
    # halo pack: slot counts must be whole pseudo-elements (NfqNf = 48)
    assert L.wadg_halo_pack(h, 0, None, None, 0, None) == 0
    assert L.wadg_halo_pack(h, 47, 8, 8, 100, 8) == 1
    assert b"multiple" in L.wadg_last_error()
    assert L.wadg_halo_pack(h, -48, 8, 8, 100, 8) == 1
    assert L.wadg_halo_pack(h, 48, None, 8, 100, 8) == 1
    L.wadg_ctx_destroy(h)


def test_state_check_and_shape_validation(L):
    """wadg_check_state and wadg_kernel_shape reject bad arguments before any
    CUDA call; an empty state is physical."""
    ops = R.load(3, 3)
    h = ctypes.c_void_p()
    p = capi.params_for(ops)
    assert L.wadg_ctx_create(ctypes.byref(p), ctypes.byref(h)) == 0
    nbad, first = ctypes.c_int(7), ctypes.c_int(7)
    assert L.wadg_check_state(h, 0, None, None, ctypes.byref(nbad), ctypes.byref(first)) == 0
    assert nbad.value == 0 and first.value == -1
    assert L.wadg_check_state(h, -1, None, None, None, None) == capi.ERR_INVALID
    assert L.wadg_check_state(h, 4, None, 8, None, None) == capi.ERR_INVALID
    assert L.wadg_check_state(None, 4, 8, 8, None, None) == capi.ERR_INVALID
    E, g = ctypes.c_int(), ctypes.c_int()
    assert L.wadg_kernel_shape(h, 9, 0, 10, ctypes.byref(E), ctypes.byref(g)) == capi.ERR_INVALID
    assert b"unknown kernel" in L.wadg_last_error()
    assert L.wadg_kernel_shape(h, 0, 0, -1, ctypes.byref(E), ctypes.byref(g)) == capi.ERR_INVALID
    assert L.wadg_kernel_shape(h, 0, 0, 10, None, ctypes.byref(g)) == capi.ERR_INVALID
    L.wadg_ctx_destroy(h)
