"""The allocation-free OC entry point (edge_oc_update_static) against edge_oc_update.

The file name puts it last in collection, so in a full run it also exercises the library
after every other GPU test has used it on the same device; it passes on its own as well.
"""
import ctypes

import numpy as np
import pytest
import torch

import edge_to_b200 as eb
from edge_to_b200 import _lib

MAX_EL = 1 << 20


def _inputs(n, seed, zero_dr=False):
    g = torch.Generator().manual_seed(seed)
    rho = 0.02 + 0.96 * torch.rand(n, generator=g, dtype=torch.float64)
    dr = torch.zeros(n, dtype=torch.float64) if zero_dr else -10.0 * torch.rand(n, generator=g, dtype=torch.float64)
    return rho.cuda(), dr.cuda()


def _with_handle(k, rho, dr, A, vol, vf, move):
    out = torch.empty_like(rho)
    lam, steps, chg = ctypes.c_double(), ctypes.c_int(), ctypes.c_double()
    k._bind_stream()
    _lib.call("edge_oc_update", k.handle, _lib.ptr(rho), _lib.ptr(dr), A, vol, vf, move, _lib.ptr(out),
              ctypes.byref(lam), ctypes.byref(steps), ctypes.byref(chg))
    return out, lam.value, steps.value, chg.value


def _static(rho, dr, A, vol, vf, move):
    out = torch.empty_like(rho)
    lam, steps, chg = ctypes.c_double(), ctypes.c_int(), ctypes.c_double()
    _lib.call("edge_oc_update_static", rho.numel(), _lib.ptr(rho), _lib.ptr(dr), A, vol, vf, move, _lib.ptr(out),
              ctypes.byref(lam), ctypes.byref(steps), ctypes.byref(chg), _lib.stream_ptr())
    return out, lam.value, steps.value, chg.value


def _check_pair(a, b):
    out_a, lam_a, steps_a, chg_a = a
    out_b, lam_b, steps_b, chg_b = b
    assert steps_a == steps_b
    assert lam_a == pytest.approx(lam_b, rel=1e-12, abs=0)
    assert chg_a == pytest.approx(chg_b, rel=1e-9, abs=1e-300)
    torch.testing.assert_close(out_a, out_b, rtol=0, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(64, 32, 32), (120, 40), (1024, 1024)])
def test_static_oc_matches_handle_entry_two_calls(shape):
    """Two consecutive updates (the second from the first's design, as in the SIMP loop)
    through both entry points; (1024, 1024) is the largest size the workspace takes."""
    mesh = eb.CuStructuredMesh3D(*shape, *map(float, shape)) if len(shape) == 3 else \
        eb.CuStructuredMesh2D(*shape, *map(float, shape))
    k = eb.CuStructuredStiffnessKernel(mesh)
    n = k.n_elements
    assert n <= MAX_EL
    A = float(np.asarray(mesh.As).reshape(-1)[0])
    vol = float(mesh.volume)
    rho, dr = _inputs(n, seed=n)
    for call in range(2):
        ref = _with_handle(k, rho, dr, A, vol, 0.3, 0.2)
        got = _static(rho, dr, A, vol, 0.3, 0.2)
        _check_pair(got, ref)
        assert ref[2] > 10
        rho = got[0].clone()
        dr = _inputs(n, seed=n + call + 1)[1]


@pytest.mark.gpu
def test_static_oc_zero_sensitivity_fallback():
    """All-zero sensitivities take the reference's ocP = 1e-3 fallback in both entries."""
    mesh = eb.CuStructuredMesh2D(60, 20, 60.0, 20.0)
    k = eb.CuStructuredStiffnessKernel(mesh)
    n = k.n_elements
    A = float(np.asarray(mesh.As).reshape(-1)[0])
    rho, dr = _inputs(n, seed=3, zero_dr=True)
    for _ in range(2):
        _check_pair(_static(rho, dr, A, float(mesh.volume), 0.5, 0.2),
                    _with_handle(k, rho, dr, A, float(mesh.volume), 0.5, 0.2))


def test_static_oc_rejects_sizes_beyond_workspace():
    """Argument checks come before any device work, so this runs without a GPU."""
    dummy = ctypes.c_void_p(256)
    lam, steps, chg = ctypes.c_double(), ctypes.c_int(), ctypes.c_double()
    with pytest.raises(ValueError, match="exceeds the fixed OC workspace"):
        _lib.call("edge_oc_update_static", MAX_EL + 1, dummy, dummy, 1.0, 1.0, 0.5, 0.2, dummy, ctypes.byref(lam),
                  ctypes.byref(steps), ctypes.byref(chg), None)
    with pytest.raises(ValueError, match="n must be positive"):
        _lib.call("edge_oc_update_static", 0, dummy, dummy, 1.0, 1.0, 0.5, 0.2, dummy, ctypes.byref(lam),
                  ctypes.byref(steps), ctypes.byref(chg), None)
