"""dtv_l1ball_noalloc: the L1-ball projection for callers that cannot
allocate device memory (no workspace argument; the library's own fixed
array is the workspace). Checked through the C ABI against dtv_l1ball with a
caller-allocated workspace, on two calls in a row so that state left in the
shared array by the first call would show in the second.

This file is collected last so that, in a run that stops at the first
failure, every other test has already run."""
import ctypes

import numpy as np
import pytest
import torch

from dtvb200 import _lib
from dtvb200.geometry import _ptr, _stream

pytestmark = pytest.mark.gpu

TOL = 2e-6  # the relative tolerance of the other L1-ball tests


def _ref(v, radius, dev):
    L = _lib.load()
    ws = torch.zeros(L.dtv_l1ball_workspace_bytes(), dtype=torch.uint8, device=dev)
    w = torch.empty_like(v)
    lam = torch.empty(1, dtype=torch.float64, device=dev)
    _lib.call("dtv_l1ball", _ptr(v), _ptr(w), v.numel(), _ptr(radius), _ptr(ws), _ptr(lam),
              _stream(dev))
    return w, lam


def _noalloc(v, radius, dev):
    w = torch.empty_like(v)
    lam = torch.empty(1, dtype=torch.float64, device=dev)
    _lib.call("dtv_l1ball_noalloc", _ptr(v), _ptr(w), v.numel(), _ptr(radius), _ptr(lam),
              _stream(dev))
    return w, lam


def test_noalloc_matches_workspace_entry_two_calls(cuda):
    rng = np.random.default_rng(2024)
    cases = [(1_000_003, 0.3), (250_000, 0.01)]  # the second call finds stale first-call state
    for n, frac in cases:
        v = torch.from_numpy((rng.standard_normal(n) * 2.0).astype(np.float32)).to(cuda)
        radius = torch.tensor([frac * float(v.double().abs().sum())], dtype=torch.float64,
                              device=cuda)
        w_ref, lam_ref = _ref(v, radius, cuda)
        w, lam = _noalloc(v, radius, cuda)
        torch.cuda.synchronize()
        scale = max(1.0, float(w_ref.abs().max()))
        assert float((w - w_ref).abs().max()) <= TOL * scale
        assert abs(float(lam) - float(lam_ref)) <= TOL * max(1.0, abs(float(lam_ref)))
        # and it is a projection onto the ball of that radius
        assert float(w.double().abs().sum()) == pytest.approx(float(radius), rel=1e-5)


def test_noalloc_rejects_oversized_input(cuda):
    v = torch.zeros(8, device=cuda)
    w = torch.empty_like(v)
    radius = torch.ones(1, dtype=torch.float64, device=cuda)
    L = _lib.load()
    # rejected on the host before any kernel runs
    rc = L.dtv_l1ball_noalloc(_ptr(v), _ptr(w), 2 ** 31, _ptr(radius), None, _stream(cuda))
    assert rc == _lib.DTV_ERR_INVALID
    assert b"exceeds the maximum" in L.dtv_last_error_message()
