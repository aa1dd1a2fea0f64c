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


def test_noalloc_against_fp64_after_an_early_exit(cuda):
    """Checked against the FP64 threshold of the oracle rather than against the
    kernels it shares with dtv_l1ball. The first call has sum|v| < radius (the
    search stops at level 1 and returns v); the next call on the same shared
    array is an ordinary projection."""
    import oracle as O
    rng = np.random.default_rng(7)
    v1 = torch.from_numpy(rng.standard_normal(50_000).astype(np.float32)).to(cuda)
    big = torch.tensor([2.0 * float(v1.double().abs().sum())], dtype=torch.float64, device=cuda)
    w1, lam1 = _noalloc(v1, big, cuda)
    torch.cuda.synchronize()
    assert torch.equal(w1, v1) and float(lam1) == 0.0
    v2 = (rng.standard_normal(400_000) * 0.5).astype(np.float32)
    v2[rng.random(v2.size) < 0.1] = 0.0
    b = 0.25 * float(np.abs(v2.astype(np.float64)).sum())
    w2, lam2 = _noalloc(torch.from_numpy(v2).to(cuda),
                        torch.tensor([b], dtype=torch.float64, device=cuda), cuda)
    torch.cuda.synchronize()
    lam_ref = O.l1ball_lambda_exact(v2, b)
    assert abs(float(lam2) - lam_ref) <= 1e-6 * lam_ref
    ref = np.sign(v2) * np.maximum(np.abs(v2.astype(np.float64)) - lam_ref, 0.0)
    assert float(np.abs(w2.cpu().numpy() - ref).max()) <= TOL * max(1.0, float(np.abs(ref).max()))


def test_noalloc_rejects_oversized_input(cuda):
    v = torch.zeros(8, device=cuda)
    w = torch.empty_like(v)
    radius = torch.ones(1, dtype=torch.float64, device=cuda)
    L = _lib.load()
    # rejected on the host before any kernel runs
    rc = L.dtv_l1ball_noalloc(_ptr(v), _ptr(w), 2 ** 31, _ptr(radius), None, _stream(cuda))
    assert rc == _lib.DTV_ERR_INVALID
    assert b"exceeds the maximum" in L.dtv_last_error_message()
