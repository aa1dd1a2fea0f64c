"""Directional finite differences and the L1-ball projection on the GPU.

Restates model/PDHG/Utils/Gradients.py (sparse D_x, D_y, D_z and their
transposes, applied per batch item) and model/PDHG/Utils/L1ball.py as
kernels of the C ABI. ``quirk=True`` keeps the reference's y operator
(offset volumeSize[1] over the flat index, wrapping the last row of a slice
into the next slice, Gradients.py:18-25).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import call
from .geometry import _ptr, _stream, check_input


def size_of(t: torch.Tensor):
    """(X, Y, Z) of a [..., Z, Y, X] tensor and the batch count."""
    Z, Y, X = t.shape[-3:]
    return (X, Y, Z), t.numel() // (X * Y * Z)


def diff(f: torch.Tensor, axis: int, transpose: bool = False, quirk: bool = True,
         out: torch.Tensor = None) -> torch.Tensor:
    """D_axis f (or D_axis^T f) per batch item; axis 0,1,2 = x,y,z."""
    check_input(f, "f")
    size, b = size_of(f)
    if out is None:
        out = torch.empty_like(f)
    call("dtv_diff", _ptr(f), _ptr(out), _lib.ivec(size), b, int(axis), int(bool(transpose)),
         int(bool(quirk)), _stream(f.device))
    return out


def diff_abs_sums(f: torch.Tensor, quirk: bool = True, out: torch.Tensor = None) -> torch.Tensor:
    """[sum|D_x f|, sum|D_y f|, sum|D_z f|] as a float64 CUDA tensor (adds into out)."""
    check_input(f, "f", dtypes=(torch.float32, torch.float16))
    size, b = size_of(f)
    if out is None:
        out = torch.zeros(3, dtype=torch.float64, device=f.device)
    dt = _lib.DTV_F32 if f.dtype == torch.float32 else _lib.DTV_F16
    call("dtv_diff_abs_sums", _ptr(f), dt, _lib.ivec(size), b, int(bool(quirk)), _ptr(out),
         _stream(f.device))
    return out


_l1_ws = {}


def l1ball(v: torch.Tensor, b, workspace: torch.Tensor = None):
    """Projection onto {||w||_1 <= b} as L1ball.py:4-17 defines it: w = v when
    sum|v| < b, else sign(v)*max(|v| - lambda, 0) with sum max(|v|-lambda,0) = b.
    Returns (w, lambda) with lambda a float64 CUDA scalar tensor."""
    check_input(v, "v")
    dev = v.device
    if not torch.is_tensor(b):
        b = torch.tensor([float(b)], dtype=torch.float64, device=dev)
    check_input(b, "b", dtypes=(torch.float64,))
    if workspace is None:
        ws = _l1_ws.get(dev.index)
        if ws is None:
            nbytes = _lib.load().dtv_l1ball_workspace_bytes()
            ws = torch.zeros(nbytes, dtype=torch.uint8, device=dev)
            _l1_ws[dev.index] = ws
        workspace = ws
    w = torch.empty_like(v)
    lam = torch.empty(1, dtype=torch.float64, device=dev)
    call("dtv_l1ball", _ptr(v), _ptr(w), v.numel(), _ptr(b), _ptr(workspace), _ptr(lam),
         _stream(dev))
    return w, lam
