"""Projector operators for torch: autograd Functions and the geometry layers.

Mirrors model/ConeBeamLayers/Standard/StandardGeometry.py and
model/ConeBeamLayers/Beijing/BeijingGeometry.py. Two pairings exist:

* the reference pairing (``matched=False``): ForwardProjection's gradient is
  the FDK backprojector and BackProjection's gradient is the forward
  projector, exactly as StandardGeometry.py:10-34 wires them (the FDK
  backprojector is NOT the transpose of the forward projector);
* the matched pairing (``matched=True``): the forward projector's gradient is
  its exact transpose (dtv_backward_adjoint), so unrolled networks get true
  gradients; checked by the dot-product test.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import call
from .geometry import Geometry, Plan, _ptr, _stream, check_input


class Projector:
    """Plans of one geometry, created lazily per (device, sampler) and grown
    to the largest batch seen."""

    def __init__(self, geometry: Geometry, sampler: str = "soft", stage_f16: bool = False,
                 max_batch: int = 1):
        self.geometry = geometry
        self.sampler = sampler
        self.stage_f16 = stage_f16
        self.max_batch = max_batch
        self._plans = {}

    def plan(self, device: torch.device, batch: int = 1, sampler: str = None) -> Plan:
        sampler = sampler or self.sampler
        key = (device.index, sampler)
        p = self._plans.get(key)
        if p is None or p.max_batch < batch:
            if p is not None:
                p.close()
            p = Plan(self.geometry, max(batch, self.max_batch), sampler, self.stage_f16, device,
                     adjoint=(sampler == "soft"))
            self._plans[key] = p
        return p

    def batch_of(self, t: torch.Tensor, volume: bool) -> int:
        per = int(np.prod(self.geometry.vol_shape(1) if volume else self.geometry.sino_shape(1)))
        return max(1, t.numel() // per)

    def fp(self, x: torch.Tensor) -> torch.Tensor:
        x = x.contiguous()
        return self.plan(x.device, self.batch_of(x, True)).forward(x)

    def bp(self, s: torch.Tensor) -> torch.Tensor:
        s = s.contiguous()
        return self.plan(s.device, self.batch_of(s, False)).backward(s)

    def adjoint(self, s: torch.Tensor) -> torch.Tensor:
        s = s.contiguous()
        return self.plan(s.device, self.batch_of(s, False), sampler="soft").adjoint(s)

    def fp_soft(self, x: torch.Tensor) -> torch.Tensor:
        x = x.contiguous()
        return self.plan(x.device, self.batch_of(x, True), sampler="soft").forward(x)


def plane_layout(geometry: Geometry, planes: int = None):
    """(to_layer, from_layer): the Beijing layers' sinogram layout.

    The projector's sinogram is [B,1,A*P,H,W] in (angle, plane, row, column)
    order. With ``planes`` = P, the Beijing layers hand out the same shape
    holding (angle, row, plane, column): each angle's H rows run across all P
    sub-detectors, as BeijingGeometry.py:18,23,31,39 permute it. Without
    ``planes`` both maps are the identity."""
    if not planes:
        return (lambda s: s), (lambda s: s)
    W, H = geometry.detector_size
    N = geometry.n_views
    if N % planes:
        raise ValueError(f"{N} views are not a whole number of angles of {planes} planes")
    A, P = N // planes, int(planes)

    def to_layer(s):
        B = s.shape[0]
        return s.reshape(B, A, P, H, W).permute(0, 1, 3, 2, 4).reshape(B, 1, N, H, W)

    def from_layer(s):
        B = s.shape[0]
        return s.reshape(B, A, H, P, W).permute(0, 1, 3, 2, 4).reshape(B, 1, N, H, W)

    return to_layer, from_layer


def make_functions(projector: Projector, matched: bool = False, planes: int = None,
                   sample_interval: float = 1.0):
    """(ForwardProjection, BackProjection) autograd Functions bound to a
    projector, with the reference pairing or the matched-adjoint pairing.

    ``planes`` and ``sample_interval`` give the Beijing layers' conventions
    (BeijingGeometry.py:13-39): sinograms in the layout of ``plane_layout``,
    and the forward projection scaled by the sample interval. As in the
    reference pairing, that scale multiplies ForwardProjection.forward and
    BackProjection.backward only (the FDK backprojector is unscaled); in the
    matched pairing the transposes carry it, so each pair stays exact."""
    to_layer, from_layer = plane_layout(projector.geometry, planes)
    s = float(sample_interval)

    def scaled(t):
        return t if s == 1.0 else t * s

    def fwd(x):
        return to_layer(scaled(projector.fp_soft(x) if matched else projector.fp(x)))

    def back(y):
        y = from_layer(y)
        return scaled(projector.adjoint(y)) if matched else projector.bp(y)

    class ForwardProjection(torch.autograd.Function):
        """StandardGeometry.py:10-21, BeijingGeometry.py:13-26."""

        @staticmethod
        def forward(ctx, input):
            return fwd(input)

        @staticmethod
        def backward(ctx, grad):
            return back(grad)

    class BackProjection(torch.autograd.Function):
        """StandardGeometry.py:23-34, BeijingGeometry.py:28-39 (matched: the
        adjoint A^T)."""

        @staticmethod
        def forward(ctx, input):
            return back(input)

        @staticmethod
        def backward(ctx, grad):
            return fwd(grad)

    return ForwardProjection, BackProjection


class StandardGeometry(torch.nn.Module):
    """x - lamb * BP(FP(x) - p)  (StandardGeometry.py:36-43)."""

    def __init__(self, projector: Projector, matched: bool = False, lamb: float = 1.0):
        super().__init__()
        self.FP, self.BP = make_functions(projector, matched)
        self.lamb = lamb

    def forward(self, x, p):
        residual = self.FP.apply(x) - p
        return x - self.lamb * self.BP.apply(residual)


class BeijingGeometry(torch.nn.Module):
    """-lamb * BP(FP(x) - p)  (BeijingGeometry.py:41-48), with the Beijing
    autograd pair: the forward projection times ``sample_interval`` and, with
    ``planes``, sinograms in the (angle, row, plane, column) layout the
    reference's layer uses (``plane_layout``)."""

    def __init__(self, projector: Projector, matched: bool = False, lamb: float = 10e-3,
                 sample_interval: float = 1.0, planes: int = None):
        super().__init__()
        self.FP, self.BP = make_functions(projector, matched, planes, sample_interval)
        self.lamb = lamb
        self.sample_interval = sample_interval
        self.planes = planes

    def forward(self, x, p):
        residual = self.FP.apply(x) - p
        return -self.lamb * self.BP.apply(residual)


def ramp_kernel(width: int) -> torch.Tensor:
    """Spatial Ram-Lak kernel of width+1 taps: 1/8 at the centre, 0 at even
    offsets, -1/(2 pi^2 n^2) at odd offsets n (StandardGeometry.py:83-93)."""
    f = np.ones((1, 1, 1, width + 1), dtype=np.float32)
    mid = np.floor(width / 2)
    for i in range(width + 1):
        if (i - mid) % 2 == 0:
            f[..., i] = 0
        else:
            f[..., i] = -0.5 / (np.pi * np.pi * (i - mid) * (i - mid))
        if i == mid:
            f[..., i] = 1 / 8
    return torch.from_numpy(f)


def cos_weight(n_views: int, detector_size, sdd: float) -> torch.Tensor:
    """sdd / sqrt(sdd^2 + (i-H/2)^2 + (j-W/2)^2) over the detector
    (StandardGeometry.py:68-74)."""
    W, H = detector_size
    i = np.arange(H)[:, None] - H / 2
    j = np.arange(W)[None, :] - W / 2
    w = (sdd / np.sqrt(sdd ** 2 + i ** 2 + j ** 2)).astype(np.float32)
    return torch.from_numpy(np.broadcast_to(w, (1, 1, n_views, H, W)).copy())


def fbp_filter(rows: torch.Tensor, sdd: float, rows_per_view: int, mid_i: float, mid_j: float,
               adjoint: bool = False) -> torch.Tensor:
    """Cosine weight and Ram-Lak ramp of the FBP layers in one kernel
    (dtv_fbp_filter): rows of the last dimension (even width), the cosine row
    index is (row number) mod rows_per_view."""
    check_input(rows, "rows")
    width = rows.shape[-1]
    out = torch.empty_like(rows)
    call("dtv_fbp_filter", _ptr(rows), _ptr(out), rows.numel() // width, int(rows_per_view),
         int(width), float(sdd), float(mid_i), float(mid_j), int(bool(adjoint)),
         _stream(rows.device))
    return out


class RampFilter(torch.autograd.Function):
    """The FBP filter as a differentiable op; its gradient is the transpose
    (ramp, then the cosine weight)."""

    @staticmethod
    def forward(ctx, rows, sdd, rows_per_view, mid_i, mid_j):
        ctx.args = (sdd, rows_per_view, mid_i, mid_j)
        return fbp_filter(rows.contiguous(), sdd, rows_per_view, mid_i, mid_j)

    @staticmethod
    def backward(ctx, grad):
        return (fbp_filter(grad.contiguous(), *ctx.args, adjoint=True), None, None, None, None)


class StandardGeometryWithFBP(torch.nn.Module):
    """lamb * BP(ramp * (cos * (FP(x) - p)))  (StandardGeometry.py:45-66).
    ``cosWeight`` and ``ramp`` are kept as the reference's frozen parameters
    (same state_dict keys); the weighting and filtering run fused in
    dtv_fbp_filter."""

    def __init__(self, projector: Projector, sdd: float, matched: bool = False):
        super().__init__()
        g = projector.geometry
        self.FP, self.BP = make_functions(projector, matched)
        self.lamb = torch.nn.Parameter(torch.tensor(1.0), requires_grad=False)
        self.cosWeight = torch.nn.Parameter(cos_weight(g.n_views, g.detector_size, sdd),
                                            requires_grad=False)
        self.ramp = torch.nn.Parameter(ramp_kernel(g.detector_size[0]), requires_grad=False)
        self.width, self.height = g.detector_size
        self.sdd = float(sdd)

    def forward(self, x, p):
        residual = self.FP.apply(x) - p
        residual = RampFilter.apply(residual, self.sdd, self.height, self.height / 2,
                                    self.width / 2)
        return self.lamb * self.BP.apply(residual)


class BeijingGeometryWithFBP(torch.nn.Module):
    """x - lamb * BP(filtered residual)  (BeijingGeometry.py:50-72). The
    residual comes in the layer layout (angle, row, plane, column), so each
    angle's rows span the W*planes columns of all sub-detectors; as in the
    reference it is weighted with the reference's midpoints (row offset from
    W*planes/2, column offset from H/2, BeijingGeometry.py:66-72) and
    ramp-filtered along those rows, then backprojected through the layer's
    BackProjection (which undoes the layout)."""

    def __init__(self, projector: Projector, sdd: float, planes: int, matched: bool = False,
                 sample_interval: float = 1.0):
        super().__init__()
        g = projector.geometry
        if g.n_views % planes:
            raise ValueError("the view count must be a multiple of planes")
        self.FP, self.BP = make_functions(projector, matched, planes, sample_interval)
        self.lamb = torch.nn.Parameter(torch.tensor(1.0), requires_grad=False)
        self.width, self.height = g.detector_size
        self.planes, self.angles = int(planes), g.n_views // planes
        self.sdd = float(sdd)
        row = self.width * self.planes
        i = np.arange(self.height)[:, None] - row / 2
        j = np.arange(row)[None, :] - self.height / 2
        cw = (self.sdd / np.sqrt(self.sdd ** 2 + i ** 2 + j ** 2)).astype(np.float32)
        self.cosWeight = torch.nn.Parameter(
            torch.from_numpy(np.broadcast_to(cw, (1, 1, self.angles, self.height, row)).copy()),
            requires_grad=False)
        self.ramp = torch.nn.Parameter(ramp_kernel(row), requires_grad=False)

    def forward(self, x, p):
        residual = self.FP.apply(x) - p
        shape = residual.shape
        rows = residual.reshape(shape[0], 1, self.angles, self.height, self.width * self.planes)
        rows = RampFilter.apply(rows, self.sdd, self.height, self.width * self.planes / 2,
                                self.height / 2)
        return x - self.lamb * self.BP.apply(rows.reshape(shape))
