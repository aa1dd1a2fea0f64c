"""GPU parity of the fused FBP filter (cosine weight + Ram-Lak ramp) against
the FP64 oracle restatement, its transpose, and the two FBP layers against the
reference's own torch formulation (StandardGeometry.py:51-65,
BeijingGeometry.py:57-64) on the same projector."""
import numpy as np
import pytest
import torch

import dtvb200
import oracle as O
from helpers import rel_rmse, vector_views

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,sdd", [((2, 1, 5, 7, 40), 1000.0), ((1, 1, 3, 16, 384), 800.0),
                                       ((1, 1, 2, 4, 6000), 1143.0)])
def test_filter_matches_oracle(cuda, shape, sdd):
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape).astype(np.float32)
    H, W = shape[-2], shape[-1]
    out = dtvb200.fbp_filter(torch.from_numpy(x).to(cuda), sdd, H, H / 2, W / 2).cpu().numpy()
    ref = O.fbp_filter(x, H, sdd, H / 2, W / 2)
    assert rel_rmse(out, ref) < 1e-6
    adj = dtvb200.fbp_filter(torch.from_numpy(x).to(cuda), sdd, H, H / 2, W / 2,
                             adjoint=True).cpu().numpy()
    assert rel_rmse(adj, O.fbp_filter(x, H, sdd, H / 2, W / 2, adjoint=True)) < 1e-6


def test_filter_transpose_and_errors(cuda):
    g = torch.Generator(device=cuda).manual_seed(2)
    x = torch.randn(1, 1, 4, 9, 64, device=cuda, generator=g)
    y = torch.randn(1, 1, 4, 9, 64, device=cuda, generator=g)
    fx = dtvb200.fbp_filter(x, 500.0, 9, 4.5, 32.0)
    fty = dtvb200.fbp_filter(y, 500.0, 9, 4.5, 32.0, adjoint=True)
    lhs, rhs = float((fx.double() * y.double()).sum()), float((x.double() * fty.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-5
    with pytest.raises(dtvb200.DtvError):
        dtvb200.fbp_filter(torch.zeros(1, 1, 2, 3, 33, device=cuda), 500.0, 3, 1.5, 16.5)


def _standard_case(cuda):
    ang = np.linspace(0, 360, 12, endpoint=False).astype(np.float32)
    geo = dtvb200.standard(ang, (24, 24, 12), (40, 16), 500.0, 1000.0)
    return geo, dtvb200.Projector(geo)


def test_standard_fbp_layer_matches_reference_formulation(cuda):
    geo, proj = _standard_case(cuda)
    layer = dtvb200.StandardGeometryWithFBP(proj, 1000.0).to(cuda)
    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.random(geo.vol_shape(1)).astype(np.float32)).to(cuda)
    p = torch.from_numpy(rng.random(geo.sino_shape(1)).astype(np.float32)).to(cuda)
    out = layer(x, p)
    # the reference's lines, in FP32 torch ops on the same projector
    res = proj.fp(x) - p
    res = res * layer.cosWeight
    b, c, a, h, w = res.shape
    prev = torch.backends.cudnn.allow_tf32
    torch.backends.cudnn.allow_tf32 = False
    try:
        res = torch.nn.functional.conv2d(res.view(b, c, a * h, w), layer.ramp, padding=(0, w // 2))
    finally:
        torch.backends.cudnn.allow_tf32 = prev
    ref = layer.lamb * proj.bp(res.view(b, c, a, h, w).contiguous())
    assert rel_rmse(out.cpu().numpy(), ref.cpu().numpy()) < 1e-5


def test_fbp_layer_gradient_is_the_transpose(cuda):
    geo, proj = _standard_case(cuda)
    rng = np.random.default_rng(4)
    s = torch.from_numpy(rng.random(geo.sino_shape(1)).astype(np.float32)).to(cuda)
    s.requires_grad_()
    y = torch.from_numpy(rng.random(geo.sino_shape(1)).astype(np.float32)).to(cuda)
    H, W = geo.detector_size[1], geo.detector_size[0]
    out = dtvb200.RampFilter.apply(s, 1000.0, H, H / 2, W / 2)
    (out * y).sum().backward()
    ref = O.fbp_filter(y.cpu().numpy(), H, 1000.0, H / 2, W / 2, adjoint=True)
    assert rel_rmse(s.grad.cpu().numpy(), ref) < 1e-6


def test_beijing_fbp_layer_matches_reference_formulation(cuda):
    """BeijingGeometry.py:17-18,31,38-39,57-64 restated in torch ops on the same
    projector: FP x sampleInterval, (view, plane) permutation, cosine weight
    and ramp along rows of W*planes, permutation back, FDK BP."""
    planes, angles, W, H, si = 3, 7, 10, 8, 1.7
    pv = vector_views(angles * planes, 40.0, 70.0, 1.6, 1.7)
    geo = dtvb200.vector(pv, (16, 14, 10), (W, H))
    proj = dtvb200.Projector(geo)
    layer = dtvb200.BeijingGeometryWithFBP(proj, 70.0, planes, sample_interval=si).to(cuda)
    rng = np.random.default_rng(5)
    x = torch.from_numpy(rng.random(geo.vol_shape(1)).astype(np.float32)).to(cuda)
    p = torch.from_numpy(rng.random(geo.sino_shape(1)).astype(np.float32)).to(cuda)
    out = layer(x, p)
    fp = (proj.fp(x) * si).reshape(angles, planes, H, W).permute(0, 2, 1, 3)
    res = (fp.reshape(1, 1, angles * planes, H, W) - p).view(1, 1, angles, H, W * planes)
    res = res * layer.cosWeight
    prev = torch.backends.cudnn.allow_tf32
    torch.backends.cudnn.allow_tf32 = False
    try:
        res = torch.nn.functional.conv2d(res.view(1, 1, angles * H, W * planes), layer.ramp,
                                         padding=(0, W * planes // 2))
    finally:
        torch.backends.cudnn.allow_tf32 = prev
    back = res.reshape(angles, H, planes, W).permute(0, 2, 1, 3).reshape(1, 1, angles * planes,
                                                                            H, W)
    ref = x - layer.lamb * proj.bp(back.contiguous())
    assert rel_rmse(out.cpu().numpy(), ref.cpu().numpy()) < 1e-5
