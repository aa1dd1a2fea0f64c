"""The correction passes of a texture-filtered z-pair plan ("pairs") against
the exact-weight plan ("exact") of the same geometry: the one-launch forward
and backward passes give the bits of the separate projections and
element-wise steps (the backward difference above 640 views within rounding),
DTVCP gives the same reconstruction either way, and mismatched plans are
refused."""
import numpy as np
import pytest
import torch

import dtvb200
from dtvb200 import _lib
from dtvb200.phantom import ellipsoids

pytestmark = pytest.mark.gpu


def plans(cuda, n=40, views=20, batch=1):
    ang = np.linspace(0, 360, views, endpoint=False)
    geo = dtvb200.circular(ang, (n, n, n), (1.0,) * 3, (60, 52), (1.2, 1.2), 500.0, 1000.0)
    fast = dtvb200.Plan(geo, max_batch=batch, sampler="pairs", device=cuda)
    exact = dtvb200.Plan(geo, max_batch=batch, sampler="exact", device=cuda)
    return fast, exact


def volumes(cuda, n, batch, dtype=torch.float32):
    v = torch.stack([ellipsoids((n, n, n), seed=s) for s in range(batch)]).unsqueeze(1)
    return v.to(cuda, dtype)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16])
@pytest.mark.parametrize("batch", [1, 2])
def test_forward_refresh_equals_separate_passes(cuda, dtype, batch):
    fast, exact = plans(cuda, batch=batch)
    vol = volumes(cuda, 40, batch, dtype)
    g = torch.rand(fast.sino_shape(batch), device=cuda) * 30
    w0 = torch.randn(fast.sino_shape(batch), device=cuda)
    sigma = 0.3
    e = exact.forward(vol)
    a = fast.forward(vol)
    w = w0.clone()
    g_eff = torch.full_like(g, float("nan"))
    s = torch.zeros(1, dtype=torch.float64, device=cuda)
    dtvb200.forward_refresh(fast, exact, vol, g, w, g_eff, sigma, s)
    assert torch.equal(g_eff, g + (a - e))
    # the dual step exactly as dtv_pdhg_sino_dual computes it
    w_ref = w0.clone()
    s_ref = torch.zeros(1, dtype=torch.float64, device=cuda)
    _lib.call("dtv_pdhg_sino_dual", w_ref.data_ptr(), e.data_ptr(), g.data_ptr(), sigma,
              w_ref.numel(), s_ref.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert torch.equal(w, w_ref)
    assert abs(s.item() - s_ref.item()) <= 1e-12 * s_ref.item()


@pytest.mark.parametrize("views,batch", [(20, 1), (20, 2), (700, 1)])  # 700: two view chunks
def test_backward_refresh_equals_separate_passes(cuda, views, batch):
    n = 40 if views == 20 else 16
    fast, exact = plans(cuda, n=n, views=views, batch=batch)
    sino = torch.rand(fast.sino_shape(batch), device=cuda)
    out = torch.full(fast.vol_shape(batch), float("nan"), device=cuda)
    e_b = torch.full_like(out, float("nan"))
    dtvb200.backward_refresh(fast, exact, sino, out, e_b)
    be = exact.backward(sino)
    bf = fast.backward(sino)
    assert torch.equal(out, be)
    if views <= 640:
        assert torch.equal(e_b, be - bf)
    else:
        # per chunk of 640 views, e_b adds that chunk's difference: the same
        # sum, rounded per chunk
        tol = 4 * torch.finfo(torch.float32).eps * be.abs().max()
        assert (e_b - (be - bf)).abs().max() <= tol


def test_refresh_passes_on_vector_geometry(cuda):
    """Per-view vector geometry with tilted detector rows (the backprojector's
    general projective path, not the z-affine one) and a wobbling source."""
    from helpers import vector_views
    geo = dtvb200.vector(vector_views(18, 40.0, 70.0, 1.6, 1.7, 1.5), (16, 14, 10), (20, 12))
    fast = dtvb200.Plan(geo, sampler="pairs", device=cuda)
    exact = dtvb200.Plan(geo, sampler="exact", device=cuda)
    rng = np.random.default_rng(4)
    vol = torch.from_numpy(rng.random(fast.vol_shape(1)).astype(np.float32)).to(cuda)
    g = torch.rand(fast.sino_shape(1), device=cuda)
    w = torch.zeros_like(g)
    g_eff = torch.empty_like(g)
    dtvb200.forward_refresh(fast, exact, vol, g, w, g_eff, 0.2)
    assert torch.equal(g_eff, g + (fast.forward(vol) - exact.forward(vol)))
    out, e_b = torch.empty_like(vol), torch.empty_like(vol)
    dtvb200.backward_refresh(fast, exact, w, out, e_b)
    be = exact.backward(w)
    assert torch.equal(out, be)
    assert torch.equal(e_b, be - fast.backward(w))


def test_backward_onto(cuda):
    fast, _ = plans(cuda)
    sino = torch.rand(fast.sino_shape(1), device=cuda)
    base = torch.randn(fast.vol_shape(1), device=cuda)
    ref = base + fast.backward(sino)
    out = fast.backward(sino, out=torch.empty_like(base), base=base)
    assert torch.equal(out, ref)
    same = base.clone()
    fast.backward(sino, out=same, base=same)  # base may be the output
    assert torch.equal(same, ref)


@pytest.mark.parametrize("use_graph,f_dtype", [(False, torch.float32), (True, torch.float32),
                                               (True, torch.float16)])
def test_dtvcp_fused_correction_equals_separate(cuda, use_graph, f_dtype):
    fast, exact = plans(cuda, n=40, views=24)
    truth = volumes(cuda, 40, 1)
    sino = fast.forward(truth)
    kw = dict(sigma=2e-3, tau=2e-3, mu=1.0, v=(0.5,) * 3, quirk=False, use_graph=use_graph,
              exact=exact, correct_every=3, f_dtype=f_dtype)
    fused = dtvb200.DTVCP(fast, 10, **kw)
    assert fused._fused()
    sep = dtvb200.DTVCP(fast, 10, **kw)
    sep.unfused = True
    f0 = torch.zeros(fast.vol_shape(1), device=cuda)
    a = fused.run(f0, sino)
    b = sep.run(f0, sino)
    assert torch.equal(a, b)
    la, lb = fused.losses.cpu(), sep.losses.cpu()
    assert torch.allclose(la, lb, rtol=1e-12, atol=0)


def test_refresh_refuses_mismatched_plans(cuda):
    fast, exact = plans(cuda)
    other_fast, other_exact = plans(cuda, views=21)
    vol = volumes(cuda, 40, 1)
    g = torch.zeros(fast.sino_shape(1), device=cuda)
    w, g_eff = torch.zeros_like(g), torch.zeros_like(g)
    with pytest.raises(dtvb200.DtvError, match="geometries differ"):
        dtvb200.forward_refresh(fast, other_exact, vol, g, w, g_eff, 0.1)
    with pytest.raises(dtvb200.DtvError, match="DTV_PLAN_PAIRS_EXACT"):
        dtvb200.forward_refresh(fast, fast, vol, g, w, g_eff, 0.1)
    with pytest.raises(dtvb200.DtvError, match="DTV_PLAN_TEX_PAIRS"):
        dtvb200.backward_refresh(exact, exact, g, torch.zeros(fast.vol_shape(1), device=cuda),
                                 torch.zeros(fast.vol_shape(1), device=cuda))
    vol_out = torch.zeros(fast.vol_shape(1), device=cuda)
    with pytest.raises(dtvb200.DtvError, match="different buffers"):
        dtvb200.backward_refresh(fast, exact, g, vol_out, vol_out)
    del other_fast
