"""GPU parity tests of the projector kernels through the C ABI: against the
FP64 oracle (same geometry), against the reference CUDA kernels' golden
outputs, the dot-product adjoint test, precision modes, epilogues, batching,
edge cases and the drop-in modules."""
import os

import numpy as np
import pytest
import torch

import dtvb200
import oracle as O
from dtvb200 import _lib
from helpers import blob_volume, rel_max, rel_rmse, vector_views

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def make_case(kind):
    """(library geometry, oracle geometry) pairs covering every phase rule."""
    if kind == "standard":
        ang = np.linspace(0, 360, 12, endpoint=False).astype(np.float32)
        vs, ds = (24, 20, 10), (33, 17)
        return (dtvb200.standard(ang, vs, ds, 500.0, 1000.0),
                O.standard_geometry(ang.astype(np.float64), vs, ds, 500.0, 1000.0))
    if kind == "standard_odd":
        ang = np.linspace(0, 360, 7, endpoint=False).astype(np.float32)
        vs, ds = (17, 23, 9), (29, 13)
        return (dtvb200.standard(ang, vs, ds, 300.0, 800.0),
                O.standard_geometry(ang.astype(np.float64), vs, ds, 300.0, 800.0))
    if kind == "vector":
        pv = vector_views(42, 40.0, 70.0, 1.6, 1.7, 1.5)
        vs, ds = (16, 14, 10), (20, 12)
        return dtvb200.vector(pv, vs, ds), O.vector_geometry(pv, vs, ds)
    if kind == "box":
        ang = np.linspace(0, 360, 10, endpoint=False)
        vs, ds, vox, pitch = (20, 18, 12), (28, 20), (1.0, 0.9, 1.2), (1.2, 1.1)
        return (dtvb200.circular(ang, vs, vox, ds, pitch, 500, 1000),
                O.circular_geometry(ang, vs, vox, ds, pitch, 500, 1000))
    raise ValueError(kind)


KINDS = ["standard", "standard_odd", "vector", "box"]


def to_dev(a, dev, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev, dtype)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("batch", [1, 2])
def test_forward_soft_matches_oracle(cuda, kind, batch):
    g, og = make_case(kind)
    plan = dtvb200.Plan(g, max_batch=2, device=cuda)
    rng = np.random.default_rng(10)
    vol = blob_volume(rng, og.vol_shape, batch)
    out = plan.forward(to_dev(vol, cuda)).cpu().numpy()
    ref = O.forward(og, vol).reshape(out.shape)
    # FP32 ray sums against FP64: tolerance 1e-5 relative RMSE, 1e-4 relative max
    assert rel_rmse(out, ref) < 1e-5
    assert rel_max(out, ref) < 1e-4


@pytest.mark.parametrize("kind", KINDS)
def test_forward_tex_matches_oracle_tex_mode(cuda, kind):
    g, og = make_case(kind)
    plan = dtvb200.Plan(g, max_batch=1, sampler="tex", device=cuda)
    vol = blob_volume(np.random.default_rng(11), og.vol_shape, 1)
    out = plan.forward(to_dev(vol, cuda)).cpu().numpy()
    refq = O.forward(og, vol, q=True).reshape(out.shape)
    ref = O.forward(og, vol).reshape(out.shape)
    # hardware filtering keeps 8 fractional weight bits
    assert rel_rmse(out, refq) < 5e-4
    assert rel_rmse(out, ref) < 5e-3


@pytest.mark.parametrize("kind", KINDS)
def test_forward_pairs_matches_oracle(cuda, kind):
    """z-pair sampler: FP16 planes, 1/256 x/y weights, exact z weights."""
    g, og = make_case(kind)
    plan = dtvb200.Plan(g, max_batch=2, sampler="pairs", device=cuda)
    vol = blob_volume(np.random.default_rng(21), og.vol_shape, 2)
    v16 = vol.astype(np.float16).astype(np.float32)
    out = plan.forward(to_dev(vol, cuda)).cpu().numpy()
    assert rel_rmse(out, O.forward(og, v16, q=2).reshape(out.shape)) < 5e-4
    assert rel_rmse(out, O.forward(og, vol).reshape(out.shape)) < 1e-3


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("share", [0, 3])
@pytest.mark.parametrize("batch", [1, 2])
def test_forward_tma_matches_oracle(cuda, kind, share, batch):
    """Shared-memory z-pair sampler: FP16 planes, FP16 x/y and FP32 z weights;
    with a share of the tiles through the texture unit (1/256 x/y weights)."""
    g, og = make_case(kind)
    plan = dtvb200.Plan(g, max_batch=2, sampler="tma", device=cuda)
    plan.set_tuning(_lib.DTV_TUNE_FP_TEX_SHARE, share)
    vol = blob_volume(np.random.default_rng(23), og.vol_shape, batch)
    v16 = vol.astype(np.float16).astype(np.float32)
    out = plan.forward(to_dev(vol, cuda)).cpu().numpy()
    assert plan.device_status() == 0
    assert rel_rmse(out, O.forward(og, v16).reshape(out.shape)) < (1e-4 if share == 0 else 5e-4)
    assert rel_rmse(out, O.forward(og, vol).reshape(out.shape)) < 1e-3


def test_forward_tma_all_texture_equals_pairs(cuda):
    g, og = make_case("standard_odd")
    vol = to_dev(blob_volume(np.random.default_rng(24), og.vol_shape, 1), cuda)
    tma = dtvb200.Plan(g, sampler="tma", device=cuda)
    tma.set_tuning(_lib.DTV_TUNE_FP_TEX_SHARE, 8)
    assert torch.equal(tma.forward(vol), dtvb200.Plan(g, sampler="pairs", device=cuda).forward(vol))
    with pytest.raises(dtvb200.DtvError):
        dtvb200.Plan(g, sampler="pairs", device=cuda).set_tuning(_lib.DTV_TUNE_FP_TEX_SHARE, 1)
    with pytest.raises(dtvb200.DtvError):
        tma.set_tuning(_lib.DTV_TUNE_FP_TEX_SHARE, 9)


def test_forward_tma_full_size_views(cuda):
    """Chunk schedules of a 128^3 volume on a 192^2 detector at every
    orientation class (axis-aligned, 45 degrees, both chunk axes and
    directions) against the soft sampler on the FP16-rounded volume."""
    n, nd = 128, 192
    ang = np.arange(0, 360, 7.5)
    g = dtvb200.circular(ang, (n, n, n), (1.0,) * 3, (nd, nd), (1.2, 1.2), 500.0, 1000.0)
    from dtvb200.phantom import ellipsoids
    x = ellipsoids((n, n, n), seed=5, device=cuda).half().float()
    ref = dtvb200.Plan(g, sampler="soft", device=cuda).forward(x).double()
    tma = dtvb200.Plan(g, sampler="tma", device=cuda)
    out = tma.forward(x).double()
    assert tma.device_status() == 0
    assert float(((out - ref) ** 2).mean().sqrt() / (ref ** 2).mean().sqrt()) < 1e-4
    assert float((out - ref).abs().max() / ref.abs().max()) < 1e-3


@pytest.mark.parametrize("sampler", ["soft", "tex", "pairs"])
def test_forward_ray_tiles_agree(cuda, sampler):
    """Every ray tile computes the same per-ray sums (bit-identical), with
    detector sizes that leave partial tiles in u and v."""
    g, og = make_case("standard_odd")
    plan = dtvb200.Plan(g, max_batch=2, sampler=sampler, device=cuda)
    vol = to_dev(blob_volume(np.random.default_rng(22), og.vol_shape, 2), cuda)
    key = _lib.DTV_TUNE_FP_RAY_TILE
    assert plan.get_tuning(key) == 0
    ref = plan.forward(vol).clone()
    for t in range(1, dtvb200.autotune.N_RAY_TILES):
        plan.set_tuning(key, t)
        assert torch.equal(plan.forward(vol), ref), t


@pytest.mark.parametrize("sampler", ["soft", "tex", "pairs"])
def test_forward_band_orders_agree(cuda, sampler):
    """Every forward block order (view by view, or bands of tile rows across
    views, with a partial last band) computes the same per-ray sums."""
    g, og = make_case("standard_odd")
    plan = dtvb200.Plan(g, max_batch=2, sampler=sampler, device=cuda)
    vol = to_dev(blob_volume(np.random.default_rng(25), og.vol_shape, 2), cuda)
    key = _lib.DTV_TUNE_FP_BAND
    assert plan.get_tuning(key) == 0  # a small staged volume runs view by view
    ref = plan.forward(vol).clone()
    for tile in (0, 6, 2):  # 16x16, 64x4 (four tile rows), 32x8 ray tiles
        plan.set_tuning(_lib.DTV_TUNE_FP_RAY_TILE, tile)
        for band in (0, 1, 3, 4096):
            plan.set_tuning(key, band)
            assert torch.equal(plan.forward(vol), ref), (tile, band)
    for bad in (-1, 4097):
        with pytest.raises(dtvb200.DtvError):
            plan.set_tuning(key, bad)
    with pytest.raises(dtvb200.DtvError):
        dtvb200.Plan(g, sampler="tma", device=cuda).set_tuning(key, 1)
    # a staged volume above 32 MB (FP32 quad records of 128^3) runs in bands
    big = dtvb200.circular([0.0, 90.0], (128, 128, 128), (1.0,) * 3, (64, 64), (2.0, 2.0), 500, 1000)
    assert dtvb200.Plan(big, sampler="soft", device=cuda).get_tuning(key) == 4
    t = dtvb200.autotune.tune(plan, key=key, reps=2, warmup=1, use_cache=False)
    assert sorted(t) == list(dtvb200.autotune.CANDIDATES[key])
    assert plan.get_tuning(key) == min(t, key=t.get)


def test_tuning_keys_and_autotune(cuda):
    g, og = make_case("standard")
    plan = dtvb200.Plan(g, sampler="pairs", device=cuda)
    key = _lib.DTV_TUNE_FP_RAY_TILE
    for bad in (-1, dtvb200.autotune.N_RAY_TILES):
        with pytest.raises(dtvb200.DtvError):
            plan.set_tuning(key, bad)
    with pytest.raises(dtvb200.DtvError):
        plan.set_tuning(99, 0)
    dtvb200.autotune.clear_cache()
    times = dtvb200.autotune.tune(plan, reps=3, warmup=1)
    assert sorted(times) == list(range(dtvb200.autotune.N_RAY_TILES))
    assert plan.get_tuning(key) == min(times, key=times.get)
    other = dtvb200.Plan(g, sampler="pairs", device=cuda)
    assert dtvb200.autotune.tune(other) == times  # cached: applied without timing
    assert other.get_tuning(key) == plan.get_tuning(key)
    adj = dtvb200.Plan(g, device=cuda, adjoint=True)
    t_adj = dtvb200.autotune.tune(adj, key=_lib.DTV_TUNE_ADJOINT, reps=2, warmup=1)
    assert sorted(t_adj) == [0, 1]
    assert adj.get_tuning(_lib.DTV_TUNE_ADJOINT) == min(t_adj, key=t_adj.get)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("sampler", ["soft", "tex", "pairs", "tma"])
def test_backward_fdk_matches_oracle(cuda, kind, sampler):
    g, og = make_case(kind)
    plan = dtvb200.Plan(g, max_batch=2, sampler=sampler, device=cuda)
    rng = np.random.default_rng(12)
    sino = rng.random((2, 1) + og.sino_shape).astype(np.float32)
    out = plan.backward(to_dev(sino, cuda)).cpu().numpy()
    if sampler == "soft":
        ref = O.backward(og, sino).reshape(out.shape)
        assert rel_rmse(out, ref) < 1e-5
        assert rel_max(out, ref) < 1e-4
    else:  # "tex" and "pairs" sample the sinogram through the same texture
        ref = O.backward(og, sino, q=True).reshape(out.shape)
        assert rel_rmse(out, ref) < 5e-4


@pytest.mark.parametrize("kind", ["standard_odd", "vector"])
@pytest.mark.parametrize("sampler", ["soft", "pairs"])
def test_backward_warp_layouts_agree(cuda, kind, sampler):
    """Every backprojector warp / quad layout computes the same voxels
    (z-affine and general maps, software and texture sampling)."""
    g, og = make_case(kind)
    plan = dtvb200.Plan(g, max_batch=2, sampler=sampler, device=cuda)
    key = _lib.DTV_TUNE_BP_WARP
    assert plan.get_tuning(key) == 4
    sino = to_dev(np.random.default_rng(26).random((2, 1) + og.sino_shape), cuda)
    ref = plan.backward(sino).clone()
    for w in range(5):
        plan.set_tuning(key, w)
        assert torch.equal(plan.backward(sino), ref), w
    for bad in (-1, 5):
        with pytest.raises(dtvb200.DtvError):
            plan.set_tuning(key, bad)
    t = dtvb200.autotune.tune(plan, key=key, reps=2, warmup=1, use_cache=False)
    assert sorted(t) == list(range(5)) and plan.get_tuning(key) == min(t, key=t.get)


def test_backward_accumulate(cuda):
    g, og = make_case("standard")
    plan = dtvb200.Plan(g, device=cuda)
    sino = to_dev(np.random.default_rng(13).random((1, 1) + og.sino_shape), cuda)
    a = plan.backward(sino)
    b = a.clone()
    plan.backward(sino, out=b, accumulate=True)
    assert torch.allclose(b, 2 * a, rtol=1e-6, atol=0)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("table,method", [(False, 0), (True, 0), (True, 1)])
def test_adjoint_matches_oracle_and_dot_test(cuda, kind, table, method):
    """method 0: brick scatter through shared memory; 1: cell records with
    vector atomics (needs the plan's adjoint tables)."""
    g, og = make_case(kind)
    plan = dtvb200.Plan(g, max_batch=2, device=cuda, adjoint=table)
    if table:
        plan.set_tuning(_lib.DTV_TUNE_ADJOINT, method)
    assert plan.get_tuning(_lib.DTV_TUNE_ADJOINT) == method
    rng = np.random.default_rng(14)
    y = rng.random((2, 1) + og.sino_shape).astype(np.float32)
    x = rng.random((2, 1) + og.vol_shape).astype(np.float32)
    aty = plan.adjoint(to_dev(y, cuda)).cpu().numpy()
    ref = O.adjoint(og, y).reshape(aty.shape)
    assert rel_rmse(aty, ref) < 1e-5
    ax = plan.forward(to_dev(x, cuda)).cpu().numpy()
    lhs = float((ax.astype(np.float64) * y).sum())
    rhs = float((x.astype(np.float64) * aty).sum())
    # <Ax, y> = <x, A^T y> to 1e-5 relative
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


@pytest.mark.parametrize("vdt", [torch.float16, torch.bfloat16])
def test_forward_16bit_inputs(cuda, vdt):
    g, og = make_case("box")
    plan = dtvb200.Plan(g, device=cuda)
    vol = blob_volume(np.random.default_rng(15), og.vol_shape, 1)
    v16 = to_dev(vol, cuda, vdt)
    out = plan.forward(v16).cpu().numpy()
    ref = O.forward(og, v16.float().cpu().numpy()).reshape(out.shape)
    assert rel_rmse(out, ref) < 1e-5  # exact on the rounded input
    assert rel_rmse(out, O.forward(og, vol).reshape(out.shape)) < (2e-3 if vdt == torch.float16 else 8e-3)


def test_forward_stage_f16(cuda):
    g, og = make_case("standard")
    plan = dtvb200.Plan(g, stage_f16=True, device=cuda)
    vol = blob_volume(np.random.default_rng(16), og.vol_shape, 1)
    out = plan.forward(to_dev(vol, cuda)).cpu().numpy()
    assert rel_rmse(out, O.forward(og, vol).reshape(out.shape)) < 1e-3


@pytest.mark.parametrize("sampler", ["soft", "tma"])
def test_forward_epilogues(cuda, sampler):
    g, og = make_case("standard_odd")
    plan = dtvb200.Plan(g, sampler=sampler, device=cuda)
    rng = np.random.default_rng(17)
    vol = to_dev(blob_volume(rng, og.vol_shape, 1), cuda)
    gs = to_dev(rng.random((1, 1) + og.sino_shape), cuda)
    fp = plan.forward(vol)
    acc = torch.zeros(1, dtype=torch.float64, device=cuda)
    res = plan.forward(vol, epilogue=_lib.DTV_EPI_RESIDUAL, g=gs, abs_sum=acc)
    assert torch.allclose(res, fp - gs, atol=1e-6)
    assert float(acc) == pytest.approx(float((fp - gs).abs().double().sum()), rel=1e-6)
    w0 = to_dev(rng.random((1, 1) + og.sino_shape), cuda)
    w = w0.clone()
    sigma = 0.3
    plan.forward(vol, out=w, epilogue=_lib.DTV_EPI_PDHG, g=gs, sigma=sigma)
    assert torch.allclose(w, (w0 + sigma * (fp - gs)) / (1 + sigma), atol=1e-6)


@pytest.mark.parametrize("sampler", ["soft", "tma"])
def test_rays_missing_the_volume_give_zero(cuda, sampler):
    # detector shifted far off axis: no ray meets the volume
    ang = np.array([0.0, 90.0], dtype=np.float32)
    g = dtvb200.standard(ang, (8, 8, 4), (16, 16), 500.0, 1000.0)
    g.views[:, 5] += 5000.0  # move the detector centres up along z
    plan = dtvb200.Plan(g, sampler=sampler, device=cuda)
    out = plan.forward(torch.ones(g.vol_shape(1), device=cuda))
    assert float(out.abs().max()) == 0.0


def test_determinism(cuda):
    g, og = make_case("box")
    plan = dtvb200.Plan(g, device=cuda)
    rng = np.random.default_rng(18)
    vol = to_dev(blob_volume(rng, og.vol_shape, 1), cuda)
    sino = to_dev(rng.random((1, 1) + og.sino_shape), cuda)
    assert torch.equal(plan.forward(vol), plan.forward(vol))
    assert torch.equal(plan.backward(sino), plan.backward(sino))
    a, b = plan.adjoint(sino), plan.adjoint(sino)  # float atomics: order may vary
    assert rel_max(a.cpu().numpy(), b.cpu().numpy()) < 1e-5


def test_input_validation(cuda):
    g, og = make_case("standard")
    plan = dtvb200.Plan(g, max_batch=1, device=cuda)
    vol = torch.zeros(g.vol_shape(1), device=cuda)
    with pytest.raises(RuntimeError, match="contiguous"):
        plan.forward(vol.transpose(3, 4))
    with pytest.raises(RuntimeError, match="max_batch"):
        plan.forward(torch.zeros(g.vol_shape(2), device=cuda))
    with pytest.raises(RuntimeError, match="CUDA"):
        plan.forward(vol.cpu())
    with pytest.raises(dtvb200.DtvError):
        plan.forward(vol, epilogue=_lib.DTV_EPI_RESIDUAL)  # needs g


def test_fp_samples_match_oracle(cuda):
    for kind in KINDS:
        g, og = make_case(kind)
        plan = dtvb200.Plan(g, device=cuda)
        assert plan.fp_samples() == O.fp_samples(og)


# ----------------------------------------------------------- reference golden outputs
def _ref_proj():
    p = os.path.join(GOLDEN, "ref_projectors.npz")
    if not os.path.exists(p):
        pytest.skip("ref_projectors.npz not generated yet")
    return np.load(p)


@pytest.mark.parametrize("name", ["s1", "s2", "s3"])
@pytest.mark.parametrize("sampler", ["soft", "tex", "pairs"])
def test_matches_reference_kernels_standard(cuda, name, sampler):
    """Through the drop-in module with the reference's argument list."""
    z = _ref_proj()
    import JITStandardGeometry as J
    X, Y, Z, W, H, n, b = (int(v) for v in z[f"{name}_sizes"])
    sid, sdd = (float(v) for v in z[f"{name}_geom"])
    ang = torch.from_numpy(z[f"{name}_angles"]).to(cuda)
    vs, ds = torch.tensor([X, Y, Z]).to(cuda), torch.tensor([W, H]).to(cuda)
    old = J._SAMPLER
    J._SAMPLER, J._plans = sampler, {}
    try:
        fp = J.forward(to_dev(z[f"{name}_vol"], cuda), ang, vs, ds, sid, sdd, 0)
        bp = J.backward(to_dev(z[f"{name}_sino_in"], cuda), ang, vs, ds, sid, sdd, 0)
    finally:
        J._SAMPLER, J._plans = old, {}
    assert fp.shape == z[f"{name}_fp"].shape and bp.shape == z[f"{name}_bp"].shape
    # the reference filters with 1/256 weights in float32 coordinates; "pairs"
    # also rounds the volume to FP16
    tol = {"tex": 5e-4, "soft": 5e-3, "pairs": 2e-3}[sampler]
    assert rel_rmse(fp.cpu().numpy(), z[f"{name}_fp"]) < tol
    assert rel_rmse(bp.cpu().numpy(), z[f"{name}_bp"]) < tol


@pytest.mark.parametrize("sampler", ["soft", "tex", "pairs"])
def test_matches_reference_kernels_vector(cuda, sampler):
    z = _ref_proj()
    import JITBeijingGeometry as J
    import JITStandardGeometry as JS
    X, Y, Z, W, H, n, b = (int(v) for v in z["v_sizes"])
    vs, ds = torch.IntTensor([X, Y, Z]).to(cuda), torch.IntTensor([W, H]).to(cuda)
    pv = torch.from_numpy(z["v_pv"]).to(cuda)
    import JITBeijingGeometry
    JITBeijingGeometry._SAMPLER, J._plans = sampler, {}
    try:
        fp = J.forward(to_dev(z["v_vol"], cuda), vs, ds, pv, 0)
        bp = J.backward(to_dev(z["v_sino_in"], cuda), vs, ds, pv, 0)
    finally:
        JITBeijingGeometry._SAMPLER, J._plans = JS._SAMPLER, {}
    tol = {"tex": 5e-4, "soft": 5e-3, "pairs": 2e-3}[sampler]
    assert rel_rmse(fp.cpu().numpy(), z["v_fp"]) < tol
    assert rel_rmse(bp.cpu().numpy(), z["v_bp"]) < tol


@pytest.mark.parametrize("name", ["s1", "s2", "s3"])
def test_reference_pairing_gradient_matches_reference_kernels(cuda, name):
    """The reference's own gradient: its ForwardProjection.backward is the FDK
    backprojection of the incoming gradient (StandardGeometry.py:17-21). The
    gradient of FP through the reference pairing, with the golden sinogram as
    the incoming gradient, equals what the reference kernels' backprojector
    gave for that sinogram."""
    z = _ref_proj()
    X, Y, Z, W, H, n, b = (int(v) for v in z[f"{name}_sizes"])
    sid, sdd = (float(v) for v in z[f"{name}_geom"])
    geo = dtvb200.standard(z[f"{name}_angles"].astype(np.float32), (X, Y, Z), (W, H), sid, sdd)
    FP, _ = dtvb200.make_functions(dtvb200.Projector(geo, sampler="tex", max_batch=b),
                                   matched=False)
    x = to_dev(z[f"{name}_vol"], cuda).requires_grad_()
    FP.apply(x).backward(to_dev(z[f"{name}_sino_in"], cuda))
    assert rel_rmse(x.grad.cpu().numpy(), z[f"{name}_bp"]) < 5e-4


def test_standard_layers_autograd(cuda):
    """Reference pairing: grad of FP is the FDK BP (StandardGeometry.py:17-21);
    matched pairing: grad of FP is the exact adjoint."""
    g, og = make_case("standard")
    proj = dtvb200.Projector(g)
    FP, BP = dtvb200.make_functions(proj, matched=False)
    x = to_dev(blob_volume(np.random.default_rng(19), og.vol_shape, 1), cuda).requires_grad_()
    y = FP.apply(x)
    gy = torch.rand_like(y)
    y.backward(gy)
    assert torch.allclose(x.grad, proj.bp(gy), rtol=1e-6, atol=1e-6)
    FPm, BPm = dtvb200.make_functions(proj, matched=True)
    x.grad = None
    FPm.apply(x).backward(gy)
    assert torch.allclose(x.grad, proj.adjoint(gy), rtol=1e-4, atol=1e-5)
    p = torch.rand_like(y)
    # the layer's value: x - lamb * BP(FP(x) - p)  (StandardGeometry.py:41-43)
    xn, pn = x.detach().cpu().numpy(), p.cpu().numpy()
    for matched, bp in ((False, O.backward), (True, O.adjoint)):
        layer = dtvb200.StandardGeometry(proj, matched=matched, lamb=0.7)
        out = layer(x.detach(), p)
        res = O.forward(og, xn).reshape(pn.shape) - pn
        ref = xn - 0.7 * bp(og, res).reshape(xn.shape)
        assert rel_rmse(out.cpu().numpy(), ref) < 1e-5


def test_gradcheck_matched_on_random_voxels(cuda):
    """Finite differences of L(x) = 0.5||Ax - p||^2 on 16 random voxels agree
    with the autograd gradient through the matched adjoint."""
    g, og = make_case("box")
    proj = dtvb200.Projector(g)
    FP, _ = dtvb200.make_functions(proj, matched=True)
    rng = np.random.default_rng(20)
    x = to_dev(blob_volume(rng, og.vol_shape, 1), cuda).double()
    p = torch.rand(g.sino_shape(1), device=cuda, dtype=torch.float64)

    def loss(xx):
        return 0.5 * float(((FP.apply(xx.float()).double() - p) ** 2).sum())

    xg = x.float().clone().requires_grad_()
    (0.5 * ((FP.apply(xg).double() - p) ** 2).sum()).backward()
    grad = xg.grad.double().flatten()
    idx = rng.choice(x.numel(), 16, replace=False)
    h = 1e-2
    for i in idx:
        e = torch.zeros_like(x).flatten()
        e[i] = h
        e = e.reshape(x.shape)
        fd = (loss(x + e) - loss(x - e)) / (2 * h)
        assert abs(fd - float(grad[i])) <= 2e-3 * max(1.0, abs(fd))
