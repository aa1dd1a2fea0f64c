"""Precision gates against the FP64 oracle (relative RMSE <= 1e-3 for every
projection and reconstruction mode), on a reduced copy of the sparse-view DTV
configuration, plus size-independent properties at the full configuration
(256^3, 64 views of 384^2 at 1.2 mm)."""
import numpy as np
import pytest
import torch

import dtvb200
from dtvb200 import _lib
import oracle as O
from dtvb200.phantom import ellipsoids
from helpers import rel_rmse

pytestmark = pytest.mark.gpu

GATE = 1e-3  # relative RMSE against FP64


def reduced(cuda, n=48, views=12):
    nd = int(n * 1.5)
    ang = np.linspace(0, 360, views, endpoint=False)
    args = (ang, (n, n, n), (1.0, 1.0, 1.0), (nd, nd), (1.2, 1.2), 500.0, 1000.0)
    geo = dtvb200.circular(*args)
    og = O.circular_geometry(*args)
    truth = ellipsoids((n, n, n), seed=3).numpy()
    return geo, og, truth


@pytest.mark.parametrize("sampler", ["soft", "tex", "pairs", "tma"])
def test_projection_gate(cuda, sampler):
    geo, og, truth = reduced(cuda)
    plan = dtvb200.Plan(geo, sampler=sampler, device=cuda)
    out = plan.forward(torch.from_numpy(truth).to(cuda)).cpu().numpy()
    ref = O.forward(og, truth).reshape(out.shape)
    assert rel_rmse(out, ref) < GATE
    sino = ref.astype(np.float32)
    bp = plan.backward(torch.from_numpy(sino).to(cuda)).cpu().numpy()
    assert rel_rmse(bp, O.backward(og, sino).reshape(bp.shape)) < GATE


@pytest.mark.parametrize("sampler,fdt", [("soft", torch.float32), ("tex", torch.float32),
                                         ("pairs", torch.float32), ("tex", torch.float16),
                                         ("pairs", torch.float16), ("pairs", torch.bfloat16),
                                         ("tma", torch.float32), ("tma", torch.float16)])
def test_dtv_reconstruction_gate(cuda, sampler, fdt):
    geo, og, truth = reduced(cuda)
    sino = O.forward(og, truth).reshape(1, 1, *og.sino_shape)
    iters, sigma = 15, 2e-3
    prm = dict(sigma=sigma, tau=sigma, mu=1.0, v=(0.5, 0.5, 0.5), quirk=False)
    fp = lambda x: O.forward(og, x).reshape(x.shape[0], 1, *og.sino_shape)  # noqa: E731
    bp = lambda s: O.backward(og, s).reshape(s.shape[0], 1, *og.vol_shape)  # noqa: E731
    ref = O.dtvcp_run(fp, bp, np.zeros((1, 1) + og.vol_shape), sino, geo.volume_size, iters,
                      sigma, sigma, 1.0, (0.5, 0.5, 0.5), quirk=False)
    plan = dtvb200.Plan(geo, sampler=sampler, device=cuda)
    alg = dtvb200.DTVCP(plan, iters, f_dtype=fdt, use_graph=True, **prm)
    f = alg.run(torch.zeros(plan.vol_shape(1), device=cuda),
                torch.from_numpy(sino.astype(np.float32)).to(cuda)).cpu().numpy()
    assert float(np.abs(ref).max()) > 0
    assert rel_rmse(f, ref) < GATE


@pytest.fixture(scope="module")
def full(cuda):
    n, nd = 256, 384
    ang = np.linspace(0, 360, 64, endpoint=False)
    geo = dtvb200.circular(ang, (n, n, n), (1.0,) * 3, (nd, nd), (1.2, 1.2), 500.0, 1000.0)
    x = ellipsoids((n, n, n), seed=7, device=cuda)
    return geo, x


def test_full_size_linearity_and_samplers(cuda, full):
    geo, x = full
    soft = dtvb200.Plan(geo, sampler="soft", device=cuda)
    y = torch.rand_like(x)
    a, b = 0.7, -1.3
    lhs = soft.forward(a * x + b * y)
    rhs = a * soft.forward(x) + b * soft.forward(y)
    assert float(((lhs - rhs).double() ** 2).mean().sqrt() / (rhs.double() ** 2).mean().sqrt()) < 1e-5
    ref = soft.forward(x).double()
    for sampler in ("tex", "pairs", "tma"):
        out = dtvb200.Plan(geo, sampler=sampler, device=cuda).forward(x).double()
        assert float(((out - ref) ** 2).mean().sqrt() / (ref ** 2).mean().sqrt()) < GATE


@pytest.mark.parametrize("table,method", [(False, 0), (True, 1)])
def test_full_size_adjoint_dot_test(cuda, full, table, method):
    geo, x = full
    soft = dtvb200.Plan(geo, sampler="soft", device=cuda, adjoint=table)
    if table:
        soft.set_tuning(_lib.DTV_TUNE_ADJOINT, method)
    g = torch.Generator(device=cuda).manual_seed(3)
    y = torch.rand(soft.sino_shape(1), device=cuda, generator=g)
    lhs = float((soft.forward(x).double() * y.double()).sum())
    rhs = float((x.double() * soft.adjoint(y).double()).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_full_size_chords_of_a_uniform_volume(cuda, full):
    """FP of the all-ones volume is each ray's chord length through the box
    (to within one sample step)."""
    geo, x = full
    soft = dtvb200.Plan(geo, sampler="soft", device=cuda)
    ones = torch.ones_like(x)
    s = soft.forward(ones)
    assert float(s.max()) <= 256 * np.sqrt(3) + 1.0
    assert float(s.max()) >= 256.0
    # the central ray of view 0 crosses 256 voxels
    nd = 384
    centre = s[0, 0, 0, nd // 2 - 1:nd // 2 + 1, nd // 2 - 1:nd // 2 + 1]
    assert torch.all((centre - 256.0).abs() < 2.0)


def test_large_scan_downsample_gate(cuda):
    """The 512^3 / 1024x768 @ 0.8 mm configuration downsampled to 128^3 and 64
    views (voxel 4 mm, detector 256x192 at 3.2 mm: the same field of view):
    projections, FDK backprojection and 10 DTV iterations with BF16-stored
    volumes against the FP64 oracle."""
    ang = np.linspace(0, 360, 64, endpoint=False)
    args = (ang, (128, 128, 128), (4.0,) * 3, (256, 192), (3.2, 3.2), 500.0, 1000.0)
    geo, og = dtvb200.circular(*args), O.circular_geometry(*args)
    truth = ellipsoids((128, 128, 128), seed=9).numpy()
    plan = dtvb200.Plan(geo, sampler="pairs", device=cuda)
    x16 = torch.from_numpy(truth).to(cuda, torch.bfloat16)
    sino = plan.forward(x16).cpu().numpy()
    ref = O.forward(og, truth).reshape(sino.shape)
    # BF16 storage of the volume (8 significand bits), FP32 accumulation
    assert rel_rmse(sino, ref) < GATE
    assert rel_rmse(sino, O.forward(og, x16.float().cpu().numpy()).reshape(sino.shape)) < GATE
    bp = plan.backward(torch.from_numpy(ref.astype(np.float32)).to(cuda)).cpu().numpy()
    assert rel_rmse(bp, O.backward(og, ref.astype(np.float32)).reshape(bp.shape)) < GATE
    iters, sigma = 10, 2e-4
    fp = lambda x: O.forward(og, x).reshape(x.shape[0], 1, *og.sino_shape)  # noqa: E731
    bpo = lambda s: O.backward(og, s).reshape(s.shape[0], 1, *og.vol_shape)  # noqa: E731
    rec_ref = O.dtvcp_run(fp, bpo, np.zeros((1, 1) + og.vol_shape), ref, geo.volume_size, iters,
                          sigma, sigma, 1.0, (0.5, 0.5, 0.5), quirk=False)
    alg = dtvb200.DTVCP(plan, iters, sigma=sigma, tau=sigma, mu=1.0, v=(0.5, 0.5, 0.5),
                        quirk=False, f_dtype=torch.bfloat16, use_graph=True)
    rec = alg.run(torch.zeros(plan.vol_shape(1), device=cuda),
                  torch.from_numpy(ref.astype(np.float32)).to(cuda)).cpu().numpy()
    assert rel_rmse(rec, rec_ref) < GATE



def test_headline_fp64_check(cuda):
    """The FP64 check that bench.py prints beside the headline number, run as a
    test: the sparse-view DTV workload's forward projection and FDK
    backprojection of its phantom at full size (16 of 64 views), and its
    100-iteration reconstruction on the same-FOV 64^3 downsample, with FP32
    and FP16 fbar storage and the texture-filtered operators corrected by the
    exact-weight plan every 8 iterations, each within 1e-3 relative RMSE of
    the FP64 oracle. Uncorrected, the texture filter's 8-bit weights leave
    the reconstruction several 1e-3 away (recorded, not gated)."""
    import bench
    c = dict(bench.CFG)
    geo, truth, _ = bench.make_problem(cuda, c, c["seed"])
    plan = dtvb200.Plan(geo, max_batch=1, sampler="pairs", device=cuda)
    sino_clean = plan.forward(truth)
    chk = bench.fp64_check(c, cuda, "pairs", plan, truth, sino_clean,
                           [("fp32_f", torch.float32, 8), ("fp16_fbar", torch.float16, 8),
                            ("uncorrected", torch.float32, 0)])
    print("headline FP64 check:", chk["forward_full_size"], chk["backward_full_size"],
          chk["reconstruction"])
    assert chk["forward_full_size"] < GATE and chk["backward_full_size"] < GATE
    for name in ("fp32_f", "fp16_fbar"):
        assert chk["reconstruction"][name] < GATE, (name, chk["reconstruction"])
    assert chk["reconstruction"]["uncorrected"] > chk["reconstruction"]["fp32_f"]


@pytest.mark.parametrize("sampler", ["exact", "soft"])
def test_exact_weight_reconstruction_gate(cuda, sampler):
    """Samplers with FP32 interpolation weights in both directions: the
    100-iteration reconstruction of the same-FOV downsample within 1e-4 of
    FP64 (FP16-stored z pairs for "exact", FP32 for "soft")."""
    import bench
    from dtvb200.phantom import poisson_noise
    ang = np.linspace(0, 360, 64, endpoint=False)
    args = (ang, (64, 64, 64), (4.0,) * 3, (96, 96), (4.8, 4.8), 500.0, 1000.0)
    geo, og = dtvb200.circular(*args), O.circular_geometry(*args)
    plan = dtvb200.Plan(geo, sampler=sampler, device=cuda)
    truth = ellipsoids((64, 64, 64), seed=2024, device=cuda)
    sino = poisson_noise(plan.forward(truth), 1e5, seed=2024)
    prm = bench.dtv_params(plan, cuda)
    fp = lambda x: O.forward(og, x).reshape(x.shape[0], 1, *og.sino_shape)  # noqa: E731
    bp = lambda s: O.backward(og, s).reshape(s.shape[0], 1, *og.vol_shape)  # noqa: E731
    ref = O.dtvcp_run(fp, bp, np.zeros((1, 1, 64, 64, 64)), sino.cpu().numpy(), (64, 64, 64),
                      100, prm["sigma"], prm["tau"], prm["mu"], prm["v"], quirk=False)
    alg = dtvb200.DTVCP(plan, 100, use_graph=True, **prm)
    f = alg.run(torch.zeros(plan.vol_shape(1), device=cuda), sino).cpu().numpy()
    assert rel_rmse(f, ref) < 1e-4


def test_exact_sampler_parity(cuda):
    """The exact sampler against the FP64 oracle on the FP16-rounded volume
    (forward, every phase rule) and on the sinogram (backward)."""
    from helpers import vector_views
    ang = np.linspace(0, 360, 10, endpoint=False)
    cases = [
        (dtvb200.circular(ang, (20, 18, 12), (1.0, 0.9, 1.2), (28, 20), (1.2, 1.1), 500, 1000),
         O.circular_geometry(ang, (20, 18, 12), (1.0, 0.9, 1.2), (28, 20), (1.2, 1.1), 500,
                             1000)),
        (dtvb200.standard(ang.astype(np.float32), (24, 20, 10), (33, 17), 500.0, 1000.0),
         O.standard_geometry(ang, (24, 20, 10), (33, 17), 500.0, 1000.0)),
    ]
    pv = vector_views(42, 40.0, 70.0, 1.6, 1.7, 1.5)
    cases.append((dtvb200.vector(pv, (16, 14, 10), (20, 12)),
                  O.vector_geometry(pv, (16, 14, 10), (20, 12))))
    rng = np.random.default_rng(8)
    for geo, og in cases:
        plan = dtvb200.Plan(geo, sampler="exact", device=cuda)
        x = rng.random((1, 1) + og.vol_shape).astype(np.float32)
        out = plan.forward(torch.from_numpy(x).to(cuda)).cpu().numpy()
        x16 = x.astype(np.float16).astype(np.float64)
        assert rel_rmse(out, O.forward(og, x16).reshape(out.shape)) < 1e-6
        s = rng.random(out.shape).astype(np.float32)
        bp = plan.backward(torch.from_numpy(s).to(cuda)).cpu().numpy()
        assert rel_rmse(bp, O.backward(og, s).reshape(bp.shape)) < 1e-6
