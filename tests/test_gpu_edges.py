"""GPU parity tests on degenerate and ragged shapes: one voxel, one z-slice,
a one-voxel column, one detector pixel, one detector row, one view, and sizes
one past every tile edge of the kernels (64 x 4 update tiles, 16 x 16
projector tiles, 8-slice z runs). Every sampler, the FDK backprojector, both
exact adjoints and the PDHG / L1-ball updates are compared with the FP64
oracle on the same inputs.

The exact (software) sampler and both adjoints are held to 1e-5 here, as on
the larger cases. The texture-filtered paths keep 8 fractional weight bits, so
each fetch may be off by up to 2^-9 of its neighbours' differences. With one
to three views, or a handful of samples per ray, that rounding does not
average out, so they are held to QTOL (their quantisation model is pinned at
5e-4 on the larger cases of test_gpu_projectors.py). The shared-memory z-pair
sampler's FP16 x/y weights are held to 5e-4."""
import ctypes

import numpy as np
import pytest
import torch

import dtvb200
import oracle as O
from dtvb200 import _lib
from helpers import blob_volume, rel_max, rel_rmse, vector_views

pytestmark = pytest.mark.gpu


def edge_case(kind):
    """(library geometry, oracle geometry) for one degenerate shape."""
    ang = lambda n: np.linspace(0, 360, n, endpoint=False)  # noqa: E731
    if kind == "voxel":  # a single voxel
        vs, ds = (1, 1, 1), (6, 5)
        a = ang(5).astype(np.float32)
        return (dtvb200.standard(a, vs, ds, 500.0, 1000.0),
                O.standard_geometry(a.astype(np.float64), vs, ds, 500.0, 1000.0))
    if kind == "slice":  # one z-slice
        vs, vox, ds, pitch = (13, 11, 1), (1.0, 1.0, 1.0), (21, 5), (1.1, 1.3)
        return (dtvb200.circular(ang(6), vs, vox, ds, pitch, 500, 1000),
                O.circular_geometry(ang(6), vs, vox, ds, pitch, 500, 1000))
    if kind == "column":  # a 1 x 1 x nz column
        vs, vox, ds, pitch = (1, 1, 19), (1.0, 1.0, 1.0), (5, 27), (1.0, 1.0)
        return (dtvb200.circular(ang(4), vs, vox, ds, pitch, 500, 1000),
                O.circular_geometry(ang(4), vs, vox, ds, pitch, 500, 1000))
    if kind == "pixel":  # a single detector pixel
        vs, ds = (7, 6, 5), (1, 1)
        a = ang(9).astype(np.float32)
        return (dtvb200.standard(a, vs, ds, 500.0, 1000.0),
                O.standard_geometry(a.astype(np.float64), vs, ds, 500.0, 1000.0))
    if kind == "row":  # a single detector row (21 views: one backprojector block)
        pv = vector_views(21, 40.0, 70.0, 1.6, 1.7)
        vs, ds = (9, 8, 6), (17, 1)
        return dtvb200.vector(pv, vs, ds), O.vector_geometry(pv, vs, ds)
    if kind == "one_view":
        vs, vox, ds, pitch = (10, 9, 7), (1.0, 0.9, 1.1), (13, 11), (1.6, 1.7)
        return (dtvb200.circular([30.0], vs, vox, ds, pitch, 500, 1000),
                O.circular_geometry(np.array([30.0]), vs, vox, ds, pitch, 500, 1000))
    if kind == "ragged":  # one past the 32/16/8 tile edges in x, y, z, u, v
        vs, vox, ds, pitch = (33, 17, 9), (1.0, 1.0, 1.0), (33, 17), (1.9, 1.9)
        return (dtvb200.circular(ang(3), vs, vox, ds, pitch, 500, 1000),
                O.circular_geometry(ang(3), vs, vox, ds, pitch, 500, 1000))
    raise ValueError(kind)


EDGES = ["voxel", "slice", "column", "pixel", "row", "one_view", "ragged"]
QTOL = 5e-3


def to_dev(a, dev, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev, dtype)


def _volume(og, seed, batch):
    rng = np.random.default_rng(seed)
    # blobs need at least a few voxels per axis; tiny axes get random values
    if min(og.vol_shape) >= 3:
        return blob_volume(rng, og.vol_shape, batch)
    return rng.uniform(0.1, 1.0, (batch, 1) + tuple(og.vol_shape)).astype(np.float32)


@pytest.mark.parametrize("kind", EDGES)
def test_edge_oracle_rays_are_not_empty(kind):
    """Every case has rays that meet the volume (the comparisons below are not
    of all-zero sinograms)."""
    _, og = edge_case(kind)
    assert O.fp_samples(og) > 0


@pytest.mark.parametrize("kind", EDGES)
def test_edge_forward_all_samplers(cuda, kind):
    g, og = edge_case(kind)
    vol = _volume(og, 31, 2)
    v16 = vol.astype(np.float16).astype(np.float32)
    ref = O.forward(og, vol).reshape((2, 1) + tuple(og.sino_shape))
    assert np.abs(ref).max() > 0
    soft = dtvb200.Plan(g, max_batch=2, sampler="soft", device=cuda).forward(to_dev(vol, cuda))
    assert rel_rmse(soft.cpu().numpy(), ref) < 1e-5
    assert rel_max(soft.cpu().numpy(), ref) < 1e-4
    tex = dtvb200.Plan(g, max_batch=2, sampler="tex", device=cuda).forward(to_dev(vol, cuda))
    assert rel_rmse(tex.cpu().numpy(), O.forward(og, vol, q=True).reshape(ref.shape)) < QTOL
    pairs = dtvb200.Plan(g, max_batch=2, sampler="pairs", device=cuda).forward(to_dev(vol, cuda))
    assert rel_rmse(pairs.cpu().numpy(), O.forward(og, v16, q=2).reshape(ref.shape)) < QTOL
    tma_plan = dtvb200.Plan(g, max_batch=2, sampler="tma", device=cuda)
    tma = tma_plan.forward(to_dev(vol, cuda))
    assert tma_plan.device_status() == 0
    assert rel_rmse(tma.cpu().numpy(), O.forward(og, v16).reshape(ref.shape)) < 5e-4


@pytest.mark.parametrize("kind", EDGES)
def test_edge_backward(cuda, kind):
    g, og = edge_case(kind)
    sino = np.random.default_rng(32).random((2, 1) + tuple(og.sino_shape)).astype(np.float32)
    ref = O.backward(og, sino).reshape((2, 1) + tuple(og.vol_shape))
    refq = O.backward(og, sino, q=True).reshape(ref.shape)
    assert np.abs(ref).max() > 0
    out = dtvb200.Plan(g, max_batch=2, sampler="soft", device=cuda).backward(to_dev(sino, cuda))
    assert rel_rmse(out.cpu().numpy(), ref) < 1e-5
    assert rel_max(out.cpu().numpy(), ref) < 1e-4
    for sampler in ("tex", "pairs"):
        out = dtvb200.Plan(g, max_batch=2, sampler=sampler, device=cuda).backward(
            to_dev(sino, cuda))
        assert rel_rmse(out.cpu().numpy(), refq) < QTOL, sampler


def test_vector_backward_with_fewer_than_21_views_is_zero(cuda):
    """The vector-geometry backprojector scales by 2*pi / (N / 21) in integer
    division (Beijing/plug/kernel/backwardKernel.cu:43,96); with N < 21 the
    reference divides by zero, this library returns a zero volume."""
    pv = vector_views(3, 40.0, 70.0, 1.6, 1.7)
    g = dtvb200.vector(pv, (9, 8, 6), (17, 5))
    sino = torch.rand((1, 1, 3, 5, 17), device=cuda)
    for sampler in ("soft", "tex", "pairs"):
        out = dtvb200.Plan(g, sampler=sampler, device=cuda).backward(sino)
        assert float(out.abs().max()) == 0.0, sampler


@pytest.mark.parametrize("kind", EDGES)
@pytest.mark.parametrize("table,method", [(False, 0), (True, 1)])
def test_edge_adjoint_and_dot_test(cuda, kind, table, method):
    g, og = edge_case(kind)
    plan = dtvb200.Plan(g, max_batch=2, device=cuda, adjoint=table)
    if table:
        plan.set_tuning(_lib.DTV_TUNE_ADJOINT, method)
    rng = np.random.default_rng(33)
    y = rng.random((2, 1) + tuple(og.sino_shape)).astype(np.float32)
    x = rng.random((2, 1) + tuple(og.vol_shape)).astype(np.float32)
    aty = plan.adjoint(to_dev(y, cuda)).cpu().numpy()
    ref = O.adjoint(og, y).reshape(aty.shape)
    assert np.abs(ref).max() > 0
    assert rel_rmse(aty, ref) < 1e-5
    ax = plan.forward(to_dev(x, cuda)).cpu().numpy()
    lhs = float((ax.astype(np.float64) * y).sum())
    rhs = float((x.astype(np.float64) * aty).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


EDGE_VOLS = [(1, 1, 1), (1, 1, 9), (7, 1, 1), (1, 6, 1), (33, 9, 17), (32, 8, 8), (65, 5, 9)]


@pytest.mark.parametrize("vs", EDGE_VOLS)
@pytest.mark.parametrize("quirk", [True, False])
def test_edge_pdhg_steps(cuda, vs, quirk):
    """One fused dual step (stencils, ascent, the three exact L1-ball
    thresholds) and one primal step against the reference's update order
    (DTVCP.py:41-54) in FP64."""
    from dtvb200.geometry import _ptr, _stream
    X, Y, Z = vs
    rng = np.random.default_rng(34)
    shp = (1, 1, Z, Y, X)
    fbar, f = rng.random(shp).astype(np.float32), rng.random(shp).astype(np.float32)
    p, q, s, c = [(rng.standard_normal(shp) * 0.01).astype(np.float32) for _ in range(4)]
    recon = (rng.standard_normal(shp) * 0.01).astype(np.float32)
    sg, tau, mu, v = 0.05, 0.02, 0.7, (0.4, 0.3, 0.2)
    t = [np.abs(O.diff(f, vs, a, quirk)).sum() * 0.5 for a in range(3)]
    duals = []
    for a, d in enumerate((p, q, s)):
        d_ = d + v[a] * sg * O.diff(fbar, vs, a, quirk)
        lam = O.l1ball_lambda_exact(np.abs(d_) / sg, v[a] * t[a])
        duals.append(d_ - sg * np.sign(d_) * np.maximum(np.abs(d_) / sg - lam, 0))
    c_ref = -np.maximum(-c - sg * mu * fbar, 0)
    reg = sum(v[a] * O.diff(duals[a], vs, a, quirk, True) for a in range(3)) + mu * c_ref
    fnew = f - recon - tau * reg

    prm = _lib.dtv_pdhg_params()
    prm.sigma, prm.tau, prm.mu = sg, tau, mu
    prm.v[:] = v
    prm.quirk = int(quirk)
    prm.f_dtype = _lib.DTV_F32
    T = {k: to_dev(a, cuda) for k, a in dict(fbar=fbar, f=f, p=p, q=q, s=s, c=c,
                                             recon=recon).items()}
    tt = torch.tensor(t, dtype=torch.float64, device=cuda)
    ws = torch.zeros(_lib.load().dtv_pdhg_workspace_bytes(), dtype=torch.uint8, device=cuda)
    size = _lib.ivec(vs)
    st = _stream(cuda)
    _lib.call("dtv_pdhg_dual", _ptr(T["fbar"]), _ptr(T["p"]), _ptr(T["q"]), _ptr(T["s"]),
              _ptr(T["c"]), size, 1, ctypes.byref(prm), _ptr(tt), _ptr(ws), st)
    _lib.call("dtv_pdhg_primal", _ptr(T["f"]), _ptr(T["fbar"]), _ptr(T["recon"]), _ptr(T["p"]),
              _ptr(T["q"]), _ptr(T["s"]), _ptr(T["c"]), size, 1, ctypes.byref(prm), _ptr(ws), st)
    for a, k in enumerate("pqs"):
        assert np.abs(T[k].cpu().numpy() - duals[a]).max() <= 1e-5 * max(np.abs(duals[a]).max(),
                                                                            1e-3), k
    assert np.abs(T["c"].cpu().numpy() - c_ref).max() <= 1e-7
    assert rel_max(T["f"].cpu().numpy(), fnew) < 1e-5
    assert rel_max(T["fbar"].cpu().numpy(), 2 * fnew - f) < 1e-5


@pytest.mark.parametrize("vs", EDGE_VOLS)
def test_edge_diff(cuda, vs):
    X, Y, Z = vs
    f = np.random.default_rng(35).standard_normal((2, 1, Z, Y, X)).astype(np.float32)
    for quirk in (True, False):
        for ax in range(3):
            for tr in (False, True):
                out = dtvb200.diff(to_dev(f, cuda), ax, tr, quirk).cpu().numpy()
                assert np.abs(out - O.diff(f, vs, ax, quirk, tr)).max() < 1e-5


@pytest.mark.parametrize("v,frac", [([0.75], 0.5), ([-2.0, 1.0], 0.0), ([0.0, 0.0, 0.0], 0.0),
                                    ([0.0, -0.0, 3.0], 0.25), ([1.0, 1.0, 1.0, 1.0], 0.5),
                                    ([5.0, -5.0], 1.0)])
def test_edge_l1ball(cuda, v, frac):
    """Tiny inputs, ties, zero radius, all zeros, radius equal to the norm."""
    v = np.asarray(v, dtype=np.float32)
    b = frac * float(np.abs(v.astype(np.float64)).sum())
    out, lam = dtvb200.l1ball(to_dev(v, cuda), b)
    lam_ref = O.l1ball_lambda_exact(v, b)
    w_ref = np.sign(v) * np.maximum(np.abs(v.astype(np.float64)) - lam_ref, 0)
    if np.abs(v).sum() < b:
        w_ref = v
    assert np.abs(out.cpu().numpy() - w_ref).max() <= 1e-6 * max(np.abs(v).max(), 1.0)
