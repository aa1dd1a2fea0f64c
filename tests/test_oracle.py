"""CPU tests of the FP64 oracle: its general form against its literal
restatements, its adjoint, and its pins against the reference's own code
(tests/golden/ref_projectors.npz from the reference CUDA kernels;
tests/golden/ref_utils.npz from the reference Python modules)."""
import os

import numpy as np
import pytest

import oracle as O
from helpers import blob_volume, rel_max, rel_rmse, vector_views

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("q", [0, 1])
@pytest.mark.parametrize("vs,ds,n,sid,sdd", [((12, 10, 8), (16, 12), 7, 500.0, 1000.0),
                                             ((9, 13, 5), (11, 7), 5, 300.0, 800.0)])
def test_standard_general_matches_literal(q, vs, ds, n, sid, sdd):
    rng = np.random.default_rng(0)
    X, Y, Z = vs
    W, H = ds
    ang = np.linspace(0, 360, n, endpoint=False).astype(np.float32).astype(np.float64)
    g = O.standard_geometry(ang, vs, ds, sid, sdd)
    vol = blob_volume(rng, (Z, Y, X), 2)
    a = O.forward(g, vol, q)
    b = O.forward_standard_literal(vol, ang, vs, ds, sid, sdd, q)
    assert rel_max(a, b) < 1e-12
    sino = rng.random((2, n, H, W))
    a = O.backward(g, sino, q)
    b = O.backward_standard_literal(sino, ang, vs, ds, sid, sdd, q)
    assert rel_max(a, b) < 1e-12


@pytest.mark.parametrize("q", [0, 1])
def test_vector_general_matches_literal(q):
    rng = np.random.default_rng(1)
    vs, ds, n = (12, 10, 8), (16, 12), 42
    pv = vector_views(n, 30.0, 60.0, 1.3, 1.2, 1.0)
    g = O.vector_geometry(pv, vs, ds)
    vol = blob_volume(rng, (8, 10, 12), 1)
    assert rel_max(O.forward(g, vol, q), O.forward_vector_literal(vol, pv, vs, ds, q)) < 1e-12
    sino = rng.random((1, n, 12, 16))
    assert rel_max(O.backward(g, sino, q), O.backward_vector_literal(sino, pv, vs, ds, q)) < 1e-12


@pytest.mark.parametrize("kind", ["standard", "box", "vector"])
def test_oracle_adjoint_dot(kind):
    rng = np.random.default_rng(2)
    vs, ds = (10, 9, 6), (14, 8)
    if kind == "standard":
        g = O.standard_geometry(np.linspace(0, 360, 6, endpoint=False), vs, ds, 500, 1000)
    elif kind == "box":
        g = O.circular_geometry(np.linspace(0, 360, 6, endpoint=False), vs, (1.0, 0.8, 1.3), ds,
                                (1.2, 1.1), 500, 1000)
    else:
        g = O.vector_geometry(vector_views(21, 30.0, 60.0, 1.3, 1.2, 1.0), vs, ds)
    x = rng.random((1,) + g.vol_shape)
    y = rng.random((1,) + g.sino_shape)
    lhs = (O.forward(g, x) * y).sum()
    rhs = (x * O.adjoint(g, y)).sum()
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_fp_samples_counts_box_chords():
    g = O.circular_geometry([0.0, 45.0], (8, 8, 8), (1, 1, 1), (16, 16), (1.0, 1.0), 100, 200)
    n = O.fp_samples(g)
    # every sample of the BOX phase lies inside the box: the per-ray sample
    # counts of the forward projector sum to the same number
    assert n > 0
    x = np.ones((1, 8, 8, 8))
    # interior rays through a unit volume integrate to about the chord length
    s = O.forward(g, x)
    assert s.max() <= np.sqrt(3) * 8 + 1.0


# ---------------------------------------------------------------- pins to the reference
def _ref_proj():
    p = os.path.join(GOLDEN, "ref_projectors.npz")
    if not os.path.exists(p):
        pytest.skip("ref_projectors.npz not generated yet")
    return np.load(p)


@pytest.mark.parametrize("name", ["s1", "s2", "s3"])
def test_oracle_pinned_to_reference_standard(name):
    z = _ref_proj()
    X, Y, Z, W, H, n, b = (int(v) for v in z[f"{name}_sizes"])
    sid, sdd = (float(v) for v in z[f"{name}_geom"])
    ang = z[f"{name}_angles"].astype(np.float32).astype(np.float64)
    fp = O.forward_standard_literal(z[f"{name}_vol"], ang, (X, Y, Z), (W, H), sid, sdd, q=1)
    bp = O.backward_standard_literal(z[f"{name}_sino_in"], ang, (X, Y, Z), (W, H), sid, sdd, q=1)
    # The reference kernels filter with 1/256 texture weights and compute their
    # coordinates in float32 (sample positions ~1e3 voxels from the origin in the
    # forward projector, products ~1e6 in the line intersection of the
    # backprojector). Measured: 1.5e-4 - 4e-4 relative RMSE with quantised
    # weights, <= 5.3e-4 with exact weights.
    assert rel_rmse(fp, z[f"{name}_fp"].reshape(fp.shape)) < 6e-4
    assert rel_rmse(bp, z[f"{name}_bp"].reshape(bp.shape)) < 6e-4
    fpe = O.forward_standard_literal(z[f"{name}_vol"], ang, (X, Y, Z), (W, H), sid, sdd, q=0)
    bpe = O.backward_standard_literal(z[f"{name}_sino_in"], ang, (X, Y, Z), (W, H), sid, sdd, q=0)
    assert rel_rmse(fpe, z[f"{name}_fp"].reshape(fp.shape)) < 1e-3
    assert rel_rmse(bpe, z[f"{name}_bp"].reshape(bp.shape)) < 1e-3


def test_oracle_pinned_to_reference_vector():
    z = _ref_proj()
    X, Y, Z, W, H, n, b = (int(v) for v in z["v_sizes"])
    pv = z["v_pv"]
    fp = O.forward_vector_literal(z["v_vol"], pv, (X, Y, Z), (W, H), q=1)
    bp = O.backward_vector_literal(z["v_sino_in"], pv, (X, Y, Z), (W, H), q=1)
    assert rel_rmse(fp, z["v_fp"].reshape(fp.shape)) < 6e-4
    assert rel_rmse(bp, z["v_bp"].reshape(bp.shape)) < 6e-4


def _ref_utils():
    return np.load(os.path.join(GOLDEN, "ref_utils.npz"))


@pytest.mark.parametrize("tag", ["a", "b"])
def test_diff_pinned_to_reference(tag):
    z = _ref_utils()
    vs = tuple(int(v) for v in z[f"d{tag}_size"])
    f = z[f"d{tag}_f"].reshape(vs[::-1])
    for ax in range(3):
        assert np.abs(O.diff(f, vs, ax, True).ravel() - z[f"d{tag}_D{ax}"]).max() < 1e-6
        assert np.abs(O.diff(f, vs, ax, True, True).ravel() - z[f"d{tag}_DT{ax}"]).max() < 1e-6


@pytest.mark.parametrize("i", range(5))
def test_l1ball_pinned_to_reference(i):
    z = _ref_utils()
    v, b, w = z[f"l1_{i}_v"], float(z[f"l1_{i}_b"]), z[f"l1_{i}_w"]
    wn, _ = O.l1ball_newton(v, b)
    assert np.abs(wn - w).max() <= 1e-6 * max(1.0, np.abs(w).max())
    lam = O.l1ball_lambda_exact(v, b)
    we = v if np.abs(v).sum() < b else np.sign(v) * np.maximum(np.abs(v) - lam, 0)
    assert np.abs(we - w).max() <= 1e-6 * max(1.0, np.abs(w).max())


def _loop_ops(z):
    import make_ref_utils as M
    geo = M.loop_geometry()
    fp = lambda x: O.forward(geo, x).reshape(x.shape[0], 1, *geo.sino_shape)  # noqa: E731
    bp = lambda s: O.backward(geo, s).reshape(s.shape[0], 1, *geo.vol_shape)  # noqa: E731
    img0 = np.zeros((1, 1) + geo.vol_shape)
    return M, fp, bp, img0, z["loop_sino"].astype(np.float64)


def test_loops_pinned_to_reference():
    z = _ref_utils()
    M, fp, bp, img0, sino = _loop_ops(z)
    sg, ta, mu, v1, v2, v3, n = z["dtvcp_params"]
    f = O.dtvcp_run(fp, bp, img0, sino, M.LOOP_VS, int(n), sg, ta, mu, (v1, v2, v3))
    assert rel_max(f, z["dtvcp_f"]) < 1e-5
    lamb, L, n = z["fista_params"]
    assert rel_max(O.fista_run(fp, bp, img0, sino, int(n), L, lamb), z["fista_f"]) < 1e-5
    p = z["dtvfista_params"]
    f = O.dtvfista_run(fp, bp, img0, sino, M.LOOP_VS, int(p[7]), p[0], p[1:4], p[4:7])
    assert rel_max(f, z["dtvfista_f"]) < 1e-5
    p = z["asd_params"]
    f = O.asdpocs_run(fp, bp, img0, sino, M.LOOP_VS, int(p[5]), beta=p[0], beta_red=p[1],
                      ng=int(p[2]), alpha=p[3], rmax=p[4])
    assert rel_max(f, z["asd_f"]) < 1e-5


def test_fbp_filter_oracle_matches_reference_torch_lines():
    """oracle.fbp_filter against the reference's own torch formulation
    (cosine weight then conv2d with padding W/2, StandardGeometry.py:51-65) on
    CPU in FP64, and its transpose by the dot test."""
    import torch
    rng = np.random.default_rng(0)
    x = rng.random((2, 1, 3, 5, 16))
    H, W, sdd = 5, 16, 1000.0
    i = np.arange(H)[:, None] - H / 2
    j = np.arange(W)[None, :] - W / 2
    cw = sdd / np.sqrt(sdd ** 2 + i ** 2 + j ** 2)
    k = torch.from_numpy(O.ramp_taps(W).astype(np.float64)).reshape(1, 1, 1, W + 1)
    y = torch.nn.functional.conv2d(torch.from_numpy(x * cw).reshape(2, 1, 3 * H, W), k,
                                   padding=(0, W // 2)).reshape(x.shape).numpy()
    assert np.abs(y - O.fbp_filter(x, H, sdd, H / 2, W / 2)).max() < 1e-12
    z = rng.random(x.shape)
    lhs = np.sum(O.fbp_filter(x, H, sdd, H / 2, W / 2) * z)
    rhs = np.sum(x * O.fbp_filter(z, H, sdd, H / 2, W / 2, adjoint=True))
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)
    taps = O.ramp_taps(8)
    assert taps[4] == np.float32(1 / 8) and taps[2] == 0 and taps[3] == np.float32(-0.5 / np.pi ** 2)

