"""GPU parity tests of the update kernels: finite differences, the L1-ball
threshold search, the fused PDHG steps and the four reconstruction loops,
against the FP64 oracle (itself pinned to the reference's Python code)."""
import os

import numpy as np
import pytest
import torch

import dtvb200
import oracle as O
from dtvb200 import _lib
from helpers import rel_max, rel_rmse

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def dev_t(a, cuda, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda, dtype)


@pytest.mark.parametrize("vs", [(5, 4, 3), (4, 4, 3), (33, 17, 9)])
@pytest.mark.parametrize("quirk", [True, False])
def test_diff_matches_oracle(cuda, vs, quirk):
    X, Y, Z = vs
    f = np.random.default_rng(0).standard_normal((2, 1, Z, Y, X)).astype(np.float32)
    ft = dev_t(f, cuda)
    for ax in range(3):
        for tr in (False, True):
            out = dtvb200.diff(ft, ax, tr, quirk).cpu().numpy()
            ref = O.diff(f, vs, ax, quirk, tr)
            assert np.abs(out - ref).max() < 1e-5


def test_diff_matches_reference_golden(cuda):
    z = np.load(os.path.join(GOLDEN, "ref_utils.npz"))
    for tag in "ab":
        vs = tuple(int(v) for v in z[f"d{tag}_size"])
        f = dev_t(z[f"d{tag}_f"].reshape(1, 1, *vs[::-1]), cuda)
        for ax in range(3):
            assert np.abs(dtvb200.diff(f, ax, False, True).cpu().numpy().ravel()
                          - z[f"d{tag}_D{ax}"]).max() < 1e-6
            assert np.abs(dtvb200.diff(f, ax, True, True).cpu().numpy().ravel()
                          - z[f"d{tag}_DT{ax}"]).max() < 1e-6


@pytest.mark.parametrize("fdt", [torch.float32, torch.float16])
def test_diff_abs_sums(cuda, fdt):
    vs = (40, 30, 20)
    f = np.random.default_rng(1).random((1, 1, 20, 30, 40)).astype(np.float32)
    ft = dev_t(f, cuda, fdt)
    s = dtvb200.diff_abs_sums(ft, quirk=True).cpu().numpy()
    fr = ft.float().cpu().numpy()
    ref = [np.abs(O.diff(fr, vs, a, True)).sum() for a in range(3)]
    assert np.allclose(s, ref, rtol=1e-6)


@pytest.mark.parametrize("i", range(5))
def test_l1ball_matches_reference_golden(cuda, i):
    z = np.load(os.path.join(GOLDEN, "ref_utils.npz"))
    v, b, w = z[f"l1_{i}_v"], float(z[f"l1_{i}_b"]), z[f"l1_{i}_w"]
    out, lam = dtvb200.l1ball(dev_t(v, cuda), b)
    assert np.abs(out.cpu().numpy() - w).max() <= 2e-6 * max(1.0, np.abs(w).max())


@pytest.mark.parametrize("n,scale,frac", [(1_000_003, 1.0, 0.3), (4_000_000, 1e-3, 0.01),
                                          (777, 5.0, 0.9), (100_000, 1.0, 0.0),
                                          (100_000, 1.0, 2.0)])
def test_l1ball_exact_on_large_inputs(cuda, n, scale, frac):
    rng = np.random.default_rng(n)
    v = (rng.standard_normal(n) * scale).astype(np.float32)
    v[rng.random(n) < 0.2] = 0.0  # many exact zeros (one hot bin)
    b = frac * float(np.abs(v.astype(np.float64)).sum())
    out, lam = dtvb200.l1ball(dev_t(v, cuda), b)
    lam_ref = O.l1ball_lambda_exact(v, b)
    if np.abs(v).sum() < b:
        assert torch.equal(out.cpu(), torch.from_numpy(v))
    else:
        assert abs(float(lam) - lam_ref) <= 1e-6 * max(lam_ref, 1e-30) + 1e-12
        s = float(out.double().abs().sum())
        if b > 0:
            assert s == pytest.approx(b, rel=1e-5)
        else:
            assert s == 0.0


def _l1ball_ws(v, radius, ws, cuda):
    from dtvb200.geometry import _ptr, _stream
    w = torch.empty_like(v)
    lam = torch.empty(1, dtype=torch.float64, device=cuda)
    _lib.call("dtv_l1ball", _ptr(v), _ptr(w), v.numel(), _ptr(radius), _ptr(ws), _ptr(lam),
              _stream(cuda))
    return w, lam


@pytest.mark.parametrize("fill", [0xFF, 0x5A, 0x01])
def test_l1ball_workspace_of_any_contents(cuda, fill):
    """A caller's workspace need not be zeroed (a fresh cudaMalloc, or one a
    previous search left part-way): the call clears what it uses."""
    rng = np.random.default_rng(fill)
    n = 300_001
    v = dev_t((rng.standard_normal(n) * 3.0).astype(np.float32), cuda)
    nbytes = _lib.load().dtv_l1ball_workspace_bytes()
    for frac in (0.2, 0.7):
        radius = torch.tensor([frac * float(v.double().abs().sum())], dtype=torch.float64,
                              device=cuda)
        w0, l0 = _l1ball_ws(v, radius, torch.zeros(nbytes, dtype=torch.uint8, device=cuda), cuda)
        dirty = torch.full((nbytes,), fill, dtype=torch.uint8, device=cuda)
        w1, l1 = _l1ball_ws(v, radius, dirty, cuda)
        assert torch.equal(w0, w1) and torch.equal(l0, l1)
        lam_ref = O.l1ball_lambda_exact(v.cpu().numpy(), float(radius))
        assert abs(float(l1) - lam_ref) <= 1e-6 * lam_ref


@pytest.mark.parametrize("edge", [0.5, 0.25, 2.0 ** -20])
def test_l1ball_radius_on_a_bin_edge(cuda, edge):
    """lambda falls exactly on a power of two, the lower edge of a bin at every
    level of the radix search."""
    k = 17
    v = np.concatenate([np.full(k, 2 * edge), np.full(k, -edge), np.full(5, edge / 2),
                        np.zeros(9)]).astype(np.float32)
    np.random.default_rng(3).shuffle(v)
    b = k * edge  # sum max(|v| - edge, 0) = k * edge
    out, lam = dtvb200.l1ball(dev_t(v, cuda), b)
    assert float(lam) == pytest.approx(edge, rel=1e-7)
    ref = np.sign(v) * np.maximum(np.abs(v) - edge, 0)
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-7 * edge


def test_pdhg_dual_workspace_of_any_contents(cuda):
    import ctypes
    from dtvb200.geometry import _ptr, _stream
    vs, fbar, f, (p, q, s, c), recon, prm, t = _pdhg_case(cuda)
    tt = torch.tensor(t, dtype=torch.float64, device=cuda)
    nbytes = _lib.load().dtv_pdhg_workspace_bytes()
    outs = []
    for fill in (0x00, 0xFF, 0x3C):
        ws = torch.full((nbytes,), fill, dtype=torch.uint8, device=cuda)
        T = {k: dev_t(x, cuda) for k, x in dict(fbar=fbar, f=f, p=p, q=q, s=s, c=c,
                                                  recon=recon).items()}
        size = _lib.ivec(vs)
        _lib.call("dtv_pdhg_dual", _ptr(T["fbar"]), _ptr(T["p"]), _ptr(T["q"]), _ptr(T["s"]),
                  _ptr(T["c"]), size, 1, ctypes.byref(prm), _ptr(tt), _ptr(ws), _stream(cuda))
        _lib.call("dtv_pdhg_primal", _ptr(T["f"]), _ptr(T["fbar"]), _ptr(T["recon"]),
                  _ptr(T["p"]), _ptr(T["q"]), _ptr(T["s"]), _ptr(T["c"]), size, 1,
                  ctypes.byref(prm), _ptr(ws), _stream(cuda))
        torch.cuda.synchronize()
        outs.append([T[k].cpu() for k in ("p", "q", "s", "c", "f", "fbar")])
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            assert torch.equal(a, b)


@pytest.mark.parametrize("fdt", [torch.float32, torch.float16])
@pytest.mark.parametrize("quirk", [True, False])
def test_pdhg_dual_vector_path_equals_scalar_path(cuda, fdt, quirk):
    """Rows of a multiple of 4 voxels take the dual step four x at a time
    (16-byte duals); an f-bar or c that is not 16-byte (8-byte) aligned sends
    it down the one-voxel path. Both give the same bits, thresholds included."""
    import ctypes
    from dtvb200.geometry import _ptr, _stream
    rng = np.random.default_rng(11)
    vs = (24, 16, 10)
    X, Y, Z = vs
    n = X * Y * Z
    fbar = rng.random(n).astype(np.float32)
    duals = [(rng.standard_normal(n) * 0.01).astype(np.float32) for _ in range(4)]
    duals[3] = -np.abs(duals[3])  # c <= 0
    prm = _lib.dtv_pdhg_params()
    prm.sigma, prm.tau, prm.mu = 0.05, 0.02, 0.7
    prm.v[:] = (0.4, 0.3, 0.2)
    prm.quirk = int(quirk)
    prm.f_dtype = _lib.DTV_F32 if fdt == torch.float32 else _lib.DTV_F16
    tt = torch.tensor([3.0, 2.0, 1.5], dtype=torch.float64, device=cuda)
    nbytes = _lib.load().dtv_pdhg_workspace_bytes()
    res = []
    for off in (0, 1):  # element offset 1: f-bar and c 4-byte (2-byte) aligned
        fb = torch.zeros(n + 4, dtype=fdt, device=cuda)[off:off + n]
        fb.copy_(torch.from_numpy(fbar))
        arrs = []
        for j, d in enumerate(duals):
            o = off if j == 3 else 0  # p, q, s stay 16-byte aligned, as required
            a = torch.zeros(n + 4, device=cuda)[o:o + n]
            a.copy_(torch.from_numpy(d))
            arrs.append(a)
        ws = torch.zeros(nbytes, dtype=torch.uint8, device=cuda)
        _lib.call("dtv_pdhg_dual", _ptr(fb), *[_ptr(a) for a in arrs], _lib.ivec(vs), 1,
                  ctypes.byref(prm), _ptr(tt), _ptr(ws), _stream(cuda))
        torch.cuda.synchronize()
        thr = [ws[k * nbytes // 3 + 44:k * nbytes // 3 + 48].cpu() for k in range(3)]
        res.append(([a.cpu() for a in arrs], thr))
    for a, b in zip(res[0][0], res[1][0]):
        assert torch.equal(a, b)
    for a, b in zip(res[0][1], res[1][1]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("fdt", [torch.float32, torch.float16])
@pytest.mark.parametrize("quirk", [True, False])
def test_pdhg_primal_vector_path_equals_scalar_path(cuda, fdt, quirk):
    """The primal step four x at a time (16-byte loads) against the one-voxel
    path (taken when f-bar or c is not aligned): the same bits of f, f-bar
    and the clipped duals."""
    import ctypes
    from dtvb200.geometry import _ptr, _stream
    rng = np.random.default_rng(12)
    vs = (24, 16, 10)
    X, Y, Z = vs
    n = X * Y * Z
    host = {k: rng.random(n).astype(np.float32) for k in ("f", "fbar")}
    host["recon"] = (rng.standard_normal(n) * 0.01).astype(np.float32)
    for k in ("p", "q", "s"):
        host[k] = (rng.standard_normal(n) * 0.05).astype(np.float32)
    host["c"] = -np.abs(rng.standard_normal(n) * 0.01).astype(np.float32)
    prm = _lib.dtv_pdhg_params()
    prm.sigma, prm.tau, prm.mu = 0.05, 0.02, 0.7
    prm.v[:] = (0.4, 0.3, 0.2)
    prm.quirk = int(quirk)
    prm.f_dtype = _lib.DTV_F32 if fdt == torch.float32 else _lib.DTV_F16
    nbytes = _lib.load().dtv_pdhg_workspace_bytes()
    ws = torch.zeros(nbytes, dtype=torch.uint8, device=cuda)
    for k, thr in enumerate((0.03, 0.02, 0.04)):  # the three channels' thresholds
        ws[k * nbytes // 3 + 44:k * nbytes // 3 + 48] = torch.from_numpy(
            np.array([thr], np.float32).view(np.uint8)).to(cuda)
    res = []
    for off in (0, 1):
        T = {}
        for k, a in host.items():
            o = off if k in ("fbar", "c") else 0
            dt = fdt if k == "fbar" else torch.float32
            t = torch.zeros(n + 4, dtype=dt, device=cuda)[o:o + n]
            t.copy_(torch.from_numpy(a))
            T[k] = t
        _lib.call("dtv_pdhg_primal", _ptr(T["f"]), _ptr(T["fbar"]), _ptr(T["recon"]),
                  _ptr(T["p"]), _ptr(T["q"]), _ptr(T["s"]), _ptr(T["c"]), _lib.ivec(vs), 1,
                  ctypes.byref(prm), _ptr(ws), _stream(cuda))
        torch.cuda.synchronize()
        res.append({k: T[k].cpu() for k in ("f", "fbar", "p", "q", "s")})
    for k in res[0]:
        assert torch.equal(res[0][k], res[1][k]), k


def _pdhg_case(cuda, fdt=torch.float32, quirk=True):
    rng = np.random.default_rng(5)
    vs = (20, 16, 12)
    X, Y, Z = vs
    fbar = rng.random((1, 1, Z, Y, X)).astype(np.float32)
    f = rng.random((1, 1, Z, Y, X)).astype(np.float32)
    duals = [(rng.standard_normal((1, 1, Z, Y, X)) * 0.01).astype(np.float32) for _ in range(4)]
    recon = (rng.standard_normal((1, 1, Z, Y, X)) * 0.01).astype(np.float32)
    prm = _lib.dtv_pdhg_params()
    prm.sigma, prm.tau, prm.mu = 0.05, 0.02, 0.7
    prm.v[:] = (0.4, 0.3, 0.2)
    prm.quirk = int(quirk)
    prm.f_dtype = _lib.DTV_F32 if fdt == torch.float32 else _lib.DTV_F16
    t = np.array([np.abs(O.diff(f, vs, a, quirk)).sum() * 0.5 for a in range(3)])
    return vs, fbar, f, duals, recon, prm, t


@pytest.mark.parametrize("quirk", [True, False])
def test_pdhg_steps_match_oracle(cuda, quirk):
    import ctypes
    from dtvb200.geometry import _ptr, _stream
    vs, fbar, f, (p, q, s, c), recon, prm, t = _pdhg_case(cuda, quirk=quirk)
    sg, tau, mu, v = prm.sigma, prm.tau, prm.mu, tuple(prm.v)
    # oracle (DTVCP.py:41-54)
    duals = []
    for a, d in enumerate((p, q, s)):
        d_ = d + v[a] * sg * O.diff(fbar, vs, a, quirk)
        proj, _ = O.l1ball_newton(np.abs(d_) / sg, v[a] * t[a])
        duals.append(d_ - sg * np.sign(d_) * proj)
    c_ref = -np.maximum(-c - sg * mu * fbar, 0)
    reg = sum(v[a] * O.diff(duals[a], vs, a, quirk, True) for a in range(3)) + mu * c_ref
    fnew = f - recon - tau * reg
    # kernels
    T = {k: dev_t(x, cuda) for k, x in dict(fbar=fbar, f=f, p=p, q=q, s=s, c=c,
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
        assert rel_max(T[k].cpu().numpy(), duals[a]) < 1e-5
    assert rel_max(T["c"].cpu().numpy(), c_ref) < 1e-6
    assert rel_max(T["f"].cpu().numpy(), fnew) < 1e-5
    assert rel_max(T["fbar"].cpu().numpy(), 2 * fnew - f) < 1e-5
    # the histogram workspace is left zeroed: a second identical search agrees
    T2 = {k: dev_t(x, cuda) for k, x in dict(fbar=fbar, p=p, q=q, s=s, c=c).items()}
    _lib.call("dtv_pdhg_dual", _ptr(T2["fbar"]), _ptr(T2["p"]), _ptr(T2["q"]), _ptr(T2["s"]),
              _ptr(T2["c"]), size, 1, ctypes.byref(prm), _ptr(tt), _ptr(ws), st)
    ws2 = torch.zeros_like(ws)
    T3 = {k: dev_t(x, cuda) for k, x in dict(fbar=fbar, p=p, q=q, s=s, c=c).items()}
    _lib.call("dtv_pdhg_dual", _ptr(T3["fbar"]), _ptr(T3["p"]), _ptr(T3["q"]), _ptr(T3["s"]),
              _ptr(T3["c"]), size, 1, ctypes.byref(prm), _ptr(tt), _ptr(ws2), st)
    torch.cuda.synchronize()
    hdr = 48
    assert torch.equal(ws[:hdr], ws2[:hdr])


# ------------------------------------------------------------------ loops
def _loop(cuda):
    import make_ref_utils as M
    z = np.load(os.path.join(GOLDEN, "ref_utils.npz"))
    geo = dtvb200.standard(M.LOOP_ANGLES, M.LOOP_VS, M.LOOP_DS, M.LOOP_SID, M.LOOP_SDD)
    plan = dtvb200.Plan(geo, device=cuda)
    og = M.loop_geometry()
    fp = lambda x: O.forward(og, x).reshape(x.shape[0], 1, *og.sino_shape)  # noqa: E731
    bp = lambda s: O.backward(og, s).reshape(s.shape[0], 1, *og.vol_shape)  # noqa: E731
    return M, z, plan, fp, bp


@pytest.mark.parametrize("use_graph", [False, True])
def test_dtvcp_matches_oracle_and_reference(cuda, use_graph):
    M, z, plan, fp, bp = _loop(cuda)
    sg, ta, mu, v1, v2, v3, n = z["dtvcp_params"]
    alg = dtvb200.DTVCP(plan, int(n), sigma=sg, tau=ta, mu=mu, v=(v1, v2, v3), quirk=True,
                        use_graph=use_graph)
    img = torch.zeros(plan.vol_shape(1), device=cuda)
    sino = dev_t(z["loop_sino"], cuda)
    f = alg.run(img, sino).cpu().numpy()
    f2 = alg.run(img, sino).cpu().numpy()  # replay / re-run: same result
    assert np.array_equal(f, f2)
    ref = z["dtvcp_f"]  # the reference's own DTVCP.run on oracle projectors
    assert rel_rmse(f, ref) < 1e-4
    fo = O.dtvcp_run(fp, bp, np.zeros((1, 1) + plan.vol_shape(1)[2:]), z["loop_sino"],
                     M.LOOP_VS, int(n), sg, ta, mu, (v1, v2, v3))
    assert rel_rmse(f, fo) < 1e-4
    losses = alg.losses.cpu().numpy()
    assert losses.shape == (int(n),) and np.all(losses > 0)


def test_dtvcp_fp16_storage(cuda):
    M, z, plan, fp, bp = _loop(cuda)
    sg, ta, mu, v1, v2, v3, n = z["dtvcp_params"]
    alg = dtvb200.DTVCP(plan, int(n), sigma=sg, tau=ta, mu=mu, v=(v1, v2, v3),
                        f_dtype=torch.float16)
    f = alg.run(torch.zeros(plan.vol_shape(1), device=cuda), dev_t(z["loop_sino"], cuda))
    assert rel_rmse(f.cpu().numpy(), z["dtvcp_f"]) < 1e-3


@pytest.mark.parametrize("use_graph", [False, True])
def test_fista_matches_reference(cuda, use_graph):
    M, z, plan, fp, bp = _loop(cuda)
    lamb, L, n = z["fista_params"]
    alg = dtvb200.FISTA(plan, int(n), lamb=lamb, L=L, use_graph=use_graph)
    f = alg.run(torch.zeros(plan.vol_shape(1), device=cuda), dev_t(z["loop_sino"], cuda))
    assert rel_rmse(f.cpu().numpy(), z["fista_f"]) < 1e-4


@pytest.mark.parametrize("quirk", [True, False])
def test_dtvfista_matches_oracle(cuda, quirk):
    M, z, plan, fp, bp = _loop(cuda)
    p = z["dtvfista_params"]
    alg = dtvb200.DTVFISTA(plan, int(p[7]), sigma=p[0], v=p[1:4], t=p[4:7], quirk=quirk)
    f = alg.run(torch.zeros(plan.vol_shape(1), device=cuda),
                dev_t(z["loop_sino"], cuda)).cpu().numpy()
    fo = O.dtvfista_run(fp, bp, np.zeros((1, 1) + plan.vol_shape(1)[2:]), z["loop_sino"],
                        M.LOOP_VS, int(p[7]), p[0], p[1:4], p[4:7], quirk=quirk)
    assert rel_rmse(f, fo) < 1e-4
    if quirk:
        assert rel_rmse(f, z["dtvfista_f"]) < 1e-4


def test_asdpocs_matches_reference(cuda):
    M, z, plan, fp, bp = _loop(cuda)
    p = z["asd_params"]
    alg = dtvb200.ASDPOCS(plan, int(p[5]), beta=p[0], beta_red=p[1], ng=int(p[2]), alpha=p[3],
                          rmax=p[4])
    f = alg.run(torch.zeros(plan.vol_shape(1), device=cuda), dev_t(z["loop_sino"], cuda))
    assert rel_rmse(f.cpu().numpy(), z["asd_f"]) < 1e-4


@pytest.mark.parametrize("alpha", [0.001, 0.2])
@pytest.mark.parametrize("use_graph", [False, True])
def test_asdpocs_clean_mode_matches_oracle(cuda, alpha, use_graph):
    """quirk=False: f0 is a real copy, so the TV-change test of ASDPOCS.py:44-45
    runs (with alpha = 0.2 it fires and shrinks davg; the result then differs
    from the aliased reference run by about 2%), and D_y does not wrap."""
    M, z, plan, fp, bp = _loop(cuda)
    p = z["asd_params"]
    alg = dtvb200.ASDPOCS(plan, int(p[5]), beta=p[0], beta_red=p[1], ng=int(p[2]), alpha=alpha,
                          rmax=p[4], quirk=False, use_graph=use_graph)
    f = alg.run(torch.zeros(plan.vol_shape(1), device=cuda), dev_t(z["loop_sino"], cuda))
    img = np.zeros((1, 1) + plan.vol_shape(1)[2:])
    fo = O.asdpocs_run(fp, bp, img, z["loop_sino"], M.LOOP_VS, int(p[5]), p[0], p[1], int(p[2]),
                       alpha, p[4], quirk=False)
    assert rel_rmse(f.cpu().numpy(), fo) < 1e-4
    if alpha == 0.2:
        fq = O.asdpocs_run(fp, bp, img, z["loop_sino"], M.LOOP_VS, int(p[5]), p[0], p[1],
                           int(p[2]), alpha, p[4], quirk=True)
        assert rel_rmse(f.cpu().numpy(), fq) > 1e-2


def test_power_norm_close_to_two(cuda):
    # ||D_x|| of a long chain is just under 2 (Gradients.py power method)
    n = dtvb200.power_norm((32, 16, 8), 0, device=cuda, iters=50)
    assert 1.9 < n <= 2.0 + 1e-6


@pytest.mark.parametrize("use_graph", [False, True])
def test_batched_heterogeneous_equals_individual(cuda, use_graph):
    """Reconstructions of different sizes and view counts run as one batch
    (one stream each, one graph) give the same result as run one by one."""
    from dtvb200.phantom import ellipsoids
    cases = [(24, 10), (32, 17), (20, 7)]
    algs, imgs, sinos, singles = [], [], [], []
    for n, views in cases:
        ang = np.linspace(0, 360, views, endpoint=False)
        d = int(1.5 * n)
        geo = dtvb200.circular(ang, (n, n, n), (1.0,) * 3, (d, d), (1.5, 1.5), 500.0, 1000.0)
        plan = dtvb200.Plan(geo, sampler="pairs", device=cuda)
        truth = ellipsoids((n, n, n), seed=n, device=cuda)
        sino = plan.forward(truth)
        alg = dtvb200.FISTA(plan, 6, lamb=0.05, L=2e-3)
        singles.append(alg.run(torch.zeros_like(truth), sino).clone())
        algs.append(dtvb200.FISTA(plan, 6, lamb=0.05, L=2e-3))
        imgs.append(torch.zeros_like(truth))
        sinos.append(sino)
    batch = dtvb200.Batched(algs, use_graph=use_graph)
    for _ in range(2):  # second run replays the graph
        outs = batch.run(imgs, sinos)
        for o, ref in zip(outs, singles):
            assert torch.equal(o, ref)
