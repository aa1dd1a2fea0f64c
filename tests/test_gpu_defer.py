"""The PDHG update steps with the duals' clip deferred into the next dual step
(dtv_pdhg_dual_defer / dtv_pdhg_primal_defer) give the bits of the storing
steps (dtv_pdhg_dual / dtv_pdhg_primal): every array after a sequence of
iterations in which the L1-ball constraints clip, on the four-x and the
one-voxel paths, batched, with and without the D_y wrap; and DTVCP gives the
same reconstruction and final duals either way (the losses within the
rounding of their atomic sums)."""
import ctypes

import numpy as np
import pytest
import torch

import dtvb200
from dtvb200 import _lib
from dtvb200.geometry import _ptr, _stream
from dtvb200.phantom import ellipsoids

pytestmark = pytest.mark.gpu


def _state(cuda, vs, batch, fdt, seed):
    X, Y, Z = vs
    n = X * Y * Z * batch
    rng = np.random.default_rng(seed)
    T = {
        "fbar": torch.from_numpy(rng.random(n).astype(np.float32)).to(cuda, fdt),
        "f": torch.from_numpy(rng.random(n).astype(np.float32)).to(cuda),
        "recon": torch.from_numpy((rng.standard_normal(n) * 0.05).astype(np.float32)).to(cuda),
    }
    for k in ("p", "q", "s"):
        T[k] = torch.from_numpy((rng.standard_normal(n) * 0.2).astype(np.float32)).to(cuda)
    T["c"] = torch.zeros(n, device=cuda)
    return T


def _run(cuda, T, vs, batch, prm, t, defer, iters):
    nbytes = _lib.load().dtv_pdhg_workspace_bytes()
    ws = torch.zeros(nbytes, dtype=torch.uint8, device=cuda)
    carry = torch.full((3,), float("nan"), device=cuda)
    size = _lib.ivec(vs)
    st = _stream(cuda)
    duals = (_ptr(T["p"]), _ptr(T["q"]), _ptr(T["s"]), _ptr(T["c"]), size, batch,
             ctypes.byref(prm))
    clipping = []
    for it in range(iters):
        if defer:
            _lib.call("dtv_pdhg_dual_defer", _ptr(T["fbar"]), *duals, _ptr(t), _ptr(ws),
                      _ptr(carry) if it > 0 else None, st)
        else:
            _lib.call("dtv_pdhg_dual", _ptr(T["fbar"]), *duals, _ptr(t), _ptr(ws), st)
        # the constraint is active: a threshold below the largest |dual|
        torch.cuda.synchronize()
        thr = [ws[k * nbytes // 3 + 44:k * nbytes // 3 + 48].view(torch.float32).item()
               for k in range(3)]
        clipping.append(any(m < T[a].abs().max().item() for m, a in zip(thr, "pqs")))
        if defer and it < iters - 1:
            _lib.call("dtv_pdhg_primal_defer", _ptr(T["f"]), _ptr(T["fbar"]), _ptr(T["recon"]),
                      *duals, _ptr(ws), _ptr(carry), st)
            torch.cuda.synchronize()
            assert carry.cpu().tolist() == thr
        else:
            _lib.call("dtv_pdhg_primal", _ptr(T["f"]), _ptr(T["fbar"]), _ptr(T["recon"]),
                      *duals, _ptr(ws), st)
    torch.cuda.synchronize()
    return clipping


@pytest.mark.parametrize("vs", [(24, 16, 10), (25, 15, 9)])  # four-x path, one-voxel path
@pytest.mark.parametrize("quirk", [True, False])
@pytest.mark.parametrize("fdt", [torch.float32, torch.float16])
@pytest.mark.parametrize("batch", [1, 2])
def test_deferred_clip_equals_stored_clip(cuda, vs, quirk, fdt, batch):
    prm = _lib.dtv_pdhg_params()
    prm.sigma, prm.tau, prm.mu = 0.05, 0.02, 0.7
    prm.v[:] = (0.4, 0.3, 0.2)
    prm.quirk = int(quirk)
    prm.f_dtype = _lib.DTV_F32 if fdt == torch.float32 else _lib.DTV_F16
    # radii sigma * v_a * t_a well below sum|p|: every channel clips
    t = torch.tensor([20.0, 30.0, 40.0], dtype=torch.float64, device=cuda)
    A = _state(cuda, vs, batch, fdt, seed=5)
    B = {k: v.clone() for k, v in A.items()}
    ca = _run(cuda, A, vs, batch, prm, t, defer=False, iters=5)
    cb = _run(cuda, B, vs, batch, prm, t, defer=True, iters=5)
    assert all(ca) and ca == cb
    for k in A:
        assert torch.equal(A[k], B[k]), k


def test_dtvcp_deferred_clip_equals_stored_clip(cuda):
    n, views = 40, 24
    ang = np.linspace(0, 360, views, endpoint=False)
    geo = dtvb200.circular(ang, (n, n, n), (1.0,) * 3, (60, 52), (1.2, 1.2), 500.0, 1000.0)
    fast = dtvb200.Plan(geo, sampler="pairs", device=cuda)
    exact = dtvb200.Plan(geo, sampler="exact", device=cuda)
    truth = ellipsoids((n, n, n), seed=0).reshape(fast.vol_shape(1)).to(cuda)
    sino = fast.forward(truth)
    kw = dict(sigma=2e-3, tau=2e-3, mu=1.0, v=(0.5,) * 3, quirk=False, use_graph=True,
              exact=exact, correct_every=3, f_dtype=torch.float16, t_refresh=4)
    runs = []
    for defer in (True, False):
        alg = dtvb200.DTVCP(fast, 12, **kw)
        alg.defer_clip = defer
        f = alg.run(torch.zeros(fast.vol_shape(1), device=cuda), sino)
        st = next(iter(alg._state.values()))
        runs.append((f, alg.losses.clone(), [st[k].clone() for k in ("p", "q", "s", "c")]))
    (fa, la, da), (fb, lb, db) = runs
    assert torch.equal(fa, fb)
    # the losses are sums of double atomics, whose order varies between runs
    assert torch.allclose(la, lb, rtol=1e-12, atol=0)
    for a, b in zip(da, db):
        assert torch.equal(a, b)
