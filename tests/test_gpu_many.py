"""Several plans in one launch: dtv_forward_many / dtv_backward_many give the
same values as one call per plan (the per-ray and per-voxel computations are
the same code), over plans of different sizes, view counts and geometry kinds,
more plans than one launch takes; and the lockstep BatchedFISTA equals a
FISTA run per reconstruction."""
import numpy as np
import pytest
import torch

import dtvb200
from dtvb200 import _lib
from helpers import blob_volume, vector_views

pytestmark = pytest.mark.gpu


def _geometries():
    rng = np.random.default_rng(31)
    geos = []
    for i in range(27):
        kind = i % 3
        if kind == 0:
            n = int(rng.integers(8, 40))
            views = int(rng.integers(3, 20))
            d = int(1.5 * n)
            ang = np.linspace(0, 360, views, endpoint=False)
            geos.append(dtvb200.circular(ang, (n, n + 3, n - 2), (1.0, 0.9, 1.1), (d, d - 5),
                                         (1.2, 1.1), 500.0, 1000.0))
        elif kind == 1:
            ang = np.linspace(0, 360, int(rng.integers(4, 12)), endpoint=False).astype(np.float32)
            geos.append(dtvb200.standard(ang, (24, 20, 10), (33, 17), 500.0, 1000.0))
        else:  # tilted detector rows: not z-affine
            geos.append(dtvb200.vector(vector_views(int(rng.integers(6, 30)), 40.0, 70.0, 1.6,
                                                    1.7, 1.5), (16, 14, 10), (20, 12)))
    return geos


def _plans(cuda, sampler="pairs"):
    return [dtvb200.Plan(g, sampler=sampler, device=cuda) for g in _geometries()]


def _vols(cuda, plans, seed=5):
    rng = np.random.default_rng(seed)
    return [torch.from_numpy(blob_volume(rng, p.vol_shape(1)[2:], 1)).to(cuda) for p in plans]


def test_forward_many_equals_per_plan(cuda):
    plans = _plans(cuda)
    vols = _vols(cuda, plans)
    outs = dtvb200.forward_many(plans, vols)
    for p, v, o in zip(plans, vols, outs):
        assert torch.equal(o, p.forward(v))
    gs = [torch.rand(p.sino_shape(1), device=cuda) for p in plans]
    res = dtvb200.forward_many(plans, vols, epilogue=_lib.DTV_EPI_RESIDUAL, gs=gs)
    for p, v, g, r in zip(plans, vols, gs, res):
        assert torch.equal(r, p.forward(v, epilogue=_lib.DTV_EPI_RESIDUAL, g=g))


@pytest.mark.parametrize("sampler", ["pairs", "tex"])
def test_backward_many_equals_per_plan(cuda, sampler):
    plans = _plans(cuda, sampler)
    g = torch.Generator(device=cuda).manual_seed(6)
    sinos = [torch.rand(p.sino_shape(1), device=cuda, generator=g) for p in plans]
    outs = dtvb200.backward_many(plans, sinos)
    for p, s, o in zip(plans, sinos, outs):
        assert torch.equal(o, p.backward(s))
    acc = [o.clone() for o in outs]
    dtvb200.backward_many(plans, sinos, outs=acc, accumulate=True)
    for o, a in zip(outs, acc):
        assert torch.allclose(a, 2 * o, rtol=1e-6, atol=0)


def test_backward_many_splits_by_views(cuda):
    """Plans whose views together exceed one launch's map budget (560 views)
    run in several launches, and a plan with more views than that reads its
    maps from device memory: the values are those of one plan at a time."""
    plans = []
    for views in (250, 250, 250, 600, 40):
        ang = np.linspace(0, 360, views, endpoint=False)
        plans.append(dtvb200.Plan(dtvb200.circular(ang, (16, 18, 12), (1.0,) * 3, (24, 20),
                                                   (1.2, 1.2), 500.0, 1000.0),
                                  sampler="pairs", device=cuda))
    g = torch.Generator(device=cuda).manual_seed(8)
    sinos = [torch.rand(p.sino_shape(1), device=cuda, generator=g) for p in plans]
    outs = dtvb200.backward_many(plans, sinos)
    for p, s_, o in zip(plans, sinos, outs):
        assert torch.equal(o, p.backward(s_))


def test_many_rejects_unsupported_plans(cuda):
    plans = _plans(cuda)[:3]
    vols = _vols(cuda, plans)
    soft = dtvb200.Plan(plans[0].geometry, sampler="soft", device=cuda)
    with pytest.raises(dtvb200.DtvError):
        dtvb200.forward_many([plans[0], soft], [vols[0], vols[0]])
    with pytest.raises(dtvb200.DtvError):
        dtvb200.backward_many([soft], [torch.zeros(soft.sino_shape(1), device=cuda)])
    with pytest.raises(ValueError):
        dtvb200.forward_many([], [])
    with pytest.raises(dtvb200.DtvError):  # one staging texture per plan
        dtvb200.forward_many([plans[0], plans[0]], [vols[0], vols[0]])
    sino = torch.zeros(plans[0].sino_shape(1), device=cuda)
    with pytest.raises(dtvb200.DtvError):
        dtvb200.backward_many([plans[0], plans[0]], [sino, sino])
    with pytest.raises(ValueError):
        dtvb200.BatchedFISTA([plans[0], plans[0]], 2)
    with pytest.raises(ValueError):
        dtvb200.Batched([dtvb200.FISTA(plans[0], 2), dtvb200.FISTA(plans[0], 2)])


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("groups", [1, 3])
def test_batched_fista_equals_fista(cuda, graph, groups):
    plans = _plans(cuda)[:8]
    truths = _vols(cuda, plans, seed=7)
    sinos = [p.forward(t) for p, t in zip(plans, truths)]
    imgs = [torch.zeros_like(t) for t in truths]
    batch = dtvb200.BatchedFISTA(plans, 6, lamb=0.05, L=1e-3, use_graph=graph, groups=groups)
    out = batch.run(imgs, sinos)
    out2 = batch.run(imgs, sinos)
    for p, i, s, o, o2 in zip(plans, imgs, sinos, out, out2):
        ref = dtvb200.FISTA(p, 6, lamb=0.05, L=1e-3).run(i, s)
        assert torch.equal(o, ref)
        assert torch.equal(o2, ref)
    assert batch.launches_per_run > 0
