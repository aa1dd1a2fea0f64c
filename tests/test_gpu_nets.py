"""GPU tests of the unrolled network path: gradients through the matched
adjoint agree with finite differences on 16 random voxels, per-stage
checkpointing changes nothing, BF16 training lowers the loss."""
import numpy as np
import pytest
import torch

import dtvb200
from dtvb200.nets import LEARN, UnrolledPDHG, train
from dtvb200.phantom import ellipsoids

pytestmark = pytest.mark.gpu


def small_problem(cuda, n=32, views=12, batch=2):
    ang = np.linspace(0, 360, views, endpoint=False)
    geo = dtvb200.circular(ang, (n, n, n), (1.0, 1.0, 1.0), (48, 48), (1.5, 1.5), 500.0, 1000.0)
    proj = dtvb200.Projector(geo, max_batch=batch)
    truth = torch.cat([ellipsoids((n, n, n), seed=s, device=cuda) for s in range(batch)])
    sino = proj.fp_soft(truth)
    return proj, truth, sino


def test_finite_differences_through_the_network(cuda):
    torch.manual_seed(0)
    proj, truth, sino = small_problem(cuda)
    net = UnrolledPDHG(proj, stages=3, features=8, lamb=2e-3, tau=1e-2, bf16=False).to(cuda)
    x0 = torch.zeros_like(truth) + 0.1

    def loss(x):
        return float(((net(x, sino).double() - truth.double()) ** 2).sum())

    xg = x0.clone().requires_grad_()
    ((net(xg, sino).double() - truth.double()) ** 2).sum().backward()
    g = xg.grad.flatten().double()
    rng = np.random.default_rng(1)
    idx = rng.choice(x0.numel(), 16, replace=False)
    h = 5e-2
    with torch.no_grad():
        for i in idx:
            e = torch.zeros_like(x0).flatten()
            e[i] = h
            e = e.reshape(x0.shape)
            fd = (loss(x0 + e) - loss(x0 - e)) / (2 * h)
            assert abs(fd - float(g[i])) <= 2e-2 * max(1.0, abs(fd)), (int(i), fd, float(g[i]))


def test_checkpointing_is_transparent(cuda):
    torch.manual_seed(0)
    proj, truth, sino = small_problem(cuda)
    net = UnrolledPDHG(proj, stages=3, features=8, bf16=False).to(cuda)
    x0 = torch.zeros_like(truth)
    grads = []
    for ckpt in (True, False):
        net.checkpoint_stages = ckpt
        net.zero_grad()
        torch.mean((net(x0, sino) - truth) ** 2).backward()
        grads.append(torch.cat([p.grad.flatten() for p in net.parameters()]))
    assert torch.allclose(grads[0], grads[1], rtol=1e-4, atol=1e-7)


def test_bf16_training_lowers_the_loss(cuda):
    torch.manual_seed(0)
    proj, truth, sino = small_problem(cuda)
    net = UnrolledPDHG(proj, stages=4, features=16, lamb=2e-3, tau=1e-3).to(cuda)
    losses = train(net, torch.zeros_like(truth), sino, truth, steps=30, lr=2e-3)
    l = losses.cpu().numpy()
    assert np.all(np.isfinite(l))
    assert l[-5:].mean() < 0.8 * l[:3].mean()


def test_learn_mirror_returns_all_iterates(cuda):
    proj, truth, sino = small_problem(cuda, batch=1)
    net = LEARN(proj, cascades=3).to(cuda)
    out = net(torch.zeros_like(truth[:1]), sino[:1])
    assert len(out) == 4 and out[-1].shape == truth[:1].shape
    assert net.blocks[0] is net.blocks[2]  # weights shared across cascades (LEARN.py:11)
