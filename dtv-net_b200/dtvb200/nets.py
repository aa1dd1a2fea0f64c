"""Unrolled reconstruction networks trained through the exact projector adjoint.

The reference's unrolled networks (model/PDHG/LEARN.py:6-22,
model/FISTA/FISTAnet.py:8-23) call the geometry layer, whose autograd pairs
the forward projector with the FDK backprojector as its "gradient"
(StandardGeometry.py:17-21). Here the data-consistency step and the backward
pass go through the matched adjoint (dtv_backward_adjoint), so the gradients
are exact; each stage is checkpointed (its activations are recomputed in the
backward pass), and the convolution blocks run their activations in BF16 under
autocast while their weights stay FP32, in the channels-last 3-D layout that
cuDNN's tensor-core convolutions take without transposes.
"""
from __future__ import annotations

import torch
import torch.nn as nn
from torch.utils.checkpoint import checkpoint

from .ops import Projector, make_functions


class ConvBlock(nn.Module):
    """Conv3d(1, f) - ReLU - Conv3d(f, f) - ReLU - Conv3d(f, 1), 3x3x3 kernels
    (the shape of model/PDHG/RegularizationLayers/CNN.py:4-18 with three layers)."""

    def __init__(self, features: int = 32):
        super().__init__()
        self.body = nn.Sequential(
            nn.Conv3d(1, features, 3, padding=1), nn.ReLU(),
            nn.Conv3d(features, features, 3, padding=1), nn.ReLU(),
            nn.Conv3d(features, 1, 3, padding=1))

    def forward(self, x):
        return self.body(x)


class UnrolledPDHG(nn.Module):
    """x_{s+1} = x_s - lamb_s * A^T (A x_s - p) - tau_s * R_s(x_s), s < stages
    (LEARN.py:15-22 with the matched adjoint A^T). ``share_weights`` reuses one
    block for every stage, as the reference's ``nn.ModuleList([m] * n)`` does
    (LEARN.py:11, FISTAnet.py:12-13)."""

    def __init__(self, projector: Projector, stages: int = 10, features: int = 32,
                 lamb: float = 1e-3, tau: float = 1e-3, share_weights: bool = False,
                 checkpoint_stages: bool = True, bf16: bool = True):
        super().__init__()
        self.stages = stages
        self.FP, self.BP = make_functions(projector, matched=True)
        blocks = [ConvBlock(features)] * stages if share_weights else \
            [ConvBlock(features) for _ in range(stages)]
        self.blocks = nn.ModuleList(blocks)
        self.lamb = nn.Parameter(torch.full((stages,), float(lamb)))
        self.tau = nn.Parameter(torch.full((stages,), float(tau)))
        self.checkpoint_stages = checkpoint_stages
        self.bf16 = bf16
        self._channels_last()

    def _channels_last(self):
        for b in self.blocks:
            b.to(memory_format=torch.channels_last_3d)

    def stage(self, s: int, x: torch.Tensor, p: torch.Tensor) -> torch.Tensor:
        grad = self.BP.apply(self.FP.apply(x) - p)
        with torch.autocast("cuda", dtype=torch.bfloat16, enabled=self.bf16):
            r = self.blocks[s](x.to(memory_format=torch.channels_last_3d))
        return x - self.lamb[s] * grad - self.tau[s] * r.float()

    def forward(self, x0: torch.Tensor, p: torch.Tensor, return_all: bool = False):
        x = x0
        xs = [x0]
        for s in range(self.stages):
            if self.checkpoint_stages and torch.is_grad_enabled():
                x = checkpoint(self.stage, s, x, p, use_reentrant=False)
            else:
                x = self.stage(s, x, p)
            if return_all:
                xs.append(x)
        return xs if return_all else x


class LEARN(UnrolledPDHG):
    """model/PDHG/LEARN.py:6-22: shared 4-layer, 8-feature ``Dual`` block,
    learned lamb and tao initialised to 10e-4, all iterates returned."""

    def __init__(self, projector: Projector, cascades: int = 30, checkpoint_stages: bool = True):
        super().__init__(projector, stages=cascades, features=8, lamb=10e-4, tau=10e-4,
                         share_weights=True, checkpoint_stages=checkpoint_stages, bf16=False)
        dual = nn.Sequential(
            nn.Conv3d(1, 8, 3, padding=1), nn.ReLU(), nn.Conv3d(8, 8, 3, padding=1), nn.ReLU(),
            nn.Conv3d(8, 8, 3, padding=1), nn.ReLU(), nn.Conv3d(8, 1, 3, padding=1))
        self.blocks = nn.ModuleList([dual] * cascades)
        self._channels_last()

    def forward(self, image, sino):
        return super().forward(image, sino, return_all=True)


def train(net: nn.Module, x0: torch.Tensor, sino: torch.Tensor, target: torch.Tensor,
          steps: int = 200, lr: float = 1e-4, callback=None):
    """Adam on the L2 loss to the target (the reference trains with Adam,
    train_v1.py:20-48). Returns the per-step losses (device tensor)."""
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    losses = torch.zeros(steps, device=x0.device)
    for i in range(steps):
        opt.zero_grad(set_to_none=True)
        out = net(x0, sino)
        loss = torch.mean((out - target) ** 2)
        loss.backward()
        opt.step()
        losses[i] = loss.detach()
        if callback is not None:
            callback(i, loss)
    return losses
