"""Unrolled reconstruction networks on the B200 projector pair.

Mirrors of the reference's three unrolled networks, with the same module and
parameter names so their state dicts load (``load_reference_state_dict``):

* ``DTVNet`` (model/FISTA/DTVSTAnet.py:8-46), the paper model: per cascade a
  gradient step through the geometry layer, the directional differences
  D_x, D_y, D_z, a CNN prox per direction plus one on the image, learned
  relaxations ntx, nty, ntz, nt, and the D^T recombination. The differences
  run in the stencil kernel (dtv_diff) instead of sparse N x N matrices;
  their autograd backward is the transposed stencil, as the sparse matmul's
  is the transposed matrix.
* ``FistaNet`` (model/FISTA/FISTAnet.py:8-23): one geometry layer and one
  ``BasicBlock`` shared by every cascade, learned extrapolation mu.
* ``LEARN`` (model/PDHG/LEARN.py:6-22): learned lamb, tao and a shared
  ``Dual`` CNN.

The geometry layer is any of this package's layers (``BeijingGeometry`` for
DTVNet and FistaNet, the Standard ``make_functions`` pair for LEARN). Its
``matched`` flag picks the reference's pairing (the FDK backprojector as the
forward projector's gradient) or the exact adjoint. Cascades may be
checkpointed (their activations recomputed in the backward pass), and the
CNN blocks may run their activations in BF16 under autocast with FP32 weights.

``UnrolledPDHG`` is the generic form used by the training benchmark:
x <- x - lamb_s A^T (A x - p) - tau_s R_s(x) with a 3-layer conv block per stage.
"""
from __future__ import annotations

import torch
import torch.nn as nn
from torch.utils.checkpoint import checkpoint

from .ops import Projector, make_functions
from .tv import diff


class Diff(torch.autograd.Function):
    """D_axis x per batch item (dtv_diff); backward D_axis^T g. ``quirk`` keeps
    the reference's D_y offset of volumeSize[1] that wraps across z-slices
    (Gradients.py:18-25)."""

    @staticmethod
    def forward(ctx, x, axis: int, transpose: bool, quirk: bool):
        ctx.args = (axis, transpose, quirk)
        return diff(x.contiguous(), axis, transpose, quirk)

    @staticmethod
    def backward(ctx, g):
        axis, transpose, quirk = ctx.args
        return diff(g.contiguous(), axis, not transpose, quirk), None, None, None


def _autocast(enabled: bool, device_type: str):
    return torch.autocast(device_type, dtype=torch.bfloat16, enabled=enabled)


class BasicBlock(nn.Module):
    """The reference's 3-D encoder-decoder prox (model/FISTA/RegularizationLayers/
    BasicBlock.py:7-62), same layers and names: a 1->f conv, two stride-(1,2,2)
    downsamplings with skip connections, nearest upsampling back, an f*2->1
    conv, and relu(x + residual) (non-negative output). Y and X must be
    multiples of 4."""

    def __init__(self, features: int = 32):
        super().__init__()
        f = features
        self.Sp = nn.Softplus()  # unused, kept so state dicts match
        self.conv_D = nn.Conv3d(1, f, 3, stride=1, padding=1)
        self.conv1_forward = nn.Conv3d(f, f, 3, stride=(1, 2, 2), padding=1)
        self.conv2_forward = nn.Conv3d(f, f, 3, stride=1, padding=1)
        self.conv3_forward = nn.Conv3d(f, f, 3, stride=(1, 2, 2), padding=1)
        self.conv4_forward = nn.Conv3d(f, f, 3, stride=1, padding=1)
        self.conv1_backward = nn.Conv3d(f, f, 3, stride=1, padding=1)
        self.conv2_backward = nn.Conv3d(2 * f, f, 3, stride=1, padding=1)
        self.conv3_backward = nn.Conv3d(2 * f, f, 3, stride=1, padding=1)
        self.conv4_backward = nn.Conv3d(2 * f, f, 3, stride=1, padding=1)
        self.conv_G = nn.Conv3d(2 * f, 1, 3, stride=1, padding=1)
        self.relu = nn.ReLU(inplace=True)
        self.upsample = nn.Upsample(scale_factor=(1, 2, 2), mode="nearest")

    def forward(self, x):
        x_d = self.conv_D(x)
        l1 = self.relu(self.conv1_forward(x_d))
        l2 = self.relu(self.conv2_forward(l1))
        l3 = self.relu(self.conv3_forward(l2))
        xf = self.conv4_forward(l3)
        b1 = self.relu(self.conv1_backward(xf))
        b2 = self.relu(self.conv2_backward(torch.cat([l3, b1], 1)))
        b2 = self.upsample(b2)
        b3 = self.relu(self.conv3_backward(torch.cat([l2, b2], 1)))
        xb = self.relu(self.conv4_backward(torch.cat([l1, b3], 1)))
        xb = self.upsample(xb)
        x_g = self.conv_G(torch.cat([x_d, xb], 1))
        return torch.relu(x + x_g.to(x.dtype))


class Dual(nn.Module):
    """model/PDHG/RegularizationLayers/CNN.py:4-18: four 3x3x3 convs, 8 features."""

    def __init__(self, features: int = 8):
        super().__init__()
        f = features
        self.convolutions = nn.Sequential(
            nn.Conv3d(1, f, 3, padding=1), nn.ReLU(), nn.Conv3d(f, f, 3, padding=1), nn.ReLU(),
            nn.Conv3d(f, f, 3, padding=1), nn.ReLU(), nn.Conv3d(f, 1, 3, padding=1))

    def forward(self, image):
        return self.convolutions(image)


_SPARSE_KEYS = ("dx", "dxt", "dy", "dyt", "dz", "dzt")


def load_reference_state_dict(net: nn.Module, state: dict, strict: bool = True):
    """Load a reference checkpoint's state dict (train_v1.py:62-64 saves
    net.state_dict()): the sparse difference matrices DTVNet stored as
    frozen parameters are dropped, as this package computes them as stencils."""
    sd = {k: v for k, v in state.items() if k not in _SPARSE_KEYS}
    return net.load_state_dict(sd, strict=strict)


class _Cascades(nn.Module):
    checkpoint_stages = False
    bf16 = False

    def _run(self, fn, *args):
        if self.checkpoint_stages and torch.is_grad_enabled():
            return checkpoint(fn, *args, use_reentrant=False)
        return fn(*args)

    def _prox(self, block, x):
        with _autocast(self.bf16, x.device.type):
            return block(x).float() if self.bf16 else block(x)


class DTVNet(_Cascades):
    """model/FISTA/DTVSTAnet.py:8-46 (``ITE`` is the geometry layer,
    ``-lamb * BP(FP(x) - p)``). forward(image, sino) returns the list of all
    cascade iterates [image, t1, ..., tC], as the reference does."""

    def __init__(self, layer: nn.Module, cascades: int = 3, quirk: bool = True,
                 features: int = 32, checkpoint_stages: bool = False, bf16: bool = False):
        super().__init__()
        self.cascades = cascades
        self.ITE = layer
        self.AE = nn.ModuleList([BasicBlock(features) for _ in range(4)])
        self.ntx = nn.Parameter(torch.tensor([-0.01] * cascades))
        self.nty = nn.Parameter(torch.tensor([-0.01] * cascades))
        self.ntz = nn.Parameter(torch.tensor([-0.01] * cascades))
        self.nt = nn.Parameter(torch.tensor([-0.1] * cascades))
        self.quirk = quirk
        self.checkpoint_stages = checkpoint_stages
        self.bf16 = bf16

    def _d(self, x, axis, transpose=False):
        return Diff.apply(x, axis, transpose, self.quirk)

    def _cascade(self, k, t, p, q, s, sino):
        z = t + self.ITE(t, sino)
        pnew, qnew, snew = self._d(z, 0), self._d(z, 1), self._d(z, 2)
        p_ = self._prox(self.AE[0], pnew) - pnew
        q_ = self._prox(self.AE[1], qnew) - qnew
        s_ = self._prox(self.AE[2], snew) - snew
        znew = self._prox(self.AE[3], z)
        p = p + self.ntx[k] * (p - p_)
        q = q + self.nty[k] * (q - q_)
        s = s + self.ntz[k] * (s - s_)
        z_ = t + self.nt[k] * (t - znew)
        t_next = self._d(q, 1, True) + self._d(p, 0, True) + self._d(s, 2, True) + z_
        return t_next, p, q, s

    def forward(self, image, sino):
        t = [image]
        zero = torch.zeros_like(image)
        p = q = s = zero  # the reference starts them at the scalar 0
        for k in range(self.cascades):
            tk, p, q, s = self._run(self._cascade, k, t[k], p, q, s, sino)
            t.append(tk)
        return t


class FistaNet(_Cascades):
    """model/FISTA/FISTAnet.py:8-23: z = t + ITE(t, sino); z = AE(z);
    t_next = t + mu_k (t - z), with the geometry layer and the BasicBlock
    shared by every cascade (``nn.ModuleList([m] * n)``)."""

    def __init__(self, layer: nn.Module, cascades: int = 3, features: int = 32,
                 checkpoint_stages: bool = False, bf16: bool = False):
        super().__init__()
        self.cascades = cascades
        self.ITE = nn.ModuleList([layer] * cascades)
        self.AE = nn.ModuleList([BasicBlock(features)] * cascades)
        self.mu = nn.Parameter(torch.tensor([-0.03] * cascades))
        self.checkpoint_stages = checkpoint_stages
        self.bf16 = bf16

    def _cascade(self, k, t, sino):
        z = t + self.ITE[k](t, sino)
        z = self._prox(self.AE[k], z)
        return t + self.mu[k] * (t - z)

    def forward(self, image, sino):
        t = [image]
        for k in range(self.cascades):
            t.append(self._run(self._cascade, k, t[k], sino))
        return t


class LEARN(_Cascades):
    """model/PDHG/LEARN.py:6-22: t_next = t - lamb_k BP(FP(t) - sino)
    - tao_k Dual(t), with one ``Dual`` CNN shared by every cascade and lamb,
    tao initialised to 10e-4. ``matched`` picks the exact adjoint for the
    backprojection and its gradient instead of the reference pairing."""

    def __init__(self, projector: Projector, cascades: int = 30, matched: bool = False,
                 checkpoint_stages: bool = False, bf16: bool = False):
        super().__init__()
        self.cascades = cascades
        self.FP, self.BP = make_functions(projector, matched)
        self.Dual = nn.ModuleList([Dual()] * cascades)
        self.lamb = nn.Parameter(torch.tensor([10e-4] * cascades))
        self.tao = nn.Parameter(torch.tensor([10e-4] * cascades))
        self.checkpoint_stages = checkpoint_stages
        self.bf16 = bf16

    def _cascade(self, k, t, sino):
        w = self.lamb[k] * self.BP.apply(self.FP.apply(t) - sino)
        prox = self.tao[k] * self._prox(self.Dual[k], t)
        return t - w - prox

    def forward(self, image, sino):
        t = [image]
        for k in range(self.cascades):
            t.append(self._run(self._cascade, k, t[k], sino))
        return t


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
    (LEARN.py:11, FISTAnet.py:12-13). The blocks run channels-last 3-D, the
    layout cuDNN's tensor-core convolutions take without transposes."""

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


def train(net: nn.Module, x0: torch.Tensor, sino: torch.Tensor, target: torch.Tensor,
          steps: int = 200, lr: float = 1e-4, callback=None):
    """Adam on the L2 loss to the target (the reference trains with Adam,
    train_v1.py:20-48). Networks that return every cascade iterate are scored
    on the last one. Returns the per-step losses (device tensor)."""
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    losses = torch.zeros(steps, device=x0.device)
    for i in range(steps):
        opt.zero_grad(set_to_none=True)
        out = net(x0, sino)
        if isinstance(out, (list, tuple)):
            out = out[-1]
        loss = torch.mean((out - target) ** 2)
        loss.backward()
        opt.step()
        losses[i] = loss.detach()
        if callback is not None:
            callback(i, loss)
    return losses
