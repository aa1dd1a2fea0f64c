"""Seeded synthetic inputs: ellipsoid phantoms and Poisson-noisy projections.

The reference trained on CT data absent here; these stand in with the shapes
and value ranges of the measured configurations: 10 ellipsoids, centres
uniform in a ball of radius 0.8 * FOV/2, semi-axes uniform in [0.05, 0.4] * FOV,
uniformly random rotations (Haar quaternions), additive intensities uniform
in [-0.2, 1], rasterised at voxel centres in FP64.
"""
from __future__ import annotations

import numpy as np
import torch


def ellipsoid_params(seed: int, n: int = 10):
    rng = np.random.default_rng(seed)
    # centres: uniform in the ball of radius 0.8 (in units of FOV/2)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = 0.8 * rng.random(n) ** (1.0 / 3.0)
    centres = d * r[:, None]
    axes = rng.uniform(0.05, 0.4, size=(n, 3))  # fraction of the FOV
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)
    val = rng.uniform(-0.2, 1.0, size=n)
    return centres, axes, R, val


def ellipsoids(shape_zyx, seed: int = 0, n: int = 10, device="cpu",
               dtype=torch.float32) -> torch.Tensor:
    """[1,1,Z,Y,X] phantom; coordinates normalised so the FOV spans [-1,1] along
    the largest edge (voxels are isotropic)."""
    Z, Y, X = shape_zyx
    edge = max(X, Y, Z)
    centres, axes, R, val = ellipsoid_params(seed, n)
    dev = torch.device(device)
    out = torch.zeros((Z, Y, X), dtype=torch.float64, device=dev)
    zs = (torch.arange(Z, dtype=torch.float64, device=dev) - (Z - 1) / 2) * (2.0 / edge)
    ys = (torch.arange(Y, dtype=torch.float64, device=dev) - (Y - 1) / 2) * (2.0 / edge)
    xs = (torch.arange(X, dtype=torch.float64, device=dev) - (X - 1) / 2) * (2.0 / edge)
    for k in range(n):
        Rk = torch.as_tensor(R[k], dtype=torch.float64, device=dev)
        c = centres[k]
        # semi-axes as a fraction of the FOV (FOV = 2 in these units)
        a = torch.as_tensor(axes[k] * 2.0, dtype=torch.float64, device=dev)
        for z0 in range(0, Z, 32):
            zz = zs[z0:z0 + 32][:, None, None] - c[2]
            yy = ys[None, :, None] - c[1]
            xx = xs[None, None, :] - c[0]
            # body coordinates: R^T (p - c)
            bx = Rk[0, 0] * xx + Rk[1, 0] * yy + Rk[2, 0] * zz
            by = Rk[0, 1] * xx + Rk[1, 1] * yy + Rk[2, 1] * zz
            bz = Rk[0, 2] * xx + Rk[1, 2] * yy + Rk[2, 2] * zz
            inside = (bx / a[0]) ** 2 + (by / a[1]) ** 2 + (bz / a[2]) ** 2 <= 1.0
            out[z0:z0 + 32] += inside.to(torch.float64) * float(val[k])
    return out.to(dtype).reshape(1, 1, Z, Y, X)


def poisson_noise(sino: torch.Tensor, i0: float = 1e5, mu_scale: float = None,
                  seed: int = 0) -> torch.Tensor:
    """counts ~ Poisson(I0 exp(-mu_scale p)), p' = -ln(max(counts,1)/I0)/mu_scale.
    mu_scale defaults to 4 / max(p) (maximum attenuation line integral 4)."""
    p = sino.double()
    if mu_scale is None:
        m = float(p.max())
        mu_scale = 4.0 / m if m > 0 else 1.0
    g = torch.Generator(device=p.device).manual_seed(seed)
    lam = i0 * torch.exp(-mu_scale * p.clamp_min(0))
    counts = torch.poisson(lam, generator=g)
    return (-torch.log(counts.clamp_min(1.0) / i0) / mu_scale).to(sino.dtype)
