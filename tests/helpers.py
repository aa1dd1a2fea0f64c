"""Shared test helpers (seeded inputs, geometry cases)."""
import numpy as np


def rel_rmse(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.sqrt(np.mean((a - b) ** 2))
    n = np.sqrt(np.mean(b ** 2))
    return d / n if n > 0 else d


def rel_max(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.abs(b).max()
    return np.abs(a - b).max() / n if n > 0 else np.abs(a - b).max()


def blob_volume(rng, shape_zyx, batch=1):
    """Smooth blobs plus a sharp box (float32, [B,1,Z,Y,X])."""
    Z, Y, X = shape_zyx
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    out = []
    for _ in range(batch):
        v = np.zeros(shape_zyx)
        for _ in range(5):
            c = rng.uniform(0.2, 0.8, 3) * np.array([Z, Y, X])
            s = rng.uniform(0.1, 0.3) * min(X, Y, Z) + 0.5
            v += rng.uniform(0.2, 1.0) * np.exp(
                -((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2) / (2 * s * s))
        v[Z // 4:3 * Z // 4 + 1, Y // 3:2 * Y // 3 + 1, X // 3:2 * X // 3 + 1] += 0.5
        out.append(v)
    return np.stack(out)[:, None].astype(np.float32)


def vector_views(n, sod, sdd, du, dv, tilt=0.0):
    """[n,12] projection vectors in the Beijing layout (source, detector, v, u;
    z of source and detector stored negated)."""
    pv = np.zeros((n, 12), dtype=np.float32)
    for i in range(n):
        t = 2 * np.pi * i / n
        ex = np.array([np.cos(t), np.sin(t), 0.0])
        ey = np.array([-np.sin(t), np.cos(t), 0.0])
        ez = np.array([0.0, 0.0, 1.0])
        src = -sod * ex + np.array([0, 0, tilt * np.sin(3 * t)])
        det = (sdd - sod) * ex
        pv[i, 0:3] = src * [1, 1, -1]
        pv[i, 3:6] = det * [1, 1, -1]
        pv[i, 6:9] = dv * (ez + 0.05 * ex)
        pv[i, 9:12] = du * ey
    return pv
