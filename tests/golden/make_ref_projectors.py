"""Golden projector vectors from the reference's own CUDA kernels.

Runs on a GPU host. Loads the reference extensions JITStandardGeometry /
JITBeijingGeometry that oracle/ref_build/build_ref.py compiled from the
reference's unmodified sources into oracle/_ref/, runs them through their own
pybind API (the calls model/ConeBeamLayers/{Standard,Beijing}/*Geometry.py
make) on seeded inputs, and writes the inputs and outputs to an .npz file
(default tests/golden/ref_projectors.npz).

Usage: python tests/golden/make_ref_projectors.py [--out PATH]
"""
import argparse
import importlib.machinery
import importlib.util
import os
import sys

import numpy as np
import torch

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(REPO, "oracle", "_ref")


def load_ext(name):
    path = os.path.join(REF, name + ".so")
    loader = importlib.machinery.ExtensionFileLoader(name, path)
    spec = importlib.util.spec_from_file_location(name, path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def smooth_volume(rng, shape_zyx):
    """Random blobs plus a sharp-edged box, float32."""
    Z, Y, X = shape_zyx
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    v = np.zeros(shape_zyx)
    for _ in range(6):
        c = rng.uniform(0.2, 0.8, 3) * np.array([Z, Y, X])
        s = rng.uniform(0.1, 0.3) * min(X, Y, Z)
        v += rng.uniform(0.2, 1.0) * np.exp(-((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2)
                                             / (2 * s * s))
    v[Z // 4:3 * Z // 4, Y // 3:2 * Y // 3, X // 3:2 * X // 3] += 0.5
    return v.astype(np.float32)


def vector_views(n, sod, sdd, du, dv, tilt):
    """[n,12] per-view vectors in the layout the reference reads
    (source, detector, v, u; z stored negated, Beijing forwardKernel.cu:27-30)."""
    pv = np.zeros((n, 12), dtype=np.float32)
    for i in range(n):
        t = 2 * np.pi * i / n
        ex = np.array([np.cos(t), np.sin(t), 0.0])
        ey = np.array([-np.sin(t), np.cos(t), 0.0])
        ez = np.array([0.0, 0.0, 1.0])
        src = -sod * ex + np.array([0, 0, tilt * np.sin(3 * t)])
        det = (sdd - sod) * ex
        u = du * ey
        v = dv * (ez + 0.05 * ex)
        pv[i, 0:3] = src * [1, 1, -1]
        pv[i, 3:6] = det * [1, 1, -1]
        pv[i, 6:9] = v
        pv[i, 9:12] = u
    return pv


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(REPO, "tests", "golden", "ref_projectors.npz"))
    a = ap.parse_args()
    std = load_ext("JITStandardGeometry")
    bj = load_ext("JITBeijingGeometry")
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(1234)
    out = {}
    cases = [
        # name, (X,Y,Z), (W,H), n_views, sid, sdd, batch
        ("s1", (16, 12, 8), (24, 16), 12, 500.0, 1000.0, 2),
        ("s2", (20, 20, 10), (30, 12), 9, 300.0, 800.0, 1),
        ("s3", (64, 64, 32), (96, 48), 30, 1000.0, 2000.0, 1),
    ]
    for name, vs, ds, n, sid, sdd, b in cases:
        X, Y, Z = vs
        W, H = ds
        vol = np.stack([smooth_volume(rng, (Z, Y, X)) for _ in range(b)])[:, None]
        angles = np.linspace(0, 360, n, endpoint=False)  # StandardGeometry.py:6
        sino_in = rng.random((b, 1, n, H, W)).astype(np.float32)
        va = torch.from_numpy(vol).to(dev)
        at = torch.from_numpy(angles).to(dev)
        vst = torch.tensor(vs).to(dev)
        dst = torch.tensor(ds).to(dev)
        fp = std.forward(va, at, vst, dst, sid, sdd, 0)
        bp = std.backward(torch.from_numpy(sino_in).to(dev), at, vst, dst, sid, sdd, 0)
        torch.cuda.synchronize()
        out[f"{name}_vol"] = vol
        out[f"{name}_angles"] = angles
        out[f"{name}_sizes"] = np.array([X, Y, Z, W, H, n, b])
        out[f"{name}_geom"] = np.array([sid, sdd])
        out[f"{name}_fp"] = fp.cpu().numpy()
        out[f"{name}_sino_in"] = sino_in
        out[f"{name}_bp"] = bp.cpu().numpy()
    # vector geometry: the reference backprojector copies 1512-view texture
    # chunks (backwardKernel.cu:76-101), so the view count is a multiple of 1512
    X, Y, Z, W, H, n = 12, 12, 8, 16, 8, 1512
    pv = vector_views(n, 40.0, 70.0, 1.6, 1.7, 1.5)
    vol = smooth_volume(rng, (Z, Y, X))[None, None]
    sino_in = rng.random((1, 1, n, H, W)).astype(np.float32)
    vst = torch.IntTensor([X, Y, Z]).to(dev)
    dst = torch.IntTensor([W, H]).to(dev)
    pvt = torch.from_numpy(pv).contiguous().to(dev)
    fp = bj.forward(torch.from_numpy(vol).to(dev), vst, dst, pvt, 0)
    bp = bj.backward(torch.from_numpy(sino_in).to(dev), vst, dst, pvt, 0)
    torch.cuda.synchronize()
    out.update(v_vol=vol, v_pv=pv, v_sizes=np.array([X, Y, Z, W, H, n, 1]),
               v_fp=fp.cpu().numpy(), v_sino_in=sino_in, v_bp=bp.cpu().numpy())
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    np.savez_compressed(a.out, **out)
    print("wrote", a.out, {k: v.shape for k, v in out.items()})
    return 0


if __name__ == "__main__":
    sys.exit(main())
