"""Golden reconstructions driven by the reference's own CUDA projectors.

Runs on a GPU host. The reference's forward projector and FDK backprojector
are its unmodified kernels (model/ConeBeamLayers/Standard/plug/kernel/
{forward,backward}Kernel.cu), compiled by oracle/ref_build/build_ref.py into
oracle/_ref/ and called through their own pybind API exactly as
StandardGeometry.py calls them. The iteration loops are the oracle's FP64
restatements of the reference's DTVCP.run (model/PDHG/DTVCP.py:29-60),
DTVFista.run (model/FISTA/FISTA.py:16-27), DTVFista.run
(model/FISTA/DTVFISTA.py:23-43) and ASDPOCS.run (model/PDHG/ASDPOCS.py:28-47),
which tests/golden/ref_utils.npz pins to those Python loops to about 3e-7
(the reference's Python cannot run on the GPU host, where its tree is
absent). The phantom is a seeded 10-ellipsoid volume; its sinogram is the
reference kernels' projection of it.

Usage: python tests/golden/make_ref_recons.py [--out PATH]
"""
import argparse
import importlib.machinery
import importlib.util
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "dtv-net_b200"))
import oracle as O  # noqa: E402

# Standard layer convention (voxel = detector pixel * SID/SDD)
VS = (48, 48, 32)   # X, Y, Z
DS = (72, 40)       # W, H
N_VIEWS = 36
SID, SDD = 500.0, 1000.0
SEED = 77
ITERS = dict(dtvcp=20, fista=20, dtvfista=10, asd=8)


def load_ext(name):
    path = os.path.join(REPO, "oracle", "_ref", name + ".so")
    loader = importlib.machinery.ExtensionFileLoader(name, path)
    spec = importlib.util.spec_from_file_location(name, path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def reference_operators(dev):
    """fp(x), bp(s) on FP64 numpy arrays [B,1,...] through the reference's
    kernels (float32 in and out, as its layer passes them)."""
    ext = load_ext("JITStandardGeometry")
    angles = np.linspace(0, 360, N_VIEWS, endpoint=False)  # StandardGeometry.py:6
    at = torch.from_numpy(angles).to(dev)
    vst, dst = torch.tensor(VS).to(dev), torch.tensor(DS).to(dev)

    def fp(x):
        t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).to(dev)
        return ext.forward(t, at, vst, dst, SID, SDD, dev.index).double().cpu().numpy()

    def bp(s):
        t = torch.from_numpy(np.ascontiguousarray(s, dtype=np.float32)).to(dev)
        return ext.backward(t, at, vst, dst, SID, SDD, dev.index).double().cpu().numpy()

    return fp, bp


def spectral_radius(fp, bp, shape, iters=12):
    """||BP FP|| by the power method (seeded), for step sizes that converge."""
    x = np.random.default_rng(5).random(shape)
    lam = 1.0
    for _ in range(iters):
        y = bp(fp(x))
        lam = np.linalg.norm(y) / np.linalg.norm(x)
        x = y / np.linalg.norm(y)
    return float(lam)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_recons.npz"))
    a = ap.parse_args()
    from dtvb200.phantom import ellipsoids
    dev = torch.device("cuda", 0)
    fp, bp = reference_operators(dev)
    X, Y, Z = VS
    truth = ellipsoids((Z, Y, X), seed=SEED).numpy().astype(np.float64)
    sino = fp(truth)
    lam = spectral_radius(fp, bp, truth.shape)
    zero = np.zeros_like(truth)
    out = {"truth": truth.astype(np.float32), "sino": sino.astype(np.float32),
           "geom": np.array([*VS, *DS, N_VIEWS, SID, SDD]), "radius": np.array(lam)}
    s = 0.9 / lam
    v, mu = (0.5, 0.5, 0.5), 1.0
    out["dtvcp_params"] = np.array([s, s, mu, *v, ITERS["dtvcp"]])
    out["dtvcp_f"] = O.dtvcp_run(fp, bp, zero, sino, VS, ITERS["dtvcp"], s, s, mu, v,
                                 quirk=True).astype(np.float32)
    L, lamb = 1.0 / lam, 1e-3
    out["fista_params"] = np.array([lamb, L, ITERS["fista"]])
    out["fista_f"] = O.fista_run(fp, bp, zero, sino, ITERS["fista"], L, lamb).astype(np.float32)
    # DTV-FISTA (DTVFISTA.py:23-43) with its intended soft-thresholds: the
    # reference's torch.max quirk thresholds by a global maximum, which makes
    # the result flip with the sign of near-zero differences
    vt, t = (0.05, 0.05, 0.05), (1e-3, 1e-3, 1e-3)
    out["dtvfista_params"] = np.array([s, *vt, *t, ITERS["dtvfista"]])
    out["dtvfista_f"] = O.dtvfista_run(fp, bp, zero, sino, VS, ITERS["dtvfista"], s, vt, t,
                                       quirk=False).astype(np.float32)
    beta = 0.5 / lam
    out["asd_params"] = np.array([beta, 0.9999, 10, 0.001, 0.95, ITERS["asd"]])
    out["asd_f"] = O.asdpocs_run(fp, bp, zero, sino, VS, ITERS["asd"], beta, 0.9999, 10, 0.001,
                                 0.95, quirk=True).astype(np.float32)
    np.savez_compressed(a.out, **out)
    print("wrote", a.out, {k: (v.shape, float(np.abs(v).max())) for k, v in out.items()})
    return 0


if __name__ == "__main__":
    sys.exit(main())
