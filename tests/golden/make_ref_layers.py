"""Golden vectors of the reference's geometry layers and unrolled networks.

Imports, unmodified, from the reference tree (CPU only):
  model/ConeBeamLayers/Beijing/BeijingGeometry.py   (autograd pair with the
      (view, plane) permutation and sampleInterval, BeijingGeometry,
      BeijingGeometryWithFBP)
  model/ConeBeamLayers/Standard/StandardGeometry.py (StandardGeometry,
      StandardGeometryWithFBP)
  model/FISTA/DTVSTAnet.py (DTVNet), model/FISTA/FISTAnet.py (FistaNet),
  model/PDHG/LEARN.py (LEARN) with their CNN blocks
from a temporary directory whose options.yaml (a copy of the reference's with
small geometries) and projection-matrix .mat file they read at import time.
Only the two pybind projector extensions, which cannot run without a GPU, are
replaced: JITStandardGeometry and JITBeijingGeometry become modules whose
forward/backward are the FP64 oracle's literal restatements of the reference
kernels (oracle/oracle.c), returned as float32 like the extensions. Networks
are built under fixed torch seeds; their weights, every cascade iterate and
the gradients of a fixed scalar loss are recorded.

Usage: python tests/golden/make_ref_layers.py [--ref-root DIR] [--out PATH]
(DIR defaults to $DTV_REFERENCE_ROOT, else a `reference` checkout beside this
repository.)
"""
import argparse
import contextlib
import importlib
import os
import shutil
import sys
import tempfile
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "tests"))
import oracle as O  # noqa: E402
from helpers import vector_views  # noqa: E402

# Standard layer geometry (X, Y, Z volume; W, H detector)
STD = dict(standardAngleNum=6, standardDetectorSize=[24, 12], standardVolumeSize=[16, 16, 8],
           standardSID=500, standardSDD=1000)
# Beijing layer geometry: 7 angles x 3 planes = 21 views (the backprojector's
# 2*pi/(N//21) scale needs N >= 21), 12 x 10 sub-detectors
BJ = dict(beijingAngleNum=7, beijingPlanes=3, beijingSubDetectorSize=[12, 10],
          beijingVolumeSize=[16, 16, 8], beijingSID=40, beijingSDD=70, sampleInterval=1.7)
BJ_PV = dict(sod=40.0, sdd=70.0, du=1.6, dv=1.7, tilt=1.5)
SEEDS = dict(dtvnet=11, fistanet=12, learn=13)
CASCADES = dict(dtvnet=2, fistanet=3, learn=3)


def default_ref_root():
    return os.environ.get("DTV_REFERENCE_ROOT",
                          os.path.join(os.path.dirname(REPO), "reference"))


def beijing_vectors():
    n = BJ["beijingAngleNum"] * BJ["beijingPlanes"]
    p = BJ_PV
    return vector_views(n, p["sod"], p["sdd"], p["du"], p["dv"], p["tilt"])


def _batch_first(t):
    return t.detach().double().numpy()


def _stubs():
    std = types.ModuleType("JITStandardGeometry")
    bj = types.ModuleType("JITBeijingGeometry")

    def s_fwd(vol, angles, vs, ds, sid, sdd, device):
        out = O.forward_standard_literal(_batch_first(vol), angles.numpy(), vs.tolist(),
                                         ds.tolist(), sid, sdd)
        return torch.from_numpy(out).float().reshape(vol.shape[0], 1, *out.shape[1:])

    def s_bwd(sino, angles, vs, ds, sid, sdd, device):
        out = O.backward_standard_literal(_batch_first(sino), angles.numpy(), vs.tolist(),
                                          ds.tolist(), sid, sdd)
        return torch.from_numpy(out).float().reshape(sino.shape[0], 1, *out.shape[1:])

    def b_fwd(vol, vs, ds, pv, device):
        out = O.forward_vector_literal(_batch_first(vol), pv.numpy(), vs.tolist(), ds.tolist())
        return torch.from_numpy(out).float().reshape(vol.shape[0], 1, *out.shape[1:])

    def b_bwd(sino, vs, ds, pv, device):
        out = O.backward_vector_literal(_batch_first(sino), pv.numpy(), vs.tolist(), ds.tolist())
        return torch.from_numpy(out).float().reshape(sino.shape[0], 1, *out.shape[1:])

    std.forward, std.backward = s_fwd, s_bwd
    bj.forward, bj.backward = b_fwd, b_bwd
    return std, bj


@contextlib.contextmanager
def reference_modules(ref_root):
    """Yields a function importing reference modules by dotted name, with the
    stub projectors and the small-geometry options.yaml in place."""
    import scipy.io
    import yaml
    names = ("JITStandardGeometry", "JITBeijingGeometry", "options")
    saved = {k: sys.modules.get(k) for k in names}
    cwd = os.getcwd()
    tmp = tempfile.mkdtemp(prefix="reflayers_")
    try:
        y = yaml.load(open(os.path.join(ref_root, "options.yaml")), yaml.FullLoader)
        y.update(STD)
        y.update(BJ)
        y["beijingParameterRoot"] = os.path.join(tmp, "projection_matrix.mat")
        y["debug"] = tmp
        scipy.io.savemat(y["beijingParameterRoot"], {"projection_matrix": beijing_vectors()})
        with open(os.path.join(tmp, "options.yaml"), "w") as f:
            yaml.safe_dump(y, f)
        std, bj = _stubs()
        sys.modules["JITStandardGeometry"] = std
        sys.modules["JITBeijingGeometry"] = bj
        sys.modules.pop("options", None)
        sys.path.insert(0, ref_root)
        os.chdir(tmp)
        yield importlib.import_module
    finally:
        os.chdir(cwd)
        sys.path.remove(ref_root)
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
        for k in [m for m in sys.modules if m == "model" or m.startswith("model.")]:
            sys.modules.pop(k, None)
        shutil.rmtree(tmp, ignore_errors=True)


def inputs():
    """Seeded layer inputs: Beijing volume and layer-layout sinogram, Standard
    volume and sinogram, and the scalar-loss weights."""
    rng = np.random.default_rng(2024)
    X, Y, Z = BJ["beijingVolumeSize"]
    W, H = BJ["beijingSubDetectorSize"]
    N = BJ["beijingAngleNum"] * BJ["beijingPlanes"]
    sx, sy, sz = STD["standardVolumeSize"]
    sw, sh = STD["standardDetectorSize"]
    sn = STD["standardAngleNum"]
    f32 = np.float32
    return {
        "bj_x": rng.random((1, 1, Z, Y, X)).astype(f32),
        "bj_p": (rng.random((1, 1, N, H, W)) * 10).astype(f32),
        "bj_r": rng.standard_normal((1, 1, Z, Y, X)).astype(f32),
        "std_x": rng.random((1, 1, sz, sy, sx)).astype(f32),
        "std_p": (rng.random((1, 1, sn, sh, sw)) * 5).astype(f32),
        "std_r": rng.standard_normal((1, 1, sz, sy, sx)).astype(f32),
    }


FULL = 4096  # tensors up to this many elements are stored whole, larger ones as checksums


def summary(t):
    """[sum, sum of squares, max |.|] in FP64: enough to show two tensors are
    the same without storing them."""
    a = np.asarray(t, dtype=np.float64)
    return np.array([a.sum(), (a * a).sum(), np.abs(a).max()])


def _store(out, key, t):
    t = t.detach().numpy()
    if t.size <= FULL:
        out[key] = t.copy()
    else:
        out[key + "#sum"] = summary(t)


def _net_record(out, tag, net, image, sino, r):
    """Weights (built under a fixed seed, so a mirror built the same way must
    reproduce them), every cascade iterate and the gradients of sum(t_C * r)."""
    for k, v in net.state_dict().items():
        if not v.is_sparse:
            _store(out, f"{tag}_sd_{k}", v)
    img = torch.from_numpy(image).requires_grad_(True)
    t = net(img, torch.from_numpy(sino))
    for k, tk in enumerate(t):
        out[f"{tag}_t{k}"] = tk.detach().numpy().copy()
    (t[-1] * torch.from_numpy(r)).sum().backward()
    out[f"{tag}_grad_image"] = img.grad.numpy().copy()
    for k, v in net.named_parameters():
        if v.grad is not None and not v.is_sparse:
            _store(out, f"{tag}_grad_{k}", v.grad)


def record(ref_root):
    inp = inputs()
    out = dict(inp)
    out["bj_pv"] = beijing_vectors()
    with reference_modules(ref_root) as imp:
        bjg = imp("model.ConeBeamLayers.Beijing.BeijingGeometry")
        sg = imp("model.ConeBeamLayers.Standard.StandardGeometry")
        x, p, r = (torch.from_numpy(inp[k]) for k in ("bj_x", "bj_p", "bj_r"))
        out["bj_fp"] = bjg.ForwardProjection.apply(x).numpy()
        out["bj_bp"] = bjg.BackProjection.apply(p).numpy()
        out["bj_layer"] = bjg.BeijingGeometry()(x, p).numpy()
        xg = x.clone().requires_grad_(True)
        (bjg.BeijingGeometry()(xg, p) * r).sum().backward()
        out["bj_layer_grad"] = xg.grad.numpy()
        out["bj_fbp"] = bjg.BeijingGeometryWithFBP()(x, p).detach().numpy()
        xs, ps, rs = (torch.from_numpy(inp[k]) for k in ("std_x", "std_p", "std_r"))
        out["std_layer"] = sg.StandardGeometry()(xs, ps).numpy()
        xg = xs.clone().requires_grad_(True)
        (sg.StandardGeometry()(xg, ps) * rs).sum().backward()
        out["std_layer_grad"] = xg.grad.numpy()
        out["std_fbp"] = sg.StandardGeometryWithFBP()(xs, ps).detach().numpy()

        dtv = imp("model.FISTA.DTVSTAnet")
        torch.manual_seed(SEEDS["dtvnet"])
        net = dtv.DTVNet(tuple(BJ["beijingVolumeSize"]), CASCADES["dtvnet"])
        _net_record(out, "dtvnet", net, inp["bj_x"], inp["bj_p"], inp["bj_r"])
        fista = imp("model.FISTA.FISTAnet")
        torch.manual_seed(SEEDS["fistanet"])
        net = fista.FistaNet(CASCADES["fistanet"])
        _net_record(out, "fistanet", net, inp["bj_x"], inp["bj_p"], inp["bj_r"])
        learn = imp("model.PDHG.LEARN")
        torch.manual_seed(SEEDS["learn"])
        net = learn.LEARN(CASCADES["learn"])
        _net_record(out, "learn", net, inp["std_x"], inp["std_p"], inp["std_r"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=default_ref_root())
    ap.add_argument("--out", default=os.path.join(HERE, "ref_layers.npz"))
    a = ap.parse_args()
    out = record(a.ref_root)
    np.savez_compressed(a.out, **out)
    print("wrote", a.out, len(out), "arrays")
    return 0


if __name__ == "__main__":
    sys.exit(main())
