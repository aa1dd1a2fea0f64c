"""Golden vectors from the reference's own Python modules (run where the
reference tree is present; CPU only).

Imports, from the reference tree:
  model/PDHG/Utils/Gradients.py  (sparse D_x, D_y, D_z, their transposes)
  model/PDHG/Utils/L1ball.py     (L1-ball projection)
  model/PDHG/DTVCP.py, model/PDHG/ASDPOCS.py, model/FISTA/FISTA.py,
  model/FISTA/DTVFISTA.py        (the iteration loops)
and records their outputs on seeded inputs. The loops call
ForwardProjection/BackProjection from the reference geometry layers, whose
CUDA extension cannot run here; those two names are provided by a stub module
backed by the FP64 oracle (oracle/oracle.py), so what the fixtures pin is the
reference's loop arithmetic. `.cuda()` is made a no-op while the reference
modules build their sparse matrices on CPU.

Usage: python tests/golden/make_ref_utils.py [--ref-root DIR] [--out PATH]
"""
import argparse
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import oracle as O  # noqa: E402

# small projector shared by the loop fixtures (Standard conventions)
LOOP_VS = (6, 6, 4)  # X, Y, Z
LOOP_DS = (10, 6)
LOOP_N = 8
LOOP_SID, LOOP_SDD = 500.0, 1000.0
LOOP_ANGLES = np.linspace(0, 360, LOOP_N, endpoint=False).astype(np.float32)


def loop_geometry():
    return O.standard_geometry(LOOP_ANGLES.astype(np.float64), LOOP_VS, LOOP_DS, LOOP_SID,
                               LOOP_SDD)


def _stub_layers():
    geo = loop_geometry()

    class ForwardProjection(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x):
            return torch.from_numpy(O.forward(geo, x.detach().double().numpy())).float().reshape(
                x.shape[0], 1, *geo.sino_shape)

    class BackProjection(torch.autograd.Function):
        @staticmethod
        def forward(ctx, s):
            return torch.from_numpy(O.backward(geo, s.detach().double().numpy())).float().reshape(
                s.shape[0], 1, *geo.vol_shape)

    for name in ("model.ConeBeamLayers.Beijing.BeijingGeometry",
                 "model.ConeBeamLayers.Standard.StandardGeometry"):
        m = types.ModuleType(name)
        m.ForwardProjection = ForwardProjection
        m.BackProjection = BackProjection
        sys.modules[name] = m


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=os.environ.get(
        "DTV_REFERENCE_ROOT", os.path.join(os.path.dirname(REPO), "reference")))
    ap.add_argument("--out", default=os.path.join(HERE, "ref_utils.npz"))
    a = ap.parse_args()
    sys.path.insert(0, a.ref_root)
    _stub_layers()
    torch.Tensor.cuda = lambda self, *args, **kw: self  # CPU-only host
    from model.PDHG.Utils import Gradients, L1ball  # noqa: E402
    from model.PDHG.DTVCP import DTVCP  # noqa: E402
    from model.PDHG.ASDPOCS import ASDPOCS  # noqa: E402
    from model.FISTA.FISTA import DTVFista  # noqa: E402
    from model.FISTA.DTVFISTA import DTVFista as DTVFistaTV  # noqa: E402

    rng = np.random.default_rng(7)
    out = {}
    # --- finite differences (Gradients.py:8-34), X != Y exposes the y offset
    for tag, vs in (("a", (5, 4, 3)), ("b", (4, 4, 3))):
        N = int(np.prod(vs))
        f = rng.standard_normal(N).astype(np.float32)
        out[f"d{tag}_size"] = np.array(vs)
        out[f"d{tag}_f"] = f
        for ax, fn in enumerate((Gradients.spraseMatrixX, Gradients.spraseMatrixY,
                                 Gradients.spraseMatrixZ)):
            np.random.seed(0)
            D, DT, _ = fn(vs)
            x = torch.from_numpy(f)
            out[f"d{tag}_D{ax}"] = torch.matmul(D, x).numpy()
            out[f"d{tag}_DT{ax}"] = torch.matmul(DT, x).numpy()
    Gradients.matrixSet.clear()
    # --- L1 ball (L1ball.py:4-17)
    for i, (n, b) in enumerate(((50, 3.0), (1000, 40.0), (1000, 1e6), (4096, 0.0), (300, 7.5))):
        v = (rng.standard_normal(n) * rng.uniform(0.1, 3)).astype(np.float32)
        w = L1ball.l1ball(torch.from_numpy(v), b)
        out[f"l1_{i}_v"] = v
        out[f"l1_{i}_b"] = np.array(b)
        out[f"l1_{i}_w"] = w.numpy()
    # --- loops on the oracle projector
    X, Y, Z = LOOP_VS
    geo = loop_geometry()
    truth = np.zeros((1, 1, Z, Y, X), dtype=np.float32)
    truth[..., 1:3, 1:5, 2:5] = 1.0
    truth[..., 2, 2:4, 1:3] = 0.5
    sino = torch.from_numpy(O.forward(geo, truth)).float().reshape(1, 1, *geo.sino_shape)
    img0 = torch.zeros(1, 1, Z, Y, X)
    out["loop_truth"] = truth
    out["loop_sino"] = sino.numpy()
    out["loop_angles"] = LOOP_ANGLES
    out["loop_geom"] = np.array([*LOOP_VS, *LOOP_DS, LOOP_N, LOOP_SID, LOOP_SDD])

    np.random.seed(1)
    dtv = DTVCP(LOOP_VS, 12, False)
    dtv.sigma = dtv.tao = 2e-3   # steps that make progress on this tiny problem
    dtv.mu, dtv.v1, dtv.v2, dtv.v3 = 0.5, 0.4, 0.3, 0.2
    f = dtv.run(img0.clone(), sino)
    out["dtvcp_f"] = f.numpy()
    out["dtvcp_params"] = np.array([dtv.sigma, dtv.tao, dtv.mu, dtv.v1, dtv.v2, dtv.v3, 12])
    Gradients.matrixSet.clear()

    fista = DTVFista(15, False)
    fista.lamb, fista.L = 0.05, 2e-3
    f = fista.run(img0.clone(), sino)
    out["fista_f"] = f.numpy()
    out["fista_params"] = np.array([fista.lamb, fista.L, 15])

    np.random.seed(2)
    dfi = DTVFistaTV(LOOP_VS, 6, False)
    dfi.sigma = 2e-3
    f = dfi.run(img0.clone(), sino)
    out["dtvfista_f"] = f.numpy()
    out["dtvfista_params"] = np.array([dfi.sigma, dfi.v1, dfi.v2, dfi.v3, dfi.t1, dfi.t2, dfi.t3, 6])
    Gradients.matrixSet.clear()

    np.random.seed(3)
    asd = ASDPOCS(LOOP_VS, 5, False)
    asd.beta = 2e-3
    f = asd.run(img0.clone(), sino)
    out["asd_f"] = f.numpy()
    out["asd_params"] = np.array([2e-3, asd.beta_red, asd.ng, asd.alpha, asd.rmax, 5])
    np.savez_compressed(a.out, **out)
    print("wrote", a.out, len(out), "arrays")


if __name__ == "__main__":
    main()
