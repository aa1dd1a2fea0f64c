"""Reconstructions against the reference's own CUDA projectors.

tests/golden/ref_recons.npz (make_ref_recons.py) holds DTV-CP, FISTA,
DTV-FISTA and ASD-POCS reconstructions of a seeded 48 x 48 x 32 ellipsoid
phantom from 36 views of 72 x 40, computed with the reference's unmodified
forward projector and FDK backprojector kernels (run on a B200 through their
pybind API) inside the oracle's restatements of the reference loops. The same
reconstructions through this library's plans must match within a stated
FP32 tolerance: the reference filters with 1/256 texture weights in float32
coordinates, which the "tex" sampler reproduces (tight) and the exact "soft"
sampler does not (looser)."""
import os

import numpy as np
import pytest
import torch

import dtvb200
from helpers import rel_rmse

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_recons.npz")
# relative RMSE of each reconstruction against the reference-kernel run
TOL = {"tex": 1e-3, "soft": 5e-3}


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _plan(gold, sampler, cuda):
    X, Y, Z, W, H, n, sid, sdd = gold["geom"]
    ang = np.linspace(0, 360, int(n), endpoint=False).astype(np.float32)
    geo = dtvb200.standard(ang, (int(X), int(Y), int(Z)), (int(W), int(H)), float(sid),
                           float(sdd))
    return dtvb200.Plan(geo, sampler=sampler, device=cuda)


def _run(alg, gold, cuda):
    sino = torch.from_numpy(gold["sino"]).to(cuda)
    img = torch.zeros(tuple(gold["truth"].shape), device=cuda)
    return alg.run(img, sino).cpu().numpy()


@pytest.mark.parametrize("sampler", ["tex", "soft"])
@pytest.mark.parametrize("loop", ["dtvcp", "fista", "dtvfista", "asd"])
def test_reconstruction_matches_reference_kernels(cuda, gold, sampler, loop):
    plan = _plan(gold, sampler, cuda)
    p = gold[f"{loop}_params"]
    if loop == "dtvcp":
        alg = dtvb200.DTVCP(plan, int(p[6]), sigma=p[0], tau=p[1], mu=p[2], v=tuple(p[3:6]),
                            quirk=True, use_graph=True)
    elif loop == "fista":
        alg = dtvb200.FISTA(plan, int(p[2]), lamb=p[0], L=p[1], use_graph=True)
    elif loop == "dtvfista":
        alg = dtvb200.DTVFISTA(plan, int(p[7]), sigma=p[0], v=tuple(p[1:4]), t=tuple(p[4:7]),
                               quirk=False)
    else:
        alg = dtvb200.ASDPOCS(plan, int(p[5]), beta=p[0], beta_red=p[1], ng=int(p[2]),
                              alpha=p[3], rmax=p[4], quirk=True, use_graph=True)
    f = _run(alg, gold, cuda)
    ref = gold[f"{loop}_f"]
    assert float(np.abs(ref).max()) > 0
    assert rel_rmse(f, ref) < TOL[sampler], rel_rmse(f, ref)
