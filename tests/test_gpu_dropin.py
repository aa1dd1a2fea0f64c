"""The drop-in module as the reference's own layer code drives it.

tests/golden/dropin_calls.json holds every call that the reference's
unmodified model/ConeBeamLayers/Standard/StandardGeometry.py made into its
projector extension (ForwardProjection, BackProjection, both autograd
backwards, StandardGeometry, StandardGeometryWithFBP) with options.yaml set
to the "s3" geometry of ref_projectors.npz: argument values and types exactly
as that module passes them (float64 angles, int64 sizes, int SID/SDD, the
device index). Here each call is replayed through this library's
JITStandardGeometry and compared with what the reference's own kernels
returned for the same inputs."""
import json
import os
import warnings

import numpy as np
import pytest
import torch

from helpers import rel_rmse

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _calls():
    with open(os.path.join(GOLDEN, "dropin_calls.json")) as f:
        return json.load(f)["calls"]


def _arg(desc, dev):
    if desc["tensor"]:
        return torch.tensor(desc["values"], dtype=getattr(torch, desc["dtype"])).to(dev)
    return desc["value"]


def _replay_args(call, dev):
    device = call["device"]["value"]
    return (_arg(call["angles"], dev), _arg(call["volumeSize"], dev),
            _arg(call["detectorSize"], dev), _arg(call["sid"], dev), _arg(call["sdd"], dev),
            0 if device is None else device)


@pytest.mark.parametrize("sampler", ["soft", "tex"])
def test_replayed_reference_calls_match_reference_kernels(cuda, sampler):
    import JITStandardGeometry as J
    z = np.load(os.path.join(GOLDEN, "ref_projectors.npz"))
    vol = torch.from_numpy(z["s3_vol"]).to(cuda)
    sino = torch.from_numpy(z["s3_sino_in"]).to(cuda)
    tol = {"tex": 5e-4, "soft": 5e-3}[sampler]
    calls = _calls()
    assert [c["fn"] for c in calls].count("forward") == 4
    old = J._SAMPLER
    J._SAMPLER, J._plans = sampler, {}
    try:
        for c in calls:
            args = _replay_args(c, cuda)  # fresh device copies each call, as the reference makes
            if c["fn"] == "forward":
                assert tuple(c["input_shape"]) == tuple(vol.shape)
                out = J.forward(vol, *args)
                assert rel_rmse(out.cpu().numpy(), z["s3_fp"]) < tol
            else:
                assert tuple(c["input_shape"]) == tuple(sino.shape)
                out = J.backward(sino, *args)
                assert rel_rmse(out.cpu().numpy(), z["s3_bp"]) < tol
        assert len(J._plans) == 1  # one geometry: one plan for all eight calls
    finally:
        J._SAMPLER, J._plans = old, {}


def test_host_syncs_per_call(cuda):
    """After the first call, a call with the same geometry tensors synchronises
    nothing; fresh device copies cost one small read-back for all three."""
    import JITStandardGeometry as J
    call = _calls()[0]
    vol = torch.rand((1, 1, 32, 64, 64), device=cuda)
    args = _replay_args(call, cuda)
    J.forward(vol, *args)
    torch.cuda.synchronize()
    torch.cuda.set_sync_debug_mode("error")
    try:
        for _ in range(3):
            J.forward(vol, *args)
            J.backward(torch.rand((1, 1, 30, 48, 96), device=cuda), *args)
    finally:
        torch.cuda.set_sync_debug_mode("default")
    fresh = _replay_args(call, cuda)
    torch.cuda.synchronize()
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        torch.cuda.set_sync_debug_mode("warn")
        try:
            J.forward(vol, *fresh)
        finally:
            torch.cuda.set_sync_debug_mode("default")
    syncs = [x for x in w if "synchroniz" in str(x.message).lower()]
    assert len(syncs) == 1, [str(x.message) for x in syncs]
    torch.cuda.synchronize()
