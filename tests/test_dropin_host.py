"""Host-side checks of the drop-in against the reference's own layer module
(run where the reference tree is present; the GPU replay of the recorded
calls is tests/test_gpu_dropin.py)."""
import json
import os

import pytest
import torch

import make_dropin_calls as M

REF = M.default_ref_root()
pytestmark = pytest.mark.skipif(
    not os.path.isfile(os.path.join(REF, "model", "ConeBeamLayers", "Standard",
                                    "StandardGeometry.py")),
    reason="reference tree absent (set DTV_REFERENCE_ROOT)")
GOLDEN = os.path.dirname(os.path.abspath(M.__file__))


def test_committed_calls_match_a_fresh_recording():
    with open(os.path.join(GOLDEN, "dropin_calls.json")) as f:
        committed = json.load(f)
    assert committed["geometry"] == M.S3
    assert M.record(REF) == committed["calls"]


def test_reference_layer_imports_this_module_unchanged():
    """The reference's StandardGeometry.py, imported with this library's
    JITStandardGeometry first on the path, binds to it and reaches its
    argument checks (a host tensor fails as the reference's CHECK_INPUT did)."""
    import JITStandardGeometry as J
    with M.reference_layer(REF, J) as sg:
        assert sg.projector is J
        with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
            sg.ForwardProjection.apply(torch.zeros((1, 1, 32, 64, 64)))
        with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
            sg.BackProjection.apply(torch.zeros((1, 1, 30, 48, 96)))
