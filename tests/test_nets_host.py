"""Host-side checks of the unrolled-network mirrors: built under the seeds the
reference networks were built with (tests/golden/make_ref_layers.py), DTVNet,
FistaNet and LEARN have exactly the reference's parameters, names and values.
(The cascades themselves run on the GPU: tests/test_gpu_nets.py.)"""
import os

import numpy as np
import pytest
import torch

import dtvb200
import make_ref_layers as ML
from dtvb200.nets import LEARN, DTVNet, FistaNet

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_layers.npz")


def _build(tag, gold):
    torch.manual_seed(ML.SEEDS[tag])
    c = ML.CASCADES[tag]
    X, Y, Z = ML.BJ["beijingVolumeSize"]
    if tag in ("dtvnet", "fistanet"):
        geo = dtvb200.vector(gold["bj_pv"], (X, Y, Z), tuple(ML.BJ["beijingSubDetectorSize"]))
        layer = dtvb200.BeijingGeometry(dtvb200.Projector(geo), planes=ML.BJ["beijingPlanes"],
                                        sample_interval=ML.BJ["sampleInterval"])
        return (DTVNet if tag == "dtvnet" else FistaNet)(layer, c)
    S = ML.STD
    ang = np.linspace(0, 360, S["standardAngleNum"], endpoint=False).astype(np.float32)
    geo = dtvb200.standard(ang, S["standardVolumeSize"], S["standardDetectorSize"],
                           S["standardSID"], S["standardSDD"])
    return LEARN(dtvb200.Projector(geo), c)


@pytest.mark.parametrize("tag", ["dtvnet", "fistanet", "learn"])
def test_mirror_has_the_reference_parameters(tag):
    gold = np.load(GOLD)
    net = _build(tag, gold)
    keys = {k.split(f"{tag}_sd_", 1)[1].split("#")[0] for k in gold.files
            if k.startswith(f"{tag}_sd_")}
    sd = net.state_dict()
    assert set(sd) == keys
    for k, v in sd.items():
        v = v.double().numpy()
        if f"{tag}_sd_{k}" in gold.files:
            assert np.array_equal(v, gold[f"{tag}_sd_{k}"]), k
        else:
            assert np.array_equal(ML.summary(v), gold[f"{tag}_sd_{k}#sum"]), k
