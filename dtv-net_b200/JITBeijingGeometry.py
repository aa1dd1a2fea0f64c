"""Drop-in replacement of the reference's pybind module ``JITBeijingGeometry``
(model/ConeBeamLayers/Beijing/plug/jit.cpp:5-8, include/forward.h:3,
include/backward.h:3) on the B200 kernels:

  forward(volume, volumeSize, detectorSize, projectVector, device) -> sino
  backward(sino, volumeSize, detectorSize, projectVector, device) -> volume

projectVector [N,12] f32 per view: source(3), detector(3), v(3), u(3). The
backprojector accepts any view count (the reference needed a multiple of
1512, backwardKernel.cu:76-101) and keeps the 2*pi/(N//21) scale.
"""
import os as _os
import sys as _sys

_sys.path.insert(0, _os.path.dirname(_os.path.abspath(__file__)))

import torch as _torch  # noqa: E402

from dtvb200 import geometry as _geo  # noqa: E402
from JITStandardGeometry import _check_len, _host_values, _SAMPLER  # noqa: E402

_plans = {}


def _plan(volumeSize, detectorSize, projectVector, device, batch):
    if not isinstance(projectVector, _torch.Tensor) or projectVector.dim() != 2 or \
            projectVector.shape[1] != 12:
        raise RuntimeError("project vector's shape must be [angle's number, 12]")
    _check_len(volumeSize, 3, "volume size")
    _check_len(detectorSize, 2, "detector size")
    ph, vh, dh = _host_values([projectVector, volumeSize, detectorSize])
    pv = ph.astype("float32").reshape(-1, 12)
    vs = [int(v) for v in vh]
    ds = [int(v) for v in dh]
    key = (pv.tobytes(), tuple(vs), tuple(ds), int(device))
    p = _plans.get(key)
    if p is None or p.max_batch < batch:
        g = _geo.vector(pv, vs, ds)
        p = _geo.Plan(g, max_batch=max(batch, 1), sampler=_SAMPLER,
                      device=_torch.device("cuda", int(device)))
        _plans[key] = p
    return p


def forward(volume, volumeSize, detectorSize, projectVector, device):
    _geo.check_input(volume, "volume")
    p = _plan(volumeSize, detectorSize, projectVector, device, volume.shape[0])
    with _torch.cuda.device(p.device):
        return p.forward(volume)


def backward(sino, volumeSize, detectorSize, projectVector, device):
    _geo.check_input(sino, "sino")
    p = _plan(volumeSize, detectorSize, projectVector, device, sino.shape[0])
    with _torch.cuda.device(p.device):
        return p.backward(sino)
