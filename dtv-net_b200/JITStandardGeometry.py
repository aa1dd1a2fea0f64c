"""Drop-in replacement of the reference's pybind module ``JITStandardGeometry``
(model/ConeBeamLayers/Standard/plug/jit.cpp:5-8, include/forward.h:3,
include/backward.h:3) on the B200 kernels.

With this directory on sys.path ahead of the reference's build, the reference's
own model/ConeBeamLayers/Standard/StandardGeometry.py imports this module
unchanged. Same names, arguments, output shapes and errors:

  forward(volume, angles, volumeSize, detectorSize, sid, sdd, device) -> sino
  backward(sino, angles, volumeSize, detectorSize, sid, sdd, device) -> volume

volume [B,1,Z,Y,X] f32, sino [B,1,N,H,W] f32, angles [N] degrees, volumeSize
(X,Y,Z), detectorSize (W,H). Inputs must be contiguous CUDA tensors
(RuntimeError otherwise, as CHECK_INPUT raised). Plans are cached per
geometry and device, so repeated calls upload nothing.
"""
import os as _os
import sys as _sys

_sys.path.insert(0, _os.path.dirname(_os.path.abspath(__file__)))

import torch as _torch  # noqa: E402

from dtvb200 import geometry as _geo  # noqa: E402

_SAMPLER = _os.environ.get("DTVB200_SAMPLER", "soft")
_plans = {}


def _host_list(t, n, name):
    if not isinstance(t, _torch.Tensor):
        raise RuntimeError(f"{name} must be a tensor")
    if t.is_cuda and not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")
    if t.numel() != n:
        raise RuntimeError(f"{name}'s length must be {n}")
    return [int(v) for v in t.detach().cpu().tolist()]


def _plan(angles, volumeSize, detectorSize, sid, sdd, device, batch):
    if not isinstance(angles, _torch.Tensor):
        raise RuntimeError("angles must be a tensor")
    a = angles.detach().to("cpu", _torch.float32).contiguous()
    vs = _host_list(volumeSize, 3, "volume size")
    ds = _host_list(detectorSize, 2, "detector size")
    key = (a.numpy().tobytes(), tuple(vs), tuple(ds), float(sid), float(sdd), int(device))
    p = _plans.get(key)
    if p is None or p.max_batch < batch:
        g = _geo.standard(a.numpy(), vs, ds, sid, sdd)
        p = _geo.Plan(g, max_batch=max(batch, 1), sampler=_SAMPLER,
                      device=_torch.device("cuda", int(device)))
        _plans[key] = p
    return p


def forward(volume, angles, volumeSize, detectorSize, sid, sdd, device):
    _geo.check_input(volume, "volume")
    p = _plan(angles, volumeSize, detectorSize, sid, sdd, device, volume.shape[0])
    with _torch.cuda.device(p.device):
        return p.forward(volume)


def backward(sino, angles, volumeSize, detectorSize, sid, sdd, device):
    _geo.check_input(sino, "sino")
    p = _plan(angles, volumeSize, detectorSize, sid, sdd, device, sino.shape[0])
    with _torch.cuda.device(p.device):
        return p.backward(sino)
