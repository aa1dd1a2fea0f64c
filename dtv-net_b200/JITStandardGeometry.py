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

The geometry arguments pick the plan, so their values are needed on the host.
Tensors this module has already read (the same tensor objects, unmodified)
are not read again; host tensors need no transfer; device tensors are read
back in one small copy for all three (the reference's own callers pass
`angles.to(device)` copies of host tensors, which synchronise the stream
before this module runs).
"""
import os as _os
import sys as _sys
import weakref as _weakref

_sys.path.insert(0, _os.path.dirname(_os.path.abspath(__file__)))

import torch as _torch  # noqa: E402

from dtvb200 import geometry as _geo  # noqa: E402

_SAMPLER = _os.environ.get("DTVB200_SAMPLER", "soft")
_plans = {}


_seen = {}  # id(tensor) -> (weakref, _version, host values)


def _check_len(t, n, name):
    if not isinstance(t, _torch.Tensor):
        raise RuntimeError(f"{name} must be a tensor")
    if t.is_cuda and not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")
    if n is not None and t.numel() != n:
        raise RuntimeError(f"{name}'s length must be {n}")


def _version(t):
    try:
        return t._version
    except RuntimeError:  # inference-mode tensors keep no version counter
        return None


def _host_values(tensors):
    """Host float64 copies of small geometry tensors: cached per tensor object
    and version, host tensors read directly, device tensors in one copy."""
    out = [None] * len(tensors)
    fetch = []
    for i, t in enumerate(tensors):
        hit = _seen.get(id(t))
        if hit is not None and hit[0]() is t and hit[1] is not None and hit[1] == _version(t):
            out[i] = hit[2]
        elif t.is_cuda:
            fetch.append(i)
        else:
            out[i] = t.detach().to(_torch.float64).reshape(-1).numpy().copy()
    if fetch:
        devs = {tensors[i].device for i in fetch}
        parts = [tensors[i].detach().reshape(-1).to(_torch.float64) for i in fetch]
        host = (_torch.cat(parts).cpu() if len(devs) == 1
                else _torch.cat([q.cpu() for q in parts])).numpy()
        o = 0
        for i in fetch:
            n = tensors[i].numel()
            out[i] = host[o:o + n].copy()
            o += n
            ver = _version(tensors[i])
            if ver is not None:
                k = id(tensors[i])
                _seen[k] = (_weakref.ref(tensors[i], lambda _r, k=k: _seen.pop(k, None)), ver,
                            out[i])
    return out


def _plan(angles, volumeSize, detectorSize, sid, sdd, device, batch):
    if not isinstance(angles, _torch.Tensor):
        raise RuntimeError("angles must be a tensor")
    _check_len(volumeSize, 3, "volume size")
    _check_len(detectorSize, 2, "detector size")
    ah, vh, dh = _host_values([angles, volumeSize, detectorSize])
    a = ah.astype("float32")
    vs = [int(v) for v in vh]
    ds = [int(v) for v in dh]
    key = (a.tobytes(), tuple(vs), tuple(ds), float(sid), float(sdd), int(device))
    p = _plans.get(key)
    if p is None or p.max_batch < batch:
        g = _geo.standard(a, vs, ds, sid, sdd)
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
