"""Geometry descriptions and projector plans (host side of the C ABI).

A :class:`Geometry` is the per-view vector form of a cone-beam scan
(source, detector centre and one-pixel steps U, V per view; FP64). The
builders reproduce the reference layers' conventions:

* :func:`standard` — model/ConeBeamLayers/Standard (circular orbit; voxel =
  sample step = sid/sdd, detector pitch 1; forwardKernel.cu:30-40,63,82;
  backwardKernel.cu:29-50).
* :func:`vector` — model/ConeBeamLayers/Beijing (per-view [N,12] projection
  vectors; Beijing/plug/kernel/forwardKernel.cu:24-35, backwardKernel.cu:21-43).
* :func:`circular` — a circular orbit with explicit voxel size and detector
  pitch (the general geometry the reference cannot express).

A :class:`Plan` uploads a geometry to one GPU once; its methods run the
projectors on torch CUDA tensors on the current stream, never synchronising.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import call

_DT = {torch.float32: _lib.DTV_F32, torch.float16: _lib.DTV_F16, torch.bfloat16: _lib.DTV_BF16}


@dataclass
class Geometry:
    """FP64 per-view geometry plus the scalar conventions of a layer."""

    struct: _lib.dtv_geometry
    views: np.ndarray  # [n_views, 12] float64, kept alive for struct.views

    @property
    def volume_size(self):
        return (self.struct.nx, self.struct.ny, self.struct.nz)

    @property
    def detector_size(self):
        return (self.struct.nu, self.struct.nv)

    @property
    def n_views(self) -> int:
        return self.struct.n_views

    def vol_shape(self, batch: int = 1):
        s = self.struct
        return (batch, 1, s.nz, s.ny, s.nx)

    def sino_shape(self, batch: int = 1):
        s = self.struct
        return (batch, 1, s.n_views, s.nv, s.nu)

    def key(self):
        s = self.struct
        scal = (s.nx, s.ny, s.nz, s.nu, s.nv, s.n_views, tuple(s.voxel), tuple(s.vol_offset),
                tuple(s.det_offset), s.fp_step, s.fp_scale, s.fp_phase, s.bp_weight_power,
                s.bp_scale, s.bp_extent_check)
        return scal + (self.views.tobytes(),)


def _finish(g: _lib.dtv_geometry, views: np.ndarray) -> Geometry:
    g.views = views.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return Geometry(g, views)


def standard(angles_deg, volume_size, detector_size, sid: float, sdd: float) -> Geometry:
    """The Standard layer's circular geometry (JITStandardGeometry conventions)."""
    a = np.ascontiguousarray(np.asarray(angles_deg, dtype=np.float32).ravel())
    views = np.zeros((a.size, 12), dtype=np.float64)
    g = _lib.dtv_geometry()
    call("dtv_geometry_standard", ctypes.byref(g),
         views.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
         a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), a.size,
         _lib.ivec(volume_size), _lib.ivec(detector_size), float(sid), float(sdd))
    geo = _finish(g, views)
    geo._angles = a
    return geo


def vector(project_vector, volume_size, detector_size) -> Geometry:
    """The Beijing layer's per-view vector geometry (JITBeijingGeometry conventions)."""
    pv = np.ascontiguousarray(np.asarray(project_vector, dtype=np.float32).reshape(-1, 12))
    views = np.zeros((pv.shape[0], 12), dtype=np.float64)
    g = _lib.dtv_geometry()
    call("dtv_geometry_vector", ctypes.byref(g),
         views.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
         pv.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), pv.shape[0],
         _lib.ivec(volume_size), _lib.ivec(detector_size))
    return _finish(g, views)


def circular(angles_deg, volume_size, voxel, detector_size, pitch, sod: float,
             sdd: float) -> Geometry:
    """Circular orbit with explicit voxel size and detector pitch (centred grids,
    exact-chord sampling at step = smallest voxel edge)."""
    a = np.ascontiguousarray(np.asarray(angles_deg, dtype=np.float64).ravel())
    views = np.zeros((a.size, 12), dtype=np.float64)
    g = _lib.dtv_geometry()
    call("dtv_geometry_circular", ctypes.byref(g),
         views.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
         a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size,
         _lib.ivec(volume_size), _lib.dvec(voxel), _lib.ivec(detector_size), _lib.dvec(pitch),
         float(sod), float(sdd))
    return _finish(g, views)


def _stream(device: torch.device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def check_input(t: torch.Tensor, name: str, shape=None, dtypes=(torch.float32,)):
    """The reference's CHECK_INPUT (forwardKernel.cu:15-17) plus shape/dtype."""
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")
    if t.dtype not in dtypes:
        raise RuntimeError(f"{name} must have dtype in {dtypes}, got {t.dtype}")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise RuntimeError(f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")


SAMPLERS = ("soft", "tex", "pairs", "tma", "exact")


class Plan:
    """A geometry uploaded to one GPU with sampler staging for ``max_batch``
    volumes. ``sampler``: "soft" (software trilinear, FP32 weights; required
    for the exact adjoint), "tex" (hardware trilinear texture filtering, like
    the reference) or "pairs" (FP16 z-plane pairs in a layered texture: one
    bilinear fetch per sample, z interpolated in FP32) or "tma" (the same
    z-pairs streamed by the Tensor Memory Accelerator into shared memory per
    ray tile and interpolated there with FP32 weights; a tunable share of the
    tiles still uses the texture unit) or "exact" (the same FP16 z-pairs in a
    zero-bordered linear copy read through L1, FP32 x/y/z weights, and the
    software FP32-weight backprojector: no 8-bit texture weights anywhere,
    whose error 100-iteration reconstructions amplify past 1e-3 of FP64).
    The backprojector samples the sinogram through a texture for "tex",
    "pairs" and "tma".
    ``stage_f16`` stages projected volumes as FP16 ("soft"/"tex").
    ``adjoint`` keeps a per-ray table (32 bytes per ray and view) and cell
    records (16 bytes per voxel) that speed up :meth:`adjoint`.

    A plan stages its input in buffers of its own, so its calls are ordered
    on the stream they are made on; calls of one plan from two streams at once
    race. Use one plan per concurrent stream."""

    def __init__(self, geometry: Geometry, max_batch: int = 1, sampler: str = "soft",
                 stage_f16: bool = False, device=None, adjoint: bool = False):
        if sampler not in SAMPLERS:
            raise ValueError(f"sampler must be one of {SAMPLERS}")
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else \
            torch.device(device)
        if dev.type != "cuda":
            raise RuntimeError("a Plan needs a CUDA device")
        self.device = torch.device("cuda", dev.index if dev.index is not None
                                   else torch.cuda.current_device())
        self.geometry = geometry
        self.max_batch = int(max_batch)
        self.sampler = sampler
        self.stage_f16 = bool(stage_f16)
        flags = {"soft": 0, "tex": _lib.DTV_PLAN_TEX, "pairs": _lib.DTV_PLAN_TEX_PAIRS,
                 "tma": _lib.DTV_PLAN_TEX_PAIRS | _lib.DTV_PLAN_TMA,
                 "exact": _lib.DTV_PLAN_PAIRS_EXACT}[sampler] | \
            (_lib.DTV_PLAN_STAGE_F16 if stage_f16 else 0) | (_lib.DTV_PLAN_ADJOINT if adjoint else 0)
        h = ctypes.c_void_p()
        call("dtv_plan_create", ctypes.byref(geometry.struct), self.max_batch, flags,
             self.device.index, ctypes.byref(h))
        self._h = h

    # ------------------------------------------------------------------ shapes
    def vol_shape(self, batch: int = 1):
        return self.geometry.vol_shape(batch)

    def sino_shape(self, batch: int = 1):
        return self.geometry.sino_shape(batch)

    def set_tuning(self, key: int, value: int) -> None:
        """Set a launch parameter (DTV_TUNE_*); results do not depend on it.
        DTV_TUNE_FP_RAY_TILE (0..7): the forward projector's block and warp
        ray tile, which decides how compact each warp's texture footprint is
        ("soft", "tex", "pairs"). DTV_TUNE_FP_TEX_SHARE (0..8, "tma" plans):
        eighths of the ray tiles sampled through the texture unit."""
        call("dtv_plan_set_tuning", self._h, int(key), int(value))

    def get_tuning(self, key: int) -> int:
        out = ctypes.c_int32()
        call("dtv_plan_get_tuning", self._h, int(key), ctypes.byref(out))
        return out.value

    def device_status(self, reset: bool = True) -> int:
        """Device-side error bits of this plan's kernels (0: none); synchronises."""
        out = ctypes.c_int32()
        call("dtv_plan_device_status", self._h, ctypes.byref(out), int(bool(reset)))
        return out.value

    def fp_samples(self) -> float:
        """Forward-projector samples per volume (exact chords / step)."""
        out = ctypes.c_double()
        call("dtv_plan_fp_samples", self._h, ctypes.byref(out))
        return out.value

    def _batch_of(self, t: torch.Tensor, per_item: int) -> int:
        b = t.numel() // per_item
        if b * per_item != t.numel() or b < 1:
            raise RuntimeError(f"tensor of {t.numel()} elements is not a whole batch")
        if b > self.max_batch:
            raise RuntimeError(f"batch {b} exceeds the plan's max_batch {self.max_batch}")
        return b

    # ------------------------------------------------------------------ ops
    def forward(self, vol: torch.Tensor, out: torch.Tensor = None, epilogue: int = 0,
                g: torch.Tensor = None, sigma: float = 0.0,
                abs_sum: torch.Tensor = None) -> torch.Tensor:
        """Forward projection of [B,1,Z,Y,X] (f32/f16/bf16) -> [B,1,N,H,W] f32.
        epilogue: DTV_EPI_STORE / DTV_EPI_RESIDUAL (out = FP - g) / DTV_EPI_PDHG
        (out = (out + sigma*(FP - g))/(1+sigma)). abs_sum (float64, 1 element)
        accumulates sum|FP - g| (or sum|FP| for STORE)."""
        check_input(vol, "volume", dtypes=tuple(_DT))
        per = int(np.prod(self.vol_shape(1)))
        b = self._batch_of(vol, per)
        shape = self.sino_shape(b)
        if out is None:
            out = torch.empty(shape, device=vol.device, dtype=torch.float32)
        check_input(out, "out", shape)
        if g is not None:
            check_input(g, "g", shape)
        if abs_sum is not None:
            check_input(abs_sum, "abs_sum", dtypes=(torch.float64,))
        call("dtv_forward", self._h, _ptr(vol), _DT[vol.dtype], b, _ptr(out), int(epilogue),
             _ptr(g), float(sigma), _ptr(abs_sum), _stream(vol.device))
        return out

    def backward(self, sino: torch.Tensor, out: torch.Tensor = None,
                 accumulate: bool = False, base: torch.Tensor = None) -> torch.Tensor:
        """FDK-weighted voxel-driven backprojection [B,1,N,H,W] -> [B,1,Z,Y,X].
        ``accumulate`` adds it to out; ``base`` (volume shaped, may be out)
        gives out = base + BP(sino)."""
        check_input(sino, "sino")
        b = self._batch_of(sino, int(np.prod(self.sino_shape(1))))
        shape = self.vol_shape(b)
        if out is None:
            out = torch.empty(shape, device=sino.device, dtype=torch.float32)
            accumulate = False
        check_input(out, "out", shape)
        if base is not None:
            check_input(base, "base", shape)
            call("dtv_backward_onto", self._h, _ptr(sino), b, _ptr(base), _ptr(out),
                 _stream(sino.device))
            return out
        call("dtv_backward", self._h, _ptr(sino), b, _ptr(out), int(bool(accumulate)),
             _stream(sino.device))
        return out

    def adjoint(self, sino: torch.Tensor, out: torch.Tensor = None) -> torch.Tensor:
        """Exact transpose of forward (STORE): A^T sino."""
        check_input(sino, "sino")
        b = self._batch_of(sino, int(np.prod(self.sino_shape(1))))
        shape = self.vol_shape(b)
        if out is None:
            out = torch.empty(shape, device=sino.device, dtype=torch.float32)
        check_input(out, "out", shape)
        call("dtv_backward_adjoint", self._h, _ptr(sino), b, _ptr(out), _stream(sino.device))
        return out

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h is not None and h.value:
            _lib.load().dtv_plan_destroy(h)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr_array(ts):
    return (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


def forward_refresh(fast: Plan, exact: Plan, vol: torch.Tensor, g: torch.Tensor,
                    w: torch.Tensor, g_eff: torch.Tensor, sigma: float,
                    abs_sum: torch.Tensor = None):
    """The correction pass of a texture-filtered z-pair plan ``fast``
    (sampler "pairs") against the exact-weight plan ``exact`` (sampler
    "exact") of the same geometry, in one launch: with e and a the exact and
    fast projections of vol, g_eff = g + (a - e) and
    w = (w + sigma (e - g)) / (1 + sigma); abs_sum += sum|e - g|."""
    check_input(vol, "volume", dtypes=tuple(_DT))
    b = fast._batch_of(vol, int(np.prod(fast.vol_shape(1))))
    shape = fast.sino_shape(b)
    for t, n in ((g, "g"), (w, "w"), (g_eff, "g_eff")):
        check_input(t, n, shape)
    if abs_sum is not None:
        check_input(abs_sum, "abs_sum", dtypes=(torch.float64,))
    call("dtv_pdhg_forward_refresh", fast._h, exact._h, _ptr(vol), _DT[vol.dtype], b, _ptr(g),
         float(sigma), _ptr(w), _ptr(g_eff), _ptr(abs_sum), _stream(vol.device))


def backward_refresh(fast: Plan, exact: Plan, sino: torch.Tensor, out: torch.Tensor,
                     e_b: torch.Tensor):
    """out = exact.backward(sino), e_b = out - fast.backward(sino), in one
    launch (the plans as for forward_refresh)."""
    check_input(sino, "sino")
    b = fast._batch_of(sino, int(np.prod(fast.sino_shape(1))))
    shape = fast.vol_shape(b)
    check_input(out, "out", shape)
    check_input(e_b, "e_b", shape)
    call("dtv_backward_refresh", fast._h, exact._h, _ptr(sino), b, _ptr(out), _ptr(e_b),
         _stream(sino.device))


def forward_many(plans, vols, outs=None, epilogue: int = 0, gs=None, sigma: float = 0.0):
    """Forward projections of several volumes, each with its own plan (any
    sizes and view counts, "pairs" or "tma" plans on one device), in one
    kernel launch (dtv_forward_many). Returns the list of sinograms."""
    if not (len(plans) == len(vols) >= 1):
        raise ValueError("need one volume per plan")
    dt = vols[0].dtype
    for p, v in zip(plans, vols):
        check_input(v, "volume", p.vol_shape(1), dtypes=(dt,))
    if outs is None:
        outs = [torch.empty(p.sino_shape(1), device=v.device) for p, v in zip(plans, vols)]
    for p, o in zip(plans, outs):
        check_input(o, "out", p.sino_shape(1))
    if gs is not None:
        for p, g in zip(plans, gs):
            check_input(g, "g", p.sino_shape(1))
    call("dtv_forward_many", (ctypes.c_void_p * len(plans))(*[p._h.value for p in plans]),
         _ptr_array(vols), _DT[dt], _ptr_array(outs), len(plans), int(epilogue),
         _ptr_array(gs) if gs is not None else None, float(sigma), _stream(vols[0].device))
    return outs


def backward_many(plans, sinos, outs=None, accumulate: bool = False):
    """FDK backprojections of several sinograms, each with its own plan
    (texture-sampled plans on one device), in one kernel launch
    (dtv_backward_many). Returns the list of volumes."""
    if not (len(plans) == len(sinos) >= 1):
        raise ValueError("need one sinogram per plan")
    for p, s in zip(plans, sinos):
        check_input(s, "sino", p.sino_shape(1))
    if outs is None:
        outs = [torch.empty(p.vol_shape(1), device=s.device) for p, s in zip(plans, sinos)]
        accumulate = False
    for p, o in zip(plans, outs):
        check_input(o, "out", p.vol_shape(1))
    call("dtv_backward_many", (ctypes.c_void_p * len(plans))(*[p._h.value for p in plans]),
         _ptr_array(sinos), _ptr_array(outs), len(plans), int(bool(accumulate)),
         _stream(sinos[0].device))
    return outs

