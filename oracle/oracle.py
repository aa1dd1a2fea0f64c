"""FP64 oracle: ctypes front end of oracle.c plus numpy restatements of the
reference's finite differences, L1-ball projection and iteration loops.

TEST INFRASTRUCTURE ONLY. The product never imports this module; tests/,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline / reference arm
use it as the checker. Every function cites the reference file:line it
restates (paths relative to the reference project root).

Parity pin: the projector layer is checked against the reference CUDA kernels
(built unmodified, run on a GPU) through tests/golden/ref_projectors.npz, and
the difference / L1-ball layer against the reference Python modules through
tests/golden/ref_utils.npz.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

# The reference's value of pi (Standard/plug/kernel/forwardKernel.cu:14).
REF_PI = 3.14159265359

PHASE_STANDARD, PHASE_VECTOR, PHASE_BOX = 0, 1, 2


class OGeom(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("nu", ctypes.c_int32), ("nv", ctypes.c_int32), ("n_views", ctypes.c_int32),
        ("phase", ctypes.c_int32), ("bp_pow", ctypes.c_int32),
        ("bp_extent", ctypes.c_int32), ("pad", ctypes.c_int32),
        ("voxel", ctypes.c_double * 3), ("vol_off", ctypes.c_double * 3),
        ("det_off", ctypes.c_double * 2),
        ("step", ctypes.c_double), ("scale", ctypes.c_double), ("bp_scale", ctypes.c_double),
    ]


_lib = None


def build() -> str:
    """Compile liboracle.so from oracle.c (make)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or (
                os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "oracle.c"))):
            build()
        L = ctypes.CDLL(LIB_PATH)
        D = ctypes.POINTER(ctypes.c_double)
        i = ctypes.c_int
        d = ctypes.c_double
        G = ctypes.POINTER(OGeom)
        L.oracle_forward_standard_literal.argtypes = [D, i, D, i, i, i, i, i, i, d, d, i, D]
        L.oracle_backward_standard_literal.argtypes = [D, i, D, i, i, i, i, i, i, d, d, i, D]
        L.oracle_forward_vector_literal.argtypes = [D, i, D, i, i, i, i, i, i, i, D]
        L.oracle_backward_vector_literal.argtypes = [D, i, D, i, i, i, i, i, i, i, D]
        L.oracle_standard_views.argtypes = [D, i, d, d, D]
        L.oracle_circular_views.argtypes = [D, i, d, d, d, d, D]
        L.oracle_forward.argtypes = [G, D, D, i, i, D]
        L.oracle_backward.argtypes = [G, D, D, i, i, D]
        L.oracle_adjoint.argtypes = [G, D, D, i, D]
        L.oracle_fp_samples.argtypes = [G, D]
        L.oracle_fp_samples.restype = d
        L.oracle_num_threads.restype = i
        L.oracle_set_threads.argtypes = [i]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def num_threads() -> int:
    return lib().oracle_num_threads()


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


# --------------------------------------------------------------------------
# geometry (per-view vector description)
# --------------------------------------------------------------------------
class Geometry:
    """Oracle-side geometry: an OGeom plus its [n_views, 12] world vectors."""

    def __init__(self, og: OGeom, views: np.ndarray):
        self.og = og
        self.views = _c64(views).reshape(-1, 12)

    @property
    def vol_shape(self):
        return (self.og.nz, self.og.ny, self.og.nx)

    @property
    def sino_shape(self):
        return (self.og.n_views, self.og.nv, self.og.nu)


def standard_geometry(angles_deg, volume_size, detector_size, sid, sdd) -> Geometry:
    """The Standard layer's conventions (forwardKernel.cu:30-40,63,82,111-113;
    backwardKernel.cu:29-44,50): voxel = step = scale = sid/sdd, pitch 1,
    uncentred voxels and pixels, weight (sdd/L)^2 * pi/N."""
    a = _c64(angles_deg)
    n = a.size
    views = np.zeros((n, 12))
    lib().oracle_standard_views(_p(a), n, float(sid), float(sdd), _p(views))
    s = float(sid) / float(sdd)
    X, Y, Z = (int(v) for v in volume_size)
    W, H = (int(v) for v in detector_size)
    og = OGeom(nx=X, ny=Y, nz=Z, nu=W, nv=H, n_views=n, phase=PHASE_STANDARD, bp_pow=2,
               bp_extent=0)
    og.voxel[:] = (s, s, s)
    og.vol_off[:] = (0.0, 0.0, 0.0)
    og.det_off[:] = (0.0, 0.0)
    og.step, og.scale, og.bp_scale = s, s, REF_PI / n
    return Geometry(og, views)


def vector_geometry(project_vector, volume_size, detector_size) -> Geometry:
    """The Beijing layer's conventions (Beijing/plug/kernel/forwardKernel.cu:
    24-35,63-73; backwardKernel.cu:29-43): world = voxel units, step 1,
    scale 1, pixel centres at +1/2, weight SDD/L * 2*pi/(N//21)."""
    pv = _c64(project_vector).reshape(-1, 12)
    n = pv.shape[0]
    views = np.empty((n, 12))
    views[:, 0:3] = pv[:, 0:3] * [1, 1, -1]
    views[:, 3:6] = pv[:, 3:6] * [1, 1, -1]
    views[:, 6:9] = pv[:, 9:12]   # U = u
    views[:, 9:12] = pv[:, 6:9]   # V = v
    X, Y, Z = (int(v) for v in volume_size)
    W, H = (int(v) for v in detector_size)
    og = OGeom(nx=X, ny=Y, nz=Z, nu=W, nv=H, n_views=n, phase=PHASE_VECTOR, bp_pow=1,
               bp_extent=1)
    og.voxel[:] = (1.0, 1.0, 1.0)
    og.vol_off[:] = (0.0, 0.0, 0.0)
    og.det_off[:] = (0.5, 0.5)
    og.step, og.scale, og.bp_scale = 1.0, 1.0, 2 * REF_PI / (n // 21) if n >= 21 else 0.0
    return Geometry(og, views)


def circular_geometry(angles_deg, volume_size, voxel, detector_size, pitch, sod, sdd) -> Geometry:
    """General circular orbit: explicit voxel size and pitch, centred voxels and
    pixels, exact-chord sampling at step = min(voxel), weight (sdd/L)^2*pi/N."""
    a = _c64(angles_deg)
    n = a.size
    views = np.zeros((n, 12))
    lib().oracle_circular_views(_p(a), n, float(sod), float(sdd), float(pitch[0]),
                                float(pitch[1]), _p(views))
    X, Y, Z = (int(v) for v in volume_size)
    W, H = (int(v) for v in detector_size)
    og = OGeom(nx=X, ny=Y, nz=Z, nu=W, nv=H, n_views=n, phase=PHASE_BOX, bp_pow=2, bp_extent=0)
    og.voxel[:] = tuple(float(v) for v in voxel)
    og.vol_off[:] = (0.5, 0.5, 0.5)
    og.det_off[:] = (0.5, 0.5)
    step = float(min(voxel))
    og.step, og.scale, og.bp_scale = step, step, np.pi / n
    return Geometry(og, views)


def _as_batch(x: np.ndarray, shape3):
    x = _c64(x)
    b = x.size // int(np.prod(shape3))
    return x.reshape((b,) + tuple(shape3)), b


def forward(geo: Geometry, vol, q: int = 0) -> np.ndarray:
    """q: 0 exact weights, 1 all weights at 1/256 (3-D texture filtering),
    2 x/y weights at 1/256 and exact z (z-pair layered texture)."""
    v, b = _as_batch(vol, geo.vol_shape)
    out = np.empty((b,) + geo.sino_shape)
    lib().oracle_forward(ctypes.byref(geo.og), _p(geo.views), _p(v), b, int(q), _p(out))
    return out


def backward(geo: Geometry, sino, q: bool = False) -> np.ndarray:
    s, b = _as_batch(sino, geo.sino_shape)
    out = np.empty((b,) + geo.vol_shape)
    lib().oracle_backward(ctypes.byref(geo.og), _p(geo.views), _p(s), b, int(q), _p(out))
    return out


def adjoint(geo: Geometry, sino) -> np.ndarray:
    s, b = _as_batch(sino, geo.sino_shape)
    out = np.empty((b,) + geo.vol_shape)
    lib().oracle_adjoint(ctypes.byref(geo.og), _p(geo.views), _p(s), b, _p(out))
    return out


def fp_samples(geo: Geometry) -> float:
    return float(lib().oracle_fp_samples(ctypes.byref(geo.og), _p(geo.views)))


# literal restatements --------------------------------------------------------
def forward_standard_literal(vol, angles_deg, volume_size, detector_size, sid, sdd, q=False):
    X, Y, Z = (int(v) for v in volume_size)
    W, H = (int(v) for v in detector_size)
    a = _c64(angles_deg)
    v, b = _as_batch(vol, (Z, Y, X))
    out = np.empty((b, a.size, H, W))
    lib().oracle_forward_standard_literal(_p(v), b, _p(a), a.size, X, Y, Z, W, H, float(sid),
                                          float(sdd), int(q), _p(out))
    return out


def backward_standard_literal(sino, angles_deg, volume_size, detector_size, sid, sdd, q=False):
    X, Y, Z = (int(v) for v in volume_size)
    W, H = (int(v) for v in detector_size)
    a = _c64(angles_deg)
    s, b = _as_batch(sino, (a.size, H, W))
    out = np.empty((b, Z, Y, X))
    lib().oracle_backward_standard_literal(_p(s), b, _p(a), a.size, X, Y, Z, W, H, float(sid),
                                           float(sdd), int(q), _p(out))
    return out


def forward_vector_literal(vol, project_vector, volume_size, detector_size, q=False):
    X, Y, Z = (int(v) for v in volume_size)
    W, H = (int(v) for v in detector_size)
    pv = _c64(project_vector).reshape(-1, 12)
    v, b = _as_batch(vol, (Z, Y, X))
    out = np.empty((b, pv.shape[0], H, W))
    lib().oracle_forward_vector_literal(_p(v), b, _p(pv), pv.shape[0], X, Y, Z, W, H, int(q),
                                        _p(out))
    return out


def backward_vector_literal(sino, project_vector, volume_size, detector_size, q=False):
    X, Y, Z = (int(v) for v in volume_size)
    W, H = (int(v) for v in detector_size)
    pv = _c64(project_vector).reshape(-1, 12)
    s, b = _as_batch(sino, (pv.shape[0], H, W))
    out = np.empty((b, Z, Y, X))
    lib().oracle_backward_vector_literal(_p(s), b, _p(pv), pv.shape[0], X, Y, Z, W, H, int(q),
                                         _p(out))
    return out


# --------------------------------------------------------------------------
# finite differences: model/PDHG/Utils/Gradients.py:8-34 (D = shift - I)
# --------------------------------------------------------------------------
def _shift_spec(size, axis, quirk):
    """(offset, valid-row mask over the flat index) of the +1 entries."""
    X, Y, Z = size
    N = X * Y * Z
    i = np.arange(N)
    if axis == 0:                       # Gradients.py:8-16
        return 1, (i + 1) % X != 0
    if axis == 1:
        if quirk:                       # Gradients.py:18-25: offset volumeSize[1], i < N - Y
            return Y, i < N - Y
        return X, (i // X) % Y != Y - 1
    return X * Y, i < N - X * Y         # Gradients.py:27-34


def diff(f, size, axis, quirk=True, transpose=False) -> np.ndarray:
    """D_axis f or D_axis^T f for each batch item; f is [..., Z, Y, X]."""
    X, Y, Z = size
    N = X * Y * Z
    g = _c64(f)
    shp = g.shape
    g = g.reshape(-1, N)
    off, valid = _shift_spec(size, axis, quirk)
    out = -g.copy()
    if not transpose:
        idx = np.nonzero(valid)[0]
        out[:, idx] += g[:, idx + off]
    else:
        idx = np.nonzero(valid)[0]          # rows i with an entry at column i+off
        out[:, idx + off] += g[:, idx]
    return out.reshape(shp)


# --------------------------------------------------------------------------
# L1-ball projection: model/PDHG/Utils/L1ball.py:4-17
# --------------------------------------------------------------------------
def l1ball_newton(v, b):
    """The reference's Newton iteration, in FP64 (L1ball.py:4-17)."""
    v = _c64(v)
    if np.sum(np.abs(v)) < b:                                   # :5-6
        return v.copy(), 0.0
    lam = 0.0                                                   # :7
    obj = np.sum(np.maximum(np.abs(v) - lam, 0)) - b            # :8
    it = 0
    while abs(obj) > 1e-4 and it < 100:                         # :10
        obj = np.sum(np.maximum(np.abs(v) - lam, 0)) - b        # :11
        dif = -np.count_nonzero(np.abs(v) - lam > 0) + 0.001    # :12
        lam -= obj / dif                                        # :13
        it += 1
    # np.max(lam, 0) returns lam unchanged for a scalar (:15)
    return np.sign(v) * np.maximum(np.abs(v) - lam, 0), lam    # :16


def l1ball_lambda_exact(a, b) -> float:
    """Exact threshold lambda >= 0 with sum max(|a|-lambda,0) = b (sorting)."""
    u = np.sort(np.abs(_c64(a)).ravel())[::-1]
    if u.sum() < b:
        return 0.0
    if b <= 0:  # every lambda >= max|a| solves it; the smallest is max|a|
        return float(u[0]) if u.size else 0.0
    c = np.cumsum(u)
    j = np.arange(1, u.size + 1)
    rho = np.nonzero(u - (c - b) / j > 0)[0][-1]
    return float((c[rho] - b) / (rho + 1))


# --------------------------------------------------------------------------
# iteration loops (FP/BP passed in as callables on [B,Z,Y,X] / [B,N,H,W])
# --------------------------------------------------------------------------
def dtvcp_run(fp, bp, image, sino, size, cascades, sigma, tau, mu, v, quirk=True,
              callback=None):
    """DTV by Chambolle-Pock, model/PDHG/DTVCP.py:29-60, in FP64."""
    f = _c64(image).copy()
    fbar = f.copy()                                              # :32
    w = np.zeros_like(_c64(sino))                                # :30
    p = np.zeros_like(f); q = np.zeros_like(f); s = np.zeros_like(f); c = np.zeros_like(f)
    t = [0.0, 0.0, 0.0]
    for it in range(cascades):                                   # :33
        if it % 10 == 0:                                         # :34-37
            t = [np.abs(diff(f, size, a, quirk)).sum() for a in range(3)]
        res = fp(fbar) - sino                                    # :38
        w = (w + sigma * res) / (1 + sigma)                      # :39
        recon = bp(w)                                            # :40
        duals = []
        for a, d in enumerate((p, q, s)):                        # :41-46
            d_ = d + v[a] * sigma * diff(fbar, size, a, quirk)
            proj, _ = l1ball_newton(np.abs(d_) / sigma, v[a] * t[a])
            duals.append(d_ - sigma * np.sign(d_) * proj)
        p, q, s = duals
        c = -np.maximum(-c - sigma * mu * fbar, 0)               # :47
        reg = (v[0] * diff(p, size, 0, quirk, True) + v[1] * diff(q, size, 1, quirk, True)
               + v[2] * diff(s, size, 2, quirk, True) + mu * c)  # :48-51
        fnew = f - recon - tau * reg                             # :52
        fbar = 2 * fnew - f                                      # :53
        f = fnew                                                 # :54
        if callback is not None:
            callback(it, f, np.abs(res).sum())
    return f


def fista_run(fp, bp, image, sino, cascades, L, lamb):
    """FISTA with soft-thresholding, model/FISTA/FISTA.py:16-27, in FP64."""
    t = 1.0
    I = Ip = _c64(image).copy()                                  # :17-18
    y = I
    for _ in range(cascades):
        d = y - L * bp(fp(y) - sino)                             # :21
        I = np.sign(d) * np.maximum(np.abs(d) - lamb * L, 0)     # :22
        tp = (1 + np.sqrt(1 + 4 * t ** 2)) / 2                   # :23
        y = I + (t - 1) / tp * (I - Ip)                          # :24
        Ip = I                                                   # :25
        t = tp                                                   # :26
    return I


def dtvfista_run(fp, bp, image, sino, size, cascades, sigma, v, tt, quirk=True):
    """FISTA-DTV, model/FISTA/DTVFISTA.py:23-43, in FP64. With quirk the
    thresholds use torch.max(tensor) (a global max, :34-36) and the momentum
    t is never advanced (t stays 1, :25-38)."""
    f = _c64(image).copy()
    t = 1.0
    for _ in range(cascades):
        tp = (1 + np.sqrt(1 + 4 * t ** 2)) / 2                   # :28
        z = np.maximum(f - sigma * bp(fp(f) - sino), 0)          # :29-30
        acc = z.copy()
        for a in range(3):
            g = diff(z, size, a, quirk)                          # :31-33
            if quirk:
                thr = np.sign(g) * np.max(np.abs(g) - v[a])      # :34-36
            else:
                thr = np.sign(g) * np.maximum(np.abs(g) - v[a], 0)
            acc += tt[a] * diff(thr, size, a, quirk, True)       # :37
        fnew = acc
        f = fnew + (t - 1) / tp * (fnew - f)                     # :38
        if not quirk:
            t = tp
    return f


def asdpocs_run(fp, bp, image, sino, size, cascades, beta=0.00005, beta_red=0.9999, ng=10,
                alpha=0.001, rmax=0.95, quirk=True):
    """ASD-POCS, model/PDHG/ASDPOCS.py:28-47, in FP64. With quirk, f0 aliases f
    during the TV steps (:36,43), so dg is 0 and davg never shrinks."""
    f = _c64(image).copy()
    f0 = f          # the iterate the next data step starts from (:30, :36)
    davg = 1.0
    for i in range(cascades):
        f = f0 - beta * bp(fp(f0) - sino)                        # :33
        dp = np.mean(np.abs(f0 - f))                             # :34
        if i == 0:
            davg = alpha * dp                                    # :35
        f_data = f.copy()                                        # :36 (f0 = f)
        for _ in range(ng):                                      # :37-43
            ds = [diff(f, size, a, quirk) for a in range(3)]
            g = np.sqrt(ds[0] ** 2 + ds[1] ** 2 + ds[2] ** 2) + 1
            grad = sum(diff(ds[a] / g, size, a, quirk, True) for a in range(3))
            f = f - davg * grad
        # :44 — in the reference f0 aliases f and `f -= ...` is in place, so
        # l1_loss(f, f0) is 0 and the test below never fires.
        dg = 0.0 if quirk else np.mean(np.abs(f - f_data))
        if dg > rmax * dp:                                       # :45
            davg *= alpha
        beta *= beta_red                                         # :46
        f0 = f
    return np.maximum(f, 0)                                      # :47


# ----------------------------------------------------------------- FBP filter
def ramp_taps(width: int) -> np.ndarray:
    """The W+1-tap spatial Ram-Lak kernel, float32 as the reference stores it
    (Standard/StandardGeometry.py:83-93, Beijing/BeijingGeometry.py:74-84)."""
    f = np.ones(width + 1, dtype=np.float32)
    mid = np.floor(width / 2)
    for i in range(width + 1):
        if (i - mid) % 2 == 0:
            f[i] = 0
        else:
            f[i] = -0.5 / (np.pi * np.pi * (i - mid) * (i - mid))
        if i == mid:
            f[i] = 1 / 8
    return f


def fbp_filter(rows, rows_per_view, sdd, mid_i, mid_j, adjoint=False) -> np.ndarray:
    """Cosine weight then ramp cross-correlation of each row (padding W/2 on
    both sides), in FP64 (StandardGeometry.py:51-65 and :68-74; the Beijing
    layer passes its own midpoints, BeijingGeometry.py:57-72). rows: [..., W];
    the cosine row index is (row number) mod rows_per_view. adjoint applies
    the transpose: ramp first, weight after."""
    x = np.asarray(rows, dtype=np.float64)
    W = x.shape[-1]
    x2 = x.reshape(-1, W)
    i = (np.arange(x2.shape[0]) % rows_per_view)[:, None] - mid_i
    j = np.arange(W)[None, :] - mid_j
    cw = sdd / np.sqrt(sdd ** 2 + i ** 2 + j ** 2)
    k = ramp_taps(W).astype(np.float64)
    half = W // 2
    src = x2 if adjoint else x2 * cw
    pad = np.zeros((x2.shape[0], W + 2 * half))
    pad[:, half:half + W] = src
    out = np.zeros_like(x2)
    for t in range(W + 1):
        out += k[t] * pad[:, t:t + W]
    if adjoint:
        out *= cw
    return out.reshape(x.shape)
