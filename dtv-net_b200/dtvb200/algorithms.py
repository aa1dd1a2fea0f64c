"""Iterative reconstructions on the fused kernels.

Each class mirrors a reference algorithm (same update order, constants and
quirks) but runs every step as a stream-ordered kernel of the C ABI with no
host synchronisation, so a whole reconstruction can be captured once as a
CUDA graph and replayed:

* :class:`DTVCP`   — model/PDHG/DTVCP.py:7-66 (DTV by Chambolle-Pock)
* :class:`FISTA`   — model/FISTA/FISTA.py:9-27 (``DTVFista`` there)
* :class:`DTVFISTA` — model/FISTA/DTVFISTA.py:8-49
* :class:`ASDPOCS` — model/PDHG/ASDPOCS.py:8-53

``quirk=True`` reproduces the reference's behaviour where it differs from
the evident intent (the y-difference wrap, DTVFISTA's global-max threshold
and frozen momentum, ASDPOCS's aliased ``f0``).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._lib import call
from .geometry import (Plan, _ptr, _stream, backward_many, backward_refresh, check_input,
                       forward_many, forward_refresh)

_FDT = {torch.float32: _lib.DTV_F32, torch.float16: _lib.DTV_F16, torch.bfloat16: _lib.DTV_BF16}


def power_norm(size, axis: int, quirk: bool = True, iters: int = 10, seed: int = 0,
               device=None) -> float:
    """||D_axis||_2 by the power method of model/PDHG/Utils/HyperParams.py:6-13
    (10 iterations of x <- D^T D x / ||.||, then ||D x||), seeded instead of the
    reference's unseeded np.random.rand."""
    from .tv import diff
    X, Y, Z = size
    g = torch.Generator().manual_seed(seed)
    x = torch.rand((1, Z, Y, X), generator=g, dtype=torch.float32).to(device or "cuda")
    s = 0.0
    for _ in range(iters):
        x = diff(diff(x, axis, False, quirk), axis, True, quirk)
        x = x / torch.linalg.vector_norm(x.double()).float()
        s = float(torch.linalg.vector_norm(diff(x, axis, False, quirk).double()))
    return s


def _run_graph(owner, key, body):
    """Run `body` (which only enqueues work on the current stream) eagerly, or
    capture it once per `key` as a CUDA graph on `owner` and replay it. The
    number of this library's kernel launches per run is kept in
    owner.launches_per_run."""
    L = _lib.load()
    if not owner.use_graph:
        n0 = L.dtv_launch_count()
        body()
        owner.launches_per_run = L.dtv_launch_count() - n0
        return
    cache = owner.__dict__.setdefault("_graphs", {})
    g = cache.get(key)
    if g is None:
        body()  # warm-up run (sets kernel attributes, loads modules)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        n0 = L.dtv_launch_count()
        with torch.cuda.graph(g):
            body()
        owner.launches_per_run = L.dtv_launch_count() - n0
        cache[key] = g
    g.replay()


class _Graphable:
    """A reconstruction run as prepare (inputs into persistent buffers) ->
    enqueue (every iteration, stream-ordered, no host sync) -> result; the
    enqueue step runs eagerly or as one captured CUDA graph per input shape."""

    use_graph: bool = False
    launches_per_run: int = 0  # kernels of this library one run launches

    def _graph_run(self, key, body):
        _run_graph(self, key, body)

    def run(self, image: torch.Tensor, sino: torch.Tensor, out: torch.Tensor = None):
        """Reconstruct from `sino` (device or host tensor) starting at `image`.
        Returns the reconstruction as float32 (a copy in `out` if given)."""
        key, st = self._prepare(image, sino)
        self._graph_run(key, lambda: self._enqueue(st))
        return self._result(st, out)


class Batched:
    """Several reconstructions (each with its own plan, geometry and size) run
    as one unit: each one's iterations go on a stream of its own, so their
    kernels overlap on the GPU, and with ``use_graph`` the whole set is one
    captured CUDA graph (one launch per run)."""

    def __init__(self, algs, use_graph: bool = True):
        self.algs = list(algs)
        plans = [id(a.plan) for a in self.algs]
        if len(set(plans)) != len(plans):
            # a plan stages its input in buffers of its own; two streams using
            # one plan at once would overwrite each other's staging
            raise ValueError("each reconstruction of a Batched set needs a plan of its own")
        self.use_graph = use_graph
        self.launches_per_run = 0
        self._streams = None

    def run(self, images, sinos, outs=None):
        if self._streams is None:
            dev = images[0].device
            self._streams = [torch.cuda.Stream(device=dev) for _ in self.algs]
        prepared = [a._prepare(i, s) for a, i, s in zip(self.algs, images, sinos)]
        key = tuple(k for k, _ in prepared)

        def enqueue_all():
            main = torch.cuda.current_stream()
            for a, (_, st), sm in zip(self.algs, prepared, self._streams):
                sm.wait_stream(main)
                with torch.cuda.stream(sm):
                    a._enqueue(st)
            for sm in self._streams:
                main.wait_stream(sm)

        _run_graph(self, key, enqueue_all)
        outs = outs or [None] * len(self.algs)
        return [a._result(st, o) for a, (_, st), o in zip(self.algs, prepared, outs)]


class DTVCP(_Graphable):
    """DTV reconstruction by Chambolle-Pock PDHG (model/PDHG/DTVCP.py:29-60).

    Per iteration: t_a = sum|D_a f| every ``t_refresh`` iterations (:34-37);
    w <- (w + sigma (A fbar - g)) / (1 + sigma) fused into the projector (:38-39);
    recon = BP(w) (:40); dual ascent + L1-ball projections + non-negativity dual
    in one fused pass plus an exact device-side threshold search (:41-47);
    primal step and over-relaxation in one fused pass (:48-54).
    ``f_dtype`` torch.float16 / torch.bfloat16 stores fbar, the projector
    input, in 16 bits; the iterate f and all arithmetic stay FP32 (rounding f
    itself each iteration would drop updates below the 16-bit resolution).

    ``exact`` (a plan of the same geometry with sampler "exact") corrects the
    error of a texture-filtered ``plan`` ("pairs", "tex": 8-bit interpolation
    weights, which a 100-iteration reconstruction amplifies to several 1e-3
    of the FP64 result). Every ``correct_every`` iterations the exact plan
    projects and backprojects the current iterate, and the differences
    e_F = A_fast fbar - A_exact fbar and e_B = BP_exact w - BP_fast w are kept;
    the iterations in between use A_fast fbar - e_F (as data g + e_F) and
    BP_fast w + e_B. Their remaining error is the fast operators' error on
    what fbar and w moved since the last refresh. Refresh iterations use the
    exact operators themselves. ``correct_bp_every`` sets the backprojector's
    refresh interval apart (default: ``correct_every``); 1 backprojects with
    the exact plan in every iteration.

    The duals' clip to the L1-ball thresholds (:44-47) is deferred: each
    primal step but the last leaves p, q, s unclipped and keeps its three
    thresholds on the device, and the next dual step clips the duals as it
    loads them (dtv_pdhg_primal_defer / dtv_pdhg_dual_defer). Late in a
    reconstruction most duals are clipped, and this saves storing them; the
    result has the same bits. ``defer_clip = False`` runs the storing steps.
    """

    def __init__(self, plan: Plan, cascades: int = 30, sigma: float = 1e-7, tau: float = 1e-7,
                 mu: float = 1e5, v=(5e4, 5e4, 5e4), quirk: bool = True,
                 f_dtype=torch.float32, t_refresh: int = 10, use_graph: bool = False,
                 backprojector: str = "fdk", exact: Plan = None, correct_every: int = 8,
                 correct_bp_every: int = None):
        if f_dtype not in _FDT:
            raise ValueError("f_dtype must be torch.float32, torch.float16 or torch.bfloat16")
        if backprojector not in ("fdk", "adjoint"):
            raise ValueError("backprojector must be 'fdk' or 'adjoint'")
        if exact is not None:
            if (tuple(exact.vol_shape(1)) != tuple(plan.vol_shape(1))
                    or tuple(exact.sino_shape(1)) != tuple(plan.sino_shape(1))):
                raise ValueError("the exact plan must have the geometry of the plan")
            if int(correct_every) < 1 or (correct_bp_every is not None and
                                          int(correct_bp_every) < 1):
                raise ValueError("correction intervals must be at least 1")
        self.exact = exact
        self.unfused = False  # True: the correction passes as separate launches
        # True: each primal step leaves the duals unclipped and the next dual
        # step clips them as it loads them (same bits, no clip stores)
        self.defer_clip = True
        self.correct_every = int(correct_every)
        self.correct_bp_every = int(correct_bp_every) if correct_bp_every else int(correct_every)
        self.plan = plan
        self.cascades = int(cascades)
        self.sigma, self.tau, self.mu = float(sigma), float(tau), float(mu)
        self.v = tuple(float(x) for x in v)
        self.quirk = bool(quirk)
        self.f_dtype = f_dtype
        self.t_refresh = int(t_refresh)
        self.use_graph = use_graph
        self.backprojector = backprojector
        self.losses = None

    @classmethod
    def reference(cls, plan: Plan, cascades: int = 30, seed: int = 0, **kw) -> "DTVCP":
        """The reference's constants (DTVCP.py:11-27): normH = 10e4,
        v_a = normH/||D_a||, mu = normH/||I||, L = 10e6, tau = sigma = 1/L."""
        size = plan.geometry.volume_size
        normH = 10e4
        v = tuple(normH / power_norm(size, a, kw.get("quirk", True), seed=seed,
                                     device=plan.device) for a in range(3))
        L = 10e6
        return cls(plan, cascades, sigma=1.0 / L, tau=1.0 / L, mu=normH / 1.0, v=v, **kw)

    def _fused(self) -> bool:
        """Whether the correction passes run as one launch per operator
        (a "pairs" plan corrected by an "exact" plan) or as separate
        projections and element-wise steps (any other pairing)."""
        return (self.exact is not None and self.plan.sampler == "pairs"
                and self.exact.sampler == "exact" and not self.unfused)

    def _params(self):
        p = _lib.dtv_pdhg_params()
        p.sigma, p.tau, p.mu = self.sigma, self.tau, self.mu
        p.v[:] = self.v
        p.quirk = int(self.quirk)
        p.f_dtype = _FDT[self.f_dtype]
        return p

    def _alloc(self, image: torch.Tensor):
        dev = image.device
        vs = image.shape
        plan = self.plan
        b = image.numel() // int(np.prod(plan.vol_shape(1)))
        st = {
            "b": b,
            "f": torch.empty(vs, dtype=torch.float32, device=dev),
            "fbar": torch.empty(vs, dtype=self.f_dtype, device=dev),
            "p": torch.zeros(vs, dtype=torch.float32, device=dev),
            "q": torch.zeros(vs, dtype=torch.float32, device=dev),
            "s": torch.zeros(vs, dtype=torch.float32, device=dev),
            "c": torch.zeros(vs, dtype=torch.float32, device=dev),
            "recon": torch.empty(vs, dtype=torch.float32, device=dev),
            "w": torch.zeros(plan.sino_shape(b), dtype=torch.float32, device=dev),
            "g": torch.empty(plan.sino_shape(b), dtype=torch.float32, device=dev),
            "t": torch.zeros(3, dtype=torch.float64, device=dev),
            "loss": torch.zeros(self.cascades, dtype=torch.float64, device=dev),
            "carry": torch.zeros(3, dtype=torch.float32, device=dev),
            "ws": torch.zeros(_lib.load().dtv_pdhg_workspace_bytes(), dtype=torch.uint8,
                              device=dev),
        }
        if self.exact is not None:
            fused = self._fused()
            for k in ("g_eff",) if fused else ("s1", "s2", "g_eff"):
                st[k] = torch.empty(plan.sino_shape(b), dtype=torch.float32, device=dev)
            for k in ("e_b",) if fused else ("e_b", "t_vol"):
                st[k] = torch.empty(vs, dtype=torch.float32, device=dev)
        return st

    def _body(self, st, image):
        plan = self.plan
        prm = self._params()
        size = _lib.ivec(plan.geometry.volume_size)
        b = st["b"]
        dev = image.device
        f, fbar = st["f"], st["fbar"]
        f.copy_(image)
        fbar.copy_(image)
        for k in ("p", "q", "s", "c", "w", "loss"):
            st[k].zero_()
        stream = _stream(dev)
        for it in range(self.cascades):
            if it % self.t_refresh == 0:
                st["t"].zero_()
                call("dtv_diff_abs_sums", _ptr(f), _lib.DTV_F32, size, b, prm.quirk,
                     _ptr(st["t"]), stream)
            ex = self.exact
            refresh = ex is not None and it % self.correct_every == 0
            if refresh and self._fused():
                # one launch: both projections, g + e_F and the exact dual step
                forward_refresh(plan, ex, fbar, st["g"], st["w"], st["g_eff"], self.sigma,
                                st["loss"][it:it + 1])
            elif refresh:
                ns = st["w"].numel()
                ex.forward(fbar, out=st["s1"])
                plan.forward(fbar, out=st["s2"], epilogue=_lib.DTV_EPI_RESIDUAL, g=st["s1"])
                call("dtv_lincomb", _ptr(st["g"]), 1.0, _ptr(st["s2"]), 1.0, _ptr(st["g_eff"]),
                     ns, stream)  # data of the corrected projection: g + e_F
                call("dtv_pdhg_sino_dual", _ptr(st["w"]), _ptr(st["s1"]), _ptr(st["g"]),
                     self.sigma, ns, _ptr(st["loss"][it:it + 1]), stream)
            else:
                plan.forward(fbar, out=st["w"], epilogue=_lib.DTV_EPI_PDHG,
                             g=st["g_eff"] if ex is not None else st["g"], sigma=self.sigma,
                             abs_sum=st["loss"][it:it + 1])
            bp_refresh = ex is not None and it % self.correct_bp_every == 0
            if self.backprojector == "fdk":
                if ex is None:
                    plan.backward(st["w"], out=st["recon"])
                elif self.correct_bp_every == 1:
                    ex.backward(st["w"], out=st["recon"])
                elif bp_refresh and self._fused():
                    backward_refresh(plan, ex, st["w"], st["recon"], st["e_b"])
                elif bp_refresh:
                    ex.backward(st["w"], out=st["recon"])
                    plan.backward(st["w"], out=st["t_vol"])
                    call("dtv_lincomb", _ptr(st["recon"]), 1.0, _ptr(st["t_vol"]), -1.0,
                         _ptr(st["e_b"]), st["recon"].numel(), stream)
                else:
                    plan.backward(st["w"], out=st["recon"], base=st["e_b"])
            else:
                plan.adjoint(st["w"], out=st["recon"])
            duals = (_ptr(st["p"]), _ptr(st["q"]), _ptr(st["s"]), _ptr(st["c"]), size, b,
                     ctypes.byref(prm))
            if not self.defer_clip:
                call("dtv_pdhg_dual", _ptr(fbar), *duals, _ptr(st["t"]), _ptr(st["ws"]), stream)
                call("dtv_pdhg_primal", _ptr(f), _ptr(fbar), _ptr(st["recon"]), *duals,
                     _ptr(st["ws"]), stream)
                continue
            # the clip of iteration it-1's primal step happens as this dual
            # step loads the duals; the last primal step stores its clip
            call("dtv_pdhg_dual_defer", _ptr(fbar), *duals, _ptr(st["t"]), _ptr(st["ws"]),
                 _ptr(st["carry"]) if it > 0 else None, stream)
            if it == self.cascades - 1:
                call("dtv_pdhg_primal", _ptr(f), _ptr(fbar), _ptr(st["recon"]), *duals,
                     _ptr(st["ws"]), stream)
            else:
                call("dtv_pdhg_primal_defer", _ptr(f), _ptr(fbar), _ptr(st["recon"]), *duals,
                     _ptr(st["ws"]), _ptr(st["carry"]), stream)

    def _prepare(self, image, sino):
        check_input(image, "image", self.plan.vol_shape(image.shape[0]),
                    dtypes=(torch.float32, torch.float16, torch.bfloat16))
        key = (tuple(image.shape), image.device.index, self._fused(), self.defer_clip)
        st = self.__dict__.setdefault("_state", {}).get(key)
        if st is None:
            st = self._alloc(image)
            self._state[key] = st
            st["img"] = torch.empty_like(image, dtype=torch.float32)
        st["img"].copy_(image)
        st["g"].copy_(sino)
        return key, st

    def _enqueue(self, st):
        self._body(st, st["img"])

    def _result(self, st, out):
        """f (float32); per-iteration sum|A fbar - g| stays in self.losses."""
        self.losses = st["loss"]
        if out is None:
            return st["f"].float().clone()
        out.copy_(st["f"])
        return out


class FISTA(_Graphable):
    """FISTA with soft thresholding (model/FISTA/FISTA.py:16-27, class DTVFista):
    d = y - L BP(FP y - g); I = soft(d, lamb L); y = I + (t-1)/t' (I - I_prev)."""

    def __init__(self, plan: Plan, cascades: int = 30, lamb: float = 10e3, L: float = 0.0001,
                 use_graph: bool = False, backprojector: str = "fdk"):
        self.plan = plan
        self.cascades = int(cascades)
        self.lamb, self.L = float(lamb), float(L)
        self.use_graph = use_graph
        self.backprojector = backprojector

    def _body(self, st):
        plan = self.plan
        dev = st["y"].device
        stream = _stream(dev)
        st["y"].copy_(st["img"])
        st["xp"].copy_(st["img"])
        t = 1.0
        n = st["y"].numel()
        for _ in range(self.cascades):
            plan.forward(st["y"], out=st["r"], epilogue=_lib.DTV_EPI_RESIDUAL, g=st["g"])
            if self.backprojector == "fdk":
                plan.backward(st["r"], out=st["bp"])
            else:
                plan.adjoint(st["r"], out=st["bp"])
            tp = (1 + math.sqrt(1 + 4 * t ** 2)) / 2
            call("dtv_fista_update", _ptr(st["y"]), _ptr(st["xp"]), _ptr(st["bp"]), n, self.L,
                 self.lamb * self.L, (t - 1) / tp, stream)
            t = tp

    def _prepare(self, image, sino):
        check_input(image, "image", self.plan.vol_shape(image.shape[0]))
        key = (tuple(image.shape), image.device.index)
        st = self.__dict__.setdefault("_state", {}).get(key)
        if st is None:
            b = image.shape[0]
            st = {k: torch.empty_like(image) for k in ("y", "xp", "bp", "img")}
            st["r"] = torch.empty(self.plan.sino_shape(b), dtype=torch.float32,
                                  device=image.device)
            st["g"] = torch.empty_like(st["r"])
            self._state[key] = st
        st["img"].copy_(image)
        st["g"].copy_(sino)
        return key, st

    def _enqueue(self, st):
        self._body(st)

    def _result(self, st, out):
        if out is None:
            return st["xp"].clone()
        out.copy_(st["xp"])
        return out


class BatchedFISTA:
    """:class:`FISTA` on several reconstructions in lockstep: per iteration one
    forward-projector launch, one backprojector launch and one update launch
    cover every volume of a group, whatever their sizes and view counts
    (dtv_forward_many, dtv_backward_many, dtv_fista_update_many). ``groups``
    splits the volumes into that many groups of about equal work, each in
    lockstep on its own stream, so one group's backprojection runs beside
    another's forward projection. With ``use_graph`` a whole run is one
    captured CUDA graph. The plans must be "pairs" (or "tma") plans; each
    reconstruction gives the same result as its own :class:`FISTA` run."""

    def __init__(self, plans, cascades: int = 30, lamb: float = 10e3, L: float = 0.0001,
                 use_graph: bool = True, groups: int = 1):
        self.plans = list(plans)
        if len({id(p) for p in self.plans}) != len(self.plans):
            raise ValueError("each reconstruction needs a plan of its own")
        if int(groups) < 1:
            raise ValueError("groups must be at least 1")
        self.cascades = int(cascades)
        self.lamb, self.L = float(lamb), float(L)
        self.use_graph = use_graph
        self.launches_per_run = 0
        self._state = {}
        # greedy balance of (rays x edge) work over the groups, heaviest first
        work = [float(np.prod(p.sino_shape(1))) * max(p.vol_shape(1)) for p in self.plans]
        G = min(int(groups), len(self.plans))
        loads, self._groups = [0.0] * G, [[] for _ in range(G)]
        for i in sorted(range(len(self.plans)), key=lambda i: -work[i]):
            g = loads.index(min(loads))
            self._groups[g].append(i)
            loads[g] += work[i]
        self._streams = None

    def _prepare(self, images, sinos):
        key = tuple((tuple(i.shape), i.device.index) for i in images)
        st = self._state.get(key)
        if st is None:
            st = []
            for p, i in zip(self.plans, images):
                check_input(i, "image", p.vol_shape(1))
                d = {k: torch.empty_like(i) for k in ("y", "xp", "bp", "img")}
                d["r"] = torch.empty(p.sino_shape(1), device=i.device)
                d["g"] = torch.empty_like(d["r"])
                st.append(d)
            self._state[key] = st
        for d, i, s in zip(st, images, sinos):
            d["img"].copy_(i)
            d["g"].copy_(s)
        return key, st

    def _enqueue_group(self, plans, st):
        stream = _stream(st[0]["y"].device)
        ys, rs, gs, bps = ([d[k] for d in st] for k in ("y", "r", "g", "bp"))
        vp = ctypes.c_void_p * len(st)
        upd = (vp(*[d["y"].data_ptr() for d in st]), vp(*[d["xp"].data_ptr() for d in st]),
               vp(*[d["bp"].data_ptr() for d in st]),
               (ctypes.c_int64 * len(st))(*[d["y"].numel() for d in st]))
        for d in st:
            d["y"].copy_(d["img"])
            d["xp"].copy_(d["img"])
        t = 1.0
        for _ in range(self.cascades):
            forward_many(plans, ys, rs, epilogue=_lib.DTV_EPI_RESIDUAL, gs=gs)
            backward_many(plans, rs, bps)
            tp = (1 + math.sqrt(1 + 4 * t ** 2)) / 2
            call("dtv_fista_update_many", *upd, len(st), self.L, self.lamb * self.L,
                 (t - 1) / tp, stream)
            t = tp

    def _enqueue(self, st):
        if len(self._groups) == 1:
            self._enqueue_group(self.plans, st)
            return
        dev = st[0]["y"].device
        if self._streams is None:
            self._streams = [torch.cuda.Stream(device=dev) for _ in self._groups]
        main = torch.cuda.current_stream(dev)
        for idx, sm in zip(self._groups, self._streams):
            sm.wait_stream(main)
            with torch.cuda.stream(sm):
                self._enqueue_group([self.plans[i] for i in idx], [st[i] for i in idx])
        for sm in self._streams:
            main.wait_stream(sm)

    def run(self, images, sinos, outs=None):
        key, st = self._prepare(images, sinos)
        _run_graph(self, key, lambda: self._enqueue(st))
        outs = outs or [None] * len(st)
        res = []
        for d, o in zip(st, outs):
            if o is None:
                res.append(d["xp"].clone())
            else:
                o.copy_(d["xp"])
                res.append(o)
        return res


class DTVFISTA(_Graphable):
    """FISTA-DTV (model/FISTA/DTVFISTA.py:23-43): z = relu(f - sigma BP(FP f - g)),
    f_new = z + sum_a t_a D_a^T thr_a(D_a z), f = f_new + (t-1)/t' (f_new - f).
    quirk=True keeps the reference's global-max threshold and its momentum that
    never advances (t stays 1)."""

    def __init__(self, plan: Plan, cascades: int = 30, sigma: float = 1e-3, v=(1760., 1760., 1760.),
                 t=(1e-3, 1e-3, 1e-3), quirk: bool = True, use_graph: bool = False):
        self.plan = plan
        self.cascades = int(cascades)
        self.sigma = float(sigma)
        self.v = tuple(float(x) for x in v)
        self.t = tuple(float(x) for x in t)
        self.quirk = bool(quirk)
        self.use_graph = use_graph

    @classmethod
    def reference(cls, plan: Plan, cascades: int = 30, seed: int = 0, **kw) -> "DTVFISTA":
        """DTVFISTA.py:12-21: v_a = ||D_a|| / 1e-3 * 0.88, sigma = t_a = 1e-3."""
        size = plan.geometry.volume_size
        v = tuple(power_norm(size, a, kw.get("quirk", True), seed=seed, device=plan.device)
                  / 1e-3 * 0.88 for a in range(3))
        return cls(plan, cascades, sigma=1e-3, v=v, t=(1e-3,) * 3, **kw)

    def _body(self, st):
        plan = self.plan
        stream = _stream(st["f"].device)
        size = _lib.ivec(plan.geometry.volume_size)
        b = st["b"]
        n = st["f"].numel()
        st["f"].copy_(st["img"])
        t = 1.0
        vv, tt = _lib.fvec(self.v), _lib.fvec(self.t)
        for _ in range(self.cascades):
            tp = (1 + math.sqrt(1 + 4 * t ** 2)) / 2
            plan.forward(st["f"], out=st["r"], epilogue=_lib.DTV_EPI_RESIDUAL, g=st["g"])
            plan.backward(st["r"], out=st["z"])
            call("dtv_relu_step", _ptr(st["f"]), _ptr(st["z"]), _ptr(st["z"]), n, self.sigma,
                 stream)
            if self.quirk:
                call("dtv_dtvfista_maxes", _ptr(st["z"]), size, b, vv, _ptr(st["maxes"]), stream)
            call("dtv_dtvfista_update", _ptr(st["f"]), _ptr(st["z"]), size, b, vv, tt,
                 (t - 1) / tp, int(self.quirk), _ptr(st["maxes"]), stream)
            if not self.quirk:
                t = tp

    def _prepare(self, image, sino):
        check_input(image, "image", self.plan.vol_shape(image.shape[0]))
        key = (tuple(image.shape), image.device.index)
        st = self.__dict__.setdefault("_state", {}).get(key)
        if st is None:
            b = image.shape[0]
            st = {k: torch.empty_like(image) for k in ("f", "z", "img")}
            st["b"] = b
            st["r"] = torch.empty(self.plan.sino_shape(b), dtype=torch.float32,
                                  device=image.device)
            st["g"] = torch.empty_like(st["r"])
            st["maxes"] = torch.zeros(4, dtype=torch.float32, device=image.device)
            self._state[key] = st
        st["img"].copy_(image)
        st["g"].copy_(sino)
        return key, st

    def _enqueue(self, st):
        self._body(st)

    def _result(self, st, out):
        if out is None:
            return st["f"].clone()
        out.copy_(st["f"])
        return out


class ASDPOCS(_Graphable):
    """ASD-POCS (model/PDHG/ASDPOCS.py:28-47): a Landweber data step, then
    ``ng`` normalised-TV steepest-descent steps of length davg, davg = alpha*dp
    from the first data step. With quirk=True (the reference's behaviour) f0
    aliases f, the TV-change test never fires and davg stays fixed. With
    quirk=False f0 is a copy of the data-step result, dp = mean|f_prev - f|
    of every data step and dg = mean|f - f0| after the TV steps, and davg is
    multiplied by alpha whenever dg > rmax * dp (:44-45), all on the device;
    the TV steps then also use the clean D_y (no wrap into the next z-slice,
    Gradients.py:18-25), as in DTVCP's quirk=False."""

    def __init__(self, plan: Plan, cascades: int = 30, beta: float = 0.00005,
                 beta_red: float = 0.9999, ng: int = 10, alpha: float = 0.001, rmax: float = 0.95,
                 alpha_red: float = 0.95, quirk: bool = True, use_graph: bool = False):
        self.plan = plan
        self.cascades = int(cascades)
        self.beta, self.beta_red = float(beta), float(beta_red)
        self.ng, self.alpha, self.rmax, self.alpha_red = int(ng), float(alpha), float(rmax), float(
            alpha_red)
        self.quirk = quirk
        self.use_graph = use_graph

    def _body(self, st):
        plan = self.plan
        stream = _stream(st["f"].device)
        size = _lib.ivec(plan.geometry.volume_size)
        b = st["b"]
        n = st["f"].numel()
        f, f2 = st["f"], st["f2"]
        f.copy_(st["img"])
        beta = self.beta
        dy_quirk = 1 if self.quirk else 0
        for i in range(self.cascades):
            plan.forward(f, out=st["r"], epilogue=_lib.DTV_EPI_RESIDUAL, g=st["g"])
            plan.backward(st["r"], out=st["bp"])
            track = i == 0 or not self.quirk
            if track:
                st["l1"].zero_()
            call("dtv_axpy_l1", _ptr(f), _ptr(st["bp"]), beta, _ptr(st["l1"]) if track else None,
                 n, stream)
            if i == 0:  # davg = alpha * mean|f0 - f|   (:34-35)
                call("dtv_scale_scalar", _ptr(st["l1"]), self.alpha / n, _ptr(st["davg"]), stream)
            if not self.quirk:
                st["f0"].copy_(f)  # f0 = f, a copy (:36)
            for _ in range(self.ng):
                call("dtv_tv_descent", _ptr(f), _ptr(f2), size, b, dy_quirk, _ptr(st["davg"]),
                     stream)
                f, f2 = f2, f
            if not self.quirk:  # dg = mean|f - f0|; davg *= alpha if dg > rmax * dp (:44-45)
                st["dg"].zero_()
                call("dtv_l1_distance", _ptr(f), _ptr(st["f0"]), n, _ptr(st["dg"]), stream)
                call("dtv_asd_adapt", _ptr(st["l1"]), _ptr(st["dg"]), self.rmax, self.alpha,
                     _ptr(st["davg"]), stream)
            beta *= self.beta_red
        st["result"] = f

    def _prepare(self, image, sino):
        check_input(image, "image", self.plan.vol_shape(image.shape[0]))
        key = (tuple(image.shape), image.device.index)
        st = self.__dict__.setdefault("_state", {}).get(key)
        if st is None:
            b = image.shape[0]
            st = {k: torch.empty_like(image) for k in ("f", "f2", "bp", "img", "f0")}
            st["b"] = b
            st["dg"] = torch.zeros(1, dtype=torch.float64, device=image.device)
            st["r"] = torch.empty(self.plan.sino_shape(b), dtype=torch.float32,
                                  device=image.device)
            st["g"] = torch.empty_like(st["r"])
            st["l1"] = torch.zeros(1, dtype=torch.float64, device=image.device)
            st["davg"] = torch.zeros(1, dtype=torch.float32, device=image.device)
            self._state[key] = st
        st["img"].copy_(image)
        st["g"].copy_(sino)
        return key, st

    def _enqueue(self, st):
        self._body(st)

    def _result(self, st, out):
        res = torch.relu(st["result"])  # (:47)
        if out is None:
            return res
        out.copy_(res)
        return out
