"""Benchmark: sparse-view DTV reconstruction on the B200 kernels.

Workload (one "step"): a complete 100-iteration DTV (Chambolle-Pock, directional
TV along x/y/z with per-direction constraint levels) reconstruction of a
256^3 volume (1 mm voxels) from 64 views over 360 deg on a 384x384 detector
(1.2 mm pitch), source-origin 500 mm, source-detector 1000 mm, Poisson noise
at I0 = 1e5. Every iteration runs one forward projection, one FDK-weighted
backprojection and the fused dual/primal updates; the whole reconstruction is
one captured CUDA graph.

metric: GRay*samples/s fwd+back = iterations * (forward-projector ray samples
[exact chord / 1 voxel step, summed over rays] + backprojector voxel*views)
per second, whole job; recon/s alongside.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun (N > 1) every rank reconstructs its own volume (replicas, no
collective on the data path); the time is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "dtv-net_b200"))

METRIC = ("GRay·samples/s fwd+back & unrolled-DTV recon/s vs plain FP32, "
          "at ≤1e-3 RMSE vs FP64")
UNIT = "GRay·samples/s"

CFG = dict(nx=256, ny=256, nz=256, voxel=1.0, nu=384, nv=384, pitch=1.2, n_views=64,
           sod=500.0, sdd=1000.0, iters=100, i0=1e5, seed=2024)

# DRAM traffic of one forward-projector launch on this workload
# (dram__bytes_read.sum + dram__bytes_write.sum) and the texture-pipe
# utilisation of that launch, from one `ncu --set full` capture of the 13th
# forward projection of `python bench.py --profile 12`. They describe the
# kernel as captured then, not this run; "source" names the summary.
FP_NCU = {"pairs": {"traffic": 142.743040e6 + 28.150784e6, "tex_pipe_pct": 95.4,
                    "source": "profiles/fp_pair_kernel_sparse_view_dtv.md"}}

# Same-FOV downsample on which the 100-iteration reconstruction is checked
# against the FP64 oracle: 64^3 at 4 mm, 96x96 detector at 4.8 mm, 64 views.
CHECK_DOWNSAMPLE = 4


def workload_name(c):
    return (f"sparse-view DTV: {c['nx']}^3 x {c['voxel']:g} mm, {c['n_views']} views/360deg, "
            f"{c['nu']}x{c['nv']} det @ {c['pitch']:g} mm, SOD {c['sod']:g} SDD {c['sdd']:g}, "
            f"Poisson I0={c['i0']:g}, {c['iters']} DTV-PDHG iterations")


def dist_init():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def max_over_ranks(x, ws, dev):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        import statistics
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------- problem
def make_problem(dev, c, seed):
    import numpy as np
    import torch

    import dtvb200
    from dtvb200.phantom import ellipsoids, poisson_noise
    ang = np.linspace(0, 360, c["n_views"], endpoint=False)
    geo = dtvb200.circular(ang, (c["nx"], c["ny"], c["nz"]), (c["voxel"],) * 3,
                           (c["nu"], c["nv"]), (c["pitch"], c["pitch"]), c["sod"], c["sdd"])
    truth = ellipsoids((c["nz"], c["ny"], c["nx"]), seed=seed, device=dev)
    return geo, truth, ang


def dtv_params(plan, dev, iters=8):
    """Step sizes from the spectral radius of BP*A (power method, untimed)."""
    import torch
    x = torch.rand(plan.vol_shape(1), device=dev,
                   generator=torch.Generator(device=dev).manual_seed(5))
    lam = 1.0
    for _ in range(iters):
        y = plan.backward(plan.forward(x))
        lam = float(torch.linalg.vector_norm(y.double()) / torch.linalg.vector_norm(x.double()))
        x = y / torch.linalg.vector_norm(y)
    sigma = 0.9 / lam
    return dict(sigma=sigma, tau=sigma, mu=1.0, v=(0.5, 0.5, 0.5), quirk=False)


def rel_rmse(a, b):
    """Relative RMSE of a (tensor or array) against the reference b."""
    import numpy as np
    if hasattr(a, "detach"):
        a = a.detach().double().cpu().numpy()
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))


def time_steps(fn, steps, stream):
    import torch
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(steps):
        fn()
    end.record(stream)
    torch.cuda.synchronize()
    return start.elapsed_time(end) / 1e3


def op_profile(plan, alg, img, sino, dev):
    """One eager reconstruction with CUDA events around each operator (on the
    launching stream): average forward / backward / update time per iteration."""
    import ctypes

    import torch

    import dtvb200
    from dtvb200 import _lib
    from dtvb200.geometry import _ptr, _stream
    key = (tuple(img.shape), img.device.index, alg._fused(), alg.defer_clip)
    st = alg._state[key]
    prm = alg._params()
    size = _lib.ivec(plan.geometry.volume_size)
    stream = torch.cuda.current_stream(dev)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    t_fp = t_bp = t_up = 0.0
    f, fbar = st["f"], st["fbar"]
    f.copy_(img)
    fbar.copy_(img)
    for k in ("p", "q", "s", "c", "w", "loss"):
        st[k].zero_()
    pairs = []
    for it in range(alg.cascades):
        if it % alg.t_refresh == 0:
            st["t"].zero_()
            _lib.call("dtv_diff_abs_sums", _ptr(f), _lib.DTV_F32, size, 1, prm.quirk,
                      _ptr(st["t"]), _stream(dev))
        e = [ev() for _ in range(4)]
        e[0].record(stream)
        plan.forward(fbar, out=st["w"], epilogue=_lib.DTV_EPI_PDHG, g=st["g"], sigma=alg.sigma,
                     abs_sum=st["loss"][it:it + 1])
        e[1].record(stream)
        plan.backward(st["w"], out=st["recon"])
        e[2].record(stream)
        # the update steps as DTVCP runs them: the duals' clip deferred into
        # the next dual step, the last primal step storing it
        duals = (_ptr(st["p"]), _ptr(st["q"]), _ptr(st["s"]), _ptr(st["c"]), size, 1,
                 ctypes.byref(prm))
        _lib.call("dtv_pdhg_dual_defer", _ptr(fbar), *duals, _ptr(st["t"]), _ptr(st["ws"]),
                  _ptr(st["carry"]) if it > 0 else None, _stream(dev))
        if it == alg.cascades - 1:
            _lib.call("dtv_pdhg_primal", _ptr(f), _ptr(fbar), _ptr(st["recon"]), *duals,
                      _ptr(st["ws"]), _stream(dev))
        else:
            _lib.call("dtv_pdhg_primal_defer", _ptr(f), _ptr(fbar), _ptr(st["recon"]), *duals,
                      _ptr(st["ws"]), _ptr(st["carry"]), _stream(dev))
        e[3].record(stream)
        pairs.append(e)
    torch.cuda.synchronize()
    for e in pairs:
        t_fp += e[0].elapsed_time(e[1])
        t_bp += e[1].elapsed_time(e[2])
        t_up += e[2].elapsed_time(e[3])
    n = alg.cascades
    return t_fp / n, t_bp / n, t_up / n


# ----------------------------------------------------------------------------- CPU baseline
def cpu_baseline(c, truth_np, views_per_step=2, steps=1, warmup=0):
    """The FP64 oracle (OpenMP over all host cores) on a bounded sample of the
    workload: forward projection and FDK backprojection of `views_per_step`
    views per step. Returns (GRay*samples/s, cores, sample description, seconds)."""
    import numpy as np
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    ang = np.linspace(0, 360, c["n_views"], endpoint=False)
    full = O.circular_geometry(ang, (c["nx"], c["ny"], c["nz"]), (c["voxel"],) * 3,
                               (c["nu"], c["nv"]), (c["pitch"], c["pitch"]), c["sod"], c["sdd"])
    cores = O.num_threads()
    vol = np.ascontiguousarray(truth_np, dtype=np.float64)
    V = c["nx"] * c["ny"] * c["nz"]
    total_units = 0.0
    elapsed = 0.0
    for s in range(warmup + steps):
        sel = [(s * views_per_step + j) % c["n_views"] for j in range(views_per_step)]
        g = O.circular_geometry(ang[sel], (c["nx"], c["ny"], c["nz"]), (c["voxel"],) * 3,
                                (c["nu"], c["nv"]), (c["pitch"], c["pitch"]), c["sod"], c["sdd"])
        # FDK weight of the full scan (pi / N_full) keeps the sample's arithmetic identical
        g.og.bp_scale = full.og.bp_scale
        t0 = time.perf_counter()
        sino = O.forward(g, vol)
        O.backward(g, sino)
        dt = time.perf_counter() - t0
        if s >= warmup:
            elapsed += dt
            total_units += O.fp_samples(g) + V * len(sel)
    sample = (f"FP64 oracle forward + FDK backprojection of {views_per_step} of "
              f"{c['n_views']} views per step x {steps} steps (same volume, detector, geometry)")
    return total_units / elapsed / 1e9, cores, sample, elapsed


def fp64_check(c, dev, sampler, plan, truth, sino_clean, variants):
    """Checker leg, outside every timed region: relative RMSE against the FP64
    oracle of (1) the workload's forward projection of the phantom and (2) its
    FDK backprojection, both at full size on 16 of the views, and (3) the
    100-iteration reconstruction, on a same-FOV downsample by CHECK_DOWNSAMPLE
    (edge, detector and views per FOV scaled together; 64 views kept), with the
    same sampler, storage, step-size rule and noise model as the timed run.
    ``variants``: (name, f_dtype, correct_every) reconstructions to check;
    correct_every > 0 corrects the sampler's operators with an "exact" plan
    every that many iterations (DTVCP's ``exact``), 0 runs it uncorrected."""
    import numpy as np
    import torch

    import dtvb200
    from dtvb200.phantom import ellipsoids, poisson_noise
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O

    def rel(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))

    t0 = time.perf_counter()
    ang = np.linspace(0, 360, c["n_views"], endpoint=False)
    sel = list(range(0, c["n_views"], c["n_views"] // 16))
    vs = (c["nx"], c["ny"], c["nz"])
    geo_args = ((c["voxel"],) * 3, (c["nu"], c["nv"]), (c["pitch"], c["pitch"]), c["sod"], c["sdd"])
    full = O.circular_geometry(ang, vs, *geo_args)
    g_sel = O.circular_geometry(ang[sel], vs, *geo_args)
    g_sel.og.bp_scale = full.og.bp_scale  # the full scan's FDK weight pi / N
    vol = truth[0, 0].double().cpu().numpy()
    fp_gpu = sino_clean[0, 0, sel].double().cpu().numpy()
    e_fp = rel(fp_gpu, O.forward(g_sel, vol).reshape(fp_gpu.shape))
    s_in = torch.zeros_like(sino_clean)
    s_in[:, :, sel] = sino_clean[:, :, sel]
    bp_gpu = plan.backward(s_in).double().cpu().numpy().reshape(vol.shape)
    e_bp = rel(bp_gpu, O.backward(g_sel, sino_clean[0, 0, sel].cpu().numpy()).reshape(vol.shape))

    k = CHECK_DOWNSAMPLE
    d = dict(c, nx=c["nx"] // k, ny=c["ny"] // k, nz=c["nz"] // k, voxel=c["voxel"] * k,
             nu=c["nu"] // k, nv=c["nv"] // k, pitch=c["pitch"] * k)
    dvs = (d["nx"], d["ny"], d["nz"])
    dargs = ((d["voxel"],) * 3, (d["nu"], d["nv"]), (d["pitch"], d["pitch"]), d["sod"], d["sdd"])
    geo_d = dtvb200.circular(ang, dvs, *dargs)
    og_d = O.circular_geometry(ang, dvs, *dargs)
    plan_d = dtvb200.Plan(geo_d, max_batch=1, sampler=sampler, device=dev)
    truth_d = ellipsoids((d["nz"], d["ny"], d["nx"]), seed=c["seed"], device=dev)
    sino_d = poisson_noise(plan_d.forward(truth_d), c["i0"], seed=c["seed"])
    prm_d = dtv_params(plan_d, dev)
    sino_np = sino_d.cpu().numpy()
    fpo = lambda x: O.forward(og_d, x).reshape(x.shape[0], 1, *og_d.sino_shape)  # noqa: E731
    bpo = lambda s: O.backward(og_d, s).reshape(s.shape[0], 1, *og_d.vol_shape)  # noqa: E731
    ref = O.dtvcp_run(fpo, bpo, np.zeros((1, 1) + og_d.vol_shape), sino_np, dvs, c["iters"],
                      prm_d["sigma"], prm_d["tau"], prm_d["mu"], prm_d["v"], quirk=prm_d["quirk"])
    recon = {}
    exact_d = None
    for name, fdt, every in variants:
        pl = plan_d if fdt == torch.float32 or sampler != "pairs" else \
            dtvb200.Plan(geo_d, max_batch=1, sampler=sampler, stage_f16=True, device=dev)
        if every and exact_d is None:
            exact_d = dtvb200.Plan(geo_d, max_batch=1, sampler="exact", device=dev)
        alg = dtvb200.DTVCP(pl, c["iters"], t_refresh=10, use_graph=True, f_dtype=fdt,
                            exact=exact_d if every else None, correct_every=max(every, 1),
                            **prm_d)
        recon[name] = rel(alg.run(torch.zeros(pl.vol_shape(1), device=dev), sino_d).cpu().numpy(),
                          ref)
    return {
        "forward_full_size": e_fp, "backward_full_size": e_bp,
        "reconstruction": recon, "gate": 1e-3,
        "how": (f"relative RMSE vs the FP64 oracle (OpenMP C, exact trilinear/bilinear). "
                f"Projections: the {c['nx']}^3 phantom, {len(sel)} of {c['n_views']} views at "
                f"full size. Reconstruction: {c['iters']} DTV-PDHG iterations on a same-FOV "
                f"downsample ({d['nx']}^3 x {d['voxel']:g} mm, {d['nu']}x{d['nv']} det @ "
                f"{d['pitch']:g} mm, {c['n_views']} views, Poisson I0={c['i0']:g}), same "
                f"sampler, storage and step-size rule as the timed run; the oracle runs the "
                f"reference loop (DTVCP.py:29-60) on the same noisy sinogram"),
        "seconds": time.perf_counter() - t0,
    }


def reference_cuda_baseline(c, dev, truth, steps=3):
    """Baseline leg: the reference's own CUDA projectors (its unmodified
    forwardKernel.cu / backwardKernel.cu, compiled with the texture-object
    shim into oracle/_ref) called through their pybind API exactly as
    StandardGeometry.py calls them: one launch per view with a host .item()
    read before each, a cudaArray copy of the input per call. Timed per call
    beside this library's Standard-geometry plans on the same arrays, in the
    reference's geometry convention (voxel = detector pixel x SID/SDD)."""
    import importlib.machinery
    import importlib.util

    import numpy as np
    import torch

    import dtvb200
    path = os.path.join(REPO, "oracle", "_ref", "JITStandardGeometry.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/JITStandardGeometry.so not built"}
    loader = importlib.machinery.ExtensionFileLoader("JITStandardGeometry", path)
    spec = importlib.util.spec_from_file_location("JITStandardGeometry", path, loader=loader)
    ref = importlib.util.module_from_spec(spec)
    loader.exec_module(ref)
    vs, ds = (c["nx"], c["ny"], c["nz"]), (c["nu"], c["nv"])
    angles = np.linspace(0, 360, c["n_views"], endpoint=False)  # StandardGeometry.py:6
    at = torch.from_numpy(angles).to(dev)
    vst, dst = torch.tensor(vs).to(dev), torch.tensor(ds).to(dev)
    sid, sdd = c["sod"], c["sdd"]
    stream = torch.cuda.current_stream(dev)
    geo = dtvb200.standard(angles.astype(np.float32), vs, ds, sid, sdd)
    samples = dtvb200.Plan(geo, max_batch=1, sampler="soft", device=dev).fp_samples()
    bp_units = float(np.prod(vs)) * c["n_views"]
    sino = torch.empty((1, 1, c["n_views"], ds[1], ds[0]), device=dev)

    def timed(fwd, bwd):
        fwd()
        bwd()
        tf = time_steps(fwd, steps, stream) / steps
        tb = time_steps(bwd, steps, stream) / steps
        return {"forward_ms": tf * 1e3, "backward_ms": tb * 1e3,
                "value": (samples + bp_units) / (tf + tb) / 1e9}

    out = {"unit": UNIT, "geometry": (f"reference convention: {vs[0]}^3 voxels of SID/SDD "
                                      f"detector pixels, {c['n_views']} views of "
                                      f"{ds[0]}x{ds[1]}, SID {sid:g}, SDD {sdd:g}"),
           "note": ("samples counted as this library's plan counts them for that geometry "
                    "(the reference marches about twice as many, from its alpha-range rule)")}
    sino_ref = ref.forward(truth, at, vst, dst, sid, sdd, dev.index)
    out["reference"] = timed(lambda: ref.forward(truth, at, vst, dst, sid, sdd, dev.index),
                             lambda: ref.backward(sino_ref, at, vst, dst, sid, sdd, dev.index))
    for smp in ("tex", "pairs"):
        pl = dtvb200.Plan(geo, max_batch=1, sampler=smp, device=dev)
        vol_out = torch.empty_like(truth)
        out[f"ours_{smp}"] = timed(lambda: pl.forward(truth, out=sino),
                                   lambda: pl.backward(sino_ref, out=vol_out))
        diff = float(((pl.forward(truth) - sino_ref).double() ** 2).mean().sqrt()
                     / (sino_ref.double() ** 2).mean().sqrt())
        out[f"ours_{smp}"]["forward_rel_rmse_vs_reference"] = diff
        del pl
    out["speedup_pairs_vs_reference"] = out["ours_pairs"]["value"] / out["reference"]["value"]
    return out


def run_reference(args):
    ws, rank, local = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return 0
    import torch
    c = dict(CFG)
    sys.path.insert(0, os.path.join(REPO, "dtv-net_b200"))
    from dtvb200.phantom import ellipsoids
    truth = ellipsoids((c["nz"], c["ny"], c["nx"]), seed=c["seed"], device="cpu").numpy()
    value, cores, sample, secs = cpu_baseline(c, truth[0, 0], views_per_step=8, steps=args.steps,
                                              warmup=args.warmup)
    samples_per_iter = None
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": secs / max(args.steps, 1) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(c), "inputs": "seeded ellipsoid phantom"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("the reference implements this path only as CUDA kernels (texture "
                 "references); its CPU path is this FP64 restatement of the same formulas"),
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- ours
def run_ours(args):
    import numpy as np
    import torch

    import dtvb200
    from dtvb200.phantom import poisson_noise
    ws, rank, local = dist_init()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    c = dict(CFG)
    if args.small:
        c.update(nx=64, ny=64, nz=64, nu=96, nv=96, n_views=16, iters=10)
    geo, truth, _ = make_problem(dev, c, c["seed"] + rank)
    tex_peak = dtvb200._lib.measure_texture_fetch_rate(32)
    plan = dtvb200.Plan(geo, max_batch=1, sampler=args.sampler, device=dev)
    sino_clean = plan.forward(truth)
    sino = poisson_noise(sino_clean, c["i0"], seed=c["seed"] + rank)
    prm = dtv_params(plan, dev)
    # texture-filtered samplers are corrected by the exact-weight plan every
    # K iterations, which keeps the reconstruction within 1e-3 of FP64
    K = args.correct_every if args.sampler in ("pairs", "tex", "tma") else 0
    xplan = dtvb200.Plan(geo, max_batch=1, sampler="exact", device=dev) if K else None
    corr = dict(exact=xplan, correct_every=max(K, 1))
    # the projected iterate fbar is stored in FP16 (--fbar f16) or FP32; the
    # iterate f, the duals and all arithmetic stay FP32
    fdt = torch.float16 if args.fbar == "f16" else torch.float32
    alg = dtvb200.DTVCP(plan, c["iters"], t_refresh=10, use_graph=True, f_dtype=fdt, **corr,
                        **prm)
    img = torch.zeros(plan.vol_shape(1), device=dev)
    stream = torch.cuda.current_stream(dev)

    # capture (counts the kernels of one replay), then warm up
    alg.run(img, sino)
    launches = alg.launches_per_run
    for _ in range(max(args.warmup - 1, 0)):
        alg.run(img, sino)
    fp_samples = plan.fp_samples()
    V = c["nx"] * c["ny"] * c["nz"]
    units = c["iters"] * (fp_samples + V * c["n_views"])  # per reconstruction

    # ---- device-resident timing
    barrier(ws)
    with ClockSampler(local) as clk:
        secs = time_steps(lambda: alg.run(img, sino), args.steps, stream)
    secs = max_over_ranks(secs, ws, dev)
    barrier(ws)
    value = ws * units * args.steps / secs / 1e9
    recon_s = ws * args.steps / secs

    # ---- end to end through the public API with host buffers
    sino_h = sino.cpu().pin_memory()
    out_h = torch.empty(plan.vol_shape(1), dtype=torch.float32).pin_memory()
    res_d = torch.empty(plan.vol_shape(1), device=dev)

    def e2e_step():
        alg.run(img, sino_h, out=res_d)  # H2D of the sinogram inside run()
        out_h.copy_(res_d, non_blocking=True)

    e2e_step()
    barrier(ws)
    e_secs = max_over_ranks(time_steps(e2e_step, args.steps, stream), ws, dev)
    e2e_value = ws * units * args.steps / e_secs / 1e9

    # ---- per-operator profile (eager pass with events on the launching stream)
    t_fp, t_bp, t_up = op_profile(plan, alg, img, sino, dev)
    t_xfp = t_xbp = 0.0
    if xplan is not None and alg._fused():  # the one-launch correction passes, timed alone
        vol = img + 0.5
        w_, ge_ = torch.zeros_like(sino), torch.empty_like(sino)
        xv, eb_ = torch.empty(plan.vol_shape(1), device=dev), torch.empty(plan.vol_shape(1),
                                                                            device=dev)
        t_xfp = time_steps(lambda: dtvb200.forward_refresh(plan, xplan, vol, sino, w_, ge_, 0.1),
                           5, stream) / 5 * 1e3
        t_xbp = time_steps(lambda: dtvb200.backward_refresh(plan, xplan, sino, xv, eb_), 5,
                           stream) / 5 * 1e3
    elif xplan is not None:  # the exact operators of each correction, timed alone
        xs = torch.empty(plan.sino_shape(1), device=dev)
        xv = torch.empty(plan.vol_shape(1), device=dev)
        t_xfp = time_steps(lambda: xplan.forward(img + 0.5, out=xs), 5, stream) / 5 * 1e3
        t_xbp = time_steps(lambda: xplan.backward(sino, out=xv), 5, stream) / 5 * 1e3
    n_views, P = c["n_views"], c["n_views"] * c["nu"] * c["nv"]
    fp_bytes = n_views * V * 4 + P * 4  # one volume pass per view + sinogram write (FP32)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    achieved = fp_bytes / (t_fp * 1e-3) / 1e9

    # ---- the other fbar storage and the plain FP32 single-volume path
    extra = {}
    if not args.no_variants:
        f_head = alg.run(img, sino)
        odt = torch.float32 if fdt == torch.float16 else torch.float16
        alt = dtvb200.DTVCP(plan, c["iters"], t_refresh=10, use_graph=True, f_dtype=odt, **corr,
                            **prm)
        alt.run(img, sino)
        s_alt = time_steps(lambda: alt.run(img, sino), args.steps, stream)
        f_alt = alt.run(img, sino)
        f32_ref, other = (f_alt, f_head) if odt == torch.float32 else (f_head, f_alt)
        err16 = float(torch.sqrt(((other - f32_ref).double() ** 2).mean()
                                 / (f32_ref.double() ** 2).mean()))
        extra = {
            ("fp32_fbar_storage" if odt == torch.float32 else "fp16_fbar_storage"): {
                "value": units * args.steps / s_alt / 1e9, "recon_per_s": args.steps / s_alt},
            "rel_rmse_fp16_vs_fp32_fbar_storage": err16,
        }
        del alt
        # the plain FP32 single-volume path: FP32 staging and FP32 weights,
        # one launch per operator, no graph ("soft"); and the same through an
        # FP32 3-D texture, as the reference samples ("tex")
        for name, smp in (("plain_fp32_eager", "soft"), ("plain_fp32_tex_eager", "tex")):
            pplan = dtvb200.Plan(geo, max_batch=1, sampler=smp, device=dev)
            plain = dtvb200.DTVCP(pplan, c["iters"], t_refresh=10, use_graph=False, **prm)
            plain.run(img, sino)
            sp = time_steps(lambda: plain.run(img, sino), args.steps, stream)
            extra[name] = {"value": units * args.steps / sp / 1e9, "recon_per_s": args.steps / sp,
                           "sampler": smp}
            del plain, pplan
        extra["speedup_vs_plain_fp32"] = recon_s / extra["plain_fp32_eager"]["recon_per_s"]

    cpu = check = ref_cuda = None
    if rank == 0 and ws == 1 and not args.no_check:
        variants = [("fp32_f", torch.float32, K), ("fp16_fbar", torch.float16, K)]
        if K:
            variants.append(("fp32_f_uncorrected", torch.float32, 0))
        check = fp64_check(c, dev, args.sampler, plan, truth, sino_clean, variants)
        ref_cuda = reference_cuda_baseline(c, dev, truth)
    if rank == 0 and ws == 1 and not args.no_cpu:
        # 48 of the 64 views: about 10-20 s of FP64 work on the host cores
        v, cores, sample, _ = cpu_baseline(c, truth[0, 0].double().cpu().numpy(),
                                           views_per_step=16, steps=3)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "fp16-staged/fp32-acc" if args.sampler in ("pairs", "tma") else "f32",
        "data": "synthetic",
        "config": {"workload": workload_name(c), "parallelism": f"replicas x{ws}",
                   "sampler": args.sampler, "graph": "one CUDA graph per reconstruction",
                   "l2": "working set > L2 (volume, 4 dual volumes, sinograms ~0.5 GB)",
                   "storage": (f"f, duals, sinograms FP32; the projected iterate fbar stored "
                               f"{'FP16' if args.fbar == 'f16' else 'FP32'} and staged as FP16 "
                               f"z-pairs; FP32 accumulation"),
                   "correction": (f"operators corrected by the exact-weight plan every {K} "
                                  f"iterations (DTVCP exact=)" if K else None),
                   "inputs": "seeded ellipsoid phantom, Poisson noise"},
        "recon_per_s": recon_s,
        "samples_per_recon": units,
        "per_iteration_ms": {"total": secs / args.steps / c["iters"] * 1e3, "forward": t_fp,
                             "backward": t_bp, "updates": t_up,
                             ("refresh_forward" if alg._fused() else "exact_forward"):
                                 t_xfp or None,
                             ("refresh_backward" if alg._fused() else "exact_backward"):
                                 t_xbp or None,
                             "correct_every": K or None},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak,
                     "traffic": FP_NCU.get(args.sampler, {}).get("traffic"),
                     "texture_pipe_pct_of_peak": FP_NCU.get(args.sampler, {}).get("tex_pipe_pct"),
                     "traffic_source": FP_NCU.get(args.sampler, {}).get("source"),
                     "kernel": "forward projector (staging + ray kernel)",
                     "algorithmic_bytes_per_launch": fp_bytes,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                     "texture": {
                         "unit": "bilinear fetches/s",
                         "peak": tex_peak,
                         "peak_source": ("measured in this run (dtv_measure_texture_fetch_rate, "
                                         "32-bit texels)"),
                         "forward_achieved": fp_samples / (t_fp * 1e-3),
                         "forward_frac": fp_samples / (t_fp * 1e-3) / tex_peak,
                         "backward_achieved": V * n_views / (t_bp * 1e-3),
                         "backward_frac": V * n_views / (t_bp * 1e-3) / tex_peak},
                     # secondary figures of the survey's roofline: the trilinear
                     # tap rate (8 taps of 2-byte FP16 values per sample) and a
                     # whole iteration's algorithmic bytes (forward as above;
                     # single-pass backprojection P*4 + 2*V*4; DTV-PDHG update
                     # 13*V*4 + 3*P*4) over its measured time
                     "tap_rate_gbs": 8 * fp_samples * 2 / (t_fp * 1e-3) / 1e9,
                     "iteration": {
                         "algorithmic_bytes": fp_bytes + (P * 4 + 2 * V * 4)
                                              + (13 * V * 4 + 3 * P * 4),
                         "ms": secs / args.steps / c["iters"] * 1e3,
                         "achieved_gbs": (fp_bytes + P * 4 + 2 * V * 4 + 13 * V * 4 + 3 * P * 4)
                                         / (secs / args.steps / c["iters"]) / 1e9,
                         "frac": (fp_bytes + P * 4 + 2 * V * 4 + 13 * V * 4 + 3 * P * 4)
                                 / (secs / args.steps / c["iters"]) / 1e9 / hbm_peak}},
        "error_vs_fp64": check,
        "cpu_baseline": cpu,
        "reference_cuda_baseline": ref_cuda,
        "clocks": clk.summary(),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": P * 4,
                "d2h_bytes_per_step": V * 4},
        "gpu_launches": launches * args.steps,
    }
    line.update(extra)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_batch16(args):
    """16 heterogeneous reconstructions: edges seeded uniform in {96,128,192,256},
    30-120 views, square detector 1.5x the edge (pitch 1.5 mm, voxel 1 mm),
    30 FISTA iterations each. Batched = one graph with a stream per
    reconstruction; plain = the same reconstructions one after another, eager."""
    import numpy as np
    import torch

    import dtvb200
    from dtvb200.phantom import ellipsoids
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(16)
    algs, plains, imgs, sinos, units = [], [], [], [], 0.0
    specs = []
    for i in range(16):
        n = int(rng.choice([96, 128, 192, 256]))
        views = int(rng.integers(30, 121))
        d = int(round(1.5 * n))
        ang = np.linspace(0, 360, views, endpoint=False)
        geo = dtvb200.circular(ang, (n, n, n), (1.0,) * 3, (d, d), (1.5, 1.5), 500.0, 1000.0)
        plan = dtvb200.Plan(geo, sampler=args.sampler, device=dev)
        truth = ellipsoids((n, n, n), seed=100 + i, device=dev)
        sino = plan.forward(truth)
        algs.append(dtvb200.FISTA(plan, 30, lamb=0.05, L=1e-3))
        # the plain FP32 path: software sampler, eager, one reconstruction at a time
        plains.append(dtvb200.FISTA(dtvb200.Plan(geo, sampler="soft", device=dev), 30, lamb=0.05,
                                    L=1e-3))
        imgs.append(torch.zeros_like(truth))
        sinos.append(sino)
        units += 30 * (plan.fp_samples() + n ** 3 * views)
        specs.append((n, views))
    batch = dtvb200.Batched(algs, use_graph=True)
    stream = torch.cuda.current_stream(dev)
    for _ in range(max(args.warmup, 1)):
        batch.run(imgs, sinos)
    with ClockSampler(0) as clk:
        secs = time_steps(lambda: batch.run(imgs, sinos), args.steps, stream)

    # lockstep: one forward and one backprojector launch per iteration for all 16
    lock = None
    if args.sampler in ("pairs", "tma"):
        lock = dtvb200.BatchedFISTA([a.plan for a in algs], 30, lamb=0.05, L=1e-3,
                                    use_graph=True, groups=2)
        lock.run(imgs, sinos)
        ls = time_steps(lambda: lock.run(imgs, sinos), args.steps, stream)

    def plain_all():
        for a, i, s in zip(plains, imgs, sinos):
            a.run(i, s)

    plain_all()
    ps = time_steps(plain_all, args.steps, stream)

    # checker leg (outside the timed regions): the smallest reconstruction of
    # the batch against the FP64 oracle's FISTA on the same sinogram
    check = None
    if not args.no_check:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle as O
        i = min(range(16), key=lambda k: specs[k][0] * specs[k][0] * specs[k][1])
        n, views = specs[i]
        d = int(round(1.5 * n))
        og = O.circular_geometry(np.linspace(0, 360, views, endpoint=False), (n, n, n),
                                 (1.0,) * 3, (d, d), (1.5, 1.5), 500.0, 1000.0)
        t0 = time.perf_counter()
        fp = lambda x: O.forward(og, x).reshape(x.shape[0], 1, *og.sino_shape)  # noqa: E731
        bp = lambda s_: O.backward(og, s_).reshape(s_.shape[0], 1, *og.vol_shape)  # noqa: E731
        ref = O.fista_run(fp, bp, np.zeros((1, 1) + og.vol_shape),
                          sinos[i].double().cpu().numpy(), 30, 1e-3, 0.05)
        got = batch.run(imgs, sinos)[i]
        check = {"reconstruction": rel_rmse(got, ref), "gate": 1e-3, "volume": [n, views],
                 "seconds": time.perf_counter() - t0,
                 "how": "relative RMSE of the batch's smallest reconstruction (30 FISTA "
                        "iterations) against the FP64 oracle's FISTA on the same sinogram"}
    line = {
        "metric": METRIC, "value": units * args.steps / secs / 1e9, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "16 heterogeneous FISTA reconstructions (30 iterations each), "
                               "edges in {96,128,192,256}, 30-120 views, detector 1.5x edge",
                   "sizes_views": specs, "sampler": args.sampler},
        "recon_per_s": 16 * args.steps / secs,
        "plain_fp32_sequential_eager": {"value": units * args.steps / ps / 1e9,
                                        "recon_per_s": 16 * args.steps / ps, "sampler": "soft"},
        "speedup_vs_plain_fp32": ps / secs,
        "lockstep_one_launch_per_operator": None if lock is None else {
            "value": units * args.steps / ls / 1e9, "recon_per_s": 16 * args.steps / ls,
            "groups": 2, "gpu_launches_per_run": lock.launches_per_run},
        "gpu_launches": batch.launches_per_run * args.steps,
        "clocks": clk.summary(),
        "error_vs_fp64": check,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_train(args):
    """Training steps of a 10-stage unrolled PDHG network (learned steps + a
    3-layer 3x3x3 conv block with 32 channels per stage, BF16 activations,
    FP32 weights, per-stage checkpointing) on a batch of two 128^3 phantoms
    seen by 48 views of 192x192 (pitch 1.5 mm): L2 loss, Adam. The data
    steps and their gradients go through the matched projector pair."""
    import numpy as np
    import torch

    import dtvb200
    from dtvb200.nets import UnrolledPDHG
    from dtvb200.phantom import ellipsoids
    dev = torch.device("cuda", 0)
    torch.backends.cudnn.benchmark = True  # the conv shapes repeat every stage
    n, views, det, stages = 128, 48, 192, 10
    ang = np.linspace(0, 360, views, endpoint=False)
    geo = dtvb200.circular(ang, (n, n, n), (1.0,) * 3, (det, det), (1.5, 1.5), 500.0, 1000.0)
    proj = dtvb200.Projector(geo, max_batch=2)
    truth = torch.cat([ellipsoids((n, n, n), seed=s, device=dev) for s in (1, 2)])
    sino = proj.fp_soft(truth)
    torch.manual_seed(0)
    net = UnrolledPDHG(proj, stages=stages, features=32, lamb=1e-3, tau=1e-3).to(dev)
    opt = torch.optim.Adam(net.parameters(), lr=1e-4)
    x0 = torch.zeros_like(truth)

    def step():
        opt.zero_grad(set_to_none=True)
        loss = torch.mean((net(x0, sino) - truth) ** 2)
        loss.backward()
        opt.step()
        return loss

    for _ in range(max(args.warmup, 1)):
        step()
    stream = torch.cuda.current_stream(dev)
    L = dtvb200._lib.load()
    n0 = L.dtv_launch_count()
    with ClockSampler(0) as clk:
        secs = time_steps(step, args.steps, stream)
    launches = L.dtv_launch_count() - n0
    plan = proj.plan(dev, 2)
    fp_units = 2 * plan.fp_samples()  # per forward projection of the batch
    # the exact adjoint alone: each sample adds two 16-byte vector reductions
    # into L2-resident cell records, so its bound is the L2's rate of those
    # reductions, measured here with a kernel that does nothing else
    adj_in = torch.rand(plan.sino_shape(2), device=dev)
    adj_out = torch.empty(plan.vol_shape(2), device=dev)
    plan.adjoint(adj_in, out=adj_out)
    t_adj = time_steps(lambda: plan.adjoint(adj_in, out=adj_out), 10, stream) / 10
    v4_contig = dtvb200._lib.measure_atomic_v4_rate(72 << 16, 0)
    v4_scatter = dtvb200._lib.measure_atomic_v4_rate(72 << 16, 1)
    adj_rate = 2 * fp_units / t_adj
    # per training step: each stage runs FP + A^T forward, recomputes them under
    # checkpointing, and backpropagates through both (FP + A^T again)
    units = stages * 3 * 2 * fp_units
    line = {
        "metric": "unrolled-net training steps/s (projector pair through the exact adjoint)",
        "value": args.steps / secs, "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 projectors, bf16 conv activations",
        "data": "synthetic",
        "config": {"workload": "10-stage unrolled PDHG net, batch 2 x 128^3, 48 views of 192^2",
                   "checkpointing": "per stage"},
        "projector_gsamples_per_s": units * args.steps / secs / 1e9,
        "roofline": {
            "bound": "l2-atomic", "kernel": "exact adjoint (cell-record scatter + gather)",
            "unit": "float4 reductions/s", "achieved": adj_rate, "peak": v4_contig,
            "frac": adj_rate / v4_contig,
            "peak_source": ("measured in this run (dtv_measure_atomic_v4_rate: each warp's 32 "
                            "lanes on 32 consecutive 16-byte records, 75 MB of records)"),
            "scattered_peak": v4_scatter,
            "adjoint_ms": t_adj * 1e3,
            "reductions_per_launch": 2 * fp_units,
            "note": ("two reductions per forward-projector sample of the batch (samples whose "
                     "cell lies wholly in the zero border add none, so achieved is an upper "
                     "bound)")},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def run_fista64(args):
    """Plain method, small: 64^3 ellipsoid phantom (1 mm voxels), 60 views over
    360 deg on a 128x128 detector at 1.0 mm pitch, SOD 500 / SDD 1000. One step
    = forward projection of the phantom, one backprojection, then 20 FISTA-TV
    (FISTA with directional-TV thresholds) iterations, as one CUDA graph."""
    import numpy as np
    import torch

    import dtvb200
    from dtvb200.algorithms import power_norm
    dev = torch.device("cuda", 0)
    c = dict(CFG, nx=64, ny=64, nz=64, nu=128, nv=128, pitch=1.0, n_views=60, iters=20)
    geo, truth, _ = make_problem(dev, c, c["seed"])
    V = 64 ** 3

    def build(sampler, graph):
        plan = dtvb200.Plan(geo, max_batch=1, sampler=sampler, device=dev)
        sigma = dtv_params(plan, dev)["sigma"]
        v = tuple(power_norm((64, 64, 64), a, False, device=dev) for a in range(3))
        alg = dtvb200.DTVFISTA(plan, c["iters"], sigma=sigma, v=v, t=(1e-3,) * 3, quirk=False)
        out_s = torch.empty(plan.sino_shape(1), device=dev)
        out_b = torch.empty(plan.vol_shape(1), device=dev)
        img = torch.zeros(plan.vol_shape(1), device=dev)

        def body():
            plan.forward(truth, out=out_s)
            plan.backward(out_s, out=out_b)
            alg.run(img, out_s)
        if not graph:
            return plan, body
        g = torch.cuda.CUDAGraph()
        body()  # allocate state outside the capture
        torch.cuda.synchronize()
        with torch.cuda.graph(g):
            body()
        return plan, g.replay

    plan, step = build(args.sampler, True)
    units = (c["iters"] + 1) * (plan.fp_samples() + V * c["n_views"])
    stream = torch.cuda.current_stream(dev)
    L = dtvb200._lib.load()
    for _ in range(max(args.warmup, 1)):
        step()
    n0 = L.dtv_launch_count()
    step()
    torch.cuda.synchronize()
    launches = L.dtv_launch_count() - n0  # a replay counts none: count an eager pass
    _, eager = build(args.sampler, False)
    n0 = L.dtv_launch_count()
    eager()
    launches = L.dtv_launch_count() - n0
    with ClockSampler(0) as clk:
        secs = time_steps(step, args.steps, stream)
    _, plain = build("soft", False)
    plain()
    ps = time_steps(plain, args.steps, stream)
    cpu = check = None
    if not args.no_cpu:
        sigma = dtv_params(plan, dev)["sigma"]
        v = tuple(power_norm((64, 64, 64), a, False, device=dev) for a in range(3))
        cpu, ref = fista64_cpu(c, truth[0, 0].double().cpu().numpy(), sigma, v)
        # this library's outputs of the same step (eager, outside the timed region)
        alg = dtvb200.DTVFISTA(plan, c["iters"], sigma=sigma, v=v, t=(1e-3,) * 3, quirk=False)
        s_gpu = plan.forward(truth)
        b_gpu = plan.backward(s_gpu)
        r_gpu = alg.run(torch.zeros(plan.vol_shape(1), device=dev), s_gpu)
        check = {"forward": rel_rmse(s_gpu, ref["sino"]), "backward": rel_rmse(b_gpu, ref["bp"]),
                 "reconstruction": rel_rmse(r_gpu, ref["recon"]), "gate": 1e-3,
                 "how": "relative RMSE of each output of the step against the FP64 oracle's "
                        "run of the same step (its own FP64 projections) at full size"}
    line = {
        "metric": METRIC, "value": units * args.steps / secs / 1e9, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "64^3 x 1 mm, 60 views/360deg, 128x128 det @ 1.0 mm, SOD 500 "
                               "SDD 1000: FP + BP + 20 FISTA-TV iterations",
                   "sampler": args.sampler, "graph": "one CUDA graph per step"},
        "recon_per_s": args.steps / secs,
        "plain_fp32_eager": {"value": units * args.steps / ps / 1e9, "recon_per_s": args.steps / ps,
                             "sampler": "soft"},
        "gpu_launches": launches * args.steps,
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
        "error_vs_fp64": check,
    }
    print(json.dumps(line), flush=True)
    return 0


def fista64_cpu(c, truth_np, sigma, v):
    """The whole 64^3 step (FP, BP, 20 FISTA-DTV iterations) by the FP64
    oracle on all host cores, timed once."""
    import numpy as np
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    ang = np.linspace(0, 360, c["n_views"], endpoint=False)
    og = O.circular_geometry(ang, (c["nx"], c["ny"], c["nz"]), (c["voxel"],) * 3,
                             (c["nu"], c["nv"]), (c["pitch"], c["pitch"]), c["sod"], c["sdd"])
    vol = np.ascontiguousarray(truth_np, dtype=np.float64)
    fp = lambda x: O.forward(og, x).reshape(x.shape[0], 1, *og.sino_shape)  # noqa: E731
    bp = lambda s: O.backward(og, s).reshape(s.shape[0], 1, *og.vol_shape)  # noqa: E731
    t0 = time.perf_counter()
    sino = fp(vol.reshape(1, 1, *vol.shape))
    bsino = bp(sino)
    recon = O.dtvfista_run(fp, bp, np.zeros((1, 1) + og.vol_shape), sino,
                           (c["nx"], c["ny"], c["nz"]), c["iters"], sigma, v, (1e-3,) * 3,
                           quirk=False)
    secs = time.perf_counter() - t0
    units = (c["iters"] + 1) * (O.fp_samples(og) + c["nx"] * c["ny"] * c["nz"] * c["n_views"])
    return ({"value": units / secs / 1e9, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
             "recon_per_s": 1.0 / secs,
             "sample": "the whole step (FP + BP + 20 FISTA-DTV iterations), FP64 oracle, once"},
            {"sino": sino, "bp": bsino, "recon": recon})


def fp64_check_large(dev, sampler, K, iters):
    """Checker leg of the large workload, outside its timed region, on its
    stated downsample: 128^3 x 4 mm with a 256x192 detector at 3.2 mm (the
    field of view of 512^3 x 1 mm, 1024x768 @ 0.8 mm) and 64 views. Relative
    RMSE vs the FP64 oracle of the forward projection (FP32- and BF16-stored
    volume), the FDK backprojection, and the `iters`-iteration DTV
    reconstruction with FP32 and BF16 fbar, corrected every K iterations as
    the timed run."""
    import numpy as np
    import torch

    import dtvb200
    from dtvb200.phantom import ellipsoids
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O

    def rel(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))

    t0 = time.perf_counter()
    ang = np.linspace(0, 360, 64, endpoint=False)
    args = (ang, (128, 128, 128), (4.0,) * 3, (256, 192), (3.2, 3.2), 500.0, 1000.0)
    geo, og = dtvb200.circular(*args), O.circular_geometry(*args)
    truth = ellipsoids((128, 128, 128), seed=CFG["seed"], device=dev)
    plan = dtvb200.Plan(geo, max_batch=1, sampler=sampler, device=dev)
    xplan = dtvb200.Plan(geo, max_batch=1, sampler="exact", device=dev) if K else None
    tn = truth.cpu().numpy()
    ref = O.forward(og, tn).reshape(1, 1, *og.sino_shape)
    out = {"forward_fp32_volume": rel(plan.forward(truth).cpu().numpy(), ref),
           "forward_bf16_volume": rel(plan.forward(truth.to(torch.bfloat16)).cpu().numpy(), ref)}
    sino = torch.from_numpy(ref.astype(np.float32)).to(dev)
    out["backward"] = rel(plan.backward(sino).cpu().numpy(),
                          O.backward(og, ref).reshape(1, 1, *og.vol_shape))
    prm = dtv_params(plan, dev)
    fpo = lambda x: O.forward(og, x).reshape(x.shape[0], 1, *og.sino_shape)  # noqa: E731
    bpo = lambda s: O.backward(og, s).reshape(s.shape[0], 1, *og.vol_shape)  # noqa: E731
    rec = O.dtvcp_run(fpo, bpo, np.zeros((1, 1) + og.vol_shape), ref, (128, 128, 128), iters,
                      prm["sigma"], prm["tau"], prm["mu"], prm["v"], quirk=prm["quirk"])
    for name, dt in (("reconstruction_fp32_fbar", torch.float32),
                     ("reconstruction_bf16_fbar", torch.bfloat16)):
        alg = dtvb200.DTVCP(plan, iters, t_refresh=10, use_graph=True, f_dtype=dt, exact=xplan,
                            correct_every=max(K, 1), **prm)
        out[name] = rel(alg.run(torch.zeros(plan.vol_shape(1), device=dev), sino).cpu().numpy(),
                        rec)
    out.update(gate=1e-3, seconds=time.perf_counter() - t0,
               how=(f"relative RMSE vs the FP64 oracle on the stated downsample: 128^3 x 4 mm, "
                    f"256x192 det @ 3.2 mm, 64 views over 360 deg; {iters} DTV-PDHG iterations "
                    f"from the noiseless projection of the same phantom"))
    return out


def run_large512(args):
    """Large: 512^3 ellipsoid phantom (1 mm voxels), 1024x768 detector at
    0.8 mm pitch, SOD 500 / SDD 1000. One step = the 360-view full-scan forward
    projection plus 50 DTV iterations from the 90-view sparse subset (every
    4th view), FP32-stored and BF16-stored (the volume and fbar in BF16; FP32
    iterates and accumulation)."""
    import numpy as np
    import torch

    import dtvb200
    from dtvb200.phantom import ellipsoids
    dev = torch.device("cuda", 0)
    n, nu, nv, pitch, views, sparse, iters = 512, 1024, 768, 0.8, 360, 90, 50
    ang = np.linspace(0, 360, views, endpoint=False)
    geo = dtvb200.circular(ang, (n, n, n), (1.0,) * 3, (nu, nv), (pitch, pitch), 500.0, 1000.0)
    geo_s = dtvb200.circular(ang[::views // sparse], (n, n, n), (1.0,) * 3, (nu, nv),
                             (pitch, pitch), 500.0, 1000.0)
    truth = ellipsoids((n, n, n), seed=CFG["seed"], device=dev)
    full = dtvb200.Plan(geo, max_batch=1, sampler=args.sampler, device=dev)
    plan = dtvb200.Plan(geo_s, max_batch=1, sampler=args.sampler, device=dev)
    prm = dtv_params(plan, dev, iters=4)
    K = args.correct_every if args.sampler in ("pairs", "tex", "tma") else 0
    corr = dict(exact=dtvb200.Plan(geo_s, max_batch=1, sampler="exact", device=dev) if K else None,
                correct_every=max(K, 1))
    sino_full = torch.empty(full.sino_shape(1), device=dev)
    V = n ** 3
    units = full.fp_samples() + iters * (plan.fp_samples() + V * sparse)
    stream = torch.cuda.current_stream(dev)
    res = {}
    for name, dt in (("fp32", torch.float32), ("bf16", torch.bfloat16)):
        vol = truth.to(dt)
        alg = dtvb200.DTVCP(plan, iters, t_refresh=10, use_graph=True, f_dtype=dt, **corr, **prm)
        img = torch.zeros(plan.vol_shape(1), device=dev)

        def step():
            full.forward(vol, out=sino_full)
            return alg.run(img, sino_full[:, :, ::views // sparse].contiguous())
        for _ in range(max(args.warmup, 1)):
            f = step()
        with ClockSampler(0) as clk:
            secs = time_steps(step, args.steps, stream)
        res[name] = {"secs": secs, "clocks": clk.summary(), "f": step(),
                     "launches": alg.launches_per_run + 2}
    err = float(torch.sqrt(((res["bf16"]["f"] - res["fp32"]["f"]).double() ** 2).mean()
                           / (res["fp32"]["f"].double() ** 2).mean()))
    secs, bf16_secs = res["fp32"]["secs"], res["bf16"]["secs"]
    launches, clocks = res["fp32"]["launches"], res["fp32"]["clocks"]
    del res, full, plan, corr, sino_full
    check = None if args.no_check else fp64_check_large(dev, args.sampler, K, iters)
    line = {
        "metric": METRIC, "value": units * args.steps / secs / 1e9, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "512^3 x 1 mm, 1024x768 det @ 0.8 mm, SOD 500 SDD 1000: 360-view "
                               "full-scan FP + 50 DTV iterations on the 90-view subset",
                   "sampler": args.sampler, "graph": "one CUDA graph per reconstruction",
                   "correction": (f"operators corrected by the exact-weight plan every {K} "
                                  f"iterations" if K else None)},
        "recon_per_s": args.steps / secs,
        "bf16_storage": {"value": units * args.steps / bf16_secs / 1e9,
                         "recon_per_s": args.steps / bf16_secs,
                         "rel_rmse_vs_fp32_storage": err},
        "error_vs_fp64": check,
        "gpu_launches": launches * args.steps,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_peaks(args):
    """The roofline denominators of the projectors and the adjoint, measured on
    this GPU (each rate three times): bilinear texture fetches of 32- and
    64-bit texels from a layered texture, bilinear fetches and gathers from a
    tiled 2-D texture, and 16-byte L2 vector reductions."""
    import torch

    import dtvb200
    L = dtvb200._lib
    torch.cuda.init()
    rates = {
        "bilinear_layered_32bit": [L.measure_texture_fetch_rate(32) for _ in range(3)],
        "bilinear_layered_64bit": [L.measure_texture_fetch_rate(64) for _ in range(3)],
        "bilinear_tiled2d_32bit": [L.measure_texture_gather_rate(0) for _ in range(3)],
        "gather_tiled2d_32bit": [L.measure_texture_gather_rate(1) for _ in range(3)],
        "atomic_v4_contiguous": [L.measure_atomic_v4_rate(72 << 16, 0) for _ in range(3)],
        "atomic_v4_scattered": [L.measure_atomic_v4_rate(72 << 16, 1) for _ in range(3)],
    }
    print(json.dumps({"unit": "per second", "sm_count": torch.cuda.get_device_properties(
        0).multi_processor_count, "rates": rates,
        "projector_concurrency_ms": projector_concurrency()}), flush=True)
    return 0


def projector_concurrency(reps=10):
    """Whether the SM-side samplers add throughput to the texture unit: the
    headline forward projection by the z-pair texture plan, the exact-record
    plan (16-byte loads through L1) and the shared-memory (TMA) plan with no
    tiles on the texture unit, each alone and two at a time on two streams
    (ms per pair of launches; independent units would give the slower one's
    time, a shared one the sum)."""
    import torch

    import dtvb200
    dev = torch.device("cuda", 0)
    c = dict(CFG)
    geo, truth, _ = make_problem(dev, c, c["seed"])
    P = {s: dtvb200.Plan(geo, sampler=s, device=dev) for s in ("pairs", "exact", "tma")}
    P["tma"].set_tuning(dtvb200._lib.DTV_TUNE_FP_TEX_SHARE, 0)
    out = {s: torch.empty(P["pairs"].sino_shape(1), device=dev) for s in P}
    streams = [torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)]
    main = torch.cuda.current_stream(dev)

    def launch(names):
        for st in streams:
            st.wait_stream(main)
        for i, s in enumerate(names):
            with torch.cuda.stream(streams[i]):
                P[s].forward(truth, out=out[s])
        for st in streams:
            main.wait_stream(st)

    def timed(names):
        for _ in range(2):
            launch(names)
        return time_steps(lambda: launch(names), reps, main) / reps * 1e3

    res = {"+".join(v): timed(v) for v in (["pairs"], ["exact"], ["tma"], ["pairs", "exact"],
                                           ["pairs", "tma"], ["pairs", "pairs"])}
    for s in P.values():
        s.close()
    return res


def run_profile(args):
    """N eager iterations of the workload (for ncu): forward projector,
    backprojector and fused updates, one launch each per iteration. With
    --workload large512 the volume is 512^3 and the scan 90 views of 1024x768
    at 0.8 mm (the sparse subset of that workload); --fp-band overrides the
    plan's forward block order (DTV_TUNE_FP_BAND)."""
    import torch

    import dtvb200
    from dtvb200.phantom import poisson_noise
    dev = torch.device("cuda", 0)
    c = dict(CFG)
    if args.small:
        c.update(nx=64, ny=64, nz=64, nu=96, nv=96, n_views=16)
    elif args.workload == "large512":
        c.update(nx=512, ny=512, nz=512, nu=1024, nv=768, pitch=0.8, n_views=90)
    geo, truth, _ = make_problem(dev, c, c["seed"])
    plan = dtvb200.Plan(geo, max_batch=1, sampler=args.sampler, device=dev)
    if args.fp_band is not None:
        plan.set_tuning(dtvb200._lib.DTV_TUNE_FP_BAND, args.fp_band)
    sino = poisson_noise(plan.forward(truth), c["i0"], seed=c["seed"])
    prm = dtv_params(plan, dev)
    K = args.correct_every if args.sampler in ("pairs", "tex", "tma") else 0
    xplan = dtvb200.Plan(geo, max_batch=1, sampler="exact", device=dev) if K else None
    alg = dtvb200.DTVCP(plan, args.profile, t_refresh=10, use_graph=False, exact=xplan,
                        correct_every=max(K, 1),
                        f_dtype=torch.float16 if args.fbar == "f16" else torch.float32, **prm)
    f = alg.run(torch.zeros(plan.vol_shape(1), device=dev), sino)
    torch.cuda.synchronize()
    print(json.dumps({"profile_iterations": args.profile, "sampler": args.sampler,
                      "loss_first_last": [float(alg.losses[0]), float(alg.losses[-1])],
                      "f_abs_sum": float(f.abs().sum())}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--sampler", choices=["soft", "tex", "pairs", "tma"], default="pairs")
    ap.add_argument("--small", action="store_true", help="64^3 smoke-size workload")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--fbar", choices=("f16", "f32"), default="f16",
                    help="storage of DTV's projected iterate fbar (headline workload)")
    ap.add_argument("--correct-every", type=int, default=8, metavar="K",
                    help="refresh the exact-weight correction of a texture-filtered sampler "
                         "every K DTV iterations (0: uncorrected)")
    ap.add_argument("--no-check", action="store_true",
                    help="skip the FP64 error check and the reference-CUDA baseline")
    ap.add_argument("--workload", choices=["sparse_dtv", "batch16", "train", "fista64",
                                           "large512", "peaks"],
                    default="sparse_dtv",
                    help="sparse_dtv: the headline workload; batch16: 16 heterogeneous FISTA "
                         "reconstructions batched into one graph; train: training steps of a "
                         "10-stage unrolled network through the exact adjoint; fista64: 64^3 "
                         "FP + BP + 20 FISTA-TV iterations; large512: 512^3 360-view scan + "
                         "50 DTV iterations on 90 views, FP32 and BF16 storage")
    ap.add_argument("--profile", type=int, default=0, metavar="N",
                    help="profiling run: N eager DTV iterations of the workload, no timing "
                         "(sparse_dtv, or large512's 90-view subset)")
    ap.add_argument("--fp-band", type=int, default=None, metavar="B",
                    help="profiling run: forward block order (0: view by view; B: bands of "
                         "B tile rows)")
    args = ap.parse_args()
    if args.warmup < 3 and not args.small:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        return run_reference(args)
    if args.profile:
        return run_profile(args)
    if args.workload == "batch16":
        return run_batch16(args)
    if args.workload == "train":
        return run_train(args)
    if args.workload == "fista64":
        return run_fista64(args)
    if args.workload == "large512":
        return run_large512(args)
    if args.workload == "peaks":
        return run_peaks(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
