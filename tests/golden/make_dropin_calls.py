"""Record the calls the reference's own layer module makes into its projector
extension, as a fixture for the drop-in test.

Imports the reference's unmodified model/ConeBeamLayers/Standard/
StandardGeometry.py (which reads ./options.yaml through options.py at import
time) from a temporary directory holding a copy of the reference's
options.yaml with the standard-geometry keys set to the "s3" case of
ref_projectors.npz (64 x 64 x 32 volume, 96 x 48 detector, 30 views, SID 1000,
SDD 2000). A recording stand-in named JITStandardGeometry takes the place of
the extension, so every forward/backward call the reference makes - through
ForwardProjection, BackProjection, their autograd backward, StandardGeometry
and StandardGeometryWithFBP - is written down with its exact argument values
and types. The GPU test replays those calls through this library's
JITStandardGeometry and compares them with the reference kernels' outputs.

Runs on a CPU host with the reference tree; the fixture travels, the
reference does not.

Usage: python tests/golden/make_dropin_calls.py [--ref-root DIR] [--out PATH]
(DIR defaults to $DTV_REFERENCE_ROOT, else a `reference` checkout beside this
repository.)
"""
import argparse
import contextlib
import json
import os
import shutil
import sys
import tempfile
import types

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

# the s3 case of ref_projectors.npz
S3 = dict(standardAngleNum=30, standardDetectorSize=[96, 48], standardVolumeSize=[64, 64, 32],
          standardSID=1000, standardSDD=2000)


def default_ref_root():
    return os.environ.get("DTV_REFERENCE_ROOT",
                          os.path.join(os.path.dirname(REPO), "reference"))


def _desc(a):
    if isinstance(a, torch.Tensor):
        return {"tensor": True, "dtype": str(a.dtype).replace("torch.", ""),
                "shape": list(a.shape), "values": a.detach().reshape(-1).tolist()
                if a.numel() <= 64 else None}
    return {"tensor": False, "type": type(a).__name__, "value": a}


@contextlib.contextmanager
def reference_layer(ref_root, projector):
    """Imports the reference's StandardGeometry.py with `projector` as its
    JITStandardGeometry and the s3 geometry in ./options.yaml; yields the
    module and restores sys.modules, sys.path and the working directory."""
    import importlib

    import yaml
    saved = {k: sys.modules.get(k) for k in ("JITStandardGeometry", "options")}
    cwd = os.getcwd()
    tmp = tempfile.mkdtemp(prefix="dropin_")
    try:
        y = yaml.load(open(os.path.join(ref_root, "options.yaml")), yaml.FullLoader)
        y.update(S3)
        with open(os.path.join(tmp, "options.yaml"), "w") as f:
            yaml.safe_dump(y, f)
        sys.modules["JITStandardGeometry"] = projector
        sys.modules.pop("options", None)
        sys.path.insert(0, ref_root)
        os.chdir(tmp)
        yield importlib.import_module("model.ConeBeamLayers.Standard.StandardGeometry")
    finally:
        os.chdir(cwd)
        sys.path.remove(ref_root)
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
        for k in [m for m in sys.modules if m == "model" or m.startswith("model.")]:
            sys.modules.pop(k, None)
        shutil.rmtree(tmp, ignore_errors=True)


def record(ref_root):
    """Returns the list of recorded calls (name + argument descriptions)."""
    calls = []

    def make(name):
        def fn(t, angles, volumeSize, detectorSize, sid, sdd, device):
            calls.append({"fn": name, "input_shape": list(t.shape),
                          "angles": _desc(angles), "volumeSize": _desc(volumeSize),
                          "detectorSize": _desc(detectorSize), "sid": _desc(sid),
                          "sdd": _desc(sdd), "device": _desc(device)})
            X, Y, Z = (int(v) for v in volumeSize.tolist())
            W, H = (int(v) for v in detectorSize.tolist())
            n = angles.numel()
            shape = (t.shape[0], 1, n, H, W) if name == "forward" else (t.shape[0], 1, Z, Y, X)
            return torch.zeros(shape, dtype=torch.float32)
        return fn

    stub = types.ModuleType("JITStandardGeometry")
    stub.forward = make("forward")
    stub.backward = make("backward")
    with reference_layer(ref_root, stub) as sg:
        x = torch.zeros((1, 1, 32, 64, 64), requires_grad=True)
        p = torch.zeros((1, 1, 30, 48, 96))
        sg.ForwardProjection.apply(x).sum().backward()
        sg.BackProjection.apply(p.clone().requires_grad_(True)).sum().backward()
        sg.StandardGeometry()(x.detach(), p)
        sg.StandardGeometryWithFBP()(x.detach(), p)
    return calls


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=default_ref_root())
    ap.add_argument("--out", default=os.path.join(HERE, "dropin_calls.json"))
    a = ap.parse_args()
    calls = record(a.ref_root)
    with open(a.out, "w") as f:
        json.dump({"geometry": S3, "calls": calls}, f, indent=1)
    print("wrote", a.out, len(calls), "calls")
    return 0


if __name__ == "__main__":
    sys.exit(main())
