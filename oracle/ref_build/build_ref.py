"""Build the reference projector extensions from their unmodified sources.

Test infrastructure for the parity pin. It compiles, where they lie,
  model/ConeBeamLayers/Standard/plug/{jit.cpp,kernel/forwardKernel.cu,kernel/backwardKernel.cu}
  model/ConeBeamLayers/Beijing/plug/{jit.cpp,kernel/forwardKernel.cu,kernel/backwardKernel.cu}
with ``texref_compat.h`` force-included (the sources use texture references,
which CUDA 12 removed), into torch extensions ``JITStandardGeometry`` and
``JITBeijingGeometry`` under ``oracle/_ref/``. Nothing is copied from the
reference tree; build products go only to ``oracle/_ref/``.

Usage: python oracle/ref_build/build_ref.py [--ref-root DIR]
"""
import argparse
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(REPO, "oracle", "_ref")


def build(ref_root: str, verbose: bool = False) -> list:
    from torch.utils import cpp_extension

    shim = os.path.join(HERE, "texref_compat.h")
    built = []
    for variant, mod in (("Standard", "JITStandardGeometry"), ("Beijing", "JITBeijingGeometry")):
        plug = os.path.join(ref_root, "model", "ConeBeamLayers", variant, "plug")
        srcs = [os.path.join(plug, "jit.cpp"),
                os.path.join(plug, "kernel", "forwardKernel.cu"),
                os.path.join(plug, "kernel", "backwardKernel.cu")]
        if not all(os.path.exists(s) for s in srcs):
            raise FileNotFoundError(f"reference sources missing under {plug}")
        bdir = os.path.join(OUT, "build_" + mod)
        os.makedirs(bdir, exist_ok=True)
        cpp_extension.load(
            name=mod,
            sources=srcs,
            extra_cflags=["-O2", "-w"],
            extra_cuda_cflags=["-O3", "-include", shim, "-w",
                               "-gencode", "arch=compute_100a,code=sm_100a"],
            build_directory=bdir,
            verbose=verbose,
            with_cuda=True,
        )
        so = os.path.join(bdir, mod + ".so")
        dst = os.path.join(OUT, mod + ".so")
        shutil.copy2(so, dst)
        built.append(dst)
    return built


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=os.environ.get(
        "DTV_REFERENCE_ROOT", os.path.join(os.path.dirname(REPO), "reference")),
        help="reference checkout (default: $DTV_REFERENCE_ROOT, else ../reference beside "
             "this repository)")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0a")
    for p in build(a.ref_root, a.verbose):
        print("built", p)
    sys.exit(0)
