"""CPU tests of the host side: the C-ABI library loads and exports every
declared symbol, the geometry builders agree with the oracle's restatement
of the reference conventions, argument validation raises, and the synthetic
inputs are deterministic. No kernel runs here."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest
import torch

import dtvb200
import oracle as O
from dtvb200 import _lib
from helpers import vector_views

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "dtv_b200.h")


def header_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"DTV_API\s+[\w\s\*]*?\b(dtv_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    syms = header_symbols()
    assert len(syms) >= 25
    L = _lib.load()
    for s in syms:
        assert hasattr(L, s), s
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r"\bT (dtv_\w+)", out))
    assert set(syms) <= exported
    # and the ctypes table binds exactly the declared set
    assert set(_lib.SIGNATURES) == set(syms)


def test_version_and_error_strings():
    L = _lib.load()
    assert L.dtv_version() >= 10000
    assert L.dtv_error_string(0) == b"ok"
    assert L.dtv_error_string(1) == b"invalid argument"
    assert L.dtv_l1ball_workspace_bytes() % 16 == 0
    assert L.dtv_pdhg_workspace_bytes() == 3 * L.dtv_l1ball_workspace_bytes()


def test_standard_builder_matches_oracle_views():
    ang = np.linspace(0, 360, 17, endpoint=False).astype(np.float32)
    g = dtvb200.standard(ang, (32, 30, 12), (40, 20), 700.0, 1100.0)
    og = O.standard_geometry(ang.astype(np.float64), (32, 30, 12), (40, 20), 700.0, 1100.0)
    assert np.abs(g.views - og.views).max() < 1e-9
    s = g.struct
    assert (s.nx, s.ny, s.nz, s.nu, s.nv, s.n_views) == (32, 30, 12, 40, 20, 17)
    assert s.fp_phase == _lib.DTV_PHASE_STANDARD and s.bp_weight_power == 2
    assert abs(s.fp_step - og.og.step) < 1e-7 and abs(s.bp_scale - og.og.bp_scale) < 1e-15
    assert tuple(s.vol_offset) == (0, 0, 0) and tuple(s.det_offset) == (0, 0)


def test_vector_builder_matches_oracle_views():
    pv = vector_views(42, 30.0, 60.0, 1.3, 1.2, 1.0)
    g = dtvb200.vector(pv, (12, 10, 8), (16, 12))
    og = O.vector_geometry(pv, (12, 10, 8), (16, 12))
    assert np.abs(g.views - og.views).max() < 1e-6
    assert g.struct.bp_scale == pytest.approx(og.og.bp_scale)
    assert g.struct.bp_extent_check == 1 and tuple(g.struct.det_offset) == (0.5, 0.5)


def test_circular_builder_matches_oracle_views():
    ang = np.linspace(0, 360, 9, endpoint=False)
    g = dtvb200.circular(ang, (16, 16, 8), (1.0, 1.0, 0.5), (24, 12), (1.2, 1.3), 500, 1000)
    og = O.circular_geometry(ang, (16, 16, 8), (1.0, 1.0, 0.5), (24, 12), (1.2, 1.3), 500, 1000)
    assert np.abs(g.views - og.views).max() < 1e-9
    assert g.struct.fp_step == 0.5 and g.struct.fp_phase == _lib.DTV_PHASE_BOX


@pytest.mark.parametrize("args,msg", [
    (((0, 8, 8), (8, 8), 500, 1000), "volume size"),
    (((8, 8, 8), (8, -1), 500, 1000), "detector size"),
    (((8, 8, 8), (8, 8), 1000, 500), "sid"),
])
def test_builder_validation(args, msg):
    with pytest.raises(dtvb200.DtvError) as e:
        dtvb200.standard([0.0, 90.0], *args)
    assert e.value.code == _lib.DTV_ERR_INVALID
    assert msg in str(e.value)


def test_builder_rejects_degenerate_views():
    pv = vector_views(21, 30.0, 60.0, 1.3, 1.2)
    pv[3, 9:12] = pv[3, 6:9]  # u parallel to v
    with pytest.raises(dtvb200.DtvError, match="parallel"):
        dtvb200.vector(pv, (8, 8, 8), (8, 8))
    pv = vector_views(21, 30.0, 60.0, 1.3, 1.2)
    pv[0, 0] = np.nan
    with pytest.raises(dtvb200.DtvError, match="non-finite"):
        dtvb200.vector(pv, (8, 8, 8), (8, 8))


def test_null_arguments_are_rejected():
    L = _lib.load()
    assert L.dtv_geometry_standard(None, None, None, 0, None, None, 1.0, 2.0) == 1
    assert b"NULL" in L.dtv_last_error_message()
    assert L.dtv_forward(None, None, 0, 1, None, 0, None, 0.0, None, None) == 1
    assert L.dtv_plan_destroy(None) == 0
    assert L.dtv_diff(None, None, None, 1, 0, 0, 0, None) == 1
    assert L.dtv_l1ball(None, None, 0, None, None, None, None) == 1
    assert L.dtv_backward_onto(None, None, 1, None, None, None) == 1
    assert L.dtv_pdhg_forward_refresh(None, None, None, 0, 1, None, 0.0, None, None, None,
                                      None) == 1
    assert L.dtv_backward_refresh(None, None, None, 1, None, None, None) == 1
    assert L.dtv_pdhg_dual_defer(None, None, None, None, None, None, 1, None, None, None, None,
                                 None) == 1
    assert L.dtv_pdhg_primal_defer(None, None, None, None, None, None, None, None, 1, None, None,
                                   None, None) == 1
    assert b"NULL" in L.dtv_last_error_message()


def test_check_input_errors():
    from dtvb200.geometry import check_input
    with pytest.raises(RuntimeError, match="CUDA tensor"):
        check_input(torch.zeros(3), "volume")


def test_phantom_is_seeded_and_bounded():
    from dtvb200.phantom import ellipsoids
    a = ellipsoids((16, 20, 24), seed=3)
    b = ellipsoids((16, 20, 24), seed=3)
    c = ellipsoids((16, 20, 24), seed=4)
    assert a.shape == (1, 1, 16, 20, 24)
    assert torch.equal(a, b) and not torch.equal(a, c)
    assert float(a.min()) >= -2.0 and float(a.max()) <= 10.0 and float(a.abs().sum()) > 0


def test_poisson_noise_is_seeded():
    from dtvb200.phantom import poisson_noise
    s = torch.rand(2, 1, 3, 8, 8) * 50
    a = poisson_noise(s, 1e5, seed=1)
    b = poisson_noise(s, 1e5, seed=1)
    assert torch.equal(a, b)
    assert float((a - s).abs().max()) < 5.0


def test_ramp_kernel_matches_reference_formula():
    from dtvb200.ops import ramp_kernel
    k = ramp_kernel(8).numpy().ravel()
    assert k.size == 9 and k[4] == np.float32(1 / 8)
    assert k[3] == np.float32(-0.5 / np.pi ** 2) and k[2] == 0.0 and k[1] == np.float32(
        -0.5 / (np.pi ** 2 * 9))
