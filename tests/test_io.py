"""CPU tests of the reference's file formats (.raw float32 arrays, .mat
projection vectors) and of the datasets built on them, with a stand-in
projector (the datasets only call ``fp``)."""
import os

import numpy as np
import pytest
import torch

from dtvb200 import io


class _SumProjector:
    """fp: sum along z, standing in for the forward projector."""

    def fp(self, x):
        return x.sum(dim=2, keepdim=True)


def test_raw_round_trip_and_size_check(tmp_path):
    a = np.random.default_rng(0).random((1, 4, 6, 5)).astype(np.float32)
    p = str(tmp_path / "v.raw")
    io.write_raw(p, torch.from_numpy(a))
    assert os.path.getsize(p) == a.size * 4
    assert np.array_equal(io.read_raw(p, a.shape).numpy(), a)
    assert np.allclose(io.read_raw(p, a.shape, 1000).numpy(), a * 1000)
    with pytest.raises(ValueError):
        io.read_raw(p, (1, 4, 6, 6))


def test_projection_matrix_round_trip(tmp_path):
    pv = np.random.default_rng(1).random((7, 12)).astype(np.float32)
    p = str(tmp_path / "m.mat")
    io.write_projection_matrix(p, pv)
    assert np.array_equal(io.read_projection_matrix(p), pv)
    io.write_projection_matrix(p, pv[:, :10])
    with pytest.raises(ValueError):
        io.read_projection_matrix(p)


def test_simulated_datasets(tmp_path):
    rng = np.random.default_rng(2)
    shape = (1, 3, 4, 5)
    (tmp_path / "label").mkdir()
    (tmp_path / "input").mkdir()
    vols = {}
    for name in ("b.raw", "a.raw"):
        vols[name] = rng.random(shape).astype(np.float32)
        io.write_raw(str(tmp_path / "label" / name), vols[name])
        io.write_raw(str(tmp_path / "input" / name), vols[name] * 0.5)
    ds = io.SimulatedDataset(str(tmp_path / "label"), _SumProjector(), "cpu", scale=shape)
    assert len(ds) == 2
    inp, proj, img = ds[0]  # sorted: a.raw
    assert np.array_equal(img.numpy(), vols["a.raw"])
    assert float(inp.abs().sum()) == 0.0
    assert np.allclose(proj.numpy(), vols["a.raw"].sum(axis=1, keepdims=True))
    ds2 = io.SimulatedInputDataset(str(tmp_path / "label"), str(tmp_path / "input"),
                                   _SumProjector(), "cpu", scale=shape, amp=1000)
    inp, proj, img = ds2[1]
    assert np.allclose(img.numpy(), vols["b.raw"] * 1000)
    assert np.allclose(inp.numpy(), vols["b.raw"] * 500)


def test_real_dataset(tmp_path):
    rng = np.random.default_rng(3)
    shape, pshape = (1, 2, 3, 4), (1, 6, 3, 2)
    d = tmp_path / "scan"
    for sub in ("label", "input", "sino", "matlab"):
        (d / sub).mkdir(parents=True)
    lab = rng.standard_normal(shape).astype(np.float32)
    io.write_raw(str(d / "label" / "x.raw"), lab)
    io.write_raw(str(d / "input" / "x.raw"), lab * 2)
    sino = rng.random(pshape).astype(np.float32)
    io.write_raw(str(d / "sino" / "x.raw"), sino)
    pv = rng.random((6, 12)).astype(np.float32)
    io.write_projection_matrix(str(d / "matlab" / "x.mat"), pv)
    seen = []
    ds = io.RealDataset([str(d)], "cpu", scale=shape, p_scale=pshape, amp=2.0,
                        on_geometry=seen.append)
    inp, proj, img = ds[0]
    assert np.allclose(img.numpy(), np.maximum(lab * 2, 0))
    assert np.allclose(inp.numpy(), np.maximum(lab * 4, 0))
    assert np.allclose(proj.numpy(), sino * 2)
    assert np.array_equal(ds.parameters.numpy(), pv) and len(seen) == 1
