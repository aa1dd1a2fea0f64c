"""File formats and datasets of the reference's training and reconstruction
scripts, on top of this package's projectors.

- ``.raw``: headerless little-endian float32 arrays; volumes reshaped to
  (1, 64, 256, 256) and sinograms to (1, 144*21, 128, 80) by default
  (data/simulateLoader.py:17-18, data/realLoader.py:28-33);
- ``.mat``: the per-view projection vectors of the Beijing geometry under the
  key ``projection_matrix``, read as float32 [N, 12]
  (model/ConeBeamLayers/Beijing/BeijingGeometry.py:7-9, data/realLoader.py:40-43).

The datasets return ``(input, projections, label)`` triples as the reference's
do (simulateLoader.py:14-22, :37-48; realLoader.py:26-44), with the forward
projection computed by a :class:`dtvb200.Projector` instead of the
JIT extension.
"""
from __future__ import annotations

import os

import numpy as np
import torch
from torch.utils.data import Dataset

VOLUME_SCALE = (1, 64, 256, 256)
SINO_SCALE = (1, 144 * 21, 128, 80)


def read_raw(path: str, shape, scale: float = 1.0) -> torch.Tensor:
    """A float32 ``.raw`` file as a CPU tensor of ``shape`` times ``scale``."""
    a = np.fromfile(path, dtype="<f4")
    n = int(np.prod(shape))
    if a.size != n:
        raise ValueError(f"{path}: {a.size} float32 values, expected {n} for shape {tuple(shape)}")
    a = a.reshape(shape)
    if scale != 1.0:
        a = a * np.float32(scale)
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32))


def write_raw(path: str, t) -> None:
    """Writes a tensor or array as headerless little-endian float32."""
    a = t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)
    np.ascontiguousarray(a, dtype="<f4").tofile(path)


def read_projection_matrix(path: str) -> np.ndarray:
    """The ``projection_matrix`` entry of a ``.mat`` file as float32 [N, 12]."""
    import scipy.io as sio
    m = np.array(sio.loadmat(path)["projection_matrix"]).astype(np.float32)
    if m.ndim != 2 or m.shape[1] != 12:
        raise ValueError(f"{path}: projection_matrix has shape {m.shape}, expected [N, 12]")
    return np.ascontiguousarray(m)


def write_projection_matrix(path: str, pv) -> None:
    import scipy.io as sio
    sio.savemat(path, {"projection_matrix": np.asarray(pv, dtype=np.float32)})


def _listdir(d):
    return [os.path.join(d, f) for f in sorted(os.listdir(d))]


class SimulatedDataset(Dataset):
    """Simulated256 (simulateLoader.py:7-25): label read from ``dir``,
    projections = FP(label) on ``device``, input = zeros."""

    def __init__(self, dir: str, projector, device, scale=VOLUME_SCALE):
        self.files = _listdir(dir)
        self.projector, self.device, self.scale = projector, torch.device(device), tuple(scale)

    def __len__(self):
        return len(self.files)

    def __getitem__(self, index):
        img = read_raw(self.files[index], self.scale).unsqueeze(0).to(self.device)
        proj = self.projector.fp(img)
        return (torch.zeros_like(img).squeeze(0).cpu(), proj.squeeze(0).cpu(),
                img.squeeze(0).cpu())


class SimulatedInputDataset(Dataset):
    """Simulated256Input (simulateLoader.py:27-51): as SimulatedDataset with the
    network input read from the same file name under ``input_dir``;
    ``amp`` scales both (1000 in Simulated256InputShepp, :53-74)."""

    def __init__(self, dir: str, input_dir: str, projector, device, scale=VOLUME_SCALE,
                 amp: float = 1.0):
        names = sorted(os.listdir(dir))
        self.files = [os.path.join(dir, n) for n in names]
        self.inputs = [os.path.join(input_dir, n) for n in names]
        self.projector, self.device, self.scale = projector, torch.device(device), tuple(scale)
        self.amp = float(amp)

    def __len__(self):
        return len(self.files)

    def __getitem__(self, index):
        img = read_raw(self.files[index], self.scale, self.amp).unsqueeze(0).to(self.device)
        proj = self.projector.fp(img)
        inp = read_raw(self.inputs[index], self.scale, self.amp)
        return inp, proj.squeeze(0).cpu(), img.squeeze(0).cpu()


class RealDataset(Dataset):
    """Real256Input (realLoader.py:9-47): per item ``label``/``input``/``sino``
    ``.raw`` files and a ``matlab`` ``.mat`` of projection vectors, all scaled
    by ``amp`` (6e4) with ReLU on label and input. The reference hands each
    item's projection matrix to the geometry module through a module global
    (:40-43); here it is kept as ``self.parameters`` and passed to
    ``on_geometry`` when given."""

    def __init__(self, dirs, device, scale=VOLUME_SCALE, p_scale=SINO_SCALE, amp: float = 6e4,
                 on_geometry=None):
        self.items = []
        for d in dirs:
            for name in sorted(os.listdir(os.path.join(d, "label"))):
                self.items.append({
                    "label": os.path.join(d, "label", name),
                    "input": os.path.join(d, "input", name),
                    "sino": os.path.join(d, "sino", name),
                    "matlab": os.path.join(d, "matlab", name.replace(".raw", ".mat")),
                })
        self.device, self.scale, self.p_scale = torch.device(device), tuple(scale), tuple(p_scale)
        self.amp = float(amp)
        self.on_geometry = on_geometry
        self.parameters = None

    def __len__(self):
        return len(self.items)

    def __getitem__(self, index):
        it = self.items[index]
        img = torch.relu(read_raw(it["label"], self.scale, self.amp))
        proj = read_raw(it["sino"], self.p_scale, self.amp)
        inp = torch.relu(read_raw(it["input"], self.scale, self.amp))
        self.parameters = torch.from_numpy(read_projection_matrix(it["matlab"]))
        if self.on_geometry is not None:
            self.on_geometry(self.parameters)
        return inp, proj, img
