"""GPU tests of the unrolled network path.

Against the reference's own layer and network modules
(tests/golden/ref_layers.npz, made by make_ref_layers.py with the reference's
BeijingGeometry.py, StandardGeometry.py, DTVSTAnet.py, FISTAnet.py and
LEARN.py, their projector extensions replaced by the FP64 oracle): the Beijing
autograd pair with its (view, plane) permutation and sampleInterval, both
geometry layers and their FBP variants, and DTVNet, FistaNet and LEARN built
under the same seeds (their weights must come out identical), cascade by
cascade and through their gradients. Then: gradients through the matched
adjoint agree with finite differences on 16 random voxels, per-stage
checkpointing changes nothing, BF16 training lowers the loss."""
import os

import numpy as np
import pytest
import torch

import dtvb200
import make_ref_layers as ML
from dtvb200.nets import LEARN, DTVNet, FistaNet, UnrolledPDHG, train
from dtvb200.phantom import ellipsoids
from helpers import rel_rmse

pytestmark = pytest.mark.gpu


def small_problem(cuda, n=32, views=12, batch=2):
    ang = np.linspace(0, 360, views, endpoint=False)
    geo = dtvb200.circular(ang, (n, n, n), (1.0, 1.0, 1.0), (48, 48), (1.5, 1.5), 500.0, 1000.0)
    proj = dtvb200.Projector(geo, max_batch=batch)
    truth = torch.cat([ellipsoids((n, n, n), seed=s, device=cuda) for s in range(batch)])
    sino = proj.fp_soft(truth)
    return proj, truth, sino


def test_finite_differences_through_the_network(cuda):
    torch.manual_seed(0)
    proj, truth, sino = small_problem(cuda)
    net = UnrolledPDHG(proj, stages=3, features=8, lamb=2e-3, tau=1e-2, bf16=False).to(cuda)
    x0 = torch.zeros_like(truth) + 0.1

    def loss(x):
        return float(((net(x, sino).double() - truth.double()) ** 2).sum())

    xg = x0.clone().requires_grad_()
    ((net(xg, sino).double() - truth.double()) ** 2).sum().backward()
    g = xg.grad.flatten().double()
    rng = np.random.default_rng(1)
    idx = rng.choice(x0.numel(), 16, replace=False)
    h = 5e-2
    with torch.no_grad():
        for i in idx:
            e = torch.zeros_like(x0).flatten()
            e[i] = h
            e = e.reshape(x0.shape)
            fd = (loss(x0 + e) - loss(x0 - e)) / (2 * h)
            assert abs(fd - float(g[i])) <= 2e-2 * max(1.0, abs(fd)), (int(i), fd, float(g[i]))


def test_checkpointing_is_transparent(cuda):
    torch.manual_seed(0)
    proj, truth, sino = small_problem(cuda)
    net = UnrolledPDHG(proj, stages=3, features=8, bf16=False).to(cuda)
    x0 = torch.zeros_like(truth)
    grads = []
    for ckpt in (True, False):
        net.checkpoint_stages = ckpt
        net.zero_grad()
        torch.mean((net(x0, sino) - truth) ** 2).backward()
        grads.append(torch.cat([p.grad.flatten() for p in net.parameters()]))
    assert torch.allclose(grads[0], grads[1], rtol=1e-4, atol=1e-7)


def test_bf16_training_lowers_the_loss(cuda):
    torch.manual_seed(0)
    proj, truth, sino = small_problem(cuda)
    net = UnrolledPDHG(proj, stages=4, features=16, lamb=2e-3, tau=1e-3).to(cuda)
    losses = train(net, torch.zeros_like(truth), sino, truth, steps=30, lr=2e-3)
    l = losses.cpu().numpy()
    assert np.all(np.isfinite(l))
    assert l[-5:].mean() < 0.8 * l[:3].mean()


def test_learn_mirror_returns_all_iterates(cuda):
    proj, truth, sino = small_problem(cuda, batch=1)
    net = LEARN(proj, cascades=3).to(cuda)
    out = net(torch.zeros_like(truth[:1]), sino[:1])
    assert len(out) == 4 and out[-1].shape == truth[:1].shape
    assert net.Dual[0] is net.Dual[2]  # weights shared across cascades (LEARN.py:11)


# ------------------------------------------------------- reference layer and net goldens
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_layers.npz")
TOL = 1e-4  # FP32 kernels and cuDNN vs the FP64-projector, FP32-CPU reference run


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.fixture(autouse=True)
def _no_tf32():
    prev = torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32
    torch.backends.cudnn.allow_tf32 = torch.backends.cuda.matmul.allow_tf32 = False
    yield
    torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32 = prev


def _bj_projector(gold):
    X, Y, Z = ML.BJ["beijingVolumeSize"]
    geo = dtvb200.vector(gold["bj_pv"], (X, Y, Z), tuple(ML.BJ["beijingSubDetectorSize"]))
    return dtvb200.Projector(geo, sampler="soft")


def _bj_layer(gold, matched=False):
    return dtvb200.BeijingGeometry(_bj_projector(gold), matched=matched, lamb=10e-3,
                                   sample_interval=ML.BJ["sampleInterval"],
                                   planes=ML.BJ["beijingPlanes"])


def _std_projector():
    S = ML.STD
    ang = np.linspace(0, 360, S["standardAngleNum"], endpoint=False).astype(np.float32)
    geo = dtvb200.standard(ang, S["standardVolumeSize"], S["standardDetectorSize"],
                           S["standardSID"], S["standardSDD"])
    return dtvb200.Projector(geo, sampler="soft")


def _t(gold, key, cuda):
    return torch.from_numpy(gold[key]).to(cuda)


def test_beijing_pair_and_layers_match_reference(cuda, gold):
    proj = _bj_projector(gold)
    P, si = ML.BJ["beijingPlanes"], ML.BJ["sampleInterval"]
    FP, BP = dtvb200.make_functions(proj, False, planes=P, sample_interval=si)
    x, p, r = (_t(gold, k, cuda) for k in ("bj_x", "bj_p", "bj_r"))
    assert rel_rmse(FP.apply(x).cpu().numpy(), gold["bj_fp"]) < 1e-5
    assert rel_rmse(BP.apply(p).cpu().numpy(), gold["bj_bp"]) < 1e-5
    layer = _bj_layer(gold)
    assert rel_rmse(layer(x, p).cpu().numpy(), gold["bj_layer"]) < 1e-5
    xg = x.clone().requires_grad_()
    (layer(xg, p) * r).sum().backward()
    assert rel_rmse(xg.grad.cpu().numpy(), gold["bj_layer_grad"]) < 1e-5
    fbp = dtvb200.BeijingGeometryWithFBP(proj, float(ML.BJ["beijingSDD"]), P,
                                         sample_interval=si).to(cuda)
    assert rel_rmse(fbp(x, p).detach().cpu().numpy(), gold["bj_fbp"]) < 1e-5


def test_standard_layers_match_reference(cuda, gold):
    proj = _std_projector()
    x, p, r = (_t(gold, k, cuda) for k in ("std_x", "std_p", "std_r"))
    layer = dtvb200.StandardGeometry(proj)
    assert rel_rmse(layer(x, p).cpu().numpy(), gold["std_layer"]) < 1e-5
    xg = x.clone().requires_grad_()
    (layer(xg, p) * r).sum().backward()
    assert rel_rmse(xg.grad.cpu().numpy(), gold["std_layer_grad"]) < 1e-5
    fbp = dtvb200.StandardGeometryWithFBP(proj, float(ML.STD["standardSDD"])).to(cuda)
    assert rel_rmse(fbp(x, p).detach().cpu().numpy(), gold["std_fbp"]) < 1e-5


def _build(tag, gold):
    torch.manual_seed(ML.SEEDS[tag])  # as the reference nets were built
    c = ML.CASCADES[tag]
    if tag == "dtvnet":
        return DTVNet(_bj_layer(gold), c)
    if tag == "fistanet":
        return FistaNet(_bj_layer(gold), c)
    return LEARN(_std_projector(), c)


def _same(gold, key, t, rtol):
    t = t.detach().cpu().double().numpy()
    if key in gold.files:
        ref = gold[key]
        assert t.shape == ref.shape, key
        assert rel_rmse(t, ref) <= rtol, (key, rel_rmse(t, ref))
    else:
        s, ref = ML.summary(t), gold[key + "#sum"]
        assert abs(s[1] - ref[1]) <= rtol * ref[1] + 1e-30, (key, s, ref)
        assert abs(s[2] - ref[2]) <= rtol * ref[2] + 1e-30, (key, s, ref)


def _err(gold, key, t):
    """Relative RMSE of a tensor against its golden copy, or against the
    golden checksum (sum of squares and max |.|) of a large one."""
    t = t.detach().cpu().double().numpy()
    if key in gold.files:
        return rel_rmse(t, gold[key])
    s, ref = ML.summary(t), gold[key + "#sum"]
    if ref[1] == 0.0:  # an all-zero gradient (e.g. behind ReLUs that never open)
        return float(np.sqrt(s[1]))
    return max(abs(np.sqrt(s[1]) - np.sqrt(ref[1])) / np.sqrt(ref[1]),
               abs(s[2] - ref[2]) / ref[2])


# Parameter gradients of the CNN blocks: a bias gradient sums the upstream
# gradient over the voxels whose ReLU is open, and CPU vs GPU FP32 arithmetic
# can flip the gates of near-zero pre-activations, which moves the small bias
# gradients of the deepest layers by up to ~3e-3 of their size (measured on a
# B200; the cascade iterates and the image gradient agree to 1e-4).
GRAD_TOL = 1e-2


@pytest.mark.parametrize("tag", ["dtvnet", "fistanet", "learn"])
def test_networks_match_reference(cuda, gold, tag):
    """Same weights as the reference network built under the same seed, then
    every cascade iterate and the gradients of sum(t_C * r) (image and every
    parameter) through the reference pairing."""
    net = _build(tag, gold)
    for k, v in net.state_dict().items():
        _same(gold, f"{tag}_sd_{k}", v, 0.0)
    net = net.to(cuda)
    xk, pk, rk = ("bj_x", "bj_p", "bj_r") if tag != "learn" else ("std_x", "std_p", "std_r")
    img = _t(gold, xk, cuda).requires_grad_()
    t = net(img, _t(gold, pk, cuda))
    assert len(t) == ML.CASCADES[tag] + 1
    for k, tk in enumerate(t):
        assert rel_rmse(tk.detach().cpu().numpy(), gold[f"{tag}_t{k}"]) < TOL, k
    (t[-1] * _t(gold, rk, cuda)).sum().backward()
    assert rel_rmse(img.grad.cpu().numpy(), gold[f"{tag}_grad_image"]) < TOL
    worst = {}
    for k, v in net.named_parameters():
        worst[k] = _err(gold, f"{tag}_grad_{k}", v.grad)
    print(tag, "parameter-gradient errors:", sorted(worst.items(), key=lambda kv: -kv[1])[:8])
    for k, e in worst.items():
        assert e <= GRAD_TOL, (k, e)


def test_reference_checkpoint_loads(cuda, gold):
    """A reference state dict (sparse difference matrices included, as
    DTVSTAnet.py stores them) loads into the mirror."""
    from dtvb200.nets import load_reference_state_dict
    net = _build("dtvnet", gold)
    sd = {k: v.clone() for k, v in net.state_dict().items()}
    sd["dx"] = torch.eye(4).to_sparse()
    other = DTVNet(_bj_layer(gold), ML.CASCADES["dtvnet"])
    load_reference_state_dict(other, sd)
    for k, v in other.state_dict().items():
        assert torch.equal(v, sd[k])


def test_dtvnet_finite_differences_and_checkpointing(cuda, gold):
    """DTVNet on the matched adjoint: the autograd gradient of
    sum((t_C - target)^2) agrees with central differences on 16 random voxels,
    and per-cascade checkpointing leaves every gradient unchanged."""
    torch.manual_seed(3)
    net = DTVNet(_bj_layer(gold, matched=True), cascades=2, features=8).to(cuda)
    x0 = _t(gold, "bj_x", cuda)
    sino = _t(gold, "bj_p", cuda)
    target = torch.rand_like(x0)

    def loss(x):
        return ((net(x, sino)[-1].double() - target.double()) ** 2).sum()

    xg = x0.clone().requires_grad_()
    loss(xg).backward()
    g = xg.grad.flatten().double()
    rng = np.random.default_rng(4)
    h = 1e-2
    with torch.no_grad():
        for i in rng.choice(x0.numel(), 16, replace=False):
            e = torch.zeros_like(x0).flatten()
            e[i] = h
            e = e.reshape(x0.shape)
            fd = float(loss(x0 + e) - loss(x0 - e)) / (2 * h)
            assert abs(fd - float(g[i])) <= 2e-2 * max(1.0, abs(fd)), (int(i), fd, float(g[i]))
    grads = []
    for ckpt in (False, True):
        net.checkpoint_stages = ckpt
        net.zero_grad()
        loss(x0).backward()
        grads.append(torch.cat([p.grad.flatten() for p in net.parameters()]))
    assert torch.allclose(grads[0], grads[1], rtol=1e-4, atol=1e-7)
