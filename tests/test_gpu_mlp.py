"""GPU parity of the guiding network's tensor-core kernels against the FP64
oracle: forward outputs, loss and parameter gradients (mma.sync and tcgen05,
FP16 inputs, FP32 accumulation; tolerances below), Adam against its
definition, and training that learns a known direction field."""
import numpy as np
import pytest
import torch

from bajo_b200 import guide
from oracle import oracle

pytestmark = pytest.mark.gpu

BOX = np.array([0, 0, 0, 1, 1, 1], np.float32)


def _batch(rng, n, scale=1.0):
    pos = rng.uniform(-0.05, 1.05, (n, 3)).astype(np.float32)  # a few outside the box: clamped bins
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = (rng.uniform(0.1, 2.0, n) * scale).astype(np.float32)
    return pos, nrm.astype(np.float32), d.astype(np.float32), w


def _dev(*arrays):
    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]


def _net(seed):
    p = guide.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    p = p + rng.normal(scale=0.05, size=p.size).astype(np.float32)  # biases off zero
    p[3 * guide.LAYER + 20 * 64:3 * guide.LAYER + 32 * 64] = 0
    p[3 * guide.LAYER + 32 * 64 + 20:] = 0
    net = guide.GuideNetwork("cuda", params=p)
    return net, net.params16.double().cpu().numpy()


@pytest.mark.parametrize("n", [1, 127, 1000, 40000])
def test_forward_matches_oracle(n):
    rng = np.random.default_rng(n)
    net, p64 = _net(1)
    pos, nrm, _, _ = _batch(rng, n)
    box = torch.from_numpy(BOX).cuda()
    out = net.forward(*_dev(pos, nrm), box).cpu().numpy()
    ref = oracle.mlp_forward(p64, pos, nrm, BOX)
    # FP16 features / activations with FP32 accumulation: absolute error
    # within 1e-2 + 1e-2 * |ref|
    err = np.abs(out - ref)
    assert np.all(err <= 1e-2 + 1e-2 * np.abs(ref)), err.max()


@pytest.mark.parametrize("n", [1, 127, 128, 129, 1000, 40000, 300_001])
def test_tensor_memory_forward(n):
    """The tcgen05 forward: the oracle's tolerance, and the mma.sync forward's
    outputs up to FP32 accumulation order."""
    rng = np.random.default_rng(n + 7)
    net, p64 = _net(2)
    pos, nrm, _, _ = _batch(rng, n)
    box = torch.from_numpy(BOX).cuda()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    dp, dn = _dev(pos, nrm)
    out = net.forward(dp, dn, box, tensor_memory=True, status=status)
    base = net.forward(dp, dn, box)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    out, base = out.cpu().numpy(), base.cpu().numpy()
    assert np.all(np.isfinite(out))
    if n <= 40000:
        ref = oracle.mlp_forward(p64, pos, nrm, BOX)
        err = np.abs(out - ref)
        assert np.all(err <= 1e-2 + 1e-2 * np.abs(ref)), err.max()
    # both kernels round every activation to FP16 the same way; only the FP32
    # sums' order differs, which can flip an FP16 rounding of a hidden unit
    assert np.abs(out - base).max() <= 5e-3 + 5e-3 * np.abs(base).max()


@pytest.mark.parametrize("tensor_memory", [True, False])
@pytest.mark.parametrize("n", [1, 200, 3000])
def test_gradient_matches_oracle(n, tensor_memory):
    rng = np.random.default_rng(7 + n)
    net, p64 = _net(2)
    pos, nrm, d, w = _batch(rng, n)
    box = torch.from_numpy(BOX).cuda()
    g, loss = net.gradient(*_dev(pos, nrm, d, w), box, tensor_memory=tensor_memory)
    torch.cuda.synchronize()
    assert int(net.status.item()) == 0
    g = g.double().cpu().numpy()
    gref, lref = oracle.mlp_grad(p64, pos, nrm, d, w, BOX)
    assert float(loss.item()) == pytest.approx(lref, rel=1e-2, abs=1e-2)
    # relative L2 error of the whole gradient and of each layer's weights
    assert np.linalg.norm(g - gref) <= 3e-2 * np.linalg.norm(gref)
    for wo, bo, rows, cols in guide.offsets():
        a, b = g[wo:wo + rows * cols], gref[wo:wo + rows * cols]
        assert np.linalg.norm(a - b) <= 5e-2 * np.linalg.norm(b) + 1e-6
        a, b = g[bo:bo + rows], gref[bo:bo + rows]
        assert np.linalg.norm(a - b) <= 5e-2 * np.linalg.norm(b) + 1e-6
    # padded output rows never receive gradient
    w4, b4 = 3 * guide.LAYER, 3 * guide.LAYER + 32 * 64
    assert not np.any(g[w4 + 20 * 64:b4]) and not np.any(g[b4 + 20:])


@pytest.mark.parametrize("n", [127, 128, 129, 40000, 200003])
def test_gradient_kernels_agree(n):
    """The tcgen05 gradient (weight gradients accumulated in tensor memory
    over several tiles per CTA at the larger sizes) against the mma.sync one:
    the same FP16 operands, FP32 sums in another order."""
    rng = np.random.default_rng(11 + n)
    net, _ = _net(5)
    pos, nrm, d, w = _batch(rng, n)
    box = torch.from_numpy(BOX).cuda()
    args = _dev(pos, nrm, d, w)
    g_tc, l_tc = net.gradient(*args, box, tensor_memory=True)
    g_tc, l_tc = g_tc.clone(), float(l_tc.item())
    g_mma, l_mma = net.gradient(*args, box, tensor_memory=False)
    torch.cuda.synchronize()
    assert int(net.status.item()) == 0
    g_tc, g_mma = g_tc.double().cpu().numpy(), g_mma.double().cpu().numpy()
    assert np.all(np.isfinite(g_tc))
    assert l_tc == pytest.approx(float(l_mma.item()), rel=1e-4)
    for wo, bo, rows, cols in guide.offsets():
        a, b = g_tc[wo:wo + rows * cols], g_mma[wo:wo + rows * cols]
        assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b) + 1e-6
        a, b = g_tc[bo:bo + rows], g_mma[bo:bo + rows]
        assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b) + 1e-6


@pytest.mark.parametrize("tensor_memory", [True, False])
def test_gradient_of_empty_batch_is_zero(tensor_memory):
    net, _ = _net(3)
    box = torch.from_numpy(BOX).cuda()
    e = torch.empty(0, dtype=torch.float32, device="cuda")
    net.grad_buf.fill_(1.0)
    g, loss = net.gradient(e, e, e, e, box, tensor_memory=tensor_memory)
    assert not torch.any(g) and float(loss.item()) == 0.0


def test_adam_matches_definition():
    net, _ = _net(4)
    p0 = net.params32.double().cpu().numpy()
    rng = np.random.default_rng(5)
    m = np.zeros_like(p0)
    v = np.zeros_like(p0)
    p = p0.copy()
    pad = np.zeros(p.size, bool)
    pad[3 * guide.LAYER + 20 * 64:3 * guide.LAYER + 32 * 64] = True
    pad[3 * guide.LAYER + 32 * 64 + 20:] = True
    for step in range(1, 4):
        g = rng.normal(size=p.size)
        net.grad_buf.copy_(torch.from_numpy(g.astype(np.float32)))
        net.adam(lr=1e-2, grad_scale=0.5)
        gs = g.astype(np.float32).astype(np.float64) * 0.5
        m = 0.9 * m + 0.1 * gs
        v = 0.999 * v + 0.001 * gs * gs
        p = p - 1e-2 * (m / (1 - 0.9 ** step)) / (np.sqrt(v / (1 - 0.999 ** step)) + 1e-8)
        p[pad] = 0
    got = net.params32.double().cpu().numpy()
    assert np.allclose(got, p, rtol=1e-5, atol=1e-6)
    assert np.array_equal(net.params16.cpu().numpy(), net.params32.half().cpu().numpy())


def _vmf_sample(rng, mu, kappa):
    """Directions from vMF(mu, kappa) rows (Jakob 2012)."""
    n = mu.shape[0]
    u = rng.random(n)
    w = 1 + np.log(u + (1 - u) * np.exp(-2 * kappa)) / kappa
    phi = 2 * np.pi * rng.random(n)
    st = np.sqrt(np.maximum(0, 1 - w * w))
    # basis around mu
    a = np.where(np.abs(mu[:, 0:1]) > 0.9, np.array([[0, 1, 0]]), np.array([[1, 0, 0]]))
    t1 = np.cross(mu, a)
    t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
    t2 = np.cross(mu, t1)
    d = t1 * (st * np.cos(phi))[:, None] + t2 * (st * np.sin(phi))[:, None] + mu * w[:, None]
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def test_training_learns_a_direction_field():
    """Directions drawn from vMF(normalize(p - centre), 20): Adam on the GPU
    gradients must bring the mean NLL from the broad initial mixture (about
    log 4 pi = 2.5) close to the field's entropy (about -0.16)."""
    rng = np.random.default_rng(11)
    n = 1 << 14
    pos = rng.uniform(0.02, 0.98, (n, 3))
    mu = pos - 0.5
    mu /= np.linalg.norm(mu, axis=1, keepdims=True)
    d = _vmf_sample(rng, mu, 20.0)
    nrm = np.tile([[0.0, 1.0, 0.0]], (n, 1))
    w = np.ones(n)
    P, N, D, W = _dev(pos.astype(np.float32), nrm.astype(np.float32), d.astype(np.float32), w.astype(np.float32))
    box = torch.from_numpy(BOX).cuda()
    net = guide.GuideNetwork("cuda", seed=0)
    _, loss0 = net.gradient(P, N, D, W, box)
    first = float(loss0.item()) / n
    for _ in range(400):
        net.gradient(P, N, D, W, box)
        net.adam(lr=1e-2, grad_scale=1.0 / n)
    _, loss = net.gradient(P, N, D, W, box)
    last = float(loss.item()) / n
    assert first > 1.5 and last < 0.6, (first, last)
    # the oracle agrees on the trained network's loss
    ref = oracle.mlp_loss(net.params16.double().cpu().numpy(), pos[:2000].astype(np.float32), nrm[:2000],
                          d[:2000], w[:2000], BOX) / 2000
    _, l2 = net.gradient(P[:2000], N[:2000], D[:2000], W[:2000], box)
    assert float(l2.item()) / 2000 == pytest.approx(ref, abs=2e-2)


def test_checkpoint_resumes_training_exactly(tmp_path):
    """save() / load() keep the whole training state: after reloading, the
    same gradient gives the same Adam step, bit for bit."""
    rng = np.random.default_rng(5)
    n = 4096
    pos, nrm, d, w = _batch(rng, n)
    P, N, D, W = _dev(pos, nrm, d, w)
    box = torch.from_numpy(BOX).cuda()
    a = guide.GuideNetwork("cuda", seed=3)
    for _ in range(25):
        a.gradient(P, N, D, W, box)
        a.adam(lr=1e-2, grad_scale=1.0 / n)
    path = str(tmp_path / "guide.npz")
    a.save(path)
    b = guide.GuideNetwork.load(path)
    assert b.step == a.step == 25
    for name in ("params32", "params16", "adam_m", "adam_v"):
        assert torch.equal(getattr(a, name), getattr(b, name)), name
    a.gradient(P, N, D, W, box)
    b.grad_buf.copy_(a.grad_buf)  # one gradient for both (its atomics may sum in any order)
    a.adam(lr=1e-2, grad_scale=1.0 / n)
    b.adam(lr=1e-2, grad_scale=1.0 / n)
    torch.cuda.synchronize()
    assert torch.equal(a.params32, b.params32) and torch.equal(a.params16, b.params16)
    assert torch.equal(a.adam_m, b.adam_m) and torch.equal(a.adam_v, b.adam_v)


def test_checkpoint_of_another_network_is_refused(tmp_path):
    path = str(tmp_path / "bad.npz")
    np.savez(path, params32=np.zeros(10, np.float32), params16=np.zeros(10, np.float16),
             adam_m=np.zeros(10, np.float32), adam_v=np.zeros(10, np.float32), step=np.int64(0), n_params=np.int64(10))
    with pytest.raises(ValueError):
        guide.GuideNetwork.load(path)


def test_guide_train_matches_gradient_and_adam_steps():
    """bajo_guide_train (one gradient memset per call, Adam clearing the
    gradient and loss between steps) against explicit tcgen05 gradient +
    Adam steps over the same cyclic record batches."""
    rng = np.random.default_rng(21)
    count, batch, steps = 5000, 2048, 5
    pos, nrm, d, w = _batch(rng, count)
    box = torch.from_numpy(BOX).cuda()
    rec = guide.GuideRecords(8192)
    for name, arr in zip(("pos", "nrm", "dir", "weight"), (pos, nrm, d, w)):
        o = rec._off[name] // 4
        rec.buffer.view(torch.float32)[o:o + arr.size] = torch.from_numpy(arr.reshape(-1)).cuda()
    rec.buffer[:4].view(torch.int32)[0] = count
    a = guide.GuideNetwork("cuda", seed=6)
    b = guide.GuideNetwork("cuda", seed=6)
    a.train_records(rec, box, batch, steps, lr=1e-2)
    for s in range(steps):
        idx = (s * batch + np.arange(batch)) % count
        P, N, D, W = _dev(pos[idx], nrm[idx], d[idx], w[idx])
        b.gradient(P, N, D, W, box)
        b.adam(lr=1e-2, grad_scale=1.0 / batch)
    torch.cuda.synchronize()
    assert a.step == b.step == steps
    assert int(a.status.item()) == 0
    pa, pb = a.params32.double().cpu().numpy(), b.params32.double().cpu().numpy()
    # atomics sum in any order, so the two gradients differ by FP32 rounding;
    # Adam's first steps move every parameter by about lr whatever the
    # gradient's size, so a gradient within rounding of zero may step either
    # way: a handful of parameters may differ by up to 2 lr per step
    diff = np.abs(pa - pb)
    assert np.mean(diff > 1e-4) < 1e-3 and diff.max() <= 2e-2 * steps, (np.mean(diff > 1e-4), diff.max())
    assert float(a.loss_buf.item()) == pytest.approx(float(b.loss_buf.item()), rel=1e-3)
    ga, gb = a.grad_buf.double().cpu().numpy(), b.grad_buf.double().cpu().numpy()
    assert np.linalg.norm(ga - gb) <= 1e-3 * np.linalg.norm(gb)
