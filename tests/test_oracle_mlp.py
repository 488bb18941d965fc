"""CPU checks of the guiding network's FP64 oracle (no GPU).

The guiding network has no reference counterpart, so the oracle is pinned by
mathematics: its gradient against central finite differences of its own
loss, the vMF mixture density against numerical integration over the
sphere, and the one-blob encoding against its definition."""
import numpy as np
import pytest

from bajo_b200 import guide
from oracle import oracle


def _batch(rng, n):
    pos = rng.uniform(0.05, 0.95, (n, 3)).astype(np.float32)
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = rng.uniform(0.1, 2.0, n).astype(np.float32)
    return pos, nrm.astype(np.float32), d.astype(np.float32), w


BOX = np.array([0, 0, 0, 1, 1, 1], np.float32)


def test_param_count_matches(lib):
    import ctypes
    n = ctypes.c_uint32(0)
    assert lib.bajo_mlp_param_count(ctypes.byref(n)) == 0
    assert n.value == oracle.mlp_param_count() == guide.N_PARAMS == 14560


def test_one_blob_rows():
    rng = np.random.default_rng(1)
    for _ in range(50):
        p = rng.uniform(-0.2, 1.2, 3)
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        f = oracle.mlp_encode(p, n, BOX)
        # every group is a partition of unity with at most two non-zero bins
        for a in range(3):
            g = f[16 * a:16 * a + 16]
            assert abs(g.sum() - 1.0) < 1e-6 and np.count_nonzero(g) <= 2
        for a in range(2):
            g = f[48 + 8 * a:56 + 8 * a]
            assert abs(g.sum() - 1.0) < 1e-6 and np.count_nonzero(g) <= 2
    # the bin centre of bin k gets the whole blob
    f = oracle.mlp_encode([(3 + 0.5) / 16, 0.5, 0.5], [0, 0, 1], BOX)
    assert f[3] == 1.0


def test_octahedral_hemispheres_differ():
    up = oracle.mlp_encode([0.5] * 3, [0, 0, 1], BOX)[48:]
    down = oracle.mlp_encode([0.5] * 3, [0, 0, -1], BOX)[48:]
    assert not np.allclose(up, down)


def test_vmf_mixture_density_integrates_to_one():
    rng = np.random.default_rng(3)
    # Fibonacci sphere quadrature
    m = 200000
    i = np.arange(m) + 0.5
    z = 1 - 2 * i / m
    phi = np.pi * (1 + 5 ** 0.5) * i
    r = np.sqrt(1 - z * z)
    dirs = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1).astype(np.float32)
    for _ in range(3):
        o = rng.normal(size=20)
        o[3::5] = rng.uniform(-2, 3.5, 4)  # kappa up to ~33: resolved by the grid
        vals = np.array([oracle.vmf_mixture_pdf(o, d) for d in dirs[::20]])
        integral = vals.mean() * 4 * np.pi
        assert abs(integral - 1.0) < 2e-2


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_gradient_matches_finite_differences(seed):
    rng = np.random.default_rng(seed)
    params = guide.init_params(seed).astype(np.float64)
    # perturb biases so every unit sees both ReLU sides
    params += rng.normal(scale=0.05, size=params.size)
    pos, nrm, d, w = _batch(rng, 24)
    g, loss = oracle.mlp_grad(params, pos, nrm, d, w, BOX)
    assert np.isfinite(loss) and loss == pytest.approx(oracle.mlp_loss(params, pos, nrm, d, w, BOX), rel=1e-12)
    # output rows 20..31 of the padded layer carry no gradient
    w4, b4 = 3 * guide.LAYER, 3 * guide.LAYER + 32 * 64
    assert not np.any(g[w4 + 20 * 64:b4]) and not np.any(g[b4 + 20:])
    idx = rng.choice(np.flatnonzero(g), 60, replace=False)
    h = 1e-6
    for k in idx:
        pp, pm = params.copy(), params.copy()
        pp[k] += h
        pm[k] -= h
        fd = (oracle.mlp_loss(pp, pos, nrm, d, w, BOX) - oracle.mlp_loss(pm, pos, nrm, d, w, BOX)) / (2 * h)
        assert fd == pytest.approx(g[k], rel=2e-4, abs=1e-7)
