"""The radix-sort sweep workload at its stated sizes: uniform u32 keys (keys
only and with u32 payloads) and 63-bit Morton keys of points in 32 Gaussian
clusters (sigma 0.02) with u32 payloads, N = 2^16 ... 2^28 in powers of 4.

Bit-exact against the oracle's stable LSD sort where the oracle finishes in
seconds (2^16 - 2^22); at 2^24 - 2^28 the size-independent properties:
sorted, the payloads a permutation that carries every key, stable (equal
keys keep increasing payloads), and keys-only results equal to an
independent library sort of the same keys."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MASK32 = 0xFFFFFFFF


def _keys(kind: str, n: int, seed: int):
    from bajo_b200 import scenes
    if kind == "morton63":
        p = scenes.clustered_points_torch(n, seed=seed, device="cuda")
        k = scenes.morton63_torch(p)
        del p
        return k, 0, 63
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randint(-2**31, 2**31, (n,), dtype=torch.int32, device="cuda", generator=g), 0, 32


def _as_unsigned(k):
    """A new int64 tensor of the unsigned key values."""
    return (k.to(torch.int64) & MASK32) if k.dtype == torch.int32 else k.clone()


@pytest.mark.parametrize("lg", [16, 18, 20, 22])
@pytest.mark.parametrize("kind", ["u32", "morton63"])
def test_sweep_sizes_bit_exact(oracle, kind, lg):
    from bajo_b200 import sort
    n = 1 << lg
    keys, b, e = _keys(kind, n, seed=lg)
    host_keys = keys.cpu().numpy().view(np.uint32 if kind == "u32" else np.uint64).copy()
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    ko = keys.clone()
    ws = sort.onesweep_radix_sort_pairs(keys, vals, begin_bit=b, end_bit=e)
    ws2 = sort.onesweep_radix_sort_keys(ko, begin_bit=b, end_bit=e)
    torch.cuda.synchronize()
    assert ws.status() == 0 and ws2.status() == 0
    ok, ov = oracle.sort_pairs(host_keys, np.arange(n, dtype=np.uint32), b, e)
    dt = np.uint32 if kind == "u32" else np.uint64
    assert np.array_equal(keys.cpu().numpy().view(dt), ok)
    assert np.array_equal(vals.cpu().numpy().view(np.uint32), ov)
    assert np.array_equal(ko.cpu().numpy().view(dt), ok)


@pytest.mark.parametrize("lg", [24, 26, 28])
@pytest.mark.parametrize("kind", ["u32", "morton63"])
def test_sweep_sizes_properties(kind, lg):
    from bajo_b200 import sort
    n = 1 << lg
    keys, b, e = _keys(kind, n, seed=lg)
    orig = _as_unsigned(keys)
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    ws = sort.onesweep_radix_sort_pairs(keys, vals, begin_bit=b, end_bit=e)
    torch.cuda.synchronize()
    assert ws.status() == 0
    sk = _as_unsigned(keys)
    del keys
    assert bool((sk[1:] >= sk[:-1]).all())
    idx = vals.long()
    assert bool((orig[idx] == sk).all())
    seen = torch.zeros(n, dtype=torch.int32, device="cuda")
    seen.index_add_(0, idx, torch.ones_like(vals))
    assert bool((seen == 1).all())
    del seen, idx
    eq = sk[1:] == sk[:-1]
    assert bool((vals[1:][eq] > vals[:-1][eq]).all())
    del eq, vals, sk
    # keys only: equal to an independent library sort of the same keys
    k2 = orig.to(torch.int32) if kind == "u32" else orig.clone()
    ws2 = sort.onesweep_radix_sort_keys(k2, begin_bit=b, end_bit=e)
    torch.cuda.synchronize()
    assert ws2.status() == 0
    lib_sorted = torch.sort(orig).values  # int64 holding non-negative codes
    assert bool((_as_unsigned(k2) == lib_sorted).all())
