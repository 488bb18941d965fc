"""GPU parity of the onesweep sort against the oracle (bit-exact), the
reference's sort KATs, and size-independent properties at full sizes."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def to_dev(a: np.ndarray):
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32).copy()).cuda()
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64).copy()).cuda()
    raise TypeError(a.dtype)


def to_host(t, dtype):
    return t.cpu().numpy().view(dtype)


def gpu_sort(keys: np.ndarray, vals: np.ndarray | None, begin=0, end=None):
    from bajo_b200 import sort
    k = to_dev(keys)
    v = None if vals is None else to_dev(vals)
    ws = sort.onesweep_radix_sort_pairs(k, v, begin_bit=begin, end_bit=end) if v is not None else \
        sort.onesweep_radix_sort_keys(k, begin_bit=begin, end_bit=end)
    torch.cuda.synchronize()
    assert ws.status() == 0
    return to_host(k, keys.dtype), (None if v is None else to_host(v, np.uint32))


SIZES = [1, 2, 3, 100, 5631, 5632, 5633, 7679, 7680, 7681, 65536, 262144, 1 << 20]


@pytest.mark.parametrize("n", SIZES)
def test_u32_pairs_and_keys_match_oracle(oracle, n):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    k, v = gpu_sort(keys, vals)
    ok, ov = oracle.sort_pairs(keys, vals)
    assert np.array_equal(k, ok) and np.array_equal(v, ov)
    k2, _ = gpu_sort(keys, None)
    assert np.array_equal(k2, ok)


@pytest.mark.parametrize("n", SIZES)
def test_u64_pairs_match_oracle(oracle, n):
    from bajo_b200 import scenes
    rng = np.random.default_rng(n + 1)
    # clustered Morton keys in the high word, index tie-break material in the low word
    p = scenes.clustered_points(n, seed=n)
    codes = np.array([oracle.morton3(*xyz) for xyz in p[: min(n, 4096)]], np.uint64)
    codes = np.resize(codes, n)
    keys = (codes << np.uint64(32)) | rng.integers(0, 2**32, size=n, dtype=np.uint64)
    vals = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    k, v = gpu_sort(keys, vals)
    ok, ov = oracle.sort_pairs(keys, vals)
    assert np.array_equal(k, ok) and np.array_equal(v, ov)
    k2, _ = gpu_sort(keys, None)
    assert np.array_equal(k2, ok)


@pytest.mark.parametrize("begin,end", [(0, 8), (0, 24), (8, 32), (3, 29), (0, 0)])
def test_u32_bit_ranges(oracle, begin, end):
    n = 50_000
    rng = np.random.default_rng(begin * 100 + end)
    keys = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    k, v = gpu_sort(keys, vals, begin, end)
    ok, ov = oracle.sort_pairs(keys, vals, begin, end)
    assert np.array_equal(k, ok) and np.array_equal(v, ov)


@pytest.mark.parametrize("begin,end", [(0, 30), (0, 44), (32, 64), (0, 40)])
def test_u64_bit_ranges(oracle, begin, end):
    n = 70_000
    rng = np.random.default_rng(end)
    keys = rng.integers(0, 2**63, size=n, dtype=np.uint64) * np.uint64(2) + np.uint64(1)
    vals = np.arange(n, dtype=np.uint32)
    k, v = gpu_sort(keys, vals, begin, end)
    ok, ov = oracle.sort_pairs(keys, vals, begin, end)
    assert np.array_equal(k, ok) and np.array_equal(v, ov)


def test_reference_sort_kats(golden_dir):
    """test/sort/test_onesweep.mojo:18-207 and test_radix_sort.mojo:316-344."""
    g = json.load(open(os.path.join(golden_dir, "sort_kats.json")))
    n = g["hist_u32"]["n"]
    i = np.arange(n, dtype=np.uint64)
    keys = (((i * 13) ^ (i << 16) ^ (i >> 3)) & 0xFFFFFFFF).astype(np.uint32)
    _, v = gpu_sort(keys, np.arange(n, dtype=np.uint32))
    assert _sha(v.astype("<u4")) == g["hist_u32"]["perm_sha256"]
    n = g["pass_u32"]["n"]
    i = np.arange(n, dtype=np.uint64)
    keys = (((i * 17) ^ (i << 13) ^ (i >> 5)) & 0xFFFFFFFF).astype(np.uint32)
    _, v = gpu_sort(keys, np.arange(n, dtype=np.uint32), 0, 8)
    assert _sha(v.astype("<u4")) == g["pass_u32"]["perm_sha256"]
    n = g["composite_u64"]["n"]
    i = np.arange(n, dtype=np.uint64)
    seg = (i * 7) % 19
    mort = ((i * 2654435761) & 0xFFFFFFFF) ^ ((i << 11) & 0xFFFFFFFF) ^ (i >> 3)
    keys = ((seg << 32) | (mort & 0xFFFFFFFF)).astype(np.uint64)
    k, v = gpu_sort(keys, np.arange(n, dtype=np.uint32))
    assert _sha(v.astype("<u4")) == g["composite_u64"]["perm_sha256"]
    assert np.array_equal(k, keys[v])


@pytest.mark.parametrize("n,kind", [(1 << 24, "u32"), (1 << 26, "u32"), (1 << 24, "u64"), (1 << 26, "u64")])
def test_full_size_properties(n, kind):
    """Sortedness, payload consistency and permutation at full sweep sizes."""
    from bajo_b200 import sort
    g = torch.Generator(device="cuda").manual_seed(n)
    if kind == "u32":
        keys = torch.randint(-2**31, 2**31, (n,), dtype=torch.int32, device="cuda", generator=g)
        ukeys = keys.to(torch.int64) & 0xFFFFFFFF
    else:
        keys = torch.randint(-2**63, 2**63 - 1, (n,), dtype=torch.int64, device="cuda", generator=g)
        keys = keys & 0x0FFFFFFFFFFFFFFF  # 60 live bits, non-negative as int64
        ukeys = keys
    orig = ukeys.clone()
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    ws = sort.onesweep_radix_sort_pairs(keys, vals)
    torch.cuda.synchronize()
    assert ws.status() == 0
    sk = (keys.to(torch.int64) & 0xFFFFFFFF) if kind == "u32" else keys
    assert bool((sk[1:] >= sk[:-1]).all())
    assert bool((orig[vals.long()] == sk).all())
    seen = torch.zeros(n, dtype=torch.int32, device="cuda")
    seen.index_add_(0, vals.long(), torch.ones_like(vals))
    assert bool((seen == 1).all())
    # stability: equal keys keep increasing payloads
    eq = sk[1:] == sk[:-1]
    assert bool((vals[1:][eq] > vals[:-1][eq]).all())


@pytest.mark.parametrize("kind,variant", [("u32", v) for v in range(7)] + [("u64", v) for v in (0, 1, 2, 3, 5, 6)])
def test_every_tile_variant_matches_oracle(oracle, variant, kind):
    """Each compiled tile shape the autotuner may pick sorts exactly (the
    early-count passes: 32-bit variants 4-6, 64-bit variants 5-6)."""
    from bajo_b200 import _lib
    L = _lib.load()
    kb = 4 if kind == "u32" else 8
    rng = np.random.default_rng(variant)
    try:
        for n in (1000, 70_001, 300_000):
            lg = int(np.ceil(np.log2(n)))
            assert L.bajo_sort_tuning_set(kb, 1, lg, variant) == _lib.OK
            assert L.bajo_sort_tuning_set(kb, 0, lg, variant) == _lib.OK
            if kb == 4:
                keys = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
            else:
                keys = rng.integers(0, 2**62, size=n, dtype=np.uint64)
            keys[: n // 4] = keys[0]  # long runs of equal keys
            vals = np.arange(n, dtype=np.uint32)
            k, v = gpu_sort(keys, vals)
            ok, ov = oracle.sort_pairs(keys, vals)
            assert np.array_equal(k, ok) and np.array_equal(v, ov)
            k2, _ = gpu_sort(keys, None)
            assert np.array_equal(k2, ok)
    finally:
        for lg in range(33):
            L.bajo_sort_tuning_set(kb, 1, lg, -1)
            L.bajo_sort_tuning_set(kb, 0, lg, -1)


@pytest.mark.parametrize("bits", [(0, 30), (0, 44), (0, 64), (5, 37), (32, 40)])
def test_wide_digit_variant_matches_oracle(oracle, bits):
    """Variant 4 of the 64-bit keys sorts 10-bit digits (passes of
    [begin, begin + 10), ... with a shorter last pass); any bit range, pairs
    and keys only, bit-exact with the oracle and stable."""
    from bajo_b200 import _lib
    L = _lib.load()
    begin, end = bits
    rng = np.random.default_rng(begin * 100 + end)
    try:
        for n in (1, 2, 1000, 1025, 70_001, 262_144):
            lg = int(np.ceil(np.log2(max(n, 2))))
            assert L.bajo_sort_tuning_set(8, 1, lg, 4) == _lib.OK
            assert L.bajo_sort_tuning_set(8, 0, lg, 4) == _lib.OK
            keys = rng.integers(0, 2**63, size=n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=n).astype(np.uint64)
            keys[: n // 4] = keys[0]  # long runs of equal keys
            vals = np.arange(n, dtype=np.uint32)
            k, v = gpu_sort(keys, vals, begin, end)
            ok, ov = oracle.sort_pairs(keys, vals, begin, end)
            assert np.array_equal(k, ok) and np.array_equal(v, ov)
            k2, _ = gpu_sort(keys, None, begin, end)
            assert np.array_equal(k2, ok)
    finally:
        for lg in range(33):
            L.bajo_sort_tuning_set(8, 1, lg, -1)
            L.bajo_sort_tuning_set(8, 0, lg, -1)


def test_wide_digit_variant_limits():
    from bajo_b200 import _lib
    L = _lib.load()
    assert L.bajo_sort_tuning_set(4, 1, 16, _lib.SORT_VARIANTS_U32) == _lib.ERR_INVALID_ARGUMENT  # 32-bit: 7
    assert L.bajo_sort_tuning_set(8, 1, 16, _lib.SORT_VARIANTS_U64) == _lib.ERR_INVALID_ARGUMENT  # 64-bit: 5
    assert L.bajo_sort_tuning_set(8, 1, 19, 4) == _lib.ERR_INVALID_ARGUMENT   # up to 2^18 keys
    assert L.bajo_sort_tuning_set(8, 1, 18, 4) == _lib.OK
    assert L.bajo_sort_tuning_set(8, 1, 18, -1) == _lib.OK


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6])
def test_lbvh_build_with_every_variant(oracle, variant):
    from bajo_b200 import _lib, bvh, scenes
    L = _lib.load()
    v = scenes.random_triangles(50_000, seed=variant)
    lg = int(np.ceil(np.log2(50_000)))
    try:
        assert L.bajo_sort_tuning_set(8, 1, lg, variant) == _lib.OK
        b = bvh.build_triangle_bvh(torch.from_numpy(v).cuda())
        torch.cuda.synchronize()
        o = oracle.lbvh_build(v)
        assert np.array_equal(b.leaf_ids.cpu().numpy().view(np.uint32), o.leaf_ids)
        assert np.array_equal(b.node_meta.cpu().numpy().view(np.uint32)[: 4 * 49_999], o.node_meta[: 4 * 49_999])
    finally:
        L.bajo_sort_tuning_set(8, 1, lg, -1)
