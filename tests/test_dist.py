"""Multi-process host logic on CPU: two gloo ranks run the same barrier,
max-over-ranks timing and sharding the multi-GPU benchmark uses (no GPU:
the kernels are per rank and exchange nothing)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bajo_b200 import dist


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, counts, n_pixels, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    w, r, _ = dist.init(backend="gloo", timeout_s=60)
    assert (w, r) == (world, rank)
    dist.barrier(w)
    slowest = dist.max_over_ranks(w, 10.0 + rank)
    total = dist.sum_over_ranks(w, 1.0)
    mine = dist.shard_scenes(counts, w, r)
    pix = dist.shard_pixels(n_pixels, w, r)
    dist.barrier(w)
    dist.finish(w)
    q.put((rank, slowest, total, mine.tolist(), pix))


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_agree_on_timing_and_shards(world):
    rng = np.random.default_rng(0)
    counts = np.exp(rng.uniform(np.log(256), np.log(65536), 97)).astype(np.int64)
    n_pixels = 1280 * 720 + 7
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, counts, n_pixels, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(o[1] == 10.0 + world - 1 for o in out)  # max over ranks
    assert all(o[2] == float(world) for o in out)
    scenes = np.concatenate([o[3] for o in out])
    assert np.array_equal(np.sort(scenes), np.arange(counts.size))  # every scene exactly once
    loads = [counts[o[3]].sum() for o in out]
    assert max(loads) - min(loads) <= counts.max()  # greedy balance bound
    spans = [o[4] for o in out]
    assert spans[0][0] == 0 and spans[-1][1] == n_pixels
    assert all(spans[k][1] == spans[k + 1][0] for k in range(world - 1))


def test_single_process_is_a_no_op():
    assert dist.max_over_ranks(1, 3.5) == 3.5
    assert dist.shard_pixels(10, 1, 0) == (0, 10)
    assert list(dist.shard_scenes([5, 1, 3], 1, 0)) == [0, 1, 2]
    idx, so = dist.subset_offsets([0, 2, 5, 9], [2, 0])
    assert list(idx) == [5, 6, 7, 8, 0, 1] and list(so) == [0, 4, 6]
