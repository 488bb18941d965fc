"""Failure detection without a GPU fault.  Faults are injected on the host
(corrupted tree records, undersized workspaces, bad segment tables, a flag
that nothing sets); every device wait and index is bounded, so each case
ends with a status word or an error code and the context stays usable."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import _lib, bvh, scenes, sort  # noqa: E402



def _tree(n=1000, seed=1):
    return bvh.build_triangle_bvh(torch.from_numpy(scenes.random_triangles(n, seed=seed)).cuda())


def _trace_status(tree, n_rays=4096):
    rng = np.random.default_rng(0)
    rays = np.zeros((8, n_rays), np.float32)
    rays[0:3] = rng.uniform(-0.5, 1.5, (3, n_rays))
    d = rng.normal(size=(3, n_rays))
    rays[4:7] = d / np.linalg.norm(d, axis=0)
    rays[7] = 10.0
    hits = torch.empty(8 * n_rays, dtype=torch.float32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    tree.launch_rays(torch.from_numpy(rays.reshape(-1)).cuda(), hits, n_rays, d_status=st)
    torch.cuda.synchronize()
    return int(st.item())


def _still_usable():
    k = torch.randint(-2**31, 2**31, (100_000,), dtype=torch.int32, device="cuda")
    v = torch.arange(100_000, dtype=torch.int32, device="cuda")
    ws = sort.onesweep_radix_sort_pairs(k, v)
    torch.cuda.synchronize()
    assert ws.status() == 0
    ku = k.cpu().numpy().view(np.uint32)
    assert np.all(ku[1:] >= ku[:-1])


@pytest.mark.parametrize("fault", ["cycle", "internal_out_of_range"])
def test_corrupted_tree_reports_bad_topology(fault):
    """The traversal bounds its node visits by the node count and checks
    every internal ref before loading it (leaf refs, written only by the
    build, are trusted as in the reference)."""
    tree = _tree()
    assert _trace_status(tree) == 0
    root = int(tree.roots[0].item())
    meta = tree.node_meta.view(-1, 4)
    if fault == "cycle":          # the root is its own left child: visits are bounded by the node count
        meta[root, 1] = root
    else:                          # an internal ref past the nodes is never dereferenced
        meta[root, 2] = 0x7FFFFFF0
    assert _trace_status(tree) & _lib.STATUS_BAD_TOPOLOGY
    _still_usable()


def test_bounded_wait_gives_up_with_a_status():
    L = _lib.load()
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")   # nothing ever sets it
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.bajo_wait_selftest(flag.data_ptr(), 1, 2000, st.data_ptr(), None) == _lib.OK
    torch.cuda.synchronize()
    assert int(st.item()) == _lib.STATUS_WAIT_TIMEOUT
    # a flag that is set ends the wait at once, with no status
    flag.fill_(1)
    st.zero_()
    assert L.bajo_wait_selftest(flag.data_ptr(), 1, 2000, st.data_ptr(), None) == _lib.OK
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    assert L.bajo_wait_selftest(flag.data_ptr(), 1, 2_000_000, st.data_ptr(), None) == _lib.ERR_INVALID_ARGUMENT
    _still_usable()


def test_undersized_workspaces_are_refused():
    L = _lib.load()
    n = 5000
    v = torch.from_numpy(scenes.random_triangles(n, seed=2)).cuda()
    tree = bvh.build_triangle_bvh(v)
    c = tree.c_struct()
    need = bvh.lbvh_sizes(n)["workspace"]
    small = torch.zeros(need - 256, dtype=torch.uint8, device="cuda")
    assert L.bajo_lbvh_build(v.data_ptr(), ctypes.byref(c), small.data_ptr(), small.numel(), None) == \
        _lib.ERR_WORKSPACE_TOO_SMALL
    keys = torch.zeros(n, dtype=torch.int32, device="cuda")
    nb = ctypes.c_size_t(0)
    assert L.bajo_sort_workspace_size(n, 4, 0, 0, 32, ctypes.byref(nb)) == _lib.OK
    ws = torch.zeros(nb.value - 16, dtype=torch.uint8, device="cuda")
    assert L.bajo_sort_keys_u32(keys.data_ptr(), n, 0, 32, ws.data_ptr(), ws.numel(), None) == \
        _lib.ERR_WORKSPACE_TOO_SMALL
    _still_usable()


@pytest.mark.parametrize("offsets", [[1, 100], [0, 50, 40, 100], [0, 99], [0, 101]])
def test_bad_segment_tables_are_refused_on_the_host(offsets):
    v = torch.from_numpy(scenes.random_triangles(100, seed=3)).cuda()
    with pytest.raises(ValueError):
        bvh.build_triangle_bvh(v, np.array(offsets))
