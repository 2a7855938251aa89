"""nxm_sort_blocks_noalloc: the block sort for callers that may not allocate
GPU memory (a host program that reserves its device memory at start-up and
forbids allocations in its frame loop; a plugin handed device buffers but no
allocator).  Its grid tables live in a fixed device array of the library, so this
checks, through the C ABI, that two calls in a row (on different scenes, so
that state left in the shared array would show) give the same active blocks
and the same per-block primary particles, in z-slab order, as the sort of
the existing entry point (nxm_debug_sort on a state), and that sizes beyond
the fixed limits are rejected (too many particles, more blocks than
max_blocks, more distinct blocks than the fixed hash holds).  Integer results: compared bit for bit.

Named to be collected last, so a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.mpm import MpmPipeline, state_from_scene, NXM_E_CAPACITY, NXM_OK

pytestmark = pytest.mark.gpu


def _noalloc_sort(lib, torch, pos_xyz: np.ndarray, dx: float, max_blocks: int):
    n = pos_xyz.shape[0]
    pos4 = np.zeros((n, 4), np.float32)
    pos4[:, :3] = pos_xyz
    d_pos = torch.from_numpy(pos4).cuda()
    d_sorted = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    d_vids = torch.zeros((max_blocks, 4), dtype=torch.int32, device="cuda")
    d_ranges = torch.zeros((max_blocks, 2), dtype=torch.int32, device="cuda")
    nb = C.c_uint32(0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.nxm_sort_blocks_noalloc(d_pos.data_ptr(), n, dx, d_sorted.data_ptr(), d_vids.data_ptr(),
                                     d_ranges.data_ptr(), max_blocks, C.byref(nb), stream)
    return rc, nb.value, d_sorted.cpu().numpy(), d_vids.cpu().numpy(), d_ranges.cpu().numpy()


def _primaries_by_block(vids, first, count, sorted_ids):
    return {tuple(int(v) for v in vids[b, :3]): sorted_ids[first[b]:first[b] + count[b]] for b in range(len(vids))}


def _check_against_existing_entry_point(gpu_lib, torch, scene):
    pipe = MpmPipeline()
    st = state_from_scene(scene)
    pipe.debug_sort(st)
    h = st.headers()
    ref = _primaries_by_block(h[:, :3], h[:, 3], h[:, 4], st.sorted_ids())

    rc, nb, sorted_ids, vids, ranges = _noalloc_sort(gpu_lib, torch, scene.particles.pos, scene.dx, 4096)
    assert rc == NXM_OK
    assert nb == len(h)
    got = _primaries_by_block(vids[:nb], ranges[:nb, 0], ranges[:nb, 1], sorted_ids)
    assert set(got) == set(ref)
    for vid, ids in ref.items():
        assert np.array_equal(np.sort(got[vid]), np.sort(ids)), vid
    # every particle is listed exactly once, and inside a block in z-slab order
    assert np.array_equal(np.sort(sorted_ids[:scene.n]), np.arange(scene.n))
    pos = scene.particles.pos
    slab = ((np.round(pos / np.float32(scene.dx)) - 1) % 4).astype(np.int64)[:, 2]
    for vid, ids in got.items():
        assert np.all(np.diff(slab[ids]) >= 0), vid


def test_noalloc_sort_matches_existing_sort_twice_in_a_row(gpu_lib, oracle_built):
    import torch
    torch.cuda.init()
    _check_against_existing_entry_point(gpu_lib, torch, scenes.elastic_cube(n_side=16))
    _check_against_existing_entry_point(gpu_lib, torch, scenes.mixed_materials(n_side=6))


def test_noalloc_sort_rejects_sizes_beyond_its_limits(gpu_lib):
    import torch
    sc = scenes.elastic_cube(n_side=16)
    rc, nb, *_ = _noalloc_sort(gpu_lib, torch, sc.particles.pos, sc.dx, 4)
    assert rc == NXM_E_CAPACITY and nb == 0
    # too many particles is refused before any GPU work
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    n = C.c_uint32(0)
    rc = gpu_lib.nxm_sort_blocks_noalloc(dummy.data_ptr(), (1 << 26) + 1, 0.1, dummy.data_ptr(), dummy.data_ptr(),
                                         dummy.data_ptr(), 1, C.byref(n), None)
    assert rc == NXM_E_CAPACITY
    # more distinct blocks than the fixed hash has slots (2 x 16384): particles
    # 8 cells apart, so that each one's 2x2x2 block neighbourhood is its own
    dx = 1.0 / 64.0
    k = np.arange(18, dtype=np.float32)
    grid = np.stack(np.meshgrid(k, k, k, indexing="ij"), -1).reshape(-1, 3)
    spread = ((grid * 8.0 + 2.5) * np.float32(dx)).astype(np.float32)
    assert 8 * len(spread) > 2 * 16384
    rc, nb, *_ = _noalloc_sort(gpu_lib, torch, spread, dx, 16384)
    assert rc == NXM_E_CAPACITY and nb == 0
    # a valid call right after a rejected one still matches the existing sort
    _check_against_existing_entry_point(gpu_lib, torch, sc)
