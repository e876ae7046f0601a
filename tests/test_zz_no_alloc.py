"""The allocation-free sort entry point (psb_sort_cells_noalloc).

It exists for callers that may not allocate device memory: applications that
give the whole GPU to their own memory pool, and per-frame loops that cannot
stall on cudaMalloc/cudaFree. Its scratch is a static array inside the
library, so this test checks that its output equals the regular path's
(psb_build_neighbors' sorted keys and particle ids) bit for bit -- the
work is integer, the tolerance is zero -- on two calls in a row, the second
smaller than the first so that stale scratch contents would show.

This file is named to be collected last; it needs nothing from the others
and passes on its own in a fresh process.
"""
import ctypes
import math

import numpy as np
import pytest

import psb_project_b200 as P
from psb_project_b200 import runtime as R

pytestmark = pytest.mark.gpu


def key_bits(sc):
    return max(1, math.ceil(math.log2(int(np.prod(sc.dims)))))


def regular_path(sc):
    """Sorted keys and ids from the regular entry point, plus its id-order keys."""
    with P.Simulation(sc) as sim:
        sim.upload(P.scene_positions(sc))
        sim.build_neighbors()
        return (sim.read_field(R.FIELD_CELL_KEY), sim.read_field(R.FIELD_SORTED_KEY),
                sim.read_field(R.FIELD_SORTED_ID))


def noalloc_sort(keys, vals, bits, in_place=False):
    import torch
    dev = torch.device("cuda", 0)
    k_in = torch.from_numpy(keys.view(np.int32)).to(dev)
    v_in = torch.from_numpy(vals.view(np.int32)).to(dev)
    k_out = k_in if in_place else torch.full_like(k_in, -1)
    v_out = v_in if in_place else torch.full_like(v_in, -1)
    stream = torch.cuda.current_stream(dev)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = R.lib().psb_sort_cells_noalloc(vp(k_in), vp(v_in), vp(k_out), vp(v_out), keys.shape[0], bits,
                                        ctypes.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return rc, k_out.cpu().numpy().view(np.uint32), v_out.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_regular_path_twice():
    pytest.importorskip("torch")
    # 16,384 then 960 pairs; 16 key bits (two passes, result lands in the
    # caller's buffer) then 24 (three passes, result copied back from scratch)
    for sc, bits in ((P.config_scene("C0"), None), (P.ref_scene(), 24)):
        keys_by_id, sorted_keys, sorted_ids = regular_path(sc)
        ids = np.arange(sc.n, dtype=np.uint32)
        rc, k, v = noalloc_sort(keys_by_id, ids, bits or key_bits(sc))
        assert rc == R.OK
        assert np.array_equal(k, sorted_keys)
        assert np.array_equal(v, sorted_ids.astype(np.uint32))


def test_noalloc_sort_in_place():
    """keys_out == keys_in and vals_out == vals_in: the sort runs in the
    caller's buffers (the copy-in is skipped) and gives the same result."""
    pytest.importorskip("torch")
    sc = P.config_scene("C0")
    keys_by_id, sorted_keys, sorted_ids = regular_path(sc)
    rc, k, v = noalloc_sort(keys_by_id, np.arange(sc.n, dtype=np.uint32), key_bits(sc), in_place=True)
    assert rc == R.OK
    assert np.array_equal(k, sorted_keys)
    assert np.array_equal(v, sorted_ids.astype(np.uint32))


def test_noalloc_sort_rejects_partial_overlap():
    """Outputs that overlap an input other than itself, or each other, are
    refused before anything runs (the pointers are never dereferenced)."""
    L = R.lib()
    n = 1024
    a, b = ctypes.c_void_p(1 << 20), ctypes.c_void_p((1 << 20) + 64)
    c, d = ctypes.c_void_p(1 << 24), ctypes.c_void_p(1 << 26)
    assert L.psb_sort_cells_noalloc(a, c, b, d, n, 20, None) == R.EINVAL     # keys_out overlaps keys_in
    assert L.psb_sort_cells_noalloc(a, c, d, d, n, 20, None) == R.EINVAL     # keys_out == vals_out


def test_noalloc_sort_rejects_sizes_beyond_its_scratch():
    L = R.lib()
    n = R.NOALLOC_MAX_N + 1
    dummy = ctypes.c_void_p(16)      # never dereferenced: the size check comes first
    assert L.psb_sort_cells_noalloc(dummy, dummy, dummy, dummy, n, 20, None) == R.EINVAL
