"""The allocation-free entry sort (gs_sort_entries_static) against the
trainer's own binning (gs_debug_binning), through the C ABI (B200 required).

The entry point exists for callers that cannot call cudaMalloc (their device
memory belongs to another runtime's pool, or an allocation's implicit
synchronisation is not allowed on their path); its scratch is a static
device array, so these checks also run it twice on the same scratch.

The input is built the way the trainer builds its entries: splats in
(depth bits, id) order, each expanding to the tiles of its rectangle in row
order, key = tile id, value = splat id.  A stable sort on the tile id must
give exactly the trainer's per-tile id lists.  Two calls in a row (one and
two radix passes) run on the same static scratch."""
import ctypes as C

import numpy as np
import pytest

from splat_b200 import native as N
from test_gpu_parity import config0, gpu_raster, make

pytestmark = pytest.mark.gpu


def host_entries(params, rect, cam, tile, W):
    """(tile id, splat id) entries in presorted order, from the trainer's rectangles."""
    n = len(params) // 16
    P = params.reshape(n, 16)
    R = np.asarray(cam["R"], np.float32).reshape(3, 3)
    t2 = np.float32(cam["t"][2])
    # depth = (R2.p) + t2, left to right without fusion, as the projection computes it
    z = (R[2, 0] * P[:, 0] + R[2, 1] * P[:, 1]) + R[2, 2] * P[:, 2]
    z = (z + t2).astype(np.float32)
    valid = rect[0::2] != 0xFFFFFFFF
    ids = np.nonzero(valid)[0].astype(np.uint32)
    order = ids[np.lexsort((ids, z[ids].view(np.uint32)))]
    tilesX = (W + tile - 1) // tile
    keys, vals = [], []
    for i in order:
        r0, r1 = int(rect[2 * i]), int(rect[2 * i + 1])
        x0, y0, x1, y1 = r0 & 0xFFFF, r0 >> 16, r1 & 0xFFFF, r1 >> 16
        ty, tx = np.meshgrid(np.arange(y0, y1 + 1), np.arange(x0, x1 + 1), indexing="ij")
        tk = (ty * tilesX + tx).reshape(-1).astype(np.uint32)
        keys.append(tk)
        vals.append(np.full(tk.size, i, np.uint32))
    return np.concatenate(keys), np.concatenate(vals)


def test_static_sort_matches_trainer_binning_twice():
    import torch
    params, sh, cams, rgbs = config0()
    n = len(params) // 16
    # full rectangle lists (no tile cull), which host_entries reproduces
    t, targets, metas = make(params, sh, cams, rgbs, dict(shDeg=2, tileCull=0), radius=1.0)
    gpu_raster(t, [0], 1)
    L = N.lib()
    rect = np.zeros(n * 2, np.uint32)
    N.check(L.gs_debug_records(t._h, 0, None, N.ptr(rect, C.c_uint32)), t._h)
    tiles = 16 * 16
    tileCnt = np.zeros(tiles, np.uint32)
    ranges = np.zeros(2 * tiles, np.uint32)
    total = C.c_uint64()
    N.check(L.gs_debug_binning(t._h, 0, N.ptr(tileCnt, C.c_uint32), N.ptr(ranges, C.c_uint32), None, 0,
                               C.byref(total)), t._h)
    ids = np.zeros(int(total.value), np.uint32)
    N.check(L.gs_debug_binning(t._h, 0, None, None, N.ptr(ids, C.c_uint32), ids.size, C.byref(total)), t._h)

    keys, vals = host_entries(params, rect, cams[0], 16, 256)
    assert keys.size == ids.size and 0 < keys.size <= N.STATIC_SORT_MAX
    want_keys = np.sort(keys, kind="stable")
    want_vals = vals[np.argsort(keys, kind="stable")]
    np.testing.assert_array_equal(want_vals, ids)  # the host expansion is the trainer's input

    for bits in (8, 16):  # one radix pass (result copied back from scratch), then two
        dk = torch.from_numpy(keys.view(np.int32)).cuda()
        dv = torch.from_numpy(vals.view(np.int32)).cuda()
        torch.cuda.synchronize()
        rc = L.gs_sort_entries_static(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), keys.size, bits, None)
        assert rc == 0, rc
        got_k = dk.cpu().numpy().view(np.uint32)
        got_v = dv.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got_k, want_keys)
        np.testing.assert_array_equal(got_v, ids)


def test_static_sort_edge_sizes():
    """Empty input, a ragged tail (not a multiple of the 4096-entry block) and
    equal keys (stability) against numpy's stable sort."""
    import torch
    L = N.lib()
    assert L.gs_sort_entries_static(None, None, 0, 8, None) == 0
    rng = np.random.default_rng(5)
    for n, hi in ((1, 4), (4097, 3), (70001, 1 << 20)):
        keys = rng.integers(0, hi, n, dtype=np.uint32)
        vals = np.arange(n, dtype=np.uint32)
        dk = torch.from_numpy(keys.view(np.int32)).cuda()
        dv = torch.from_numpy(vals.view(np.int32)).cuda()
        torch.cuda.synchronize()
        bits = max(1, int(hi - 1).bit_length())
        rc = L.gs_sort_entries_static(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), n, bits, None)
        assert rc == 0, rc
        o = np.argsort(keys, kind="stable")
        np.testing.assert_array_equal(dk.cpu().numpy().view(np.uint32), keys[o])
        np.testing.assert_array_equal(dv.cpu().numpy().view(np.uint32), vals[o])


def test_static_sort_at_the_limit_allocates_nothing():
    """A call of exactly GS_STATIC_SORT_MAX entries (3 radix passes, so the
    result is copied back from the scratch half) sorts correctly and leaves
    the device's free memory unchanged; one entry more is refused with
    GS_E_LIMIT before any device work."""
    import torch
    L = N.lib()
    n = N.STATIC_SORT_MAX
    rng = np.random.default_rng(11)
    keys = rng.integers(0, 1 << 20, n, dtype=np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    dk = torch.from_numpy(keys.view(np.int32)).cuda()
    dv = torch.from_numpy(vals.view(np.int32)).cuda()
    wk, wv = dk.clone(), dv.clone()
    torch.cuda.synchronize()
    # warm-up call: loads the library's kernels on this device (lazy module loading)
    assert L.gs_sort_entries_static(C.c_void_p(wk.data_ptr()), C.c_void_p(wv.data_ptr()), n, 20, None) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc = L.gs_sort_entries_static(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), n, 20, None)
    free1, _ = torch.cuda.mem_get_info()
    assert rc == 0, rc
    assert free1 == free0, (free0, free1)
    o = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(dk.cpu().numpy().view(np.uint32), keys[o])
    np.testing.assert_array_equal(dv.cpu().numpy().view(np.uint32), vals[o])
    assert L.gs_sort_entries_static(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), n + 1, 20, None) == -5
