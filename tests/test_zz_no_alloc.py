"""srcu_voxel_centroid_noalloc: the allocation-free voxel entry point.

Callers such as real-time LiDAR loops that may not allocate device memory
after start-up, or hosts whose device memory belongs to another allocator,
use this entry point; its scratch is a fixed __device__ array inside the
library.  The tests call it through the C ABI, several times in a row, and
check every result against srcu_voxel_centroid (bit-exact keys and counts,
centroids within 1e-5 * leaf -- the voxel tests' tolerance -- and in fact
identical) and directly against the oracle.  This file is collected last."""
import ctypes

import numpy as np
import pytest

import oracle
from spatialrust_b200 import _native, synthetic

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _attrs(cloud, n_attrs):
    """n_attrs attribute columns: intensity, then derived columns."""
    base = [cloud.intensity, (cloud.x * np.float32(0.5)).astype(np.float32),
            (cloud.intensity * np.float32(3.0) + np.float32(1.0)).astype(np.float32)]
    return base[:n_attrs]


def _mode(mode):
    return {"centroid": dict(), "first": dict(attribute_first=True),
            "approximate": dict(approximate=True)}[mode]


def run_noalloc(lib, torch, cloud, leaf, n_attrs=1, mode="centroid", want_counts=True,
                want_keys=True):
    attrs = _attrs(cloud, n_attrs)
    cols = [_dev(torch, a) for a in (cloud.x, cloud.y, cloud.z, *attrs)]
    n = cloud.n
    outs = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(3 + n_attrs)]
    keys = torch.empty((n, 3), dtype=torch.int64, device="cuda")
    counts = torch.empty(n, dtype=torch.int32, device="cuda")
    attr_in = (ctypes.c_void_p * max(n_attrs, 1))(*[t.data_ptr() for t in cols[3:]])
    attr_out = (ctypes.c_void_p * max(n_attrs, 1))(*[t.data_ptr() for t in outs[3:]])
    c = _native.SrcuCloud(cols[0].data_ptr(), cols[1].data_ptr(), cols[2].data_ptr(),
                          ctypes.cast(attr_in, ctypes.c_void_p), n_attrs, 1, n)
    o = _native.SrcuVoxelOut(outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(),
                             ctypes.cast(attr_out, ctypes.c_void_p),
                             keys.data_ptr() if want_keys else 0,
                             counts.data_ptr() if want_counts else 0, 1)
    p = _native._voxel_params(leaf, None, **_mode(mode))
    nv = ctypes.c_uint64(0)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    reserved_before = torch.cuda.memory_reserved()
    free_before = torch.cuda.mem_get_info()[0]
    st = lib.srcu_voxel_centroid_noalloc(ctypes.byref(c), ctypes.byref(p), ctypes.byref(o),
                                         ctypes.byref(nv), ctypes.c_void_p(stream))
    free_after = torch.cuda.mem_get_info()[0]
    assert torch.cuda.memory_reserved() == reserved_before
    assert st == _native.SRCU_OK, _native.STATUS_NAMES.get(st, st)
    v = int(nv.value)
    res = ([t[:v].cpu().numpy() for t in outs],
           keys[:v].cpu().numpy() if want_keys else None,
           counts[:v].cpu().numpy().astype(np.uint32) if want_counts else None)
    return res, free_before - free_after


def check_against_context(cuda_ctx, cloud, leaf, res, n_attrs=1, mode="centroid"):
    cols, keys, counts = res
    m = _mode(mode)
    ref_cols, ref_keys, ref_counts = cuda_ctx.voxel_centroid(
        cloud.x, cloud.y, cloud.z, _attrs(cloud, n_attrs), leaf=leaf, want_keys=True, **m)
    if keys is not None:
        assert np.array_equal(keys, ref_keys)
    if counts is not None:
        assert np.array_equal(counts, ref_counts)
    assert len(cols[0]) == len(ref_counts)
    for a, b in zip(cols, ref_cols):
        assert np.max(np.abs(a.astype(np.float64) - b)) <= 1e-5 * leaf
        assert np.array_equal(a, b)


def check_against_oracle(cloud, leaf, res, n_attrs=1, mode="centroid"):
    cols, keys, counts = res
    attrs = _attrs(cloud, n_attrs)
    if mode == "centroid":
        ref = oracle.voxel_centroid(cloud.x, cloud.y, cloud.z, attrs, leaf=leaf)
    else:
        ref = oracle.voxel_general(cloud.x, cloud.y, cloud.z, attrs, leaf=leaf, **_mode(mode))
    if keys is not None:
        assert np.array_equal(keys, ref.keys)
    if counts is not None:
        assert np.array_equal(counts, ref.counts)
    for a, b in zip(cols, ref.fields):
        assert np.max(np.abs(a.astype(np.float64) - b)) <= 1e-5 * leaf


def test_noalloc_matches_context_entry_point_twice(cuda_ctx):
    import torch
    lib = _native.load()
    frame = synthetic.georef_scan(131_072, seed=41)        # one 64 x 2048 LiDAR frame's worth
    other = synthetic.uniform_cube(50_000, seed=42, extent=30.0)
    first, _ = run_noalloc(lib, torch, frame, 0.2)
    second, grown = run_noalloc(lib, torch, other, 0.5)    # scratch keeps the previous call's data
    check_against_context(cuda_ctx, frame, 0.2, first)
    check_against_context(cuda_ctx, other, 0.5, second)
    check_against_oracle(frame, 0.2, first)
    check_against_oracle(other, 0.5, second)
    assert grown == 0, "the second call changed free device memory"
    third, grown = run_noalloc(lib, torch, frame, 0.2)
    for a, b in zip(first[0], third[0]):
        assert np.array_equal(a, b)
    assert grown == 0


@pytest.mark.parametrize("n_attrs,mode,want_counts,want_keys", [
    (0, "centroid", True, True),
    (3, "centroid", True, False),
    (1, "first", False, True),
    (3, "approximate", False, False),
    (0, "approximate", True, True),
])
def test_noalloc_columns_modes_and_optional_outputs(cuda_ctx, n_attrs, mode, want_counts,
                                                    want_keys):
    import torch
    lib = _native.load()
    cloud = synthetic.georef_scan(90_000, seed=43)
    for leaf in (0.1, 0.5):  # two calls in a row on the shared scratch
        res, grown = run_noalloc(lib, torch, cloud, leaf, n_attrs, mode, want_counts, want_keys)
        check_against_context(cuda_ctx, cloud, leaf, res, n_attrs, mode)
        check_against_oracle(cloud, leaf, res, n_attrs, mode)
        assert grown == 0


def test_noalloc_epoch_restart_before_the_wrap(cuda_ctx):
    # The scratch's look-back tags advance by 64 per call; placed just below
    # the 32-bit wrap, the calls must clear the tagged words and restart the
    # epoch, and every result must still equal the context path's.
    import torch
    lib = _native.load()
    big = synthetic.georef_scan(131_072, seed=44)
    small = synthetic.georef_scan(20_000, seed=45)
    run_noalloc(lib, torch, big, 0.2)  # set-up on this device
    e0 = ctypes.c_uint32(0)
    r0 = ctypes.c_uint64(0)
    assert lib.srcu_noalloc_debug_get_epoch(ctypes.byref(e0), ctypes.byref(r0)) == _native.SRCU_OK
    assert lib.srcu_noalloc_debug_set_epoch(ctypes.c_uint32(0xFFFFFF40)) == _native.SRCU_OK
    for cloud in (big, small, big, small):
        res, _ = run_noalloc(lib, torch, cloud, 0.2)
        check_against_context(cuda_ctx, cloud, 0.2, res)
    e = ctypes.c_uint32(0)
    r = ctypes.c_uint64(0)
    assert lib.srcu_noalloc_debug_get_epoch(ctypes.byref(e), ctypes.byref(r)) == _native.SRCU_OK
    assert r.value == r0.value + 1 and e.value == 128


def test_noalloc_rejects_clouds_beyond_its_scratch():
    import torch
    lib = _native.load()
    n = 131_073
    x = torch.zeros(n, dtype=torch.float32, device="cuda")
    c = _native.SrcuCloud(x.data_ptr(), x.data_ptr(), x.data_ptr(), 0, 0, 1, n)
    o = _native.SrcuVoxelOut(x.data_ptr(), x.data_ptr(), x.data_ptr(), 0, 0, 0, 1)
    p = _native._voxel_params(1.0, None)
    nv = ctypes.c_uint64(7)
    st = lib.srcu_voxel_centroid_noalloc(ctypes.byref(c), ctypes.byref(p), ctypes.byref(o),
                                         ctypes.byref(nv), None)
    assert st == _native.SRCU_ERR_INVALID_ARGUMENT and nv.value == 0
