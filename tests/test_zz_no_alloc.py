"""srcu_voxel_centroid_noalloc: the allocation-free voxel entry point.

Callers such as real-time LiDAR loops that may not allocate device memory
after start-up, or hosts whose device memory belongs to another allocator,
use this entry point; its scratch is a fixed __device__ array inside the
library.  The test calls it through the C ABI twice in a row and checks both
results against srcu_voxel_centroid (bit-exact keys and counts, centroids
within 1e-5 * leaf -- the voxel tests' tolerance -- and in fact identical).
It lives in its own file so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

from spatialrust_b200 import _native, synthetic

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_noalloc(lib, torch, cloud, leaf):
    cols = [_dev(torch, a) for a in (cloud.x, cloud.y, cloud.z, cloud.intensity)]
    n = cloud.n
    outs = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(4)]
    keys = torch.empty((n, 3), dtype=torch.int64, device="cuda")
    counts = torch.empty(n, dtype=torch.int32, device="cuda")
    attr_in = (ctypes.c_void_p * 1)(cols[3].data_ptr())
    attr_out = (ctypes.c_void_p * 1)(outs[3].data_ptr())
    c = _native.SrcuCloud(cols[0].data_ptr(), cols[1].data_ptr(), cols[2].data_ptr(),
                          ctypes.cast(attr_in, ctypes.c_void_p), 1, 1, n)
    o = _native.SrcuVoxelOut(outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(),
                             ctypes.cast(attr_out, ctypes.c_void_p), keys.data_ptr(),
                             counts.data_ptr(), 1)
    p = _native._voxel_params(leaf, None)
    nv = ctypes.c_uint64(0)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    st = lib.srcu_voxel_centroid_noalloc(ctypes.byref(c), ctypes.byref(p), ctypes.byref(o),
                                         ctypes.byref(nv), ctypes.c_void_p(stream))
    free_after = torch.cuda.mem_get_info()[0]
    assert st == _native.SRCU_OK, _native.STATUS_NAMES.get(st, st)
    v = int(nv.value)
    res = ([t[:v].cpu().numpy() for t in outs], keys[:v].cpu().numpy(),
           counts[:v].cpu().numpy().astype(np.uint32))
    return res, free_before - free_after


def check_against_context(cuda_ctx, cloud, leaf, res):
    cols, keys, counts = res
    ref_cols, ref_keys, ref_counts = cuda_ctx.voxel_centroid(
        cloud.x, cloud.y, cloud.z, [cloud.intensity], leaf=leaf, want_keys=True)
    assert np.array_equal(keys, ref_keys)
    assert np.array_equal(counts, ref_counts)
    for a, b in zip(cols, ref_cols):
        assert np.max(np.abs(a.astype(np.float64) - b)) <= 1e-5 * leaf
        assert np.array_equal(a, b)


def test_noalloc_matches_context_entry_point_twice(cuda_ctx):
    import torch
    lib = _native.load()
    frame = synthetic.georef_scan(131_072, seed=41)        # one 64 x 2048 LiDAR frame's worth
    other = synthetic.uniform_cube(50_000, seed=42, extent=30.0)
    first, _ = run_noalloc(lib, torch, frame, 0.2)
    second, grown = run_noalloc(lib, torch, other, 0.5)    # scratch keeps the previous call's data
    check_against_context(cuda_ctx, frame, 0.2, first)
    check_against_context(cuda_ctx, other, 0.5, second)
    assert grown == 0, "the second call changed free device memory"
    third, grown = run_noalloc(lib, torch, frame, 0.2)
    for a, b in zip(first[0], third[0]):
        assert np.array_equal(a, b)
    assert grown == 0


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
