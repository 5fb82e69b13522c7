"""The device-side failure path: a bounded wait that gives up reports
SRCU_ERR_TIMEOUT through the context's status word, nothing faults, and the
same context runs the next chain normally."""
import time

import numpy as np
import pytest

from spatialrust_b200 import InvalidArgument, _native, synthetic

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_the_context_recovers(cuda_ctx):
    c = synthetic.georef_scan(50_000, seed=80)
    before = cuda_ctx.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=0.2)[0]
    t0 = time.perf_counter()
    with pytest.raises(_native.DeviceTimeout):
        cuda_ctx.selftest_bounded_wait(2000)  # ~2 ms of polling a flag nothing sets
    assert time.perf_counter() - t0 < 10.0
    after = cuda_ctx.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=0.2)[0]
    assert len(before) == len(after)
    for a, b in zip(before, after):
        assert np.array_equal(a, b)


def test_bounded_wait_arguments(cuda_ctx):
    with pytest.raises(InvalidArgument):
        cuda_ctx.selftest_bounded_wait(0)
    with pytest.raises(InvalidArgument):
        cuda_ctx.selftest_bounded_wait(1 << 22)
