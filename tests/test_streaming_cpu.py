"""Host-side contract of the streaming voxel mirror: configuration and spool
validation (StreamingVoxelConfig::new, streaming.rs:345-363; SpoolOptions::new,
crates/spatialrust-io/src/spool.rs:21-33), chunking and push_scalar narrowing.
No GPU."""
import numpy as np
import pytest

import spatialrust_b200 as sr
from spatialrust_b200.streaming import (MemoryChunkSource, RecordsError, SpoolOptions,
                                        StreamingVoxelConfig, push_scalar)


def spool(limit=4096, tmp="/tmp"):
    return SpoolOptions(tmp, limit)


def test_config_validation():
    for leaf in (0.0, -1.0, float("inf"), float("nan")):
        with pytest.raises(RecordsError):
            StreamingVoxelConfig(leaf, 2, 2, spool())
    with pytest.raises(RecordsError):
        StreamingVoxelConfig(1.0, 0, 2, spool())
    with pytest.raises(RecordsError):
        StreamingVoxelConfig(1.0, 2, 0, spool())
    c = StreamingVoxelConfig(0.1, 3, 4, spool())
    assert c.leaf_size() == float(np.float32(0.1)) and c.run_points() == 3 and c.max_runs() == 4


def test_spool_options_validation(tmp_path):
    with pytest.raises(RecordsError):
        SpoolOptions(str(tmp_path), 0)
    with pytest.raises(RecordsError):
        SpoolOptions(str(tmp_path / "missing"), 16)
    assert SpoolOptions(str(tmp_path), 16).limit_bytes == 16


def test_memory_chunk_source_splits_in_order():
    b = sr.PointCloudBuilder.xyz()
    for i in range(5):
        b.push_point([float(i), 0.0, 0.0])
    src = MemoryChunkSource(b.build(), 2)
    sizes, xs = [], []
    while (c := src.next_chunk()) is not None:
        sizes.append(len(c))
        xs.extend(c.field("x").tolist())
    assert sizes == [2, 2, 1] and xs == [0, 1, 2, 3, 4]


def test_push_scalar_rounds_half_away_and_clamps():
    v = np.array([0.49999999999999994, 0.5, 2.5, -0.5, 300.0, -7.0, np.nan])
    assert push_scalar(v, sr.DType.U8).tolist() == [0, 1, 3, 0, 255, 0, 0]
    assert push_scalar(v, sr.DType.I32).tolist() == [0, 1, 3, -1, 300, -7, 0]
    assert push_scalar(np.array([1.0 + 2 ** -30]), sr.DType.F32)[0] == np.float32(1.0)
