"""Sort autotuner host logic: size classes, the choice, the generated header,
and the launch shapes the library exports."""
import re

from spatialrust_b200 import _native, autotune

BIG = (1 << 64) - 1


def fake(costs_by_size):
    """costs_by_size: {(points, voxels): [ms per shape]} -> a measure() result
    (voxel sort 3/4 of the cost, cell sort 1/4)."""
    n_cfg = len(next(iter(costs_by_size.values())))
    runs = [dict(points=p, voxels=v, config=c, voxel_sort_ms=ms[c] * 0.75, cell_sort_ms=ms[c] * 0.25)
            for (p, v), ms in costs_by_size.items() for c in range(n_cfg)]
    return dict(configs=[dict(items_per_thread=16, blocks_per_sm=2)] * n_cfg, runs=runs)


def test_samples_and_boundaries():
    res = fake({(100_000, 50_000): [2.0, 1.0, 3.0, 1.5],
                (400_000, 200_000): [1.0, 2.0, 3.0, 1.5],
                (800_000, 300_000): [1.0, 2.0, 3.0, 1.5]})
    v, c = autotune.samples(res, "voxel"), autotune.samples(res, "cell")
    # both kinds are keyed by the chain's point count (the launch-time bound)
    assert [k for k, _ in v] == [k for k, _ in c] == [100_000, 400_000, 800_000]
    assert v[0][1] == [1.5, 0.75, 2.25, 1.125] and c[0][1] == [0.5, 0.25, 0.75, 0.375]
    # shape 1 up to the first sample, shape 0 from the second: the boundary is
    # their geometric mean
    assert autotune.choose(res, "voxel") == [(200_000, 1), (BIG, 0)]
    assert autotune.choose(res, "cell") == [(200_000, 1), (BIG, 0)]


def test_hysteresis_keeps_the_smaller_sizes_shape():
    def run(p, v, c, ms):
        return dict(points=p, voxels=v, config=c, voxel_sort_ms=ms, cell_sort_ms=ms)
    res = dict(configs=[{}, {}], runs=[run(100_000, 50_000, 0, 2.0), run(100_000, 50_000, 1, 1.0),
                                       run(400_000, 200_000, 0, 0.995), run(400_000, 200_000, 1, 1.0)])
    # at 400k keys shape 0 is faster by less than the hysteresis: shape 1 stays
    assert autotune.choose(res, "voxel") == [(BIG, 1)]
    assert autotune.choose(res, "voxel", hysteresis=0.0) == [(200_000, 1), (BIG, 0)]


def test_choose_bounds_the_table():
    # alternating winners at every sample would exceed the entry limit: the
    # hysteresis widens until the table fits
    costs = {(1000 * (k + 1), 500 * (k + 1)): ([1.0, 1.3] if k % 2 else [1.3, 1.0]) for k in range(40)}
    t = autotune.choose(fake(costs), "voxel")
    assert 1 <= len(t) <= autotune.TABLE_MAX and t[-1][0] == BIG
    bounds = [m for m, _ in t]
    assert bounds == sorted(bounds) and len(set(bounds)) == len(bounds)
    assert autotune.choose(dict(configs=[{}], runs=[]), "cell") == [(BIG, 0)]


def test_header_is_parseable():
    res = fake({(131_072, 60_000): [2.0, 1.0, 3.0, 1.5]})
    text = autotune.header_text({"voxel": [(1 << 20, 1), (BIG, 0)], "cell": [(BIG, 2)]}, res)
    assert "kVoxelSortTuneCount = 2;" in text and "kCellSortTuneCount = 1;" in text
    assert re.search(r"kVoxelSortTuneMaxPoints\[\] = \{1048576ull, UINT64_MAX\};", text)
    assert "kVoxelSortTuneConfig[] = {1, 0};" in text and "kCellSortTuneConfig[] = {2};" in text


def test_library_shapes():
    cfgs = _native.sort_configs()
    assert len(cfgs) >= 2 and cfgs[0]["items_per_thread"] == 16
    assert all(c["threads_per_block"] in (256, 512) for c in cfgs)
    assert {c["threads_per_block"] for c in cfgs} == {256, 512}  # block size is a tuned dimension
    assert {c["digit_bits"] for c in cfgs} == {8, 9}  # and so is digit width
    # a thread per digit bin of the widest digit
    assert all(c["threads_per_block"] >= 1 << c["digit_bits"] for c in cfgs)
    assert len({(c["items_per_thread"], c["blocks_per_sm"], c["threads_per_block"], c["digit_bits"])
                for c in cfgs}) == len(cfgs)


def test_batch_kinds_sample_their_own_runs():
    def run(w, p, c, vms, cms):
        return dict(workload=w, points=p, voxels=p // 2, config=c, voxel_sort_ms=vms, cell_sort_ms=cms)
    res = dict(configs=[{}, {}], runs=[run("scan", 100_000, 0, 1.0, 0.5), run("scan", 100_000, 1, 2.0, 0.6),
                                       run("batch", 100_000, 0, 3.0, 0.9), run("batch", 100_000, 1, 2.0, 0.7)])
    assert autotune.samples(res, "voxel") == [(100_000, [1.0, 2.0])]
    assert autotune.samples(res, "batch_voxel") == [(100_000, [3.0, 2.0])]
    assert autotune.samples(res, "batch_cell") == [(100_000, [0.9, 0.7])]
    assert autotune.choose(res, "voxel") == [(BIG, 0)] and autotune.choose(res, "batch_voxel") == [(BIG, 1)]
    # runs from before the batch workload existed count as scan runs
    old = dict(configs=[{}], runs=[dict(points=5, voxels=2, config=0, voxel_sort_ms=1.0, cell_sort_ms=1.0)])
    assert autotune.samples(old, "voxel") == [(5, [1.0])] and autotune.samples(old, "batch_voxel") == []
    # without batch tables the header repeats the scan tables for the batch kinds
    text = autotune.header_text({"voxel": [(BIG, 3)], "cell": [(BIG, 2)]}, None)
    assert "kBatchVoxelSortTuneConfig[] = {3};" in text and "kBatchCellSortTuneConfig[] = {2};" in text
    text = autotune.header_text({"voxel": [(BIG, 3)], "cell": [(BIG, 2)], "batch_voxel": [(BIG, 6)],
                                 "batch_cell": [(BIG, 7)]}, None)
    assert "kBatchVoxelSortTuneConfig[] = {6};" in text and "kBatchCellSortTuneConfig[] = {7};" in text


def test_committed_header_matches_library():
    import os
    h = open(os.path.join(os.path.dirname(autotune.__file__), "csrc", "sort_tuning.h")).read()
    for name in ("Voxel", "Cell", "BatchVoxel", "BatchCell"):
        n = int(re.search(rf"k{name}SortTuneCount = (\d+);", h).group(1))
        cfg = [int(v) for v in
               re.search(rf"k{name}SortTuneConfig\[\] = \{{([^}}]*)\}};", h).group(1).split(",")]
        assert 1 <= n <= autotune.TABLE_MAX
        assert len(cfg) == n and all(0 <= c < len(_native.sort_configs()) for c in cfg)


def test_choose_staging():
    def res(pairs):
        return dict(staging=[dict(points=n, voxels=n, staging=m, normals_ms=ms)
                             for n, (a, b) in enumerate(pairs) for m, ms in ((0, a), (1, b))])
    assert autotune.choose_staging(res([(1.0, 0.9), (2.0, 1.9)])) == 1
    # one large size where staging wins by a little does not outvote the rest
    assert autotune.choose_staging(res([(0.037, 0.041), (0.149, 0.167), (0.657, 0.696),
                                        (3.629, 3.697), (7.365, 7.231)])) == 0
    assert autotune.choose_staging({}) == 0
    assert "kNeighborStaging = 1;" in autotune.header_text({"voxel": [(BIG, 0)], "cell": [(BIG, 0)]},
                                                             None, 1)


def test_choose_walk_among_three():
    def res(rows):
        return dict(staging=[dict(points=n, voxels=n, staging=m, normals_ms=ms)
                             for n, per in enumerate(rows) for m, ms in enumerate(per)])
    # the packed walk wins on the geometric mean even where staging wins one size
    assert autotune.choose_staging(res([(1.0, 1.1, 0.7), (2.0, 1.8, 1.5), (4.0, 4.2, 3.0)])) == 2
    assert autotune.choose_staging(res([(1.0, 1.1, 1.2), (2.0, 2.1, 2.3)])) == 0
    assert "kNeighborStaging = 2;" in autotune.header_text({"voxel": [(BIG, 0)], "cell": [(BIG, 0)]},
                                                             None, 2)


def test_batch_workload_holds_exactly_n_points_in_two_clouds_or_more():
    import numpy as np
    from spatialrust_b200 import synthetic
    for n in (20_000, 150_000):
        x, y, z, offsets, leaves, radii = autotune.batch_clouds(n)
        assert len(x) == len(y) == len(z) == n
        assert offsets[0] == 0 and offsets[-1] == n and np.all(np.diff(offsets) > 0)
        assert len(offsets) - 1 == len(leaves) == len(radii) >= 2
        assert np.allclose(radii, 5.0 * leaves)
    # the clouds are the first clouds of the full batch generator
    few, lv, _ = synthetic.batched_uneven(256, seed=3, max_points=50_000)
    assert len(few) >= 2 and sum(c.n for c in few) >= 50_000
    assert sum(c.n for c in few[:-1]) < 50_000 or len(few) == 2
    head, lv_all, _ = synthetic.batched_uneven(256, seed=3, scale=0.01)
    assert np.array_equal(lv, lv_all[:len(few)])
