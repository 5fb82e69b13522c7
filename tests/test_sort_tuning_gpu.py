"""Every onesweep sort launch shape (keys per thread x blocks per SM x
threads per block, 8- or 9-bit digits) on the device, and the per-context
tuning tables.

Bar: the sort is a stable LSD radix sort in every shape, so the voxel and
normal outputs are byte-identical whichever shape a context picks, and the
voxel keys and counts equal the oracle's."""
import numpy as np
import pytest

import normal_parity
import oracle
import spatialrust_b200 as sr
from spatialrust_b200 import _native, autotune, synthetic

pytestmark = pytest.mark.gpu
BIG = (1 << 64) - 1


def chain(ctx, c, config):
    ctx.set_sort_tuning([(BIG, config)])
    try:
        return ctx.voxel_normals(c.x, c.y, c.z, [c.intensity], leaf=0.1, radius=0.5,
                                 viewpoint=(0, 0, 100), want_keys=True)
    finally:
        ctx.set_sort_tuning([])


def same(a, b):
    for k in ("keys", "counts", "nx", "ny", "nz", "curvature", "neighbor_counts"):
        assert np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)), k
    for g, r in zip(a["columns"], b["columns"]):
        assert np.array_equal(g.view(np.uint32), r.view(np.uint32))


@pytest.mark.parametrize("n", [1, 4097, 300_000, 3_000_000])
def test_every_shape_gives_identical_output(cuda_ctx, n):
    c = synthetic.georef_scan(n, seed=9)
    base = chain(cuda_ctx, c, 0)
    if n <= 300_000:
        vox = oracle.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=0.1)
        assert np.array_equal(base["keys"], vox.keys) and np.array_equal(base["counts"], vox.counts)
    for cfg in range(1, len(_native.sort_configs())):
        same(chain(cuda_ctx, c, cfg), base)


def test_tuning_table_selects_by_size(cuda_ctx):
    c = synthetic.georef_scan(200_000, seed=10)
    ref = chain(cuda_ctx, c, 0)
    # one table per sort kind, with the size boundaries between the point and
    # the centroid counts
    cuda_ctx.set_sort_tuning([(150_000, 1), (BIG, 3)], "voxel")
    cuda_ctx.set_sort_tuning([(150_000, 2), (BIG, 0)], "cell")
    try:
        assert cuda_ctx.sort_tuning("voxel") == [(150_000, 1), (BIG, 3)]
        tables = cuda_ctx.sort_tuning()
        assert tables["voxel"] == [(150_000, 1), (BIG, 3)] and tables["cell"] == [(150_000, 2), (BIG, 0)]
        got = cuda_ctx.voxel_normals(c.x, c.y, c.z, [c.intensity], leaf=0.1, radius=0.5,
                                     viewpoint=(0, 0, 100), want_keys=True)
    finally:
        cuda_ctx.set_sort_tuning([])
    same(got, ref)


def test_tuning_table_arguments(cuda_ctx):
    default = cuda_ctx.sort_tuning()
    assert all(t and t[-1][0] == BIG for t in default.values())
    n_cfg = len(_native.sort_configs())
    for bad in ([(10, n_cfg)], [(10, -1)], [(100, 0), (100, 1)], [(i + 1, 0) for i in range(33)]):
        with pytest.raises(sr.InvalidArgument):
            cuda_ctx.set_sort_tuning(bad)
    assert cuda_ctx.sort_tuning() == default
    assert set(default) == {"voxel", "cell", "batch_voxel", "batch_cell"}
    cuda_ctx.set_sort_tuning([(1000, 2)], "cell")
    assert cuda_ctx.sort_tuning() == dict(default, cell=[(1000, 2)])
    cuda_ctx.set_sort_tuning([(1000, 6)], "batch_voxel")
    assert cuda_ctx.sort_tuning() == dict(default, cell=[(1000, 2)], batch_voxel=[(1000, 6)])
    cuda_ctx.set_sort_tuning([])
    assert cuda_ctx.sort_tuning() == default
    for kind in (-1, 4):
        assert (cuda_ctx._lib.srcu_set_sort_tuning(cuda_ctx._h, kind, None, None, 0)
                == _native.SRCU_ERR_INVALID_ARGUMENT)


def test_autotuner_measures_every_shape():
    res = autotune.measure(sizes=(20_000, 150_000), reps=2, warmup=1)
    n_cfg = len(res["configs"])
    # every shape on the scan and on a batch of clouds, at both sizes
    assert len(res["runs"]) == 2 * 2 * n_cfg and len(res["staging"]) == 2 * len(autotune.WALK_MODES)
    assert all(r["voxel_sort_ms"] > 0 and r["cell_sort_ms"] > 0 for r in res["runs"])
    assert all(r["clouds"] >= 2 for r in res["runs"] if r["workload"] == "batch")
    for kind in autotune.KINDS:
        table = autotune.choose(res, kind)
        assert table[-1][0] == BIG and all(0 <= c < n_cfg for _, c in table)


# ---- digit width ---------------------------------------------------------------

def wide_batch(scale=0.02, count=100):
    """Clouds of the uneven batch generator: the cloud id above each cloud's key
    makes the batch keys wide enough that 9-bit digits save a pass (34 bits
    per cloud + 7 cloud bits: 5 nine-bit passes instead of 6)."""
    import torch
    clouds, leaves, radii = synthetic.batched_uneven(count, seed=3, scale=scale)
    sizes = np.array([c.n for c in clouds])
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    cols = [torch.from_numpy(np.concatenate([getattr(c, k) for c in clouds])).cuda()
            for k in ("x", "y", "z", "intensity")]
    return clouds, leaves, radii, offsets, cols


def batch_chain(ctx, pts, offsets, leaves, radii, config):
    ctx.set_sort_tuning([(BIG, config)])
    try:
        ctx.batch_voxel_normals_enqueue(pts, offsets, leaves.tolist(), radii.tolist(), 3,
                                        [(0.0, 0.0, 100.0)] * len(leaves), count_shell=False)
        voff = ctx.batch_voxel_offsets()
        out = ctx.frame_fetch(int(voff[-1]), n_attrs=1)
        info = ctx.chain_info()
    finally:
        ctx.set_sort_tuning([])
    return out, info


def test_nine_bit_digits_save_passes_and_change_nothing(cuda_ctx):
    clouds, leaves, radii, offsets, cols = wide_batch()
    keep = _native._Keep()
    pts = _native.make_cloud(cols[0], cols[1], cols[2], [cols[3]], keep)
    cfgs = _native.sort_configs()
    base, info0 = batch_chain(cuda_ctx, pts, offsets, leaves, radii, 0)
    kv, kc = info0["voxel_key_bits"], info0["cell_key_bits"]
    assert -(-kv // 9) < -(-kv // 8), f"the batch's voxel keys ({kv} bits) must gain from 9-bit digits"
    for cfg in range(1, len(cfgs)):
        got, info = batch_chain(cuda_ctx, pts, offsets, leaves, radii, cfg)
        for k in ("counts", "nx", "ny", "nz", "curvature", "neighbor_counts"):
            assert np.array_equal(got[k].view(np.uint8), base[k].view(np.uint8)), (cfg, k)
        for g, r in zip(got["columns"], base["columns"]):
            assert np.array_equal(g.view(np.uint32), r.view(np.uint32)), cfg
        # passes: one per digit that is not the same for every key, so at most
        # ceil(bits / width), with the width the shape takes for these keys
        width = lambda bits: 9 if cfgs[cfg]["digit_bits"] == 9 and -(-bits // 9) < -(-bits // 8) else 8
        assert info["voxel_sort_passes"] <= -(-kv // width(kv)), cfg
        assert info["cell_sort_passes"] <= -(-kc // width(kc)), cfg
        if cfgs[cfg]["digit_bits"] == 9:
            assert info["voxel_sort_passes"] < info0["voxel_sort_passes"], (cfg, info, info0)
    # the batch against the oracle, cloud by cloud, for the 9-bit shape
    got, _ = batch_chain(cuda_ctx, pts, offsets, leaves, radii, 6)
    voff = cuda_ctx.batch_voxel_offsets()
    for b in (0, len(clouds) // 2, len(clouds) - 1):
        c, leaf = clouds[b], float(leaves[b])
        a, e = int(voff[b]), int(voff[b + 1])
        vox = oracle.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=leaf)
        assert np.array_equal(got["counts"][a:e], vox.counts), b
        for g, r in zip(got["columns"], vox.fields):
            assert np.max(np.abs(g[a:e].astype(np.float64) - r)) <= 1e-5 * leaf, b


def test_single_cloud_wide_keys_take_nine_bit_digits(cuda_ctx):
    # one cloud at a fine leaf: 45-bit voxel keys sort in 5 nine-bit passes
    # instead of 6 eight-bit ones, with the same output
    c = synthetic.georef_scan(400_000, seed=12)
    outs = {}
    for cfg in (0, 6, 7):
        cuda_ctx.set_sort_tuning([(BIG, cfg)])
        try:
            cols, keys, counts = cuda_ctx.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=0.004,
                                                         want_keys=True)
            outs[cfg] = (cols, keys, counts, cuda_ctx.chain_info())
        finally:
            cuda_ctx.set_sort_tuning([])
    kv = outs[0][3]["voxel_key_bits"]
    assert kv == 45
    for cfg in (6, 7):
        cols, keys, counts, info = outs[cfg]
        assert np.array_equal(keys, outs[0][1]) and np.array_equal(counts, outs[0][2])
        for g, r in zip(cols, outs[0][0]):
            assert np.array_equal(g.view(np.uint32), r.view(np.uint32))
        assert info["voxel_sort_passes"] == 5 and outs[0][3]["voxel_sort_passes"] == 6
    vox = oracle.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=0.004)
    assert np.array_equal(outs[6][1], vox.keys) and np.array_equal(outs[6][2], vox.counts)
