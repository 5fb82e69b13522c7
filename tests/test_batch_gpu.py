"""Many clouds in one chain (cloud id in the high key bits) vs each cloud alone.

Bar: every cloud's voxel keys, counts and centroids, and its normals and
neighbour counts, are bit-identical alone and in the mix -- a cloud's points
keep their relative order through the stable sorts, so its sums and its
candidate order are the same -- and agree with the oracle."""
import numpy as np
import pytest

import oracle
from spatialrust_b200 import _native, synthetic

pytestmark = pytest.mark.gpu


def device_concat(torch, clouds):
    cols = [np.concatenate([getattr(c, k) for c in clouds]) for k in ("x", "y", "z", "intensity")]
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in cols]
    offsets = np.concatenate([[0], np.cumsum([c.n for c in clouds])]).astype(np.int64)
    return dev, offsets


def run_batch(ctx, torch, clouds, leaves, radii, viewpoints=None):
    dev, offsets = device_concat(torch, clouds)
    keep = _native._Keep()
    pts = _native.make_cloud(dev[0], dev[1], dev[2], [dev[3]], keep)
    ctx.batch_voxel_normals_enqueue(pts, offsets, leaves, radii, 3, viewpoints)
    voff = ctx.batch_voxel_offsets()
    out = ctx.frame_fetch(int(offsets[-1]), n_attrs=1)
    return voff, out


def slice_out(out, a, b):
    return {k: (v[a:b] if k != "columns" else [c[a:b] for c in v])
            for k, v in out.items() if k != "stats"}


def test_batch_equals_each_cloud_alone(cuda_ctx):
    import torch
    rng = np.random.default_rng(77)
    clouds = [synthetic.georef_scan(int(n), seed=100 + i, offset=rng.uniform(0, 1e6, 3))
              for i, n in enumerate([30_000, 5_000, 120_000, 1, 64_000, 17])]
    leaves = [0.1, 0.2, 0.05, 0.1, 0.2, 0.5]
    radii = [5 * l for l in leaves]
    vps = [(0.0, 0.0, 100.0)] * len(clouds)
    voff, out = run_batch(cuda_ctx, torch, clouds, leaves, radii, vps)
    assert voff[0] == 0 and np.all(np.diff(voff) >= 0)
    alone_ctx = _native.Context(0)
    for b, c in enumerate(clouds):
        mine = slice_out(out, int(voff[b]), int(voff[b + 1]))
        ref = alone_ctx.voxel_normals(c.x, c.y, c.z, [c.intensity], leaf=leaves[b], radius=radii[b],
                                      viewpoint=vps[b])
        assert len(mine["counts"]) == len(ref["counts"]), f"cloud {b}: voxel count"
        assert np.array_equal(mine["counts"], ref["counts"])
        for g, r in zip(mine["columns"], ref["columns"]):
            assert np.array_equal(g, r), f"cloud {b}: centroids differ"
        for k in ("nx", "ny", "nz", "curvature", "neighbor_counts"):
            assert np.array_equal(mine[k], ref[k], equal_nan=True), f"cloud {b}: {k} differs"
    alone_ctx.close()


def test_batch_matches_oracle(cuda_ctx):
    import torch
    clouds = [synthetic.georef_scan(40_000, seed=5), synthetic.uniform_cube(30_000, seed=6, extent=20.0)]
    leaves, radii = [0.1, 0.5], [0.5, 1.5]
    voff, out = run_batch(cuda_ctx, torch, clouds, leaves, radii)
    for b, c in enumerate(clouds):
        mine = slice_out(out, int(voff[b]), int(voff[b + 1]))
        vox = oracle.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=leaves[b])
        assert np.array_equal(mine["counts"], vox.counts)
        for g, r in zip(mine["columns"], vox.fields):
            assert np.array_equal(g, r)
        ref = oracle.radius_normals_fp64(vox.x, vox.y, vox.z, radii[b], 3)
        assert np.array_equal(mine["neighbor_counts"], ref.counts)


def test_batch_with_empty_clouds(cuda_ctx):
    import torch
    a = synthetic.uniform_cube(10_000, seed=8, extent=10.0)
    b = synthetic.uniform_cube(12_000, seed=9, extent=10.0)
    empty = synthetic.uniform_cube(0, seed=1)
    voff, out = run_batch(cuda_ctx, torch, [empty, a, empty, empty, b, empty], [1.0] * 6, [2.0] * 6)
    assert voff[0] == voff[1] == 0
    assert voff[2] == voff[3] == voff[4] > 0
    assert voff[5] == voff[6] == len(out["counts"])
    assert int(out["counts"][: voff[2]].sum()) == a.n
    assert int(out["counts"][voff[4]:].sum()) == b.n


def test_batch_rejects_bad_offsets(cuda_ctx):
    import torch
    c = synthetic.uniform_cube(1000, seed=3)
    dev, _ = device_concat(torch, [c])
    keep = _native._Keep()
    pts = _native.make_cloud(dev[0], dev[1], dev[2], [dev[3]], keep)
    with pytest.raises(_native.BufferLengthMismatch):
        cuda_ctx.batch_voxel_normals_enqueue(pts, [0, 500], [1.0], [2.0])
    with pytest.raises(_native.InvalidArgument):
        cuda_ctx.batch_voxel_normals_enqueue(pts, [0, 600, 500, 1000], [1.0] * 3, [2.0] * 3)


def test_chain_graph_replays_match_enqueue():
    import torch
    ctx = _native.Context(0)
    clouds = [synthetic.georef_scan(20_000, seed=21), synthetic.georef_scan(7_000, seed=22)]
    leaves, radii = [0.1, 0.2], [0.5, 1.0]
    dev, offsets = device_concat(torch, clouds)
    keep = _native._Keep()
    pts = _native.make_cloud(dev[0], dev[1], dev[2], [dev[3]], keep)
    n = int(offsets[-1])
    ctx.batch_voxel_normals_enqueue(pts, offsets, leaves, radii, count_shell=False)
    ref = ctx.frame_fetch(n, n_attrs=1)
    ref_off = ctx.batch_voxel_offsets()
    g = ctx.chain_graph(pts, leaves, radii, offsets=offsets)
    for _ in range(3):
        g.launch()
    got = ctx.frame_fetch(n, n_attrs=1)
    assert np.array_equal(ctx.batch_voxel_offsets(), ref_off)
    for a, b in zip(got["columns"], ref["columns"]):
        assert np.array_equal(a, b)
    for k in ("nx", "nz", "curvature", "neighbor_counts"):
        assert np.array_equal(got[k], ref[k], equal_nan=True)
    g.close()
    # single cloud
    single = _native.make_cloud(dev[0][:clouds[0].n], dev[1][:clouds[0].n], dev[2][:clouds[0].n],
                                [dev[3][:clouds[0].n]], keep)
    g1 = ctx.chain_graph(single, [0.1], [0.5])
    g1.launch()
    got1 = ctx.frame_fetch(clouds[0].n, n_attrs=1)
    ref1 = ctx.voxel_normals(clouds[0].x, clouds[0].y, clouds[0].z, [clouds[0].intensity], leaf=0.1,
                             radius=0.5)
    assert np.array_equal(got1["columns"][0], ref1["columns"][0])
    assert np.array_equal(got1["nx"], ref1["nx"], equal_nan=True)
    g1.close()
    ctx.close()


def test_thousand_tiny_clouds_equal_alone():
    # the serving loop's shape: up to 1024 small requests in one chain, some
    # empty or single points; every cloud must match its own chain
    import torch
    rng = np.random.default_rng(91)
    sizes = rng.integers(0, 600, 1000)
    sizes[::97] = 0
    sizes[5::101] = 1
    clouds = [synthetic.georef_scan(int(n), seed=500 + i, offset=rng.uniform(0, 1e5, 3))
              if n else synthetic.uniform_cube(0, seed=1) for i, n in enumerate(sizes)]
    leaves = rng.choice([0.1, 0.2, 0.5], len(clouds)).tolist()
    radii = [4 * l for l in leaves]
    ctx = _native.Context(0)
    voff, out = run_batch(ctx, torch, clouds, leaves, radii)
    assert voff[-1] == len(out["counts"])
    alone = _native.Context(0)
    for b in rng.choice(len(clouds), 60, replace=False):
        c = clouds[b]
        mine = slice_out(out, int(voff[b]), int(voff[b + 1]))
        if c.n == 0:
            assert voff[b] == voff[b + 1]
            continue
        ref = alone.voxel_normals(c.x, c.y, c.z, [c.intensity], leaf=leaves[b], radius=radii[b])
        assert np.array_equal(mine["counts"], ref["counts"]), f"cloud {b}"
        for g, r in zip(mine["columns"], ref["columns"]):
            assert np.array_equal(g, r), f"cloud {b}"
        for k in ("nx", "ny", "nz", "curvature", "neighbor_counts"):
            assert np.array_equal(mine[k], ref[k], equal_nan=True), f"cloud {b}: {k}"
    alone.close()
    ctx.close()
