"""Every onesweep sort launch shape (keys per thread x blocks per SM) on the
device, and the per-context tuning table.

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
        assert cuda_ctx.sort_tuning() == {"voxel": [(150_000, 1), (BIG, 3)],
                                          "cell": [(150_000, 2), (BIG, 0)]}
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
    cuda_ctx.set_sort_tuning([(1000, 2)], "cell")
    assert cuda_ctx.sort_tuning() == {"voxel": default["voxel"], "cell": [(1000, 2)]}
    cuda_ctx.set_sort_tuning([])
    assert cuda_ctx.sort_tuning() == default
    assert cuda_ctx._lib.srcu_set_sort_tuning(cuda_ctx._h, 2, None, None, 0) == _native.SRCU_ERR_INVALID_ARGUMENT


def test_autotuner_measures_every_shape():
    res = autotune.measure(sizes=(20_000, 150_000), reps=2, warmup=1)
    n_cfg = len(res["configs"])
    assert len(res["runs"]) == 2 * n_cfg and len(res["staging"]) == 2 * len(autotune.WALK_MODES)
    assert all(r["voxel_sort_ms"] > 0 and r["cell_sort_ms"] > 0 for r in res["runs"])
    for kind in ("voxel", "cell"):
        table = autotune.choose(res, kind)
        assert table[-1][0] == BIG and all(0 <= c < n_cfg for _, c in table)


# ---- the normals kernel's staged neighbour gather ---------------------------

def normals_with(ctx, x, y, z, staging, **kw):
    ctx.set_neighbor_staging(staging)
    try:
        return ctx.radius_normals(x, y, z, **kw)
    finally:
        ctx.set_neighbor_staging(-1)


@pytest.mark.parametrize("case", ["georef_centroids", "dense_unstageable", "shapes"])
def test_staged_gather_is_identical(cuda_ctx, case):
    if case == "georef_centroids":
        c = synthetic.georef_scan(400_000, seed=11)
        v = oracle.voxel_centroid(c.x, c.y, c.z, leaf=0.1)
        x, y, z, kw = v.x, v.y, v.z, dict(radius=0.5, viewpoint=(0, 0, 100))
    elif case == "dense_unstageable":
        # thousands of points per column: the strips exceed the warp's staging
        # buffer and are read from global memory
        p = np.random.default_rng(12).uniform(0, 2, (200_000, 3)).astype(np.float32)
        x, y, z, kw = p[:, 0], p[:, 1], p[:, 2], dict(radius=0.5)
    else:
        c = synthetic.shapes_scene(300_000, seed=13)
        x, y, z, kw = c.x, c.y, c.z, dict(radius=0.3, viewpoint=(50, 50, 150))
    a = normals_with(cuda_ctx, x, y, z, 0, **kw)
    b = normals_with(cuda_ctx, x, y, z, 1, **kw)
    for u, w in zip(a[:5], b[:5]):
        assert np.array_equal(np.asarray(u).view(np.uint32), np.asarray(w).view(np.uint32))
    assert a[5] == b[5]


def test_staged_gather_in_the_chain_and_batches(cuda_ctx):
    c = synthetic.georef_scan(250_000, seed=14)
    cuda_ctx.set_neighbor_staging(1)
    try:
        got = cuda_ctx.voxel_normals(c.x, c.y, c.z, [c.intensity], leaf=0.1, radius=0.5,
                                     viewpoint=(0, 0, 100), want_keys=True)
    finally:
        cuda_ctx.set_neighbor_staging(-1)
    same(got, cuda_ctx.voxel_normals(c.x, c.y, c.z, [c.intensity], leaf=0.1, radius=0.5,
                                     viewpoint=(0, 0, 100), want_keys=True))


def test_staged_gather_without_shell_count(cuda_ctx):
    # the device-resident chain without shell counting (the bench's variant)
    import torch
    c = synthetic.georef_scan(300_000, seed=15)
    keep = _native._Keep()
    cloud = _native.make_cloud(*[torch.from_numpy(a).cuda() for a in (c.x, c.y, c.z)], (), keep)
    out = []
    for mode in (0, 1):
        cuda_ctx.set_neighbor_staging(mode)
        try:
            cuda_ctx.voxel_normals_enqueue(cloud, 0.1, None, 0.5, 3, (0, 0, 100), count_shell=False)
            v, stats = cuda_ctx.frame_check()
            out.append((v, stats, cuda_ctx.frame_fetch(c.n)))
        finally:
            cuda_ctx.set_neighbor_staging(-1)
    (va, sa, a), (vb, sb, b) = out
    assert va == vb and sa == sb
    for k in ("nx", "ny", "nz", "curvature", "neighbor_counts"):
        assert np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)), k


def test_staging_switch_arguments(cuda_ctx):
    builtin = cuda_ctx.neighbor_staging()
    assert builtin in (0, 1, 2)
    for mode in (0, 1, 2):
        cuda_ctx.set_neighbor_staging(mode)
        assert cuda_ctx.neighbor_staging() == mode
    for bad in (3, -2):
        with pytest.raises(sr.InvalidArgument):
            cuda_ctx.set_neighbor_staging(bad)
    cuda_ctx.set_neighbor_staging(-1)
    assert cuda_ctx.neighbor_staging() == builtin


# ---- the packed neighbour walk (the L1 walk in f32x2 arithmetic) -------------

PACKED = 2


@pytest.mark.parametrize("case", ["georef_centroids", "dense", "shapes", "include_self"])
def test_packed_walk_is_bit_identical_and_meets_the_oracle(cuda_ctx, case):
    # the same IEEE operations on each half of every packed instruction, in the
    # L1 walk's order: every output bit-identical to walk 0, and the FP64
    # oracle's bar met
    inc = case == "include_self"
    if case in ("georef_centroids", "include_self"):
        c = synthetic.georef_scan(400_000, seed=11)
        v = oracle.voxel_centroid(c.x, c.y, c.z, leaf=0.1)
        x, y, z, r, vp = v.x, v.y, v.z, 0.5, (0, 0, 100)
    elif case == "dense":  # ~2,000 neighbours per point, 3-D
        p = np.random.default_rng(12).uniform(0, 2, (30_000, 3)).astype(np.float32)
        x, y, z, r, vp = p[:, 0], p[:, 1], p[:, 2], 0.5, None
    else:
        c = synthetic.shapes_scene(300_000, seed=13)
        x, y, z, r, vp = c.x, c.y, c.z, 0.3, (50, 50, 150)
    a = normals_with(cuda_ctx, x, y, z, 0, radius=r, viewpoint=vp, include_self=inc)
    b = normals_with(cuda_ctx, x, y, z, PACKED, radius=r, viewpoint=vp, include_self=inc)
    for u, w in zip(a[:5], b[:5]):
        assert np.array_equal(np.asarray(u).view(np.uint32), np.asarray(w).view(np.uint32))
    assert a[5] == b[5]
    ref = oracle.radius_normals_fp64(x, y, z, r, 3, vp, include_self=inc)
    normal_parity.check_against_fp64(*b[:5], ref, x, y, z, vp, b[5], include_self=inc,
                                     label=f"packed {case}")


def test_packed_walk_batch_equals_alone(cuda_ctx):
    import torch
    rng = np.random.default_rng(78)
    clouds = [synthetic.georef_scan(int(n), seed=200 + i, offset=rng.uniform(0, 1e6, 3))
              for i, n in enumerate([30_000, 120_000, 7, 64_000])]
    leaves = [0.1, 0.05, 0.1, 0.2]
    radii = [5 * l for l in leaves]
    cols = [np.concatenate([getattr(c, k) for c in clouds]) for k in ("x", "y", "z", "intensity")]
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in cols]
    offsets = np.concatenate([[0], np.cumsum([c.n for c in clouds])]).astype(np.int64)
    keep = _native._Keep()
    pts = _native.make_cloud(dev[0], dev[1], dev[2], [dev[3]], keep)
    ctx = _native.Context(0)
    ctx.set_neighbor_staging(PACKED)
    ctx.batch_voxel_normals_enqueue(pts, offsets, leaves, radii, 3, [(0.0, 0.0, 100.0)] * 4)
    voff = ctx.batch_voxel_offsets()
    out = ctx.frame_fetch(int(offsets[-1]), n_attrs=1)
    for b, c in enumerate(clouds):
        ref = ctx.voxel_normals(c.x, c.y, c.z, [c.intensity], leaf=leaves[b], radius=radii[b],
                                viewpoint=(0.0, 0.0, 100.0))
        a_, e_ = int(voff[b]), int(voff[b + 1])
        for k in ("nx", "ny", "nz", "curvature", "neighbor_counts"):
            assert np.array_equal(out[k][a_:e_], ref[k], equal_nan=True), f"cloud {b}: {k}"
    ctx.close()


def test_packed_walk_plane_covariances(cuda_ctx):
    c = synthetic.georef_scan(300_000, seed=16)
    a = cuda_ctx.plane_covariances(c.x, c.y, c.z, 0.3, 1e-3)
    cuda_ctx.set_neighbor_staging(PACKED)
    try:
        b = cuda_ctx.plane_covariances(c.x, c.y, c.z, 0.3, 1e-3)
    finally:
        cuda_ctx.set_neighbor_staging(-1)
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    fb = np.all(a[:, 3:] == 0, axis=1) & np.all(a[:, :3] == a[:, :1], axis=1)
    assert np.array_equal(fb, np.all(b[:, 3:] == 0, axis=1) & np.all(b[:, :3] == b[:, :1], axis=1))
    assert np.max(np.abs(a - b)) <= 2e-4
