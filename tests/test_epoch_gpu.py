"""The look-back epoch restart before the 32-bit wrap.

Every chain tags the look-back words and hash slots it publishes with an
epoch that advances by 64 per chain.  A context placed just below the wrap
(srcu_debug_set_epoch) must clear its tagged arrays and restart the epoch
before the first chain whose tags would pass 2^32 - 1, and every result --
a large chain, then a small one whose tiles the large one's stale words
still cover -- must be bit-identical to a fresh context's."""
import numpy as np
import pytest

from spatialrust_b200 import _native, synthetic

pytestmark = pytest.mark.gpu

NEAR_WRAP = 0xFFFFFF40  # three chains below the wrap: two run, the third restarts


def chain(ctx, c, leaf):
    return ctx.voxel_normals(c.x, c.y, c.z, [c.intensity], leaf=leaf, radius=5 * leaf,
                             viewpoint=(0.0, 0.0, 100.0), want_keys=True)


def same(a, b):
    assert np.array_equal(a["keys"], b["keys"]) and np.array_equal(a["counts"], b["counts"])
    for g, r in zip(a["columns"], b["columns"]):
        assert np.array_equal(g, r)
    for k in ("nx", "ny", "nz", "curvature", "neighbor_counts"):
        assert np.array_equal(a[k], b[k], equal_nan=True), k


def test_epoch_restart_is_invisible_in_results():
    big = synthetic.georef_scan(1_000_000, seed=21)
    small = synthetic.georef_scan(60_000, seed=22)
    fresh = _native.Context(0)
    ref_big, ref_small = chain(fresh, big, 0.1), chain(fresh, small, 0.1)
    fresh.close()
    ctx = _native.Context(0)
    chain(ctx, big, 0.1)  # size every buffer at epoch 64
    ctx.debug_set_epoch(NEAR_WRAP)
    for _ in range(3):  # chains at NEAR_WRAP + 64, + 128, then the restart
        same(chain(ctx, big, 0.1), ref_big)
        same(chain(ctx, small, 0.1), ref_small)
    epoch, restarts = ctx.debug_epoch()
    assert restarts == 1
    assert epoch == 4 * 64  # four chains since the restart
    ctx.close()


def test_graph_replays_across_the_restart():
    import torch
    c = synthetic.georef_scan(300_000, seed=23)
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (c.x, c.y, c.z, c.intensity)]
    keep = _native._Keep()
    pts = _native.make_cloud(dev[0], dev[1], dev[2], [dev[3]], keep)
    ref_ctx = _native.Context(0)
    ref_ctx.voxel_normals_enqueue(pts, 0.2, None, 1.0, 3, (0.0, 0.0, 100.0), count_shell=False)
    v_ref, _ = ref_ctx.frame_check()
    ref = ref_ctx.frame_fetch(c.n, n_attrs=1)
    ref_ctx.close()
    ctx = _native.Context(0)
    g = ctx.chain_graph(pts, [0.2], [1.0], viewpoints=[(0.0, 0.0, 100.0)])
    ctx.debug_set_epoch(NEAR_WRAP)
    for _ in range(5):
        g.launch()
        v, _ = ctx.frame_check()
        assert v == v_ref
        got = ctx.frame_fetch(c.n, n_attrs=1)
        for a, b in zip(got["columns"], ref["columns"]):
            assert np.array_equal(a, b)
        for k in ("nx", "ny", "nz", "curvature", "neighbor_counts"):
            assert np.array_equal(got[k], ref[k], equal_nan=True), k
    epoch, restarts = ctx.debug_epoch()
    assert restarts == 1 and epoch == 3 * 64
    g.close()
    ctx.close()
