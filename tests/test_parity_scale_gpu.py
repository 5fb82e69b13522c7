"""Voxel and normal parity at the benchmark sizes, against the oracle.

  - the full 2,000,000-point georeferenced scan (offset (450000, 3900000, 50) m,
    f32 local coordinates), voxel leaf 0.1 and 0.5 m (1.82M and 417k
    centroids), then radius normals r 0.5 on the centroids with the viewpoint
    at origin + (0, 0, 100) -- MvpPipeline::run's chain (mvp.rs:193-226);
  - the full 5,000,000-point shapes scene, radius normals r 0.3, uncapped
    (neighbourhoods of up to ~1,000 points on the cylinders);
  - nine clouds sliced out of the real 256-cloud, 52M-point batch run as one
    batched chain: for each leaf (0.05, 0.1, 0.2 m) its smallest, median and
    largest cloud (10k-1M points), r = 5 x leaf.

Voxels: keys (where fetched) and counts bit-exact, centroids within 1e-5 x
leaf of the oracle's (voxel.rs:464-540).  Normals: the bar of
normal_parity.py on the normals stage's own input (the GPU centroids) against
the FP64 oracle (normal.rs:321-573 neighbour sets, FP64 covariance and
Jacobi): counts exact, valid set exact, <= 1e-4 rad where the eigengap is
>= 1e-3, the ill-conditioned share and its looser bound asserted."""
import numpy as np
import pytest

import normal_parity
import oracle
from spatialrust_b200 import _native, synthetic

pytestmark = pytest.mark.gpu
VIEWPOINT = (0.0, 0.0, 100.0)
# Ill-conditioned points (relative eigengap < 1e-3) of each input, from the FP64
# oracle's eigengaps on these seeded clouds: (count, solved points).
ILL_C1 = {0.1: (4, 1_629_258), 0.5: (4, 57_353)}
ILL_C3 = {74: (0, 0), 180: (6, 483), 156: (4415, 516_850), 186: (0, 4), 26: (185, 8228),
          84: (151, 733_647), 225: (2, 217), 229: (292, 111_174), 21: (9, 616_665)}


def check_voxels(cols, counts, vox, leaf, keys=None, label=""):
    if keys is not None:
        assert np.array_equal(keys, vox.keys), f"{label}: voxel keys"
    assert np.array_equal(counts, vox.counts), f"{label}: voxel counts"
    for g, r in zip(cols, vox.fields):
        assert np.max(np.abs(g.astype(np.float64) - r)) <= 1e-5 * leaf, f"{label}: centroids"


@pytest.mark.parametrize("leaf", [0.1, 0.5])
def test_georeferenced_2m_chain_full_size(leaf):
    c = synthetic.georef_scan(2_000_000, seed=1)
    ctx = _native.Context(0)
    out = ctx.voxel_normals(c.x, c.y, c.z, [c.intensity], leaf=leaf, radius=0.5,
                            viewpoint=VIEWPOINT, want_keys=True)
    ctx.close()
    vox = oracle.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=leaf)
    check_voxels(out["columns"], out["counts"], vox, leaf, out["keys"], f"C1 leaf {leaf}")
    gx, gy, gz = out["columns"][:3]
    ref = oracle.radius_normals_fp64(gx, gy, gz, 0.5, 3, VIEWPOINT)
    rep = normal_parity.check_against_fp64(out["nx"], out["ny"], out["nz"], out["curvature"],
                                           out["neighbor_counts"], ref, gx, gy, gz, VIEWPOINT,
                                           out["stats"], label=f"C1 leaf {leaf}")
    assert rep["points"] == (1_820_918 if leaf == 0.1 else 417_439)
    assert (rep["ill_conditioned"], rep["solved"]) == ILL_C1[leaf]
    print(f"C1 leaf {leaf}:", rep)


def test_shapes_5m_full_size():
    c = synthetic.shapes_scene(5_000_000, seed=2)
    ctx = _native.Context(0)
    nx, ny, nz, curv, counts, stats = ctx.radius_normals(c.x, c.y, c.z, 0.3, 3, None)
    ctx.close()
    ref = oracle.radius_normals_fp64(c.x, c.y, c.z, 0.3, 3, None)
    rep = normal_parity.check_against_fp64(nx, ny, nz, curv, counts, ref, c.x, c.y, c.z, None,
                                           stats, label="C2")
    assert counts.max() > 900  # the uncapped cylinder neighbourhoods are in the check
    assert rep["ill_conditioned"] == 0 and rep["solved"] == 5_000_000
    print("C2 shapes 5M:", rep)


def test_batched_256_clouds_sliced():
    import torch
    clouds, leaves, radii = synthetic.batched_uneven(256, seed=3)
    sizes = np.array([c.n for c in clouds])
    cols = [torch.from_numpy(np.concatenate([getattr(c, k) for c in clouds])).cuda()
            for k in ("x", "y", "z", "intensity")]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    keep = _native._Keep()
    ctx = _native.Context(0)
    pts = _native.make_cloud(cols[0], cols[1], cols[2], [cols[3]], keep)
    ctx.batch_voxel_normals_enqueue(pts, offsets, leaves.tolist(), radii.tolist(), 3,
                                    [VIEWPOINT] * len(clouds), count_shell=False)
    voff = ctx.batch_voxel_offsets()
    out = ctx.frame_fetch(int(voff[-1]), n_attrs=1)
    ctx.close()
    del cols
    picks = []
    for leaf in (0.05, 0.1, 0.2):
        idx = np.flatnonzero(np.isclose(leaves, leaf))
        idx = idx[np.argsort(sizes[idx], kind="stable")]
        picks += [int(idx[0]), int(idx[len(idx) // 2]), int(idx[-1])]
    assert sizes[picks].min() < 20_000 and sizes[picks].max() > 700_000
    for b in picks:
        c, leaf, r = clouds[b], float(leaves[b]), float(radii[b])
        a, e = int(voff[b]), int(voff[b + 1])
        label = f"C3 cloud {b} ({c.n} points, leaf {leaf})"
        vox = oracle.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=leaf)
        check_voxels([col[a:e] for col in out["columns"]], out["counts"][a:e], vox, leaf,
                     label=label)
        gx, gy, gz = (out["columns"][k][a:e] for k in range(3))
        ref = oracle.radius_normals_fp64(gx, gy, gz, r, 3, VIEWPOINT)
        rep = normal_parity.check_against_fp64(out["nx"][a:e], out["ny"][a:e], out["nz"][a:e],
                                               out["curvature"][a:e],
                                               out["neighbor_counts"][a:e], ref, gx, gy, gz,
                                               VIEWPOINT, label=label)
        assert (rep["ill_conditioned"], rep["solved"]) == ILL_C3[b], label
        print(label, rep)
