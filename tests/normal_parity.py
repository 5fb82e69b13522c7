"""Shared normal-parity checks of the GPU tests against the FP64 oracle.

Bar (every config): neighbour counts exact (the f32 predicate of
kdtree.rs:544-549 evaluated exactly as the reference does); the valid set
exact; curvature within CURV_TOL; normals within ANGLE_TOL of the FP64
eigenvector, sign-matched by viewpoint, wherever the relative eigengap
(l1 - l0) / l2 is at least GAP_MIN.  Below GAP_MIN the normal is
ill-conditioned for any solver: those points are counted, their share must
stay under the config's ill_max, and their angle must stay under
ILL_ANGLE_TOL (the kernel solves them from FP64 moments, so the bound holds
down to gaps of ~1e-9; a gap of exactly 0 leaves the normal undefined and is
only counted).  The share is a property of the input, set by the FP64
oracle's eigengaps: dense surfaces have almost none (4 of 1.6M centroids on
the 2M-point scan at leaf 0.1), sparse clouds whose neighbourhoods hold 3-5
nearly collinear points have up to ~2.3% (ILL_MAX caps it at 3%)."""
import numpy as np

ANGLE_TOL = 1e-4      # rad, gap >= GAP_MIN
ILL_ANGLE_TOL = 1e-3  # rad, GAP_UNDEFINED < gap < GAP_MIN
CURV_TOL = 1e-5
GAP_MIN = 1e-3
GAP_UNDEFINED = 1e-9
ILL_MAX = 0.03        # largest share of ill-conditioned points of any test input


def angle_between(a, b):
    """Angle in radians via atan2(|a x b|, a . b) -- accurate near 0, unlike
    arccos of a dot product, which turns float32 rounding into ~1e-4 rad."""
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    a = a / np.linalg.norm(a, axis=1, keepdims=True)
    b = b / np.linalg.norm(b, axis=1, keepdims=True)
    return np.arctan2(np.linalg.norm(np.cross(a, b), axis=1), np.sum(a * b, axis=1))


def angle_errors(gpu, ref, points, viewpoint):
    """Angle between GPU and FP64 normals; sign-free where the viewpoint does
    not decide the sign robustly (or no viewpoint is given)."""
    err = angle_between(gpu, ref)
    sign_free = np.minimum(err, np.pi - err)
    if viewpoint is None:
        return sign_free
    view = np.asarray(viewpoint, np.float64)[None, :] - points.astype(np.float64)
    cos_view = np.abs(np.sum(ref * view, axis=1)) / np.linalg.norm(view, axis=1)
    ambiguous = cos_view < 1e-3
    err[ambiguous] = sign_free[ambiguous]
    return err


def check_against_fp64(nx, ny, nz, curv, counts, ref, x, y, z, viewpoint=None, stats=None,
                       ill_max=ILL_MAX, include_self=False, label=""):
    """Asserts the bar above for GPU outputs against an oracle.radius_normals_fp64
    result on the same points; returns a report dict."""
    assert np.array_equal(counts, ref.counts), \
        f"{label}: {np.count_nonzero(counts != ref.counts)} neighbour counts differ"
    if include_self:
        # fewer than 3 points (query included): (0, 0, +-1) exactly, as the oracle
        fb = ref.counts < 3
        solved = ~fb
        for g, r in ((nx, ref.nx), (ny, ref.ny), (nz, ref.nz)):
            assert np.array_equal(g[fb].astype(np.float64), r[fb]), f"{label}: fallback normals"
        assert np.all(curv[fb] == 0)
    else:
        solved = ~np.isnan(ref.nx)
        assert np.array_equal(~np.isnan(nx), solved), f"{label}: valid sets differ"
        assert np.all(curv[~solved] == 0)
    if stats is not None:
        assert stats["valid_count"] == int(solved.sum())
        assert stats["invalid_count"] == int((~solved).sum())
    pts = np.stack([x, y, z], 1)[solved]
    g = np.stack([nx, ny, nz], 1)[solved]
    err = angle_errors(g, ref.normals[solved], pts, viewpoint)
    gap = ref.gap[solved]
    well = gap >= GAP_MIN
    ill = ~well & (gap > GAP_UNDEFINED)
    undefined = gap <= GAP_UNDEFINED
    n = int(solved.sum())
    rep = dict(points=len(x), solved=n, max_err=float(err[well].max()) if well.any() else 0.0,
               ill_conditioned=int((~well).sum()), ill_fraction=float((~well).sum() / max(n, 1)),
               ill_max_err=float(err[ill].max()) if ill.any() else 0.0,
               undefined=int(undefined.sum()), shell=int(ref.shell.sum()),
               mean_neighbours=float(ref.counts.mean()) if len(x) else 0.0)
    if well.any():
        assert err[well].max() <= ANGLE_TOL, f"{label}: max angle error {err[well].max():.3e} rad"
    assert rep["ill_fraction"] <= ill_max, f"{label}: {rep['ill_conditioned']} ill-conditioned points"
    if ill.any():
        assert err[ill].max() <= ILL_ANGLE_TOL, \
            f"{label}: ill-conditioned max angle error {err[ill].max():.3e} rad"
    if n:
        assert np.max(np.abs(curv[solved] - ref.curvature[solved])) <= CURV_TOL, f"{label}: curvature"
    return rep
