"""Autotuner for the onesweep radix sort's launch shape.

libsrcuda.so is built with several launch shapes of the persistent onesweep
sort (keys per thread, and the blocks per SM its registers are capped for;
`_native.sort_configs()` lists them).  Which one is fastest depends on the
number of keys: small sorts want many small tiles so that every SM gets work,
large ones want long tiles that amortise the per-tile look-back.  This module
measures every shape on the real chain -- voxel centroid (voxel-key sort over
the input points) then radius normals (cell-key sort over the centroids) on a
georeferenced scan -- at one input size per size class, and picks per class
the shape with the least sort time.  The shapes cover keys per thread, blocks
per SM, threads per block (256 or 512) and digit width (8 bits, or 9 bits in
512-thread shapes: a thread per digit bin).  It also times the normals
kernel's three neighbour walks (range by range through L1, range by range from
shared memory filled by bulk copies, and the L1 walk in packed f32x2
arithmetic) over the same sizes and keeps the fastest.

Shapes and digit width are tuned twice: on one georeferenced scan, and on
batches of whole clouds from the uneven-cloud generator of the 256-cloud batch
workload (leaves 0.05/0.1/0.2 m, radius 5 x leaf), cut to the same sizes.  A
batch's keys carry the cloud id above each cloud's key, so they are wider,
and the 9-bit-digit shapes save a pass on them where they save none on one
scan; a context takes its batch tables for chains of more than one cloud.

    python -m spatialrust_b200.autotune                 # measure, print the table
    python -m spatialrust_b200.autotune --write         # ... and rewrite csrc/sort_tuning.h
    python -m spatialrust_b200.autotune --json out.json
    python -m spatialrust_b200.autotune --from-json out.json --write

A context starts with the table in csrc/sort_tuning.h; `Context.set_sort_tuning`
installs a measured one at run time.  No counterpart in the reference, whose
wgpu bitonic sort has fixed workgroup sizes.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

# Point counts measured: half-octave steps from 2^16 to 2^25.  Which shape is
# fastest is not smooth in the size -- the last wave of tiles over the
# persistent grid fills a different fraction of the SMs in each shape -- so the
# samples are dense.  Each chain gives two samples: the voxel sort at the
# point count and the cell sort at the voxel count.
SAMPLE_POINTS = tuple(int(round(2 ** (16 + k / 2))) for k in range(19))
LEAF = 0.1
RADIUS = 0.5
HYSTERESIS = 0.02  # keep the smaller size's shape unless another is this much faster
WALK_MODES = (0, 1, 2)  # srcu_set_neighbor_staging: L1, staged, packed
TABLE_MAX = 32     # SRCU_SORT_TUNING_MAX
BIG = (1 << 64) - 1
L2_FLUSH_BYTES = 256 << 20  # written before every timed chain: inputs start outside L2

_HEADER = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "sort_tuning.h")


def batch_clouds(n: int, seed: int = 3):
    """The first clouds of the uneven-cloud batch generator, the last one cut so
    that they hold n points: (x, y, z, offsets, leaves, radii)."""
    from . import synthetic

    clouds, leaves, radii = synthetic.batched_uneven(256, seed=seed, max_points=n)
    cols, offsets, total = ([], [], []), [0], 0
    for c in clouds:
        take = min(c.n, n - total)
        for col, a in zip(cols, (c.x, c.y, c.z)):
            col.append(a[:take])
        total += take
        offsets.append(total)
    x, y, z = (np.concatenate(col) for col in cols)
    k = len(offsets) - 1
    return x, y, z, np.array(offsets, np.int64), leaves[:k], radii[:k]


def measure(sizes=SAMPLE_POINTS, reps: int = 10, warmup: int = 3, seed: int = 1,
            device: int = 0, batch: bool = True) -> dict:
    """Sort device time (ms per chain) of every launch shape at every size,
    on one scan and (batch) on a batch of clouds of that size, and the
    normals kernel's time with each neighbour walk on the scan.

    Returns {"configs": [...], "runs": [{"workload", "points", "voxels",
    "clouds", "config", "voxel_sort_ms", "cell_sort_ms"}], "staging":
    [{"points", "voxels", "staging", "normals_ms"}]}."""
    import torch

    from . import _native, synthetic

    configs = _native.sort_configs()
    scan = synthetic.georef_scan(max(sizes), seed=seed)
    batch_src = batch_clouds(max(sizes)) if batch else None
    dev = torch.device("cuda", device)
    ctx = _native.Context(device)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    runs, staging = [], []

    def timed(enqueue, groups):
        for _ in range(warmup):
            enqueue()
        ctx.synchronize()
        ctx.profile_read(reset=True)
        ctx.profile_enable(groups)
        for _ in range(reps):
            flush.zero_()
            torch.cuda.synchronize(dev)
            enqueue()
            ctx.synchronize()
        prof = ctx.profile_read(reset=True)
        ctx.profile_enable([])
        return {g: prof[g]["total_ms"] / reps for g in groups}

    def shapes(workload, n, clouds, enqueue):
        for c in range(len(configs)):
            ctx.set_sort_tuning([(BIG, c)])
            t = timed(enqueue, ["voxel_sort", "cell_sort"])
            runs.append(dict(workload=workload, points=n, clouds=clouds,
                             voxels=int(ctx.chain_info()["voxels"]), config=c,
                             voxel_sort_ms=t["voxel_sort"], cell_sort_ms=t["cell_sort"]))
        ctx.set_sort_tuning([])

    try:
        for n in sizes:
            keep = _native._Keep()
            cols = [keep.add(torch.from_numpy(np.ascontiguousarray(a[:n])).to(dev))
                    for a in (scan.x, scan.y, scan.z)]
            cloud = _native.make_cloud(*cols, (), keep)

            def scan_chain():
                ctx.voxel_normals_enqueue(cloud, LEAF, None, RADIUS, 3, None, count_shell=False)

            shapes("scan", n, 1, scan_chain)
            for mode in WALK_MODES:
                ctx.set_neighbor_staging(mode)
                t = timed(scan_chain, ["normals"])
                staging.append(dict(points=n, voxels=int(ctx.chain_info()["voxels"]), staging=mode,
                                    normals_ms=t["normals"]))
            ctx.set_neighbor_staging(-1)
            del cols, cloud, keep
            if batch_src is not None:
                bx, by, bz, offsets, leaves, radii = batch_src
                # clouds [0, k) hold >= n points; two clouds at least, so that
                # the chain takes the batch tables
                k = max(2, int(np.searchsorted(offsets, n, side="left")))
                offs = np.minimum(offsets[:k + 1], n)
                if offs[1] >= n:
                    offs[1] = n // 2
                keep = _native._Keep()
                cols = [keep.add(torch.from_numpy(np.ascontiguousarray(a[:n])).to(dev))
                        for a in (bx, by, bz)]
                pts = _native.make_cloud(*cols, (), keep)

                def batch_chain():
                    ctx.batch_voxel_normals_enqueue(pts, offs, leaves[:k].tolist(),
                                                    radii[:k].tolist(), 3, None, count_shell=False)

                shapes("batch", n, k, batch_chain)
                del cols, pts, keep
    finally:
        ctx.set_sort_tuning([])
        ctx.set_neighbor_staging(-1)
        ctx.close()
    return dict(configs=configs, runs=runs, staging=staging)


KINDS = ("voxel", "cell", "batch_voxel", "batch_cell")


def samples(result: dict, kind: str) -> list:
    """[(size, [ms per shape])], ascending, for one sort kind: the voxel sorts
    ("voxel") or the cell sorts ("cell") of the scan chains, or the same of the
    batch chains ("batch_voxel", "batch_cell").  The size is the chain's point
    count for both sorts: the library picks a cell sort's shape before the
    voxel count is known on the host, from the same upper bound."""
    n_cfg = len(result["configs"])
    workload = "batch" if kind.startswith("batch_") else "scan"
    field = "voxel_sort_ms" if kind.endswith("voxel") else "cell_sort_ms"
    by = {}
    for r in result["runs"]:
        if r.get("workload", "scan") != workload:
            continue
        by.setdefault(r["points"], [None] * n_cfg)[r["config"]] = r[field]
    out = [(k, ms) for k, ms in by.items() if all(m is not None for m in ms)]
    return sorted(out, key=lambda t: t[0])


def choose(result: dict, kind: str, hysteresis: float = HYSTERESIS) -> list:
    """[(max_points, shape)] for one sort kind: walking its samples from small
    to large, the shape of the previous sample is kept while it is within
    `hysteresis` of the sample's fastest, else the fastest is taken; a change
    of shape between two samples puts the table boundary at their geometric
    mean."""
    pts = samples(result, kind)
    if not pts:
        return [(BIG, 0)]
    while True:
        table, cur = [], None
        for idx, (keys, ms) in enumerate(pts):
            best = int(np.argmin(ms))
            if cur is None or ms[cur] > ms[best] * (1.0 + hysteresis):
                if cur is not None and cur != best:
                    prev = pts[idx - 1][0]
                    table.append((int(np.sqrt(float(prev) * float(keys))), cur))
                cur = best
        table.append((BIG, cur))
        if len(table) <= TABLE_MAX:
            return table
        hysteresis *= 2.0


def choose_staging(result: dict) -> int:
    """The neighbour walk whose normals time, relative to walk 0 (L1), has the
    smallest geometric mean over the measured sizes (each size weighted
    equally); 0 when no other walk is faster on that mean, or without
    measurements."""
    by_n = {}
    for r in result.get("staging", []):
        by_n.setdefault(r["points"], {})[r["staging"]] = r["normals_ms"]
    best, best_score = 0, 0.0
    for mode in sorted({m for per in by_n.values() for m in per}):
        ratios = [per[mode] / per[0] for per in by_n.values()
                  if 0 in per and mode in per and per[0] > 0]
        if not ratios:
            continue
        score = float(np.mean(np.log(ratios)))
        if score < best_score:
            best, best_score = mode, score
    return best


def header_text(tables: dict, result: dict | None = None, staging: int = 0) -> str:
    lines = [
        "// sort_tuning.h -- the sort launch shape per input size that a context starts",
        "// with.  Written by `python -m spatialrust_b200.autotune --write` from its",
        "// measurements; srcu_set_sort_tuning replaces it per context.",
        "//",
        "// One table per sort kind: the voxel-key sort over the input points and the",
        "// cell-key sort over the radius-grid points, of one cloud and (Batch) of a",
        "// batch of clouds.  Entry k applies to sorts of at most k*SortTuneMaxPoints[k]",
        "// keys (the last entry to every larger sort); k*SortTuneConfig[k] indexes the",
        "// launch shapes of radix.cuh (kSortItems, kSortMinBlocks, kSortThreads,",
        "// kSortDigitBits).",
        "// kNeighborStaging: the normals kernel's neighbour walk -- range by range",
        "// through L1 (0), range by range from shared memory filled by bulk copies (1),",
        "// or the L1 walk in packed f32x2 arithmetic (2).",
    ]
    if result is not None:
        lines.append("//")
        lines.append("// Measured sort ms (georeferenced scan, leaf "
                     f"{LEAF}, radius {RADIUS}; batches of uneven clouds, leaf 0.05-0.2,")
        lines.append("// radius 5 x leaf; L2 flushed before every chain), per shape")
        lines.append("// (keys per thread x blocks per SM x threads / digit bits):")
        cfgs = result["configs"]
        shapes = "  ".join(f"{c['items_per_thread']}x{c['blocks_per_sm']}x{c.get('threads_per_block', 256)}"
                           f"/{c.get('digit_bits', 8)}" for c in cfgs)
        for kind in KINDS:
            rows = samples(result, kind)
            if not rows:
                continue
            lines.append(f"//   {kind} sort, points: {shapes}")
            for keys, ms in rows:
                lines.append(f"//   {keys:>9}  " + "  ".join(f"{m:6.4f}" for m in ms))
        if result.get("staging"):
            lines.append("// Normals kernel ms per chain, neighbour walk L1 / staged / packed:")
            by_n = {}
            for r in result["staging"]:
                by_n.setdefault(r["points"], {})[r["staging"]] = r["normals_ms"]
            for n, per in sorted(by_n.items()):
                lines.append(f"//   {n:>9}   " + " / ".join(
                    f"{per.get(m, float('nan')):6.3f}" for m in WALK_MODES))
    lines += [
        "#pragma once",
        "",
        "#include <cstdint>",
        "",
        "namespace srcu {",
        "",
    ]
    for kind, name in (("voxel", "Voxel"), ("cell", "Cell"), ("batch_voxel", "BatchVoxel"),
                       ("batch_cell", "BatchCell")):
        # without batch measurements, a batch kind takes its scan kind's table
        table = tables.get(kind) or tables[kind.replace("batch_", "")]
        lines += [
            f"constexpr uint32_t k{name}SortTuneCount = {len(table)};",
            f"constexpr uint64_t k{name}SortTuneMaxPoints[] = {{" + ", ".join(
                "UINT64_MAX" if m >= BIG else f"{m}ull" for m, _ in table) + "};",
            f"constexpr int32_t k{name}SortTuneConfig[] = {{" + ", ".join(
                str(c) for _, c in table) + "};",
        ]
    lines += [
        "// the normals kernel's neighbour walk (srcu_set_neighbor_staging)",
        f"constexpr int32_t kNeighborStaging = {int(staging)};",
        "",
        "}  // namespace srcu",
        "",
    ]
    return "\n".join(lines)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--sizes", type=int, nargs="*", default=list(SAMPLE_POINTS))
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--no-batch", action="store_true", help="tune on the scan alone")
    ap.add_argument("--json", help="write the measurements and the chosen table here")
    ap.add_argument("--write", action="store_true", help="rewrite csrc/sort_tuning.h")
    ap.add_argument("--from-json", help="take the measurements from an earlier --json run")
    args = ap.parse_args(argv)
    if args.from_json:
        with open(args.from_json) as f:
            result = json.load(f)
    else:
        result = measure(args.sizes, reps=args.reps, batch=not args.no_batch)
    tables = {kind: choose(result, kind) for kind in KINDS
              if kind in ("voxel", "cell") or samples(result, kind)}
    staging = choose_staging(result)
    result["tables"] = {k: [[m, c] for m, c in t] for k, t in tables.items()}
    result["neighbor_staging"] = staging
    for r in result["runs"]:
        print(f"{r.get('workload', 'scan'):5} points {r['points']:>9} voxels {r['voxels']:>9} "
              f"config {r['config']}: voxel sort {r['voxel_sort_ms']:.4f} ms  "
              f"cell sort {r['cell_sort_ms']:.4f} ms")
    for r in result.get("staging", []):
        print(f"points {r['points']:>9} voxels {r['voxels']:>9} staging {r['staging']}: "
              f"normals {r['normals_ms']:.4f} ms")
    for kind, table in tables.items():
        print(f"{kind} sort table:", table)
    print("neighbor staging:", staging)
    if args.json:
        with open(args.json, "w") as f:
            json.dump(result, f, indent=1)
    if args.write:
        with open(_HEADER, "w") as f:
            f.write(header_text(tables, result, staging))
    return 0

if __name__ == "__main__":
    sys.exit(main())
