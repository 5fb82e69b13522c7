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
per SM and threads per block (256 or 512: the first 256 threads own one digit
each).  Digit width stays at 8 bits.  It also times the normals kernel's three neighbour walks
(range by range through L1, range by range from shared memory filled by bulk
copies, each lane's ranges as one list with packed f32x2 arithmetic) over the
same sizes and keeps the fastest.

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


def measure(sizes=SAMPLE_POINTS, reps: int = 10, warmup: int = 3, seed: int = 1,
            device: int = 0) -> dict:
    """Sort device time (ms per chain) of every launch shape at every size,
    and the normals kernel's time with either neighbour gather.

    Returns {"configs": [...], "runs": [{"points", "voxels", "config",
    "voxel_sort_ms", "cell_sort_ms"}], "staging": [{"points", "voxels",
    "staging", "normals_ms"}]}."""
    import torch

    from . import _native, synthetic

    configs = _native.sort_configs()
    scan = synthetic.georef_scan(max(sizes), seed=seed)
    dev = torch.device("cuda", device)
    ctx = _native.Context(device)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    runs, staging = [], []

    def timed(groups):
        for _ in range(warmup):
            ctx.voxel_normals_enqueue(cloud, LEAF, None, RADIUS, 3, None, count_shell=False)
        ctx.synchronize()
        ctx.profile_read(reset=True)
        ctx.profile_enable(groups)
        for _ in range(reps):
            flush.zero_()
            torch.cuda.synchronize(dev)
            ctx.voxel_normals_enqueue(cloud, LEAF, None, RADIUS, 3, None, count_shell=False)
            ctx.synchronize()
        prof = ctx.profile_read(reset=True)
        ctx.profile_enable([])
        return {g: prof[g]["total_ms"] / reps for g in groups}

    try:
        for n in sizes:
            keep = _native._Keep()
            cols = [keep.add(torch.from_numpy(np.ascontiguousarray(a[:n])).to(dev))
                    for a in (scan.x, scan.y, scan.z)]
            cloud = _native.make_cloud(*cols, (), keep)
            for c in range(len(configs)):
                ctx.set_sort_tuning([(BIG, c)])
                t = timed(["voxel_sort", "cell_sort"])
                runs.append(dict(points=n, voxels=int(ctx.chain_info()["voxels"]), config=c,
                                 voxel_sort_ms=t["voxel_sort"], cell_sort_ms=t["cell_sort"]))
            ctx.set_sort_tuning([])
            for mode in WALK_MODES:
                ctx.set_neighbor_staging(mode)
                t = timed(["normals"])
                staging.append(dict(points=n, voxels=int(ctx.chain_info()["voxels"]), staging=mode,
                                    normals_ms=t["normals"]))
            ctx.set_neighbor_staging(-1)
            del cols, cloud, keep
    finally:
        ctx.set_sort_tuning([])
        ctx.set_neighbor_staging(-1)
        ctx.close()
    return dict(configs=configs, runs=runs, staging=staging)


def samples(result: dict, kind: str) -> list:
    """[(size, [ms per shape])], ascending, for the voxel sorts (kind "voxel")
    or the cell sorts ("cell").  The size is the chain's point count for both:
    the library picks a cell sort's shape before the voxel count is known on
    the host, from the same upper bound."""
    n_cfg = len(result["configs"])
    by = {}
    for r in result["runs"]:
        keys, ms = ((r["points"], r["voxel_sort_ms"]) if kind == "voxel"
                    else (r["points"], r["cell_sort_ms"]))
        by.setdefault(keys, [None] * n_cfg)[r["config"]] = ms
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
        "// cell-key sort over the radius-grid points.  Entry k applies to sorts of at",
        "// most k*SortTuneMaxPoints[k] keys (the last entry to every larger sort);",
        "// k*SortTuneConfig[k] indexes kSortItems / kSortMinBlocks in radix.cuh.",
        "// kNeighborStaging: the normals kernel's neighbour walk -- range by range",
        "// through L1 (0), range by range from shared memory filled by bulk copies (1),",
        "// or the L1 walk in packed f32x2 arithmetic (2).",
    ]
    if result is not None:
        lines.append("//")
        lines.append("// Measured sort ms (georeferenced scan, leaf "
                     f"{LEAF}, radius {RADIUS}; L2 flushed before every chain):")
        cfgs = result["configs"]
        shapes = "  ".join(f"{c['items_per_thread']:>2}x{c['blocks_per_sm']}x{c.get('threads_per_block', 256)}"
                           for c in cfgs)
        for kind in ("voxel", "cell"):
            lines.append(f"//   {kind}-key sort     points  {shapes}")
            for keys, ms in samples(result, kind):
                lines.append(f"//   {'':14} {keys:>9}  " + "  ".join(f"{m:6.4f}" for m in ms))
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
    for kind, name in (("voxel", "Voxel"), ("cell", "Cell")):
        table = tables[kind]
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
    ap.add_argument("--json", help="write the measurements and the chosen table here")
    ap.add_argument("--write", action="store_true", help="rewrite csrc/sort_tuning.h")
    ap.add_argument("--from-json", help="take the measurements from an earlier --json run")
    args = ap.parse_args(argv)
    if args.from_json:
        with open(args.from_json) as f:
            result = json.load(f)
    else:
        result = measure(args.sizes, reps=args.reps)
    tables = {kind: choose(result, kind) for kind in ("voxel", "cell")}
    staging = choose_staging(result)
    result["tables"] = {k: [[m, c] for m, c in t] for k, t in tables.items()}
    result["neighbor_staging"] = staging
    for r in result["runs"]:
        print(f"points {r['points']:>9} voxels {r['voxels']:>9} config {r['config']}: "
              f"voxel sort {r['voxel_sort_ms']:.4f} ms  cell sort {r['cell_sort_ms']:.4f} ms")
    for r in result.get("staging", []):
        print(f"points {r['points']:>9} voxels {r['voxels']:>9} staging {r['staging']}: "
              f"normals {r['normals_ms']:.4f} ms")
    print("voxel-key sort table:", tables["voxel"])
    print("cell-key sort table:", tables["cell"])
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
