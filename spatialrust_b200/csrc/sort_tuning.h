// sort_tuning.h -- the sort launch shape per input size that a context starts
// with.  Written by `python -m spatialrust_b200.autotune --write` from its
// measurements; srcu_set_sort_tuning replaces it per context.
//
// One table per sort kind: the voxel-key sort over the input points and the
// cell-key sort over the radius-grid points.  Entry k applies to sorts of at
// most k*SortTuneMaxPoints[k] keys (the last entry to every larger sort);
// k*SortTuneConfig[k] indexes kSortItems / kSortMinBlocks in radix.cuh.
// kNeighborStaging: whether the normals kernel
// stages candidate records in shared memory by bulk copies (1) or reads them
// through L1 (0).
//
// Measured sort ms (georeferenced scan, leaf 0.1, radius 0.5; L2 flushed before every chain):
//   voxel-key sort       keys    16x2     8x3    12x3     8x4
//                      65536  0.0609  0.0472  0.0557  0.0470
//                      92682  0.0623  0.0480  0.0556  0.0485
//                     131072  0.0624  0.0498  0.0578  0.0498
//                     185364  0.0642  0.0516  0.0587  0.0520
//                     262144  0.0664  0.0536  0.0603  0.0539
//                     370728  0.0666  0.0584  0.0629  0.0586
//                     524288  0.0696  0.0642  0.0683  0.0642
//                     741455  0.0764  0.0779  0.0738  0.0772
//                    1048576  0.0827  0.0918  0.0918  0.1071
//                    1482910  0.1100  0.1150  0.1070  0.1274
//                    2097152  0.1308  0.1404  0.1407  0.1609
//                    2965821  0.1739  0.1799  0.1659  0.1998
//                    4194304  0.2338  0.2427  0.2259  0.2647
//                    5931642  0.3242  0.3285  0.3041  0.3499
//                    8388608  0.4434  0.4447  0.4117  0.4638
//                   11863283  0.6092  0.6128  0.5608  0.6309
//                   16777216  0.8398  0.8483  0.7703  0.8710
//                   23726566  1.1608  1.1787  1.0690  1.2085
//                   33554432  1.6223  1.6466  1.4860  1.6870
//   cell-key sort       keys    16x2     8x3    12x3     8x4
//                      65325  0.0534  0.0403  0.0455  0.0412
//                      92252  0.0542  0.0410  0.0463  0.0416
//                     130231  0.0551  0.0417  0.0478  0.0428
//                     183630  0.0551  0.0431  0.0480  0.0432
//                     258683  0.0562  0.0451  0.0495  0.0451
//                     364390  0.0564  0.0475  0.0502  0.0488
//                     511610  0.0590  0.0533  0.0555  0.0535
//                     716353  0.0639  0.0636  0.0603  0.0640
//                     998975  0.0691  0.0737  0.0744  0.0872
//                    1386254  0.0910  0.0917  0.0825  0.0983
//                    1913842  0.1088  0.1083  0.1124  0.1275
//                    2610072  0.1358  0.1384  0.1314  0.1508
//                    3512442  0.1664  0.1721  0.1646  0.1925
//                    4648599  0.2132  0.2152  0.2011  0.2373
//                    6011810  0.2763  0.2685  0.2482  0.2890
//                    7569816  0.3437  0.3297  0.3032  0.3468
//                    8875163  0.3965  0.3793  0.3492  0.3952
//                   10515699  0.4595  0.4416  0.4036  0.4590
//                   12236880  0.5264  0.5067  0.4606  0.5245
// Normals kernel ms per chain, neighbour gather through L1 / staged:
//       65536    0.023 /  0.026
//       92682    0.027 /  0.032
//      131072    0.033 /  0.038
//      185364    0.050 /  0.063
//      262144    0.064 /  0.079
//      370728    0.092 /  0.113
//      524288    0.118 /  0.140
//      741455    0.147 /  0.171
//     1048576    0.194 /  0.213
//     1482910    0.288 /  0.302
//     2097152    0.411 /  0.442
//     2965821    0.644 /  0.669
//     4194304    1.037 /  1.067
//     5931642    1.664 /  1.722
//     8388608    2.382 /  2.416
//    11863283    3.477 /  3.478
//    16777216    4.445 /  4.489
//    23726566    5.981 /  5.908
//    33554432    7.549 /  7.403
#pragma once

#include <cstdint>

namespace srcu {

constexpr uint32_t kVoxelSortTuneCount = 6;
constexpr uint64_t kVoxelSortTuneMaxPoints[] = {623486ull, 881743ull, 1246973ull, 1763487ull, 2493948ull, UINT64_MAX};
constexpr int32_t kVoxelSortTuneConfig[] = {3, 2, 0, 2, 0, 2};
constexpr uint32_t kCellSortTuneCount = 6;
constexpr uint64_t kCellSortTuneMaxPoints[] = {605386ull, 845942ull, 1176789ull, 1628825ull, 2235009ull, UINT64_MAX};
constexpr int32_t kCellSortTuneConfig[] = {1, 2, 0, 2, 1, 2};
// 1: the normals kernel gathers candidates through shared memory (bulk copies)
constexpr int32_t kNeighborStaging = 0;

}  // namespace srcu
