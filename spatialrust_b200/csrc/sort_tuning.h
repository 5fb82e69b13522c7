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
//   voxel-key sort     points    16x2     8x3    12x3     8x4
//                      65536  0.0589  0.0453  0.0537  0.0476
//                      92682  0.0597  0.0463  0.0535  0.0490
//                     131072  0.0605  0.0481  0.0546  0.0500
//                     185364  0.0622  0.0501  0.0562  0.0520
//                     262144  0.0643  0.0519  0.0582  0.0542
//                     370728  0.0645  0.0563  0.0599  0.0586
//                     524288  0.0667  0.0623  0.0644  0.0644
//                     741455  0.0723  0.0724  0.0705  0.0745
//                    1048576  0.0790  0.0851  0.0824  0.0908
//                    1482910  0.1052  0.1067  0.0988  0.1096
//                    2097152  0.1276  0.1289  0.1265  0.1356
//                    2965821  0.1670  0.1673  0.1544  0.1708
//                    4194304  0.2251  0.2272  0.2059  0.2251
//                    5931642  0.3117  0.3083  0.2784  0.3038
//                    8388608  0.4236  0.4195  0.3752  0.4048
//                   11863283  0.5822  0.5777  0.5129  0.5484
//                   16777216  0.8046  0.8001  0.7058  0.7505
//                   23726566  1.1152  1.1109  0.9771  1.0369
//                   33554432  1.5592  1.5515  1.3612  1.4412
//   cell-key sort     points    16x2     8x3    12x3     8x4
//                      65536  0.0516  0.0391  0.0456  0.0410
//                      92682  0.0519  0.0397  0.0468  0.0415
//                     131072  0.0533  0.0409  0.0474  0.0428
//                     185364  0.0535  0.0412  0.0479  0.0433
//                     262144  0.0543  0.0435  0.0491  0.0453
//                     370728  0.0545  0.0468  0.0502  0.0490
//                     524288  0.0572  0.0522  0.0550  0.0546
//                     741455  0.0617  0.0597  0.0596  0.0614
//                    1048576  0.0677  0.0699  0.0680  0.0731
//                    1482910  0.0865  0.0856  0.0791  0.0872
//                    2097152  0.1053  0.1027  0.1027  0.1069
//                    2965821  0.1304  0.1308  0.1215  0.1276
//                    4194304  0.1620  0.1636  0.1532  0.1617
//                    5931642  0.2073  0.2054  0.1897  0.2028
//                    8388608  0.2662  0.2595  0.2391  0.2541
//                   11863283  0.3320  0.3200  0.2931  0.3076
//                   16777216  0.3815  0.3684  0.3341  0.3505
//                   23726566  0.4414  0.4255  0.3838  0.4019
//                   33554432  0.5016  0.4851  0.4356  0.4555
// Normals kernel ms per chain, neighbour gather through L1 / staged:
//       65536    0.023 /  0.026
//       92682    0.027 /  0.032
//      131072    0.032 /  0.039
//      185364    0.051 /  0.062
//      262144    0.064 /  0.078
//      370728    0.091 /  0.112
//      524288    0.118 /  0.140
//      741455    0.145 /  0.168
//     1048576    0.195 /  0.212
//     1482910    0.286 /  0.301
//     2097152    0.410 /  0.448
//     2965821    0.641 /  0.672
//     4194304    1.039 /  1.055
//     5931642    1.666 /  1.713
//     8388608    2.388 /  2.436
//    11863283    3.489 /  3.480
//    16777216    4.426 /  4.486
//    23726566    5.936 /  5.917
//    33554432    7.543 /  7.378
#pragma once

#include <cstdint>

namespace srcu {

constexpr uint32_t kVoxelSortTuneCount = 4;
constexpr uint64_t kVoxelSortTuneMaxPoints[] = {623486ull, 881743ull, 1246973ull, UINT64_MAX};
constexpr int32_t kVoxelSortTuneConfig[] = {1, 2, 0, 2};
constexpr uint32_t kCellSortTuneCount = 3;
constexpr uint64_t kCellSortTuneMaxPoints[] = {881743ull, 1246973ull, UINT64_MAX};
constexpr int32_t kCellSortTuneConfig[] = {1, 0, 2};
constexpr uint32_t kBatchVoxelSortTuneCount = 4;
constexpr uint64_t kBatchVoxelSortTuneMaxPoints[] = {623486ull, 881743ull, 1246973ull, UINT64_MAX};
constexpr int32_t kBatchVoxelSortTuneConfig[] = {1, 2, 0, 2};
constexpr uint32_t kBatchCellSortTuneCount = 3;
constexpr uint64_t kBatchCellSortTuneMaxPoints[] = {881743ull, 1246973ull, UINT64_MAX};
constexpr int32_t kBatchCellSortTuneConfig[] = {1, 0, 2};
// 1: the normals kernel gathers candidates through shared memory (bulk copies)
constexpr int32_t kNeighborStaging = 0;

}  // namespace srcu
