"""spatialrust_b200: SpatialRust's uniform-grid hot path (VoxelGrid centroid
downsample + radius-mode normal estimation) as hand-written CUDA for B200
(sm_100a), behind the reference's own API shape -- with the consumers on the
same grid (Euclidean cluster roots, GICP plane covariances), the bounded
streaming voxel and LAS record decoding on either side of it.

The compute path is libsrcuda.so (C ABI: include/srcuda.h).  This Python
layer mirrors the reference's Rust API so that code written against
VoxelGridDownsample / NormalEstimator / GpuNormalEstimator reads the same.
"""
from .core import (Auto, BufferLengthMismatch, CpuParallel, CpuSingle, DeviceKind, DType,
                   ExecutionOutput, ExecutionPolicy, ExecutionReceipt, FieldSemantic, GpuCuda,
                   InvalidArgument, MissingField, PointCloud, PointCloudBuilder, PointField,
                   PointSchema, SpatialError, StandardSchemas, TransferDirection, UnsupportedDType)
from .features import (GpuNormalEstimator, NormalEstimationConfig, NormalEstimationResult,
                       NormalEstimator, build_output_cloud)
from .filtering import (AttributeAggregation, VoxelAggregationMode, VoxelGridDownsample,
                        VoxelGridDownsampleConfig)
from .segmentation import (EuclideanClusterConfig, EuclideanClusterExtractor,
                           EuclideanClusterResult, GpuEuclideanClusterExtractor,
                           GpuRansacPlaneSegmenter, PlaneModel, RansacPlaneConfig,
                           RansacPlaneSegmentation, RansacPlaneSegmenter)
from .streaming import (MemoryChunkSource, SpoolOptions, StreamingVoxelConfig,
                        StreamingVoxelSource)
from .las import LasChunkSource, LasReader, read_las
from .pipeline import MvpPipeline, MvpPipelineConfig, MvpPipelineReceipt, MvpPipelineResult
from . import gpu

__all__ = [
    "Auto", "AttributeAggregation", "BufferLengthMismatch", "CpuParallel", "CpuSingle",
    "DeviceKind", "DType", "ExecutionOutput", "ExecutionPolicy", "ExecutionReceipt",
    "FieldSemantic", "GpuCuda", "GpuNormalEstimator", "InvalidArgument", "MissingField",
    "NormalEstimationConfig", "NormalEstimationResult", "NormalEstimator", "PointCloud",
    "PointCloudBuilder", "PointField", "PointSchema", "SpatialError", "StandardSchemas",
    "TransferDirection", "UnsupportedDType", "VoxelAggregationMode", "VoxelGridDownsample",
    "VoxelGridDownsampleConfig", "build_output_cloud", "EuclideanClusterConfig",
    "EuclideanClusterExtractor", "EuclideanClusterResult", "GpuEuclideanClusterExtractor",
    "MemoryChunkSource", "SpoolOptions", "StreamingVoxelConfig", "StreamingVoxelSource",
    "LasChunkSource", "LasReader", "read_las", "gpu", "GpuRansacPlaneSegmenter", "PlaneModel",
    "RansacPlaneConfig", "RansacPlaneSegmentation", "RansacPlaneSegmenter", "MvpPipeline",
    "MvpPipelineConfig", "MvpPipelineReceipt", "MvpPipelineResult",
]
