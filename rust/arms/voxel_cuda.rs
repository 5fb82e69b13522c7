//! The `ExecutionPolicy::Gpu(DeviceKind::Cuda)` arm of
//! `VoxelGridDownsample::filter_internal`, as the child module
//! `crates/spatialrust-filtering/src/voxel/cuda.rs` of `voxel.rs`: a child
//! module sees the parent's private `read_buffer_f32` (voxel.rs:692-701),
//! `push_field` (voxel.rs:1241-1259) and `is_plain_xyz_f32_schema`.
//!
//! Wiring in voxel.rs (today the arm is rejected at voxel.rs:336-339):
//!
//! ```ignore
//! #[cfg(feature = "filter-voxel-cuda")]
//! mod cuda;
//!
//! // in filter_internal, after `let policy = self.resolve_policy(input, policy)?;`
//! // (voxel.rs:276), before the Wgpu arm; an explicit CUDA request never falls
//! // back to the CPU (voxel.rs:209-212)
//! if matches!(policy, ExecutionPolicy::Gpu(DeviceKind::Cuda)) {
//!     #[cfg(feature = "filter-voxel-cuda")]
//!     return cuda::filter_cuda(input, x, y, z, &self.config);
//!     #[cfg(not(feature = "filter-voxel-cuda"))]
//!     return Err(SpatialError::InvalidArgument(
//!         "CUDA voxel downsampling requires the filter-voxel-cuda feature".to_owned()));
//! }
//! ```
//!
//! and in `resolve_policy` (voxel.rs:370-403) `Gpu(DeviceKind::Cuda)` passes
//! through as `Gpu(Wgpu)` does.  The test that asserts the rejection
//! (voxel.rs:1510-1527) asserts parity with the CPU path instead when the
//! feature is on.

use spatialrust_core::{FieldSemantic, PointBuffer, PointBufferSet, PointCloud, SpatialResult};
use spatialrust_gpu_cuda::{CudaRuntime, VoxelMode};

use super::{
    is_plain_xyz_f32_schema, push_field, read_buffer_f32, AttributeAggregation,
    VoxelAggregationMode, VoxelGridDownsampleConfig,
};

fn is_position(semantic: FieldSemantic) -> bool {
    matches!(
        semantic,
        FieldSemantic::PositionX | FieldSemantic::PositionY | FieldSemantic::PositionZ
    )
}

/// Every mode on the device: Centroid + Average with the fast path's
/// arithmetic (voxel.rs:464-540) or, for plain-xyz clouds, the plain-xyz fast
/// path's (voxel.rs:550-636); the other modes with the general path's
/// (voxel.rs:1123-1165).  The output keeps the input schema and metadata.
pub(super) fn filter_cuda(
    input: &PointCloud,
    x: &[f32],
    y: &[f32],
    z: &[f32],
    config: &VoxelGridDownsampleConfig,
) -> SpatialResult<PointCloud> {
    let schema = input.schema().clone();
    let fields = schema.fields();
    // positions first, then every other field widened to f32 (read_buffer_f32)
    let others: Vec<_> = fields.iter().filter(|f| !is_position(f.semantic)).collect();
    let widened = others
        .iter()
        .map(|f| {
            let buffer = input.field(&f.name)?;
            Ok((0..input.len()).map(|i| read_buffer_f32(buffer, i)).collect::<Vec<f32>>())
        })
        .collect::<SpatialResult<Vec<_>>>()?;
    let mut cols: Vec<&[f32]> = vec![x, y, z];
    cols.extend(widened.iter().map(Vec::as_slice));
    let centroid_average = config.mode == VoxelAggregationMode::Centroid
        && config.attribute_policy == AttributeAggregation::Average;
    let mode = VoxelMode {
        approximate_first: config.mode == VoxelAggregationMode::ApproximateFirst,
        attribute_first: config.attribute_policy == AttributeAggregation::First,
        plain_xyz: centroid_average && is_plain_xyz_f32_schema(&schema),
    };
    let origin = config.origin.map(|o| [o.x, o.y, o.z]);
    let (out, _counts) = CudaRuntime::shared()?.voxel_centroid(&cols, config.leaf_size, origin, mode)?;

    // the column of each schema field: 0, 1, 2 for the positions, then the others in order
    let mut next_other = 3;
    let mut buffers = PointBufferSet::new();
    let voxels = out[0].len();
    for field in fields {
        buffers.insert(field.name.clone(), PointBuffer::with_capacity(field.dtype, voxels));
    }
    let column: Vec<usize> = fields
        .iter()
        .map(|f| match f.semantic {
            FieldSemantic::PositionX => 0,
            FieldSemantic::PositionY => 1,
            FieldSemantic::PositionZ => 2,
            _ => {
                next_other += 1;
                next_other - 1
            }
        })
        .collect();
    for v in 0..voxels {
        for (field, &c) in fields.iter().zip(&column) {
            push_field(&mut buffers, field, out[c][v])?;
        }
    }
    PointCloud::try_from_parts(schema, buffers, input.metadata().clone())
}
