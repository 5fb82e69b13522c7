//! The `ExecutionPolicy::Gpu(DeviceKind::Cuda)` arms of `NormalEstimator` and
//! the CUDA flavour of `GpuNormalEstimator`, as the child module
//! `crates/spatialrust-features/src/normal/cuda.rs` of `normal.rs` (it sees the
//! parent's `build_output_cloud`, normal.rs:575-599).
//!
//! Wiring in normal.rs (today `resolve_policy` rejects Cuda at normal.rs:292-294):
//!
//! ```ignore
//! #[cfg(feature = "feature-normal-cuda")]
//! mod cuda;
//!
//! // resolve_policy: Gpu(DeviceKind::Cuda) => Ok(policy) when the feature is on
//! // estimate_policy_output (normal.rs:208-230), before the Wgpu arm:
//! #[cfg(feature = "feature-normal-cuda")]
//! if matches!(self.resolve_policy(input, policy)?, ExecutionPolicy::Gpu(DeviceKind::Cuda)) {
//!     return cuda::estimate_cuda(input, &self.config).map(|(cloud, _)| cloud);
//! }
//! ```
//!
//! `estimate_with_diagnostics` (normal.rs:102-164) on the CUDA arm returns the
//! second element as its NormalEstimationResult.  The test that asserts the
//! rejection (normal.rs:705-712) asserts parity with the CPU path instead.

use spatialrust_core::{HasPositions3, PointCloud, SpatialError, SpatialResult};
use spatialrust_gpu_cuda::{CudaRuntime, RadiusNormalParams};

use super::{build_output_cloud, NormalEstimationConfig, NormalEstimationResult};

fn radius_params(config: &NormalEstimationConfig, include_self: bool) -> SpatialResult<RadiusNormalParams> {
    let radius = config.search_radius.ok_or_else(|| {
        SpatialError::InvalidArgument(
            "the CUDA arm implements radius-mode normal estimation; set search_radius".to_owned(),
        )
    })?;
    if radius < 0.0 {
        // normal.rs:109-111
        return Err(SpatialError::InvalidArgument("search_radius must be non-negative".to_owned()));
    }
    Ok(RadiusNormalParams {
        radius,
        min_neighbors: config.min_neighbors as u32,
        viewpoint: config.viewpoint.map(|v| [v.x, v.y, v.z]),
        include_self,
    })
}

/// NormalEstimator's CPU semantics on the device (normal.rs:321-573): the
/// query excluded from its own neighbourhood, NaN normal and curvature 0 below
/// min_neighbors, normals turned toward the viewpoint.
pub(super) fn estimate_cuda(
    input: &PointCloud,
    config: &NormalEstimationConfig,
) -> SpatialResult<(PointCloud, NormalEstimationResult)> {
    if input.is_empty() {
        return Ok((input.clone(), NormalEstimationResult::default()));
    }
    let params = radius_params(config, false)?;
    let (x, y, z) = input.positions3()?;
    let out = CudaRuntime::shared()?.radius_normals(x, y, z, &params)?;
    let result = NormalEstimationResult {
        valid_count: out.valid_count,
        invalid_count: out.invalid_count,
    };
    Ok((build_output_cloud(input, out.nx, out.ny, out.nz, out.curvature)?, result))
}

/// GpuNormalEstimator::estimate in radius mode on the device, with the wgpu
/// grid kernel's semantics (normals_grid.rs:86-197): the query included,
/// fewer than 3 points -> (0, 0, 1) and curvature 0, every normal turned toward
/// the viewpoint (normal_gpu.rs:63-70).
pub(crate) fn estimate_grid_cuda(
    input: &PointCloud,
    config: &NormalEstimationConfig,
) -> SpatialResult<PointCloud> {
    if input.is_empty() {
        return Ok(input.clone());
    }
    let params = radius_params(config, true)?;
    let (x, y, z) = input.positions3()?;
    let out = CudaRuntime::shared()?.radius_normals(x, y, z, &params)?;
    build_output_cloud(input, out.nx, out.ny, out.nz, out.curvature)
}
