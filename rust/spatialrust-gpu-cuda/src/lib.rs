//! Safe wrapper over libsrcuda for the `ExecutionPolicy::Gpu(DeviceKind::Cuda)`
//! arms of SpatialRust's voxel filter and normal estimators.
//!
//! One context per process, like `WgpuRuntime::shared()`
//! (crates/spatialrust-gpu/src/runtime.rs:72-95); a mutex serialises calls, as
//! the wgpu runtime's pools are behind `Mutex`.  Every call is synchronous and
//! works on host slices (pageable memory is fine); results come back as owned
//! `Vec`s.  Status codes map onto `SpatialError` as the header documents
//! (crates/spatialrust-core/src/error.rs:8-37); an explicit CUDA request never
//! falls back to the CPU (crates/spatialrust-filtering/src/voxel.rs:209-212).
#![allow(unsafe_code)]

use std::ffi::CStr;
use std::ptr;
use std::sync::{Mutex, OnceLock};

use spatialrust_core::{DType, SpatialError, SpatialResult};
use spatialrust_cuda_sys as sys;

/// The process-wide CUDA context.
pub struct CudaRuntime {
    ctx: Mutex<*mut sys::srcu_ctx>,
}

// The raw context is only touched under the mutex.
unsafe impl Send for CudaRuntime {}
unsafe impl Sync for CudaRuntime {}

/// Voxel aggregation (srcu_voxel_params.mode / .attribute_policy).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub struct VoxelMode {
    pub approximate_first: bool,
    pub attribute_first: bool,
    /// The reference's plain-xyz fast path (clouds of x, y, z only).
    pub plain_xyz: bool,
}

/// NormalEstimationConfig in radius mode.
#[derive(Clone, Copy, Debug)]
pub struct RadiusNormalParams {
    pub radius: f32,
    pub min_neighbors: u32,
    pub viewpoint: Option<[f32; 3]>,
    /// GpuNormalEstimator's grid semantics (query included, fewer than 3 -> (0, 0, 1)).
    pub include_self: bool,
}

/// Normal columns of n points, and NormalEstimationResult's counts.
#[derive(Clone, Debug, Default)]
pub struct NormalColumns {
    pub nx: Vec<f32>,
    pub ny: Vec<f32>,
    pub nz: Vec<f32>,
    pub curvature: Vec<f32>,
    pub valid_count: usize,
    pub invalid_count: usize,
}

impl CudaRuntime {
    /// The shared context on device 0, created on first use.
    pub fn shared() -> SpatialResult<&'static CudaRuntime> {
        static RT: OnceLock<Result<CudaRuntime, String>> = OnceLock::new();
        RT.get_or_init(|| {
            let mut ctx = ptr::null_mut();
            match unsafe { sys::srcu_create(0, 0, &mut ctx) } {
                sys::SRCU_OK => Ok(CudaRuntime { ctx: Mutex::new(ctx) }),
                sys::SRCU_ERR_NO_DEVICE => {
                    Err("no CUDA device of compute capability 10.x (B200)".to_owned())
                }
                code => Err(format!("srcu_create failed (status {code})")),
            }
        })
        .as_ref()
        .map_err(|e| SpatialError::InvalidArgument(e.clone()))
    }

    /// Maps a status code onto SpatialError.
    fn check(ctx: *mut sys::srcu_ctx, code: sys::srcu_status) -> SpatialResult<()> {
        if code == sys::SRCU_OK {
            return Ok(());
        }
        let msg = unsafe { CStr::from_ptr(sys::srcu_last_error(ctx)) }.to_string_lossy().into_owned();
        Err(match code {
            sys::SRCU_ERR_INVALID_ARGUMENT => SpatialError::InvalidArgument(msg),
            sys::SRCU_ERR_LENGTH_MISMATCH => {
                let (mut expected, mut found) = (0u64, 0u64);
                unsafe { sys::srcu_last_length_mismatch(ctx, &mut expected, &mut found) };
                SpatialError::BufferLengthMismatch {
                    expected: expected as usize,
                    found: found as usize,
                }
            }
            // the library reads f32 columns only; the widening happens on the Rust side
            sys::SRCU_ERR_UNSUPPORTED_DTYPE => SpatialError::UnsupportedDType(DType::F64),
            sys::SRCU_ERR_MISSING_FIELD => SpatialError::MissingField(msg),
            _ => SpatialError::InvalidArgument(format!("cuda: {msg}")),
        })
    }

    fn cloud(cols: &[&[f32]], attr_ptrs: &[*const f32]) -> sys::srcu_cloud {
        sys::srcu_cloud {
            x: cols[0].as_ptr(),
            y: cols[1].as_ptr(),
            z: cols[2].as_ptr(),
            attrs: if attr_ptrs.is_empty() { ptr::null() } else { attr_ptrs.as_ptr() },
            n_attrs: attr_ptrs.len() as u32,
            on_device: 0,
            n: cols[0].len() as u64,
            stride: 0,
            reserved: 0,
        }
    }

    fn voxel_params(leaf: f32, origin: Option<[f32; 3]>, mode: VoxelMode) -> sys::srcu_voxel_params {
        sys::srcu_voxel_params {
            leaf_size: leaf,
            has_origin: origin.is_some() as i32,
            origin: origin.unwrap_or([0.0; 3]),
            mode: if mode.approximate_first {
                sys::SRCU_VOXEL_APPROXIMATE_FIRST
            } else if mode.plain_xyz {
                sys::SRCU_VOXEL_CENTROID_XYZ
            } else {
                sys::SRCU_VOXEL_CENTROID
            },
            attribute_policy: if mode.attribute_first {
                sys::SRCU_ATTRIBUTE_FIRST
            } else {
                sys::SRCU_ATTRIBUTE_AVERAGE
            },
        }
    }

    fn normal_params(p: &RadiusNormalParams) -> sys::srcu_normal_params {
        sys::srcu_normal_params {
            radius: p.radius,
            min_neighbors: p.min_neighbors,
            has_viewpoint: p.viewpoint.is_some() as i32,
            viewpoint: p.viewpoint.unwrap_or([0.0; 3]),
            include_self: p.include_self as i32,
            count_shell: 0,
        }
    }

    /// Voxel downsample of `cols` (x, y, z, then attribute columns widened to
    /// f32, as read_buffer_f32 does, voxel.rs:692-701).  Returns the voxel
    /// columns in the reference's output order and the points per voxel.
    pub fn voxel_centroid(
        &self,
        cols: &[&[f32]],
        leaf: f32,
        origin: Option<[f32; 3]>,
        mode: VoxelMode,
    ) -> SpatialResult<(Vec<Vec<f32>>, Vec<u32>)> {
        let n = cols[0].len();
        let attrs: Vec<*const f32> = cols[3..].iter().map(|c| c.as_ptr()).collect();
        let cloud = Self::cloud(cols, &attrs);
        let params = Self::voxel_params(leaf, origin, mode);
        let mut out: Vec<Vec<f32>> = cols.iter().map(|_| vec![0.0; n]).collect();
        let mut counts = vec![0u32; n];
        let out_attrs: Vec<*mut f32> = out[3..].iter_mut().map(|c| c.as_mut_ptr()).collect();
        let vout = sys::srcu_voxel_out {
            x: out[0].as_mut_ptr(),
            y: out[1].as_mut_ptr(),
            z: out[2].as_mut_ptr(),
            attrs: if out_attrs.is_empty() { ptr::null() } else { out_attrs.as_ptr() },
            keys: ptr::null_mut(),
            counts: counts.as_mut_ptr(),
            on_device: 0,
        };
        let ctx = *self.ctx.lock().unwrap();
        let mut v = 0u64;
        Self::check(ctx, unsafe { sys::srcu_voxel_centroid(ctx, &cloud, &params, &vout, &mut v) })?;
        for c in &mut out {
            c.truncate(v as usize);
        }
        counts.truncate(v as usize);
        Ok((out, counts))
    }

    /// Radius normals of the points (x, y, z), in input order.
    pub fn radius_normals(
        &self,
        x: &[f32],
        y: &[f32],
        z: &[f32],
        params: &RadiusNormalParams,
    ) -> SpatialResult<NormalColumns> {
        let n = x.len();
        if y.len() != n || z.len() != n {
            return Err(SpatialError::BufferLengthMismatch { expected: n, found: y.len().min(z.len()) });
        }
        let cloud = Self::cloud(&[x, y, z], &[]);
        let p = Self::normal_params(params);
        let mut out = NormalColumns {
            nx: vec![0.0; n],
            ny: vec![0.0; n],
            nz: vec![0.0; n],
            curvature: vec![0.0; n],
            ..Default::default()
        };
        let nout = sys::srcu_normal_out {
            nx: out.nx.as_mut_ptr(),
            ny: out.ny.as_mut_ptr(),
            nz: out.nz.as_mut_ptr(),
            curvature: out.curvature.as_mut_ptr(),
            neighbor_counts: ptr::null_mut(),
            on_device: 0,
        };
        let mut stats = sys::srcu_normal_stats {
            valid_count: 0,
            invalid_count: 0,
            shell_points: 0,
            fp64_eigensolves: 0,
        };
        let ctx = *self.ctx.lock().unwrap();
        Self::check(ctx, unsafe { sys::srcu_radius_normals(ctx, &cloud, &p, &nout, &mut stats) })?;
        out.valid_count = stats.valid_count as usize;
        out.invalid_count = stats.invalid_count as usize;
        Ok(out)
    }

    /// MvpPipeline::run's voxel -> normals chain in one device-resident call
    /// (crates/spatialrust-pipeline/src/mvp.rs:193-226): the voxel columns and
    /// the normals of every voxel centroid.
    pub fn voxel_normals(
        &self,
        cols: &[&[f32]],
        leaf: f32,
        origin: Option<[f32; 3]>,
        mode: VoxelMode,
        params: &RadiusNormalParams,
    ) -> SpatialResult<(Vec<Vec<f32>>, NormalColumns)> {
        let n = cols[0].len();
        let attrs: Vec<*const f32> = cols[3..].iter().map(|c| c.as_ptr()).collect();
        let cloud = Self::cloud(cols, &attrs);
        let vp = Self::voxel_params(leaf, origin, mode);
        let np = Self::normal_params(params);
        let mut out: Vec<Vec<f32>> = cols.iter().map(|_| vec![0.0; n]).collect();
        let out_attrs: Vec<*mut f32> = out[3..].iter_mut().map(|c| c.as_mut_ptr()).collect();
        let vout = sys::srcu_voxel_out {
            x: out[0].as_mut_ptr(),
            y: out[1].as_mut_ptr(),
            z: out[2].as_mut_ptr(),
            attrs: if out_attrs.is_empty() { ptr::null() } else { out_attrs.as_ptr() },
            keys: ptr::null_mut(),
            counts: ptr::null_mut(),
            on_device: 0,
        };
        let mut normals = NormalColumns {
            nx: vec![0.0; n],
            ny: vec![0.0; n],
            nz: vec![0.0; n],
            curvature: vec![0.0; n],
            ..Default::default()
        };
        let nout = sys::srcu_normal_out {
            nx: normals.nx.as_mut_ptr(),
            ny: normals.ny.as_mut_ptr(),
            nz: normals.nz.as_mut_ptr(),
            curvature: normals.curvature.as_mut_ptr(),
            neighbor_counts: ptr::null_mut(),
            on_device: 0,
        };
        let mut stats = sys::srcu_normal_stats {
            valid_count: 0,
            invalid_count: 0,
            shell_points: 0,
            fp64_eigensolves: 0,
        };
        let ctx = *self.ctx.lock().unwrap();
        let mut v = 0u64;
        Self::check(ctx, unsafe {
            sys::srcu_voxel_normals(ctx, &cloud, &vp, &np, &vout, &nout, &mut v, &mut stats)
        })?;
        let v = v as usize;
        for c in out.iter_mut().chain([&mut normals.nx, &mut normals.ny, &mut normals.nz,
                                       &mut normals.curvature]) {
            c.truncate(v);
        }
        normals.valid_count = stats.valid_count as usize;
        normals.invalid_count = stats.invalid_count as usize;
        Ok((out, normals))
    }
}
