//! The `cuda` backend of paintop's `repair.poisson_blend@1` and
//! `repair.screened_poisson@1` ops, an `OpImplementation`
//! (crates/paintop-core/src/executor/op_impl.rs:51-70) over
//! libpaintop_cuda.so's `pt_op_compute_ex`. The library runs the whole op body
//! (param resolution, port reads, shape checks, solve, SolverData mapping) with
//! the reference's defaults, error classes, codes and messages
//! (crates/paintop-cpu/src/poisson_blend.rs:102-139,417-445,534-600;
//! screened_poisson.rs:66-112,361-430); this crate marshals ports in and the
//! candidate and report out.
//!
//! Two implementation ids: `cuda.poisson@1` (red-black SOR with FP64
//! refinement) and `cuda.multigrid@1` (multigrid-preconditioned CG to the same
//! bar). A missing GPU is `E_CUDA_UNAVAILABLE` (Policy class), never a CPU
//! fallback.
mod ffi;
mod mask;

pub use mask::CudaMask;

use paintop_core::executor::{InputValues, OpImplementation, OutputValues, ResourceValue};
use paintop_ir::{Error, ErrorClass, Report, ResourceDescriptor, SolverData, SolverStopReason};
use std::ffi::CString;
use std::sync::OnceLock;

/// The process's device context (device 0), created on first use. A failure to
/// create it is kept, so every later call reports the same status.
pub(crate) static CTX: OnceLock<Result<ffi::Ctx, i32>> = OnceLock::new();

pub(crate) fn ctx_ptr() -> *mut ffi::pt_ctx {
    CTX.get_or_init(|| ffi::Ctx::new(0)).as_ref().map_or(std::ptr::null_mut(), ffi::Ctx::raw)
}

/// The reference's error class tokens (crates/paintop-ir/src/error.rs:23-114).
pub(crate) fn class(tok: &str) -> ErrorClass {
    match tok {
        "schema" => ErrorClass::Schema,
        "reference" => ErrorClass::Reference,
        "type" => ErrorClass::Type,
        "semantic" => ErrorClass::Semantic,
        "policy" => ErrorClass::Policy,
        "parse" => ErrorClass::Parse,
        _ => ErrorClass::Execution,
    }
}

pub(crate) fn lib_error(err: &ffi::pt_error) -> Error {
    Error::new(class(&ffi::field_str(&err.error_class)), ffi::field_str(&err.code),
               ffi::field_str(&err.message))
}

/// The ports of an op call as `pt_port`s; the returned names must outlive them.
pub(crate) fn ports(inputs: &InputValues) -> (Vec<CString>, Vec<ffi::pt_port>) {
    let mut names = Vec::with_capacity(inputs.len());
    let mut out = Vec::with_capacity(inputs.len());
    for (name, v) in inputs {
        let (kind, w, h, ch) = match v.descriptor() {
            ResourceDescriptor::Image(d) => {
                (ffi::PT_KIND_IMAGE, d.extent.width, d.extent.height, d.layout.channel_count())
            }
            ResourceDescriptor::Mask(d) => (ffi::PT_KIND_MASK, d.extent.width, d.extent.height, 1),
            _ => (7, 0, 0, 0), // any other kind: the library rejects it with the reference's message
        };
        names.push(CString::new(name.as_str()).unwrap_or_default());
        out.push(ffi::pt_port {
            name: std::ptr::null(),
            kind,
            width: w,
            height: h,
            channels: ch,
            samples: v.samples().as_ptr(),
            sample_count: v.samples().len(),
        });
    }
    for (p, n) in out.iter_mut().zip(&names) {
        p.name = n.as_ptr();
    }
    (names, out)
}

/// `flags` 0: `cuda.poisson@1`; `ffi::PT_FLAG_MULTIGRID`: `cuda.multigrid@1`.
pub struct CudaPoisson {
    op_id: &'static str,
    kind: &'static str,
    anchor_port: &'static str,
    flags: u32,
}

impl CudaPoisson {
    pub const fn blend() -> Self {
        Self { op_id: "repair.poisson_blend@1", kind: "poisson", anchor_port: "target", flags: 0 }
    }
    pub const fn screened() -> Self {
        Self { op_id: "repair.screened_poisson@1", kind: "screened-poisson", anchor_port: "anchor",
               flags: 0 }
    }
    pub const fn multigrid(self) -> Self {
        Self { flags: ffi::PT_FLAG_MULTIGRID, ..self }
    }
}

/// The largest history the op can produce: its iteration cap
/// (crates/paintop-cpu/src/poisson_blend.rs:68-74).
const HISTORY_CAP: usize = 100_000;

impl OpImplementation for CudaPoisson {
    #[allow(unsafe_code)] // the FFI call and the zeroed C structs
    fn compute(&self, inputs: &InputValues, params: &serde_json::Value) -> Result<OutputValues, Error> {
        let (_names, ports) = ports(inputs);
        // the candidate takes the anchor's descriptor (poisson_blend.rs:417-445);
        // a missing or non-image anchor is reported by the library with the
        // reference's code, so only the buffer size is needed here
        let (desc, n) = match inputs.get(self.anchor_port).map(ResourceValue::descriptor) {
            Some(ResourceDescriptor::Image(d)) => {
                (Some(*d), (d.extent.width * d.extent.height * d.layout.channel_count()) as usize)
            }
            _ => (None, 0),
        };
        let mut candidate = vec![0.0f32; n];
        let mut hist = vec![0.0f64; HISTORY_CAP];
        // SAFETY: plain-old-data C structs; all-zero is a valid value of each
        let mut sd: ffi::pt_solver_data = unsafe { std::mem::zeroed() };
        let mut err: ffi::pt_error = unsafe { std::mem::zeroed() };
        let mut finite = 0i32;
        let op = CString::new(self.op_id).unwrap_or_default();
        let pj = CString::new(params.to_string()).unwrap_or_default();
        // SAFETY: every pointer refers to a live buffer of the stated length for
        // the duration of the call; the library keeps none of them
        let st = unsafe {
            ffi::pt_op_compute_ex(ctx_ptr(), op.as_ptr(), ports.as_ptr(), ports.len() as u32,
                pj.as_ptr(), candidate.as_mut_ptr(), n, &mut sd, hist.as_mut_ptr(),
                hist.len() as u32, &mut finite, &mut err, self.flags)
        };
        if st != ffi::PT_OK {
            return Err(lib_error(&err));
        }
        let desc = desc.ok_or_else(|| Error::new(ErrorClass::Execution, "E_POISSON_BLEND_INPUT",
                                                 "anchor image missing after a successful solve"))?;
        hist.truncate(sd.history_len as usize);
        let stop = match sd.stop_reason {
            ffi::PT_STOP_CONVERGED => SolverStopReason::Converged,
            ffi::PT_STOP_MAX_ITERATIONS => SolverStopReason::MaxIterations,
            _ => SolverStopReason::Stalled,
        };
        let solver = SolverData {
            kind: self.kind.into(),
            steps: sd.steps,
            stability_number: 0.0,
            stability_limit: 0.0,
            stable: true,
            residual_history: hist,
            total_energy: 0.0,
            iterations: Some(sd.iterations),
            stop_reason: Some(stop),
            converged: Some(sd.converged != 0),
            tolerance: Some(sd.tolerance),
            final_residual: Some(sd.final_residual),
        };
        let channels = desc.layout.channel_count();
        let mut out = OutputValues::new();
        out.insert("candidate".into(),
            ResourceValue::new(ResourceDescriptor::Image(desc), channels, candidate).map_err(|len| {
                Error::new(ErrorClass::Execution, "E_POISSON_BLEND_BUFFER",
                           format!("candidate buffer of unexpected length {len}"))
            })?);
        out.insert("report".into(), ResourceValue::report(Report {
            extent: desc.extent,
            channels,
            channel_stats: Vec::new(),
            all_finite: finite != 0,
            content_hash: String::new(),
            diff: None,
            assertion: None,
            histogram: None,
            components: None,
            frequency_energy: None,
            solver: Some(solver),
        }));
        Ok(out)
    }
}
