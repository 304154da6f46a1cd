//! The `cuda` backend of `mask.ellipse@1` and `mask.polygon@1`
//! (crates/paintop-cpu/src/ellipse.rs:506-540, mask_polygon.rs:427-452): the
//! library resolves the params with the reference's validation and messages
//! and rasterises the mask on the device. The polygon is bit-identical to the
//! reference's rasteriser (exact tier); the ellipse is held to the bounded tier
//! its manifest declares.
use crate::{ctx_ptr, ffi, lib_error};
use paintop_core::executor::{InputValues, OpImplementation, OutputValues, ResourceValue};
use paintop_ir::{
    CoordinateConvention, Error, ErrorClass, MaskDescriptor, MaskMeaning, ResourceDescriptor,
    ScalarType, ValidRange,
};
use std::ffi::CString;

pub struct CudaMask {
    op_id: &'static str,
}

impl CudaMask {
    pub const fn ellipse() -> Self { Self { op_id: "mask.ellipse@1" } }
    pub const fn polygon() -> Self { Self { op_id: "mask.polygon@1" } }
}

impl OpImplementation for CudaMask {
    #[allow(unsafe_code)] // the FFI call and the zeroed C structs
    fn compute(&self, inputs: &InputValues, params: &serde_json::Value) -> Result<OutputValues, Error> {
        // only the extent of `extent_from` is read; a missing port is reported by
        // the library with the reference's code and message
        let src = inputs.get("extent_from");
        let extent = src.map(ResourceValue::extent);
        let name = CString::new("extent_from").unwrap_or_default();
        let ports: Vec<ffi::pt_port> = src
            .iter()
            .map(|v| ffi::pt_port {
                name: name.as_ptr(),
                kind: ffi::PT_KIND_IMAGE,
                width: v.extent().width,
                height: v.extent().height,
                channels: 1,
                samples: v.samples().as_ptr(),
                sample_count: v.samples().len(),
            })
            .collect();
        let n = extent.map_or(0, |e| (e.width * e.height) as usize);
        let mut mask = vec![0.0f32; n];
        // SAFETY: a plain-old-data C struct; all-zero is a valid value
        let mut err: ffi::pt_error = unsafe { std::mem::zeroed() };
        let op = CString::new(self.op_id).unwrap_or_default();
        let pj = CString::new(params.to_string()).unwrap_or_default();
        // SAFETY: the pointers refer to live buffers of the stated lengths; a
        // mask op takes no solver record, history or finiteness flag
        let st = unsafe {
            ffi::pt_op_compute(ctx_ptr(), op.as_ptr(), ports.as_ptr(), ports.len() as u32,
                pj.as_ptr(), mask.as_mut_ptr(), n, std::ptr::null_mut(), std::ptr::null_mut(), 0,
                std::ptr::null_mut(), &mut err)
        };
        if st != ffi::PT_OK {
            return Err(lib_error(&err));
        }
        let extent = extent.ok_or_else(|| Error::new(ErrorClass::Execution, "E_POLYGON_INPUT",
                                                     "extent_from missing after a successful call"))?;
        let desc = MaskDescriptor {
            extent,
            scalar: ScalarType::F32,
            range: ValidRange::Bounded { min: 0.0, max: 1.0 },
            meaning: MaskMeaning::Coverage,
            coordinates: CoordinateConvention::PixelCenterUpperLeft,
        };
        let mut out = OutputValues::new();
        out.insert("mask".into(), ResourceValue::new(ResourceDescriptor::Mask(desc), 1, mask)
            .map_err(|len| Error::new(ErrorClass::Execution, "E_POLYGON_INPUT",
                                      format!("mask buffer of unexpected length {len}")))?);
        Ok(out)
    }
}
