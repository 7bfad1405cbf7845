//! The nhswps time-step path of the shallow-water crate on a B200 GPU.
//!
//! Modules and functions keep the reference crate's names, argument meaning and
//! array layout (src/lib.rs:4-15): `stafft`, `sta2dfft`, `spectral`, `nhswps`.  The
//! arithmetic runs in libswcuda.so (hand-written sm_100a CUDA) through the raw
//! bindings of `shallow-water-cuda-sys`; there is no CPU fallback.
//!
//! Errors: functions whose reference counterpart returns `anyhow::Result` return
//! one here, carrying the library's status and message (`SwError`).  Functions whose
//! reference counterpart returns `()` and quits the process on a numerical failure
//! (`quit::with_code(1)` in stafft/mod.rs:148, psolve.rs:349-366) print the message
//! and exit with code 1 in the same way; each has a `try_` variant that returns the
//! error instead.

pub mod nhswps;
pub mod spectral;
pub mod sta2dfft;
pub mod stafft;

use ndarray::{ArrayBase, ArrayView, ArrayViewMut, Data, Dimension};
use shallow_water_cuda_sys as sys;
use std::ffi::CStr;
use std::fmt;
use std::os::raw::c_int;

/// Precision of a context's hot path (include/sw_cuda.h).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum Precision {
    /// everything in float64
    Fp64,
    /// float64 with float32 pressure correction sweeps (within 1e-5 of Fp64)
    Mixed,
    /// float32 transforms and work fields (fastest, ~1e-4 on delta/gamma at ng=256)
    Fp32,
}

impl Precision {
    pub(crate) fn code(self) -> c_int {
        match self {
            Precision::Fp64 => sys::SW_FP64,
            Precision::Mixed => sys::SW_MIXED,
            Precision::Fp32 => sys::SW_FP32,
        }
    }
}

/// A failed library call: its status (SW_ERR_*) and message.
#[derive(Debug, Clone)]
pub struct SwError {
    pub status: i32,
    pub message: String,
}

impl fmt::Display for SwError {
    fn fmt(&self, f: &mut fmt::Formatter<'_>) -> fmt::Result {
        write!(f, "libswcuda status {}: {}", self.status, self.message)
    }
}

impl std::error::Error for SwError {}

/// The calling thread's last library error message.
pub fn last_error() -> String {
    let p = unsafe { sys::sw_last_error() };
    if p.is_null() {
        return String::new();
    }
    unsafe { CStr::from_ptr(p) }.to_string_lossy().into_owned()
}

pub(crate) fn check(status: c_int) -> anyhow::Result<()> {
    if status == sys::SW_OK {
        Ok(())
    } else {
        Err(anyhow::Error::new(SwError { status, message: last_error() }))
    }
}

/// The reference's reaction to a numerical failure: report and quit with code 1.
pub(crate) fn or_quit<T>(r: anyhow::Result<T>) -> T {
    match r {
        Ok(v) => v,
        Err(e) => {
            eprintln!("{}", e);
            std::process::exit(1)
        }
    }
}

/// The values of an array in Fortran (column-major) order, the layout of every
/// array of the reference (src/utils.rs:6-32), whatever the view's strides.
pub(crate) fn fortran_vec<S: Data<Elem = f64>, D: Dimension>(a: &ArrayBase<S, D>) -> Vec<f64> {
    a.t().iter().copied().collect()
}

/// Writes values given in Fortran order into a view of any strides.
pub(crate) fn fill_fortran<D: Dimension>(a: &mut ArrayViewMut<f64, D>, v: &[f64]) {
    assert_eq!(a.len(), v.len());
    for (d, s) in a.view_mut().reversed_axes().iter_mut().zip(v) {
        *d = *s;
    }
}

pub(crate) fn fortran_vec_view<D: Dimension>(a: &ArrayView<f64, D>) -> Vec<f64> {
    a.t().iter().copied().collect()
}
