//! spectral (reference src/spectral/mod.rs): the spectral operators and the
//! per-level spectral functions of one (ng, nz) grid.

use crate::sta2dfft::D2FFT;
use crate::{check, fill_fortran, fortran_vec_view, or_quit, Precision};
use ndarray::{Array2, Array3, ArrayView2, ArrayView3, ArrayViewMut2, ArrayViewMut3, ShapeBuilder};
use shallow_water_cuda_sys as sys;
use std::ffi::CString;
use std::os::raw::c_int;
use std::sync::{Arc, Mutex};

/// A device context (sw_ctx): an ensemble of `members` runs of one (ng, nz) on one
/// GPU.  The library requires one caller at a time per context; the mutex gives
/// that to the `&self` methods that the reference shares across rayon threads.
pub struct Context {
    raw: Mutex<*mut sys::SwCtx>,
    pub ng: usize,
    pub nz: usize,
    pub members: usize,
    pub precision: Precision,
}

unsafe impl Send for Context {}
unsafe impl Sync for Context {}

impl Context {
    pub fn new(ng: usize, nz: usize, members: usize, precision: Precision) -> anyhow::Result<Self> {
        Self::on_device(ng, nz, members, precision, 0)
    }

    pub fn on_device(ng: usize, nz: usize, members: usize, precision: Precision, device: usize)
                     -> anyhow::Result<Self> {
        let mut p: *mut sys::SwCtx = std::ptr::null_mut();
        check(unsafe {
            sys::sw_ctx_create(ng as c_int, nz as c_int, members as c_int, precision.code(), device as c_int, &mut p)
        })?;
        Ok(Context { raw: Mutex::new(p), ng, nz, members, precision })
    }

    /// Runs f on the raw context with exclusive access.
    pub fn with<T>(&self, f: impl FnOnce(*mut sys::SwCtx) -> T) -> T {
        let g = self.raw.lock().unwrap();
        f(*g)
    }

    pub fn n3(&self) -> usize {
        self.ng * self.ng * (self.nz + 1)
    }

    fn operator(&self, name: &str, n: usize) -> Vec<f64> {
        let c = CString::new(name).unwrap();
        let mut v = vec![0.0; n];
        or_quit(self.with(|p| check(unsafe { sys::sw_spectral_get(p, c.as_ptr(), v.as_mut_ptr(), n) })));
        v
    }
}

impl Drop for Context {
    fn drop(&mut self) {
        let p = *self.raw.lock().unwrap();
        unsafe { sys::sw_ctx_destroy(p) };
    }
}

fn plane(v: Vec<f64>, ng: usize) -> Array2<f64> {
    Array2::from_shape_vec((ng, ng).f(), v).unwrap()
}

/// Replaces Spectral (src/spectral/mod.rs:18-62).  The operators are built by the
/// library (in float64 by the reference's formulas) and copied out into the same
/// public fields; the functions run on the device.
pub struct Spectral {
    pub hlap: Array2<f64>,
    pub glap: Array2<f64>,
    pub rlap: Array2<f64>,
    pub helm: Array2<f64>,
    pub c2g2: Array2<f64>,
    pub simp: Array2<f64>,
    pub rope: Array2<f64>,
    pub fope: Array2<f64>,
    pub filt: Array2<f64>,
    pub diss: Array2<f64>,
    pub opak: Array2<f64>,
    pub rdis: Array2<f64>,
    pub etdv: Array3<f64>,
    pub htdv: Array3<f64>,
    pub ap: Array2<f64>,
    pub etd1: Vec<f64>,
    pub htd1: Vec<f64>,
    pub theta: Vec<f64>,
    pub weight: Vec<f64>,
    pub hrkx: Vec<f64>,
    pub hrky: Vec<f64>,
    pub rk: Vec<f64>,
    pub d2fft: D2FFT,
    pub spmf: Vec<f64>,
    pub alk: Vec<f64>,
    pub kmag: Array2<usize>,
    pub kmax: usize,
    pub kmaxred: usize,
    pub ng: usize,
    pub nz: usize,
    pub(crate) ctx: Arc<Context>,
}

impl Spectral {
    /// Replaces Spectral::new (src/spectral/mod.rs:65-299), float64.
    pub fn new(ng: usize, nz: usize) -> Self {
        Self::with_precision(ng, nz, Precision::Fp64)
    }

    /// A context of the given precision (SW_FP64, SW_MIXED or SW_FP32).
    pub fn with_precision(ng: usize, nz: usize, precision: Precision) -> Self {
        let ctx = Arc::new(or_quit(Context::new(ng, nz, 1, precision)));
        let n2 = ng * ng;
        let g = |name: &str| plane(ctx.operator(name, n2), ng);
        let mut hrkx = vec![0.0; ng];
        let mut hrky = vec![0.0; ng];
        let d2fft = D2FFT::with_context(ng, ng, 2.0 * std::f64::consts::PI, 2.0 * std::f64::consts::PI, &mut hrkx,
                                        &mut hrky, ctx.clone());
        let tri = |name: &str| Array3::from_shape_vec((ng, ng, nz).f(), ctx.operator(name, n2 * nz)).unwrap();
        let kmag = ctx.operator("kmag", n2).iter().map(|v| *v as usize).collect::<Vec<_>>();
        Spectral {
            hlap: g("hlap"), glap: g("glap"), rlap: g("rlap"), helm: g("helm"), c2g2: g("c2g2"), simp: g("simp"),
            rope: g("rope"), fope: g("fope"), filt: g("filt"), diss: g("diss"), opak: g("opak"), rdis: g("rdis"),
            etdv: tri("etdv"), htdv: tri("htdv"), ap: g("ap"),
            etd1: ctx.operator("etd1", nz), htd1: ctx.operator("htd1", nz),
            theta: ctx.operator("theta", nz + 1), weight: ctx.operator("weight", nz + 1),
            rk: ctx.operator("rk", ng), spmf: ctx.operator("spmf", ng + 1), alk: ctx.operator("alk", ng),
            hrkx, hrky, d2fft,
            kmag: Array2::from_shape_vec((ng, ng).f(), kmag).unwrap(),
            kmax: ctx.operator("kmax", 1)[0] as usize,
            kmaxred: ctx.operator("kmaxred", 1)[0] as usize,
            ng, nz, ctx,
        }
    }

    pub fn context(&self) -> &Context {
        &self.ctx
    }

    fn set_field(&self, field: c_int, a: &ArrayView3<f64>) -> anyhow::Result<()> {
        let v = fortran_vec_view(a);
        self.ctx.with(|c| check(unsafe { sys::sw_state_set(c, field, 0, v.as_ptr(), v.len()) }))
    }

    fn get_field(&self, field: c_int, a: &mut ArrayViewMut3<f64>) -> anyhow::Result<()> {
        let mut v = vec![0.0; self.ctx.n3()];
        self.ctx.with(|c| check(unsafe { sys::sw_state_get(c, field, 0, v.as_mut_ptr(), v.len()) }))?;
        fill_fortran(a, &v);
        Ok(())
    }

    /// Replaces Spectral::main_invert (src/spectral/mod.rs:305-417): qs, ds, gs
    /// (spectral) -> r, u, v, zeta (physical).
    pub fn main_invert(&self, qs: ArrayView3<f64>, ds: ArrayView3<f64>, gs: ArrayView3<f64>,
                       mut r: ArrayViewMut3<f64>, mut u: ArrayViewMut3<f64>, mut v: ArrayViewMut3<f64>,
                       mut zeta: ArrayViewMut3<f64>) {
        or_quit((|| -> anyhow::Result<()> {
            self.set_field(sys::SW_QS, &qs)?;
            self.set_field(sys::SW_DS, &ds)?;
            self.set_field(sys::SW_GS, &gs)?;
            self.ctx.with(|c| check(unsafe { sys::sw_main_invert(c) }))?;
            self.get_field(sys::SW_R, &mut r)?;
            self.get_field(sys::SW_U, &mut u)?;
            self.get_field(sys::SW_V, &mut v)?;
            self.get_field(sys::SW_ZETA, &mut zeta)
        })())
    }

    fn plane_op(&self, f: impl FnOnce(*mut sys::SwCtx, *mut f64) -> c_int, mut out: ArrayViewMut2<f64>) {
        let mut o = vec![0.0; self.ng * self.ng];
        or_quit(self.ctx.with(|c| check(f(c, o.as_mut_ptr()))));
        fill_fortran(&mut out, &o);
    }

    /// Replaces Spectral::jacob (src/spectral/mod.rs:423-453): J(aa, bb), physical
    /// inputs, spectral output.
    pub fn jacob(&self, aa: ArrayView2<f64>, bb: ArrayView2<f64>, cs: ArrayViewMut2<f64>) {
        let (a, b) = (fortran_vec_view(&aa), fortran_vec_view(&bb));
        self.plane_op(|c, o| unsafe { sys::sw_jacob(c, a.as_ptr(), b.as_ptr(), o) }, cs)
    }

    /// Replaces Spectral::divs (src/spectral/mod.rs:461-475).
    pub fn divs(&self, aa: ArrayView2<f64>, bb: ArrayView2<f64>, cs: ArrayViewMut2<f64>) {
        let (a, b) = (fortran_vec_view(&aa), fortran_vec_view(&bb));
        self.plane_op(|c, o| unsafe { sys::sw_divs(c, a.as_ptr(), b.as_ptr(), o) }, cs)
    }

    /// Replaces Spectral::ptospc3d (src/spectral/mod.rs:479-500), levels izbeg..=izend.
    pub fn ptospc3d(&self, fp: ArrayView3<f64>, mut fs: ArrayViewMut3<f64>, izbeg: usize, izend: usize) {
        let a = fortran_vec_view(&fp);
        let mut o = fortran_vec_view(&fs.view());
        or_quit(self.ctx.with(|c| check(unsafe {
            sys::sw_ptospc3d(c, a.as_ptr(), o.as_mut_ptr(), izbeg as c_int, izend as c_int)
        })));
        fill_fortran(&mut fs, &o);
    }

    /// Replaces Spectral::spctop3d (src/spectral/mod.rs:502-522).
    pub fn spctop3d(&self, fs: ArrayView3<f64>, mut fp: ArrayViewMut3<f64>, izbeg: usize, izend: usize) {
        let a = fortran_vec_view(&fs);
        let mut o = fortran_vec_view(&fp.view());
        or_quit(self.ctx.with(|c| check(unsafe {
            sys::sw_spctop3d(c, a.as_ptr(), o.as_mut_ptr(), izbeg as c_int, izend as c_int)
        })));
        fill_fortran(&mut fp, &o);
    }

    /// Replaces Spectral::deal3d (src/spectral/mod.rs:524-542), in place.
    pub fn deal3d(&self, mut fp: ArrayViewMut3<f64>) {
        let mut o = fortran_vec_view(&fp.view());
        or_quit(self.ctx.with(|c| check(unsafe { sys::sw_deal3d(c, o.as_mut_ptr()) })));
        fill_fortran(&mut fp, &o);
    }

    /// Replaces Spectral::deal2d (src/spectral/mod.rs:544-554), in place.
    pub fn deal2d(&self, mut fp: ArrayViewMut2<f64>) {
        let mut o = fortran_vec_view(&fp.view());
        or_quit(self.ctx.with(|c| check(unsafe { sys::sw_deal2d(c, o.as_mut_ptr()) })));
        fill_fortran(&mut fp, &o);
    }

    /// Replaces Spectral::spec1d (src/spectral/mod.rs:558-591): ss has ng*ng
    /// values, spec ng+1.
    pub fn spec1d(&self, ss: &[f64], spec: &mut [f64]) {
        assert_eq!(self.ng * self.ng, ss.len());
        assert_eq!(self.ng + 1, spec.len());
        or_quit(self.ctx.with(|c| check(unsafe { sys::sw_spec1d(c, ss.as_ptr(), spec.as_mut_ptr()) })));
    }
}
