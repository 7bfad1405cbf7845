//! sta2dfft (reference src/sta2dfft.rs): 2-D transforms of one ng x ng plane,
//! physical rvar(ny, nx) <-> spectral svar(nx, ny), and spectral derivatives.

use crate::spectral::Context;
use crate::stafft;
use crate::{check, fill_fortran, fortran_vec, fortran_vec_view, or_quit};
use ndarray::{ArrayView2, ArrayViewMut2};
use shallow_water_cuda_sys as sys;
use std::f64::consts::PI;
use std::sync::Arc;

/// Replaces D2FFT (src/sta2dfft.rs:22-29).  The transforms run on a device context
/// of the square grid nx = ny.
pub struct D2FFT {
    pub nx: usize,
    pub ny: usize,
    pub xfactors: [usize; 5],
    pub yfactors: [usize; 5],
    pub xtrig: Vec<f64>,
    pub ytrig: Vec<f64>,
    pub(crate) ctx: Arc<Context>,
}

impl D2FFT {
    /// Replaces D2FFT::new (src/sta2dfft.rs:37-88): the trig tables and factors of
    /// both axes and the wavenumbers kx[k-1] = (pi/lx) k, ky[k-1] = (pi/ly) k.
    pub fn new(nx: usize, ny: usize, lx: f64, ly: f64, kx: &mut [f64], ky: &mut [f64]) -> Self {
        assert_eq!(nx, ny, "the GPU transforms take square grids");
        if lx == 0.0 {
            eprintln!("Wavenumber array definition not possible, domain length in x equal to zero not allowed!");
            std::process::exit(1);
        }
        let ctx = or_quit(Context::new(nx, 2, 1, crate::Precision::Fp64));
        Self::with_context(nx, ny, lx, ly, kx, ky, Arc::new(ctx))
    }

    pub(crate) fn with_context(nx: usize, ny: usize, lx: f64, ly: f64, kx: &mut [f64], ky: &mut [f64],
                               ctx: Arc<Context>) -> Self {
        let mut d = D2FFT { nx, ny, xfactors: [0; 5], yfactors: [0; 5], xtrig: vec![0.0; 2 * nx],
                            ytrig: vec![0.0; 2 * ny], ctx };
        stafft::initfft(nx, &mut d.xfactors, &mut d.xtrig);
        stafft::initfft(ny, &mut d.yfactors, &mut d.ytrig);
        let sc = PI / lx;
        for k in 1..=nx {
            kx[k - 1] = sc * k as f64;
        }
        if ly != 0.0 {
            let sc = PI / ly;
            for k in 1..=ny {
                ky[k - 1] = sc * k as f64;
            }
        }
        d
    }

    /// Replaces D2FFT::ptospc (src/sta2dfft.rs:91-111).  rvar is left unchanged
    /// (the reference destroys it).
    pub fn ptospc(&self, rvar: ArrayViewMut2<f64>, mut svar: ArrayViewMut2<f64>) {
        let r = fortran_vec(&rvar);
        let mut s = vec![0.0; r.len()];
        or_quit(self.ctx.with(|c| check(unsafe { sys::sw_ptospc(c, r.as_ptr(), s.as_mut_ptr()) })));
        fill_fortran(&mut svar, &s);
    }

    /// Replaces D2FFT::spctop (src/sta2dfft.rs:113-123).
    pub fn spctop(&self, svar: ArrayViewMut2<f64>, mut rvar: ArrayViewMut2<f64>) {
        let s = fortran_vec(&svar);
        let mut r = vec![0.0; s.len()];
        or_quit(self.ctx.with(|c| check(unsafe { sys::sw_spctop(c, s.as_ptr(), r.as_mut_ptr()) })));
        fill_fortran(&mut rvar, &r);
    }

    /// Replaces D2FFT::xderiv (src/sta2dfft.rs:128-155).  rkx must be the wavenumber
    /// array of D2FFT::new, (pi/lx) k: the device multiplies by the integer
    /// wavenumbers of the 2 pi domain, and a domain of length lx scales the
    /// result by 2 pi / lx = 2 rkx[0].
    pub fn xderiv(&self, rkx: &[f64], var: ArrayView2<f64>, der: ArrayViewMut2<f64>) {
        self.deriv(rkx, var, der, true)
    }

    /// Replaces D2FFT::yderiv (src/sta2dfft.rs:157-184).
    pub fn yderiv(&self, rky: &[f64], var: ArrayView2<f64>, der: ArrayViewMut2<f64>) {
        self.deriv(rky, var, der, false)
    }

    fn deriv(&self, rk: &[f64], var: ArrayView2<f64>, mut der: ArrayViewMut2<f64>, x: bool) {
        for (k, v) in rk.iter().enumerate() {
            assert!((v - rk[0] * (k + 1) as f64).abs() <= 1e-12 * v.abs(), "wavenumbers must be (pi/l) k");
        }
        let scale = 2.0 * rk[0];
        let a = fortran_vec_view(&var);
        let mut d = vec![0.0; a.len()];
        or_quit(self.ctx.with(|c| {
            check(unsafe {
                if x {
                    sys::sw_xderiv(c, a.as_ptr(), d.as_mut_ptr())
                } else {
                    sys::sw_yderiv(c, a.as_ptr(), d.as_mut_ptr())
                }
            })
        }));
        if scale != 1.0 {
            for v in d.iter_mut() {
                *v *= scale;
            }
        }
        fill_fortran(&mut der, &d);
    }
}
