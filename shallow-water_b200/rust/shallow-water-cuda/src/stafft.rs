//! stafft (reference src/stafft/mod.rs): mixed-radix real FFTs in the Hermitian
//! convention, m transforms of length n on x[i + m*j] (an (m, n) array).

use crate::{check, fill_fortran, fortran_vec, or_quit};
use ndarray::ArrayViewMut2;
use shallow_water_cuda_sys as sys;
use std::os::raw::c_int;

fn to_c(factors: &[usize; 5]) -> [c_int; 5] {
    [factors[0] as c_int, factors[1] as c_int, factors[2] as c_int, factors[3] as c_int, factors[4] as c_int]
}

/// Replaces stafft::factorisen (src/stafft/mod.rs:97-150): the counts of the
/// radices [6, 4, 2, 3, 5] of n.  Quits like the reference when n has another factor.
pub fn factorisen(n: usize, factors: &mut [usize; 5]) {
    or_quit(try_factorisen(n, factors))
}

pub fn try_factorisen(n: usize, factors: &mut [usize; 5]) -> anyhow::Result<()> {
    let mut f: [c_int; 5] = [0; 5];
    check(unsafe { sys::sw_factorisen(n as c_int, f.as_mut_ptr()) })?;
    for i in 0..5 {
        factors[i] = f[i] as usize;
    }
    Ok(())
}

/// Replaces stafft::initfft (src/stafft/mod.rs:67-95): factors and the 2n-entry
/// trig table of the reference (the GPU keeps its own twiddles).
pub fn initfft(n: usize, factors: &mut [usize; 5], trig: &mut [f64]) {
    or_quit(try_initfft(n, factors, trig))
}

pub fn try_initfft(n: usize, factors: &mut [usize; 5], trig: &mut [f64]) -> anyhow::Result<()> {
    assert!(trig.len() >= 2 * n, "trig needs 2n entries");
    let mut f: [c_int; 5] = [0; 5];
    check(unsafe { sys::sw_initfft(n as c_int, f.as_mut_ptr(), trig.as_mut_ptr()) })?;
    for i in 0..5 {
        factors[i] = f[i] as usize;
    }
    Ok(())
}

/// Replaces stafft::forfft (src/stafft/mod.rs:158): forward transforms of the m
/// columns of xs (shape (m, n)), in place.
pub fn forfft(m: usize, n: usize, xs: ArrayViewMut2<f64>, trig: &[f64], factors: &[usize; 5]) {
    or_quit(try_fft(m, n, xs, trig, factors, false))
}

/// Replaces stafft::revfft (src/stafft/mod.rs:301): the inverse of forfft.
pub fn revfft(m: usize, n: usize, xs: ArrayViewMut2<f64>, trig: &[f64], factors: &[usize; 5]) {
    or_quit(try_fft(m, n, xs, trig, factors, true))
}

pub fn try_fft(m: usize, n: usize, mut xs: ArrayViewMut2<f64>, trig: &[f64], factors: &[usize; 5],
               inverse: bool) -> anyhow::Result<()> {
    assert_eq!(xs.shape(), &[m, n], "xs must have shape (m, n)");
    let mut x = fortran_vec(&xs);
    let f = to_c(factors);
    let st = unsafe {
        if inverse {
            sys::sw_revfft(m as c_int, n as c_int, x.as_mut_ptr(), trig.as_ptr(), f.as_ptr())
        } else {
            sys::sw_forfft(m as c_int, n as c_int, x.as_mut_ptr(), trig.as_ptr(), f.as_ptr())
        }
    };
    check(st)?;
    fill_fortran(&mut xs, &x);
    Ok(())
}
