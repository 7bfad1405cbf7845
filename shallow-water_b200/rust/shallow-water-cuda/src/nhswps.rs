//! nhswps (reference src/nhswps/): the state, one predictor-corrector step and
//! its parts, on the device.
//!
//! `State` keeps the reference's public fields (src/nhswps/mod.rs:87-148) in host
//! memory, so code written against the reference keeps working: each function
//! uploads the fields it needs to the state's device context, runs there and
//! downloads what it changes.  `Ensemble` is the device-resident path: the fields
//! of many members stay in HBM across steps and cross the host boundary only when
//! asked for.

use crate::spectral::{Context, Spectral};
use crate::{check, fill_fortran, fortran_vec_view, or_quit, Precision};
use ndarray::{Array3, ArrayView3, ArrayViewMut3, ShapeBuilder};
use shallow_water_cuda_sys as sys;
use std::io::Write;
use std::os::raw::{c_int, c_longlong};

/// Replaces nhswps::State (src/nhswps/mod.rs:87-148).
pub struct State {
    pub spectral: Spectral,
    pub u: Array3<f64>,
    pub v: Array3<f64>,
    pub w: Array3<f64>,
    pub z: Array3<f64>,
    pub zx: Array3<f64>,
    pub zy: Array3<f64>,
    pub r: Array3<f64>,
    pub ri: Array3<f64>,
    pub aa: Array3<f64>,
    pub zeta: Array3<f64>,
    pub pn: Array3<f64>,
    pub dpn: Array3<f64>,
    pub ps: Array3<f64>,
    pub qs: Array3<f64>,
    pub ds: Array3<f64>,
    pub gs: Array3<f64>,
    pub t: f64,
    pub ngsave: usize,
    pub itime: usize,
    pub jtime: usize,
    pub ggen: bool,
}

const FIELDS: [c_int; 16] = [
    sys::SW_U, sys::SW_V, sys::SW_W, sys::SW_Z, sys::SW_ZX, sys::SW_ZY, sys::SW_R, sys::SW_RI, sys::SW_AA,
    sys::SW_ZETA, sys::SW_PN, sys::SW_DPN, sys::SW_PS, sys::SW_QS, sys::SW_DS, sys::SW_GS,
];

impl State {
    /// All fields zero, as the reference's nhswps allocates them (mod.rs:190-235).
    pub fn new(spectral: Spectral) -> Self {
        let (ng, nz) = (spectral.ng, spectral.nz);
        let z = || Array3::<f64>::zeros((ng, ng, nz + 1).f());
        State {
            u: z(), v: z(), w: z(), z: z(), zx: z(), zy: z(), r: z(), ri: z(), aa: z(), zeta: z(), pn: z(),
            dpn: z(), ps: z(), qs: z(), ds: z(), gs: z(), t: 0.0, ngsave: 0, itime: 0, jtime: 0, ggen: false,
            spectral,
        }
    }

    fn field(&self, f: c_int) -> &Array3<f64> {
        match f {
            sys::SW_U => &self.u, sys::SW_V => &self.v, sys::SW_W => &self.w, sys::SW_Z => &self.z,
            sys::SW_ZX => &self.zx, sys::SW_ZY => &self.zy, sys::SW_R => &self.r, sys::SW_RI => &self.ri,
            sys::SW_AA => &self.aa, sys::SW_ZETA => &self.zeta, sys::SW_PN => &self.pn, sys::SW_DPN => &self.dpn,
            sys::SW_PS => &self.ps, sys::SW_QS => &self.qs, sys::SW_DS => &self.ds, _ => &self.gs,
        }
    }

    fn field_mut(&mut self, f: c_int) -> &mut Array3<f64> {
        match f {
            sys::SW_U => &mut self.u, sys::SW_V => &mut self.v, sys::SW_W => &mut self.w, sys::SW_Z => &mut self.z,
            sys::SW_ZX => &mut self.zx, sys::SW_ZY => &mut self.zy, sys::SW_R => &mut self.r,
            sys::SW_RI => &mut self.ri, sys::SW_AA => &mut self.aa, sys::SW_ZETA => &mut self.zeta,
            sys::SW_PN => &mut self.pn, sys::SW_DPN => &mut self.dpn, sys::SW_PS => &mut self.ps,
            sys::SW_QS => &mut self.qs, sys::SW_DS => &mut self.ds, _ => &mut self.gs,
        }
    }

    fn ctx(&self) -> &Context {
        self.spectral.context()
    }

    /// Copies every field and the time to the device context.
    pub fn upload(&self) -> anyhow::Result<()> {
        for f in FIELDS {
            let v = fortran_vec_view(&self.field(f).view());
            self.ctx().with(|c| check(unsafe { sys::sw_state_set(c, f, 0, v.as_ptr(), v.len()) }))?;
        }
        self.ctx().with(|c| check(unsafe { sys::sw_set_time(c, self.t) }))
    }

    /// Copies every field and the time back from the device context.
    pub fn download(&mut self) -> anyhow::Result<()> {
        let n3 = self.ctx().n3();
        for f in FIELDS {
            let mut v = vec![0.0; n3];
            self.ctx().with(|c| check(unsafe { sys::sw_state_get(c, f, 0, v.as_mut_ptr(), n3) }))?;
            fill_fortran(&mut self.field_mut(f).view_mut(), &v);
        }
        let mut t = 0.0;
        self.ctx().with(|c| check(unsafe { sys::sw_get_time(c, &mut t) }))?;
        self.t = t;
        Ok(())
    }

    fn run(&mut self, f: impl FnOnce(*mut sys::SwCtx) -> c_int) -> anyhow::Result<()> {
        self.upload()?;
        self.ctx().with(|c| check(f(c)))?;
        self.download()
    }
}

/// Replaces nhswps::advance::advance (src/nhswps/advance.rs:13-279): one
/// predictor-corrector step (main_invert + psolve first when state.ggen), with the
/// diagnose line of the step's start time written to `monitor` as in
/// src/nhswps/mod.rs:700-708.
pub fn advance(state: &mut State, monitor: &mut dyn Write) -> anyhow::Result<()> {
    let t0 = state.t;
    let ggen = state.ggen as c_int;
    state.run(|c| unsafe { sys::sw_advance(c, 1, ggen) })?;
    let mut d = [0.0f64; 4];
    let mut count: c_int = 0;
    state.ctx().with(|c| check(unsafe { sys::sw_diag_history(c, d.as_mut_ptr(), 1, &mut count) }))?;
    writeln!(monitor, "{:.5} {:.6} {:.6} {:.6} {:.6}", t0, d[0], d[1], d[2], d[3])?;
    Ok(())
}

/// Replaces nhswps::psolve::psolve (src/nhswps/psolve.rs:16-411): quits like the
/// reference when the iteration diverges or reaches its cap.
pub fn psolve(state: &mut State) {
    or_quit(try_psolve(state).map(|_| ()))
}

/// psolve returning (sweeps, final relative change) or the error status.
pub fn try_psolve(state: &mut State) -> anyhow::Result<(usize, f64)> {
    let mut it: c_int = 0;
    let mut e = 0.0f64;
    state.run(|c| unsafe { sys::sw_psolve(c, 100, &mut it, &mut e) })?;
    Ok((it as usize, e))
}

/// Replaces nhswps::vertical::vertical (src/nhswps/vertical.rs:8-143).
pub fn vertical(state: &mut State) {
    or_quit(state.run(|c| unsafe { sys::sw_vertical(c) }))
}

fn three(state: &State, f: impl FnOnce(*mut sys::SwCtx, [*mut f64; 4]) -> c_int, outs: [Option<&mut ArrayViewMut3<f64>>; 4])
         -> anyhow::Result<()> {
    state.upload()?;
    let n3 = state.ctx().n3();
    let mut bufs = [vec![0.0; n3], vec![0.0; n3], vec![0.0; n3], vec![0.0; n3]];
    let ptrs = [bufs[0].as_mut_ptr(), bufs[1].as_mut_ptr(), bufs[2].as_mut_ptr(), bufs[3].as_mut_ptr()];
    state.ctx().with(|c| check(f(c, ptrs)))?;
    for (o, b) in outs.into_iter().zip(bufs.iter()) {
        if let Some(o) = o {
            fill_fortran(o, b);
        }
    }
    Ok(())
}

/// Replaces nhswps::coeffs::coeffs (src/nhswps/coeffs.rs:8-101).
pub fn coeffs(state: &State, mut sigx: ArrayViewMut3<f64>, mut sigy: ArrayViewMut3<f64>,
              mut cpt1: ArrayViewMut3<f64>, mut cpt2: ArrayViewMut3<f64>) {
    or_quit(three(state, |c, p| unsafe { sys::sw_coeffs(c, p[0], p[1], p[2], p[3]) },
                  [Some(&mut sigx), Some(&mut sigy), Some(&mut cpt1), Some(&mut cpt2)]))
}

/// Replaces nhswps::cpsource::cpsource (src/nhswps/cpsource.rs:13-261).
pub fn cpsource(state: &State, mut sp0: ArrayViewMut3<f64>) {
    or_quit(three(state, |c, p| unsafe { sys::sw_cpsource(c, p[0]) }, [Some(&mut sp0), None, None, None]))
}

/// Replaces nhswps::source::source (src/nhswps/source.rs:19-138): the spectral
/// source terms sqs, sds, sgs.
pub fn source(state: &State, mut sqs: ArrayViewMut3<f64>, mut sds: ArrayViewMut3<f64>, mut sgs: ArrayViewMut3<f64>) {
    or_quit(three(state, |c, p| unsafe { sys::sw_source(c, p[0], p[1], p[2]) },
                  [Some(&mut sqs), Some(&mut sds), Some(&mut sgs), None]))
}

/// savegrid's energies (src/nhswps/mod.rs:365-410): {ekin, epot, etot}.
pub fn energy(state: &State) -> anyhow::Result<[f64; 3]> {
    state.upload()?;
    let mut e = [0.0f64; 3];
    state.ctx().with(|c| check(unsafe { sys::sw_energy(c, 0, e.as_mut_ptr()) }))?;
    Ok(e)
}

/// savegrid's data computed on the device in one call (src/nhswps/mod.rs:347-663):
/// energies, the three shell spectra (zeta, delta, gamma; kmax+1 values each) and
/// the float32 3-D (q, delta, gamma, r, w, p) and 2-D (d, zeta, q, g, h) snapshots
/// in Fortran order.  The caller writes the reference's text and .r4 records.
pub struct SaveData {
    pub energies: [f64; 3],
    pub spectra: Vec<f64>,
    pub fields3: Vec<f32>,
    pub fields2: Vec<f32>,
}

pub fn savegrid_data(state: &State) -> anyhow::Result<SaveData> {
    state.upload()?;
    let sp = &state.spectral;
    let (n2, n3) = (sp.ng * sp.ng, sp.ng * sp.ng * (sp.nz + 1));
    let nspec = 3 * (sp.kmax + 1);
    let mut d = SaveData { energies: [0.0; 3], spectra: vec![0.0; nspec], fields3: vec![0.0; 6 * n3],
                           fields2: vec![0.0; 5 * n2] };
    state.ctx().with(|c| check(unsafe {
        sys::sw_savegrid(c, 0, d.energies.as_mut_ptr(), d.spectra.as_mut_ptr(), nspec as c_int,
                         d.fields3.as_mut_ptr(), d.fields2.as_mut_ptr())
    }))?;
    Ok(d)
}

/// An ensemble of members of one (ng, nz) resident on one GPU: every step of every
/// member runs as one CUDA graph launch, without host copies.
pub struct Ensemble {
    ctx: Context,
}

impl Ensemble {
    pub fn new(ng: usize, nz: usize, members: usize, precision: Precision) -> anyhow::Result<Self> {
        Ok(Ensemble { ctx: Context::new(ng, nz, members, precision)? })
    }

    pub fn context(&self) -> &Context {
        &self.ctx
    }

    /// Uploads one field (SW_* index) of one member.
    pub fn set(&self, field: c_int, member: usize, a: ArrayView3<f64>) -> anyhow::Result<()> {
        let v = fortran_vec_view(&a);
        self.ctx.with(|c| check(unsafe { sys::sw_state_set(c, field, member as c_int, v.as_ptr(), v.len()) }))
    }

    /// Downloads one field (SW_* index) of one member.
    pub fn get(&self, field: c_int, member: usize, mut a: ArrayViewMut3<f64>) -> anyhow::Result<()> {
        let mut v = vec![0.0; self.ctx.n3()];
        self.ctx.with(|c| check(unsafe { sys::sw_state_get(c, field, member as c_int, v.as_mut_ptr(), v.len()) }))?;
        fill_fortran(&mut a, &v);
        Ok(())
    }

    /// main_invert of every member (after loading qs, ds, gs).
    pub fn main_invert(&self) -> anyhow::Result<()> {
        self.ctx.with(|c| check(unsafe { sys::sw_main_invert(c) }))
    }

    /// nsteps steps of every member; ggen as State::ggen for the first step.
    pub fn advance(&self, nsteps: usize, ggen: bool) -> anyhow::Result<()> {
        self.ctx.with(|c| check(unsafe { sys::sw_advance(c, nsteps as c_int, ggen as c_int) }))
    }

    /// Queues nsteps steps and returns; `sync` waits for them and returns their status.
    pub fn advance_async(&self, nsteps: usize, ggen: bool) -> anyhow::Result<()> {
        self.ctx.with(|c| check(unsafe { sys::sw_advance_async(c, nsteps as c_int, ggen as c_int) }))
    }

    pub fn sync(&self) -> anyhow::Result<()> {
        self.ctx.with(|c| check(unsafe { sys::sw_sync(c) }))
    }

    /// Pressure sweeps run so far: float64 and float32-correction sweeps.
    pub fn sweep_counts(&self) -> anyhow::Result<[i64; 2]> {
        let mut o: [c_longlong; 2] = [0, 0];
        self.ctx.with(|c| check(unsafe { sys::sw_sweep_counts(c, o.as_mut_ptr()) }))?;
        Ok([o[0] as i64, o[1] as i64])
    }

    /// Stop rule of the pressure iteration of a Mixed ensemble (default 1e-7).
    pub fn set_psolve_toler(&self, toler: f64) -> anyhow::Result<()> {
        self.ctx.with(|c| check(unsafe { sys::sw_set_psolve_toler(c, toler) }))
    }

    /// Relaxation factor in (0, 1] of the pressure iteration (default 1, the
    /// reference's iteration); the fixed point does not depend on it.
    pub fn set_psolve_relax(&self, omega: f64) -> anyhow::Result<()> {
        self.ctx.with(|c| check(unsafe { sys::sw_set_psolve_relax(c, omega) }))
    }
}
