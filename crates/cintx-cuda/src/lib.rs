//! Rust binding of `libcintx_cuda.so`, the B200 engine for cintx's two-electron Coulomb family
//! (`int2e`, `int2c2e`, `int3c2e` over Rys quadrature).
//!
//! The library exports libcint 6.1.3's C signatures for these integrals and cintx-capi's
//! `cintrs_eval` / `cintrs_query_workspace` id dispatch, so this crate is only the FFI
//! declarations of `include/cintx_cuda.h` plus small owning wrappers.  cintx-capi's shim
//! (`crates/cintx-capi/src/shim.rs:371`, `cintrs_eval`) routes a request here with [`route`]
//! before it falls back to `eval_raw` for the ids this engine does not evaluate.
//!
//! The repository that ships the library has no cargo, so this crate is written against the
//! header and is not built or tested there.

use std::os::raw::{c_char, c_int, c_void};

/// libcint's optimizer handle as this library defines it (opaque).
#[repr(C)]
pub struct CINTOpt {
    _private: [u8; 0],
}

/// A batched evaluation plan (`cintx_plan_*`).
#[repr(C)]
pub struct CintxPlan {
    _private: [u8; 0],
}

/// `CintxWorkspaceQuery` of cintx-capi (`shim.rs:52-60`), field for field.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct CintxWorkspaceQuery {
    pub bytes: usize,
    pub alignment: usize,
    pub required_bytes: usize,
    pub chunk_count: usize,
    pub work_units: usize,
}

/// `CintxEvalSummary` of cintx-capi (`shim.rs:62-68`), field for field.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct CintxEvalSummary {
    pub not0: i32,
    pub bytes_written: usize,
    pub workspace_bytes: usize,
}

/// `CintxPlanStats` of `include/cintx_cuda.h`.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct CintxPlanStats {
    pub nquartets: i64,
    pub nintegrals: i64,
    pub nchunks: i64,
    pub max_chunk_doubles: i64,
    pub nprim_quartets: i64,
    pub device_bytes: i64,
    pub nquartets_fp32: i64,
    pub flops: f64,
}

/// Integral families of a plan.
pub const CINTX_INT2E: c_int = 0;
pub const CINTX_INT3C2E: c_int = 1;
pub const CINTX_INT2C2E: c_int = 2;

#[link(name = "cintx_cuda")]
unsafe extern "C" {
    pub fn int2e_sph(out: *mut f64, dims: *mut c_int, shls: *mut c_int, atm: *mut c_int, natm: c_int,
                     bas: *mut c_int, nbas: c_int, env: *mut f64, opt: *mut CINTOpt, cache: *mut f64) -> c_int;
    pub fn int2e_cart(out: *mut f64, dims: *mut c_int, shls: *mut c_int, atm: *mut c_int, natm: c_int,
                      bas: *mut c_int, nbas: c_int, env: *mut f64, opt: *mut CINTOpt, cache: *mut f64) -> c_int;
    pub fn int2e_optimizer(opt: *mut *mut CINTOpt, atm: *mut c_int, natm: c_int, bas: *mut c_int, nbas: c_int,
                           env: *mut f64);
    pub fn int2c2e_sph(out: *mut f64, dims: *mut c_int, shls: *mut c_int, atm: *mut c_int, natm: c_int,
                       bas: *mut c_int, nbas: c_int, env: *mut f64, opt: *mut CINTOpt, cache: *mut f64) -> c_int;
    pub fn int2c2e_cart(out: *mut f64, dims: *mut c_int, shls: *mut c_int, atm: *mut c_int, natm: c_int,
                        bas: *mut c_int, nbas: c_int, env: *mut f64, opt: *mut CINTOpt, cache: *mut f64) -> c_int;
    pub fn int3c2e_sph(out: *mut f64, dims: *mut c_int, shls: *mut c_int, atm: *mut c_int, natm: c_int,
                       bas: *mut c_int, nbas: c_int, env: *mut f64, opt: *mut CINTOpt, cache: *mut f64) -> c_int;
    pub fn int3c2e_cart(out: *mut f64, dims: *mut c_int, shls: *mut c_int, atm: *mut c_int, natm: c_int,
                        bas: *mut c_int, nbas: c_int, env: *mut f64, opt: *mut CINTOpt, cache: *mut f64) -> c_int;
    pub fn CINTdel_optimizer(opt: *mut *mut CINTOpt);

    pub fn cintrs_query_workspace(api: i32, dims: *const i32, dims_len: usize, shls: *const i32, shls_len: usize,
                                  atm: *const i32, atm_len: usize, bas: *const i32, bas_len: usize,
                                  env: *const f64, env_len: usize, opt: *const CINTOpt,
                                  query_out: *mut CintxWorkspaceQuery) -> i32;
    pub fn cintrs_eval(api: i32, out: *mut f64, out_len: usize, dims: *const i32, dims_len: usize,
                       shls: *const i32, shls_len: usize, atm: *const i32, atm_len: usize, bas: *const i32,
                       bas_len: usize, env: *const f64, env_len: usize, opt: *const CINTOpt, cache: *mut f64,
                       cache_len: usize, summary_out: *mut CintxEvalSummary) -> i32;

    pub fn cintx_cuda_last_error_code() -> c_int;
    pub fn cintx_cuda_last_error_message(buf: *mut c_char, cap: usize) -> usize;
    pub fn cintx_cuda_clear_last_error();

    pub fn cintx_plan_shells(plan: *mut *mut CintxPlan, opt: *mut CINTOpt, family: c_int, shls: *const c_int,
                             n: i64, sph: c_int, offsets_out: *mut i64) -> c_int;
    pub fn cintx_plan_int2e_screened(plan: *mut *mut CintxPlan, opt: *mut CINTOpt, cutoff: f64, sph: c_int,
                                     max_chunk_doubles: i64) -> c_int;
    pub fn cintx_plan_int2e_screened_mixed(plan: *mut *mut CintxPlan, opt: *mut CINTOpt, cutoff: f64, sph: c_int,
                                           max_chunk_doubles: i64, fp32_budget: f64, prim_budget: f64) -> c_int;
    pub fn cintx_plan_stats(plan: *const CintxPlan, stats: *mut CintxPlanStats) -> c_int;
    pub fn cintx_plan_execute(plan: *mut CintxPlan, chunk: i64, out_dev: *mut f64, stream: *mut c_void) -> c_int;
    pub fn cintx_plan_execute_host(plan: *mut CintxPlan, chunk: i64, out_host: *mut f64) -> c_int;
    pub fn cintx_plan_jk(plan: *mut CintxPlan, dm: *const f64, nao: c_int, vj: *mut f64, vk: *mut f64,
                         stream: *mut c_void) -> c_int;
    pub fn cintx_plan_destroy(plan: *mut CintxPlan);
}

/// A failed call: cintx-capi's status code (`errors.rs:9-21`, the same numbers) and the
/// library's thread-local message.
#[derive(Debug, Clone)]
pub struct Error {
    pub status: i32,
    pub message: String,
}

fn last_error(status: i32) -> Error {
    let mut buf = vec![0u8; 1024];
    // SAFETY: the buffer is writable for its length; the library NUL-terminates within it.
    let n = unsafe { cintx_cuda_last_error_message(buf.as_mut_ptr() as *mut c_char, buf.len()) };
    buf.truncate(n.min(buf.len().saturating_sub(1)));
    Error { status, message: String::from_utf8_lossy(&buf).into_owned() }
}

/// An optimizer handle of this library (device-resident basis and primitive-pair tables).
pub struct Optimizer {
    raw: *mut CINTOpt,
}

impl Optimizer {
    /// `int2e_optimizer` over libcint's (atm, bas, env) arrays.
    pub fn int2e(atm: &mut [i32], bas: &mut [i32], env: &mut [f64]) -> Result<Self, Error> {
        let mut raw = std::ptr::null_mut();
        // SAFETY: the slices outlive the call; natm / nbas follow libcint's 6 and 8 slots per row.
        unsafe {
            int2e_optimizer(&mut raw, atm.as_mut_ptr(), (atm.len() / 6) as c_int, bas.as_mut_ptr(),
                            (bas.len() / 8) as c_int, env.as_mut_ptr());
        }
        if raw.is_null() {
            // SAFETY: plain query of the thread-local status.
            return Err(last_error(unsafe { cintx_cuda_last_error_code() }));
        }
        Ok(Self { raw })
    }

    pub fn as_ptr(&self) -> *mut CINTOpt {
        self.raw
    }
}

impl Drop for Optimizer {
    fn drop(&mut self) {
        // SAFETY: raw came from this library's optimizer constructor.
        unsafe { CINTdel_optimizer(&mut self.raw) };
    }
}

/// A plan over an optimizer; keeps the optimizer borrowed for its lifetime.
pub struct Plan<'a> {
    raw: *mut CintxPlan,
    _opt: &'a Optimizer,
}

impl<'a> Plan<'a> {
    /// Every 8-fold-unique int2e quartet whose Schwarz bound reaches `cutoff`
    /// (`cintx_plan_int2e_screened`).
    pub fn screened(opt: &'a Optimizer, cutoff: f64, sph: bool, max_chunk_doubles: i64) -> Result<Self, Error> {
        let mut raw = std::ptr::null_mut();
        // SAFETY: opt is a live handle of this library.
        let rc = unsafe { cintx_plan_int2e_screened(&mut raw, opt.as_ptr(), cutoff, sph as c_int, max_chunk_doubles) };
        if rc != 0 {
            return Err(last_error(rc));
        }
        Ok(Self { raw, _opt: opt })
    }

    /// An explicit list of int2e quartets (4 shell ids each); block offsets go to `offsets`.
    pub fn shells(opt: &'a Optimizer, quartets: &[i32], sph: bool, offsets: &mut [i64]) -> Result<Self, Error> {
        let n = quartets.len() / 4;
        assert!(offsets.len() >= n, "offsets must hold one entry per quartet");
        let mut raw = std::ptr::null_mut();
        // SAFETY: quartets holds 4 * n ints and offsets n entries.
        let rc = unsafe {
            cintx_plan_shells(&mut raw, opt.as_ptr(), CINTX_INT2E, quartets.as_ptr(), n as i64, sph as c_int,
                              offsets.as_mut_ptr())
        };
        if rc != 0 {
            return Err(last_error(rc));
        }
        Ok(Self { raw, _opt: opt })
    }

    pub fn stats(&self) -> CintxPlanStats {
        let mut s = CintxPlanStats::default();
        // SAFETY: raw is a live plan.
        unsafe { cintx_plan_stats(self.raw, &mut s) };
        s
    }

    /// Every chunk, back to back, into host memory (`cintx_plan_execute_host`).
    pub fn execute_host(&mut self, out: &mut [f64]) -> Result<(), Error> {
        assert!(out.len() as i64 >= self.stats().nintegrals, "out is smaller than the plan's output");
        // SAFETY: out holds at least nintegrals doubles.
        let rc = unsafe { cintx_plan_execute_host(self.raw, -1, out.as_mut_ptr()) };
        if rc != 0 { Err(last_error(rc)) } else { Ok(()) }
    }
}

impl Drop for Plan<'_> {
    fn drop(&mut self) {
        // SAFETY: raw came from a plan constructor of this library.
        unsafe { cintx_plan_destroy(self.raw) };
    }
}

/// cintx-capi api ids this engine evaluates (`shim.rs:8-50`): int2e_cart 9, int2e_sph 10,
/// int2c2e_cart 12, int2c2e_sph 13, int3c2e_ip1_cart 18, int3c2e_ip1_sph 19, int2e_ip1_cart 35,
/// int2e_ip1_sph 36.
pub fn handles_api(api: i32) -> bool {
    matches!(api, 9 | 10 | 12 | 13 | 18 | 19 | 35 | 36)
}

/// For cintx-capi's `cintrs_eval`: evaluates the request here when [`handles_api`] says so and
/// returns `Some(status)`, else `None` so that the shim falls through to `eval_raw`.  The
/// arguments are cintx-capi's own; `opt` must be NULL or an optimizer made by this library.
///
/// # Safety
/// The pointer/length pairs must describe valid memory, as for cintx-capi's `cintrs_eval`.
#[allow(clippy::too_many_arguments)]
pub unsafe fn route(api: i32, out: *mut f64, out_len: usize, dims: *const i32, dims_len: usize, shls: *const i32,
                    shls_len: usize, atm: *const i32, atm_len: usize, bas: *const i32, bas_len: usize,
                    env: *const f64, env_len: usize, opt: *const CINTOpt, cache: *mut f64, cache_len: usize,
                    summary_out: *mut CintxEvalSummary) -> Option<i32> {
    if !handles_api(api) {
        return None;
    }
    // SAFETY: forwarded unchanged under the caller's guarantees.
    Some(unsafe {
        cintrs_eval(api, out, out_len, dims, dims_len, shls, shls_len, atm, atm_len, bas, bas_len, env, env_len, opt,
                    cache, cache_len, summary_out)
    })
}
