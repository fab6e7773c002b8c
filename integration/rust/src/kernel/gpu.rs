//! The B200 backend as an entry of turboGP's kernel table, and the safe
//! wrappers the query interpreter's hand-offs call.
//!
//! Not compiled here (this image has no Rust toolchain). It is written
//! against the reference's plugin API — `trait Kernel`, `KernelParams`,
//! `KernelResult`, `Operator`, `PredicateOp`, `KernelTable`
//! (src/kernel/mod.rs:38-242), `CpuTarget` (src/kernel/cpu.rs:31-43) and
//! `MemoryTier` (src/memory/tier.rs:11-29) — and against the raw bindings in
//! `gpu_ffi.rs`.
//!
//! Registration: `KernelTable::new` (src/kernel/mod.rs:191-206) gains one call
//! after its CPU registrations, `gpu::register_gpu_kernels(&mut kernels,
//! detected_cpu)`. Each GPU kernel is keyed `(operator, detected CPU,
//! MemoryTier::Hbm)`, so `KernelTable::select(op, MemoryTier::Hbm)` finds it
//! through the reference's first lookup rule (exact match on the detected
//! CPU, mod.rs:209-221) and every other tier keeps selecting the CPU kernels.
#![allow(dead_code)]

use std::ffi::CStr;
use std::os::raw::c_void;
use std::sync::{Arc, Mutex};

use super::gpu_ffi as ffi;
use super::{CpuTarget, Kernel, KernelParams, KernelResult, MemoryTier, Operator, PredicateOp};

/// An error reported by the C ABI: the status code and the context's message.
#[derive(Debug, Clone)]
pub struct GpuError {
    pub status: i32,
    pub message: String,
}

impl std::fmt::Display for GpuError {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        write!(f, "turbogp_b200 status {}: {}", self.status, self.message)
    }
}

impl std::error::Error for GpuError {}

/// One CUDA device's context (`tgp_init` / `tgp_shutdown`). A context may be
/// used from one thread at a time, so it lives behind a mutex.
pub struct GpuContext {
    raw: Mutex<*mut ffi::tgp_ctx>,
}

// The raw pointer is only used under the mutex.
unsafe impl Send for GpuContext {}
unsafe impl Sync for GpuContext {}

impl GpuContext {
    pub fn open(device: i32) -> Result<Arc<Self>, GpuError> {
        let mut raw = std::ptr::null_mut();
        let st = unsafe { ffi::tgp_init(&mut raw, device) };
        if st != ffi::TGP_OK {
            return Err(GpuError { status: st, message: format!("tgp_init(device={device}) failed") });
        }
        Ok(Arc::new(Self { raw: Mutex::new(raw) }))
    }

    /// Runs `f` with the raw context; a nonzero status becomes a GpuError
    /// carrying tgp_last_error.
    pub fn call<F: FnOnce(*mut ffi::tgp_ctx) -> i32>(&self, f: F) -> Result<(), GpuError> {
        let guard = self.raw.lock().expect("context mutex poisoned");
        let st = f(*guard);
        if st == ffi::TGP_OK {
            return Ok(());
        }
        let msg = unsafe { CStr::from_ptr(ffi::tgp_last_error(*guard)) }.to_string_lossy().into_owned();
        Err(GpuError { status: st, message: msg })
    }
}

impl Drop for GpuContext {
    fn drop(&mut self) {
        let raw = *self.raw.get_mut().expect("context mutex poisoned");
        if !raw.is_null() {
            unsafe { ffi::tgp_shutdown(raw) };
        }
    }
}

fn operator_from_index(op: u32) -> Option<Operator> {
    Some(match op {
        ffi::TGP_OP_SCAN_EQ_U64 => Operator::ScanEqU64,
        ffi::TGP_OP_SCAN_RANGE_U64 => Operator::ScanRangeU64,
        ffi::TGP_OP_SCAN_MULTI_PREDICATE => Operator::ScanMultiPredicate,
        ffi::TGP_OP_HASH_BUILD => Operator::HashBuild,
        ffi::TGP_OP_HASH_PROBE => Operator::HashProbe,
        ffi::TGP_OP_AGGREGATE_SUM_F64 => Operator::AggregateSumF64,
        ffi::TGP_OP_AGGREGATE_COUNT_DISTINCT => Operator::AggregateCountDistinct,
        ffi::TGP_OP_SIMILARITY_HAMMING => Operator::SimilarityHamming,
        ffi::TGP_OP_LEAPFROG_JOIN => Operator::LeapfrogJoin,
        _ => return None,
    })
}

fn predicate_op_index(op: PredicateOp) -> u8 {
    match op {
        PredicateOp::Eq => ffi::TGP_PRED_EQ,
        PredicateOp::Gt => ffi::TGP_PRED_GT,
        PredicateOp::Lt => ffi::TGP_PRED_LT,
    }
}

fn params_to_c(p: &KernelParams) -> ffi::tgp_kernel_params {
    ffi::tgp_kernel_params {
        target_u64: p.target_u64,
        low_u64: p.low_u64,
        high_u64: p.high_u64,
        max_distance: p.max_distance,
        _pad0: 0,
        cell_count: p.cell_count as u64,
        target2_u64: p.target2_u64,
        target3_u64: p.target3_u64,
        pred1_op: predicate_op_index(p.pred1_op),
        pred2_op: predicate_op_index(p.pred2_op),
        pred3_op: predicate_op_index(p.pred3_op),
        predicate_count: p.predicate_count,
        _pad1: 0,
    }
}

/// One GPU operator behind the reference's `Kernel` trait.
pub struct GpuKernel {
    ctx: Arc<GpuContext>,
    op: Operator,
    op_index: u32,
    cpu: CpuTarget,
    name: &'static str,
}

impl Kernel for GpuKernel {
    fn operator(&self) -> Operator {
        self.op
    }
    /// The detected host CPU: the GPU kernels sit beside that CPU's kernels
    /// under the HBM tier (see the module comment).
    fn cpu(&self) -> CpuTarget {
        self.cpu
    }
    fn tier(&self) -> MemoryTier {
        MemoryTier::Hbm
    }
    fn name(&self) -> &'static str {
        self.name
    }
    /// `input` / `output` as the reference's kernels take them
    /// (src/kernel/scan.rs:45-62, hash.rs:135-178, aggregate.rs:36-41); host
    /// or device memory. The trait has no error channel (mod.rs:158-177): a
    /// failure panics with the library's message, as a reference kernel
    /// would on a violated safety contract.
    unsafe fn execute(&self, input: *const u8, output: *mut u8, params: &KernelParams) -> KernelResult {
        let p = params_to_c(params);
        let mut r = ffi::tgp_kernel_result::default();
        self.ctx
            .call(|ctx| ffi::tgp_kernel_execute(ctx, self.op_index, input as *const c_void, output as *mut c_void, &p, &mut r))
            .unwrap_or_else(|e| panic!("{}: {e}", self.name));
        KernelResult { count: r.count, sum: r.sum, mask: r.mask }
    }
}

/// Adds every operator the library registers (`tgp_kernel_count` /
/// `tgp_kernel_info_at`) to the kernel map of `KernelTable::new`, keyed
/// `(operator, detected_cpu, MemoryTier::Hbm)`. Operators the GPU does not
/// implement (similarity, leapfrog) are listed by the library but left out.
pub fn register_gpu_kernels(
    kernels: &mut std::collections::HashMap<(Operator, CpuTarget, MemoryTier), Arc<dyn Kernel>>,
    detected_cpu: CpuTarget,
    ctx: &Arc<GpuContext>,
) {
    let n = unsafe { ffi::tgp_kernel_count() };
    for i in 0..n {
        let mut info = std::mem::MaybeUninit::<ffi::tgp_kernel_info>::uninit();
        if unsafe { ffi::tgp_kernel_info_at(i, info.as_mut_ptr()) } != ffi::TGP_OK {
            continue;
        }
        let info = unsafe { info.assume_init() };
        if info.op == ffi::TGP_OP_SIMILARITY_HAMMING || info.op == ffi::TGP_OP_LEAPFROG_JOIN {
            continue;
        }
        let Some(op) = operator_from_index(info.op) else { continue };
        let name: &'static str =
            Box::leak(unsafe { CStr::from_ptr(info.name) }.to_string_lossy().into_owned().into_boxed_str());
        let k = GpuKernel { ctx: ctx.clone(), op, op_index: info.op, cpu: detected_cpu, name };
        kernels.insert((op, detected_cpu, MemoryTier::Hbm), Arc::new(k));
    }
}

// ---------------------------------------------------------------------------
// Safe wrappers for the interpreter's hand-offs
// ---------------------------------------------------------------------------

/// A table resident in HBM (`tgp_table_register_cells`: the reference's own
/// u64 cells and i32 sidecars, narrowed on the device).
pub struct ResidentTable {
    ctx: Arc<GpuContext>,
    pub id: u64,
    pub rows: u64,
}

impl ResidentTable {
    /// `cells[i]` is `Table::columns[i]`, `sidecars[i]` its
    /// `Table::i32_columns[i]` (src/datasource/table.rs:25-66), `coltypes[i]`
    /// the column's `ColType` as TGP_CT_*.
    pub fn from_cells(
        ctx: &Arc<GpuContext>,
        cells: &[&[u64]],
        sidecars: &[Option<&[i32]>],
        coltypes: &[u32],
    ) -> Result<Self, GpuError> {
        let rows = cells.first().map(|c| c.len()).unwrap_or(0) as u64;
        let descs: Vec<ffi::tgp_cell_column> = cells
            .iter()
            .zip(sidecars)
            .zip(coltypes)
            .map(|((c, s), ct)| ffi::tgp_cell_column {
                cells: c.as_ptr(),
                i32_sidecar: s.map(|s| s.as_ptr()).unwrap_or(std::ptr::null()),
                coltype: *ct,
                _pad: 0,
            })
            .collect();
        let mut id = 0u64;
        ctx.call(|c| unsafe { ffi::tgp_table_register_cells(c, descs.as_ptr(), descs.len() as u32, rows, &mut id) })?;
        Ok(Self { ctx: ctx.clone(), id, rows })
    }

    /// WHERE → selection bitmap (LSB-first, the reference's `Bitmap` bytes,
    /// src/exec/bitmap.rs:36-40) and its count: `build_mask`'s hand-off.
    pub fn filter(&self, program: &[ffi::tgp_pred_node]) -> Result<(Vec<u8>, u64), GpuError> {
        let mut bitmap = vec![0u8; ((self.rows + 7) / 8) as usize];
        let mut count = 0u64;
        self.ctx.call(|c| unsafe {
            ffi::tgp_filter(c, self.id, program.as_ptr(), program.len() as u32, bitmap.as_mut_ptr(),
                            std::ptr::null_mut(), 0, &mut count)
        })?;
        Ok((bitmap, count))
    }
}

impl Drop for ResidentTable {
    fn drop(&mut self) {
        let id = self.id;
        let _ = self.ctx.call(|c| unsafe { ffi::tgp_table_drop(c, id) });
    }
}

/// A grouped / scalar result: key tuples in ascending order, exact int128
/// values as (lo, hi) limbs (the reference's `ResultColumn.values: Vec<u64>`
/// cannot carry them, src/engine/result.rs:37-53).
pub struct GroupedResult {
    pub keys: Vec<u64>,
    pub values: Vec<ffi::tgp_agg_value>,
    pub ngroups: u64,
    pub rows_selected: u64,
}

/// `execute_grouped` / `try_accumulator_grouped` / `execute_scalar_agg`'s
/// hand-off (aggregate.rs:507, accum_grouped.rs:55, aggregate.rs:1270), and
/// with `join` set, `hash_join_with_keys` + `execute_grouped` fused
/// (join.rs:544): one tgp_execute, resized once if the groups outgrow the
/// first guess.
pub fn execute(
    ctx: &Arc<GpuContext>,
    table: &ResidentTable,
    program: &[ffi::tgp_pred_node],
    group: &[ffi::tgp_group_key],
    aggs: &[ffi::tgp_agg],
    join: Option<(u64, u32)>,
) -> Result<GroupedResult, GpuError> {
    let q = ffi::tgp_query {
        table: table.id,
        pred: if program.is_empty() { std::ptr::null() } else { program.as_ptr() },
        npred: program.len() as u32,
        ngroup: group.len() as u32,
        group: group.as_ptr(),
        nagg: aggs.len() as u32,
        _pad: 0,
        aggs: aggs.as_ptr(),
        join: join.map(|j| j.0).unwrap_or(0),
        probe_key_column: join.map(|j| j.1).unwrap_or(0),
        flags: 0,
    };
    let mut cap: u64 = 1024;
    loop {
        let mut keys = vec![0u64; (cap * group.len().max(1) as u64) as usize];
        let mut values = vec![ffi::tgp_agg_value::default(); (cap * aggs.len().max(1) as u64) as usize];
        let mut res = ffi::tgp_query_result::default();
        let r = ctx.call(|c| unsafe { ffi::tgp_execute(c, &q, keys.as_mut_ptr(), values.as_mut_ptr(), cap, &mut res) });
        match r {
            Err(e) if e.status == ffi::TGP_CAPACITY && res.ngroups > cap => cap = res.ngroups,
            Err(e) => return Err(e),
            Ok(()) => {
                keys.truncate((res.ngroups * group.len() as u64) as usize);
                values.truncate((res.ngroups * aggs.len() as u64) as usize);
                return Ok(GroupedResult { keys, values, ngroups: res.ngroups, rows_selected: res.rows_selected });
            }
        }
    }
}
