//! Raw bindings of the B200 backend's C ABI (`include/turbogp_gpu.h`):
//! `#[repr(C)]` twins of its structs, its constants and its functions.
//!
//! Not compiled here (this image has no Rust toolchain); the repository's
//! `tests/test_rust_shim.py` checks every struct below field by field against
//! the header's offsets and sizes (compiled with gcc), every constant against
//! the header's value, and that every `TGP_API` function is declared here with
//! the same number of arguments.
#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_int, c_void};

// ---------------------------------------------------------------------------
// Status codes (tgp_status)
// ---------------------------------------------------------------------------
pub const TGP_OK: c_int = 0;
pub const TGP_INVALID_ARG: c_int = 1;
pub const TGP_OOM: c_int = 2;
pub const TGP_UNSUPPORTED: c_int = 3;
pub const TGP_TIMEOUT: c_int = 4;
pub const TGP_DEVICE_ERROR: c_int = 5;
pub const TGP_NOT_FOUND: c_int = 6;
pub const TGP_CAPACITY: c_int = 7;
pub const TGP_PENDING: c_int = 8;

// Operators (tgp_operator), in the order of the reference's `enum Operator`.
pub const TGP_OP_SCAN_EQ_U64: u32 = 0;
pub const TGP_OP_SCAN_RANGE_U64: u32 = 1;
pub const TGP_OP_SCAN_MULTI_PREDICATE: u32 = 2;
pub const TGP_OP_HASH_BUILD: u32 = 3;
pub const TGP_OP_HASH_PROBE: u32 = 4;
pub const TGP_OP_AGGREGATE_SUM_F64: u32 = 5;
pub const TGP_OP_AGGREGATE_COUNT_DISTINCT: u32 = 6;
pub const TGP_OP_SIMILARITY_HAMMING: u32 = 7;
pub const TGP_OP_LEAPFROG_JOIN: u32 = 8;

// Predicate operators (tgp_predicate_op).
pub const TGP_PRED_EQ: u8 = 0;
pub const TGP_PRED_GT: u8 = 1;
pub const TGP_PRED_LT: u8 = 2;

// Memory tiers (tgp_memory_tier), in the order of `enum MemoryTier`.
pub const TGP_TIER_HBM: u32 = 3;
// CPU targets (tgp_cpu_target): the GPU kernels register under this one.
pub const TGP_CPU_GPU_SM100A: u32 = 5;

// Column element types (tgp_dtype) and comparison types (tgp_coltype).
pub const TGP_DT_U8: u32 = 1;
pub const TGP_DT_I32: u32 = 2;
pub const TGP_DT_I64: u32 = 3;
pub const TGP_DT_U64: u32 = 4;
pub const TGP_DT_F64: u32 = 5;
pub const TGP_CT_INT: u32 = 0;
pub const TGP_CT_DATE: u32 = 1;
pub const TGP_CT_FLOAT: u32 = 2;

// Comparisons (tgp_cmp) and predicate program nodes (tgp_pred_kind).
pub const TGP_CMP_EQ: u32 = 0;
pub const TGP_CMP_NE: u32 = 1;
pub const TGP_CMP_LT: u32 = 2;
pub const TGP_CMP_LE: u32 = 3;
pub const TGP_CMP_GT: u32 = 4;
pub const TGP_CMP_GE: u32 = 5;
pub const TGP_CMP_BETWEEN: u32 = 6;
pub const TGP_CMP_NOT_BETWEEN: u32 = 7;
pub const TGP_PN_LEAF: u32 = 0;
pub const TGP_PN_AND: u32 = 1;
pub const TGP_PN_OR: u32 = 2;
pub const TGP_PN_NOT: u32 = 3;

// Aggregates (tgp_agg_func) and column sides (tgp_side).
pub const TGP_AGG_COUNT_STAR: u32 = 0;
pub const TGP_AGG_COUNT_NONZERO: u32 = 1;
pub const TGP_AGG_SUM: u32 = 2;
pub const TGP_AGG_AVG: u32 = 3;
pub const TGP_AGG_MIN: u32 = 4;
pub const TGP_AGG_MAX: u32 = 5;
pub const TGP_SIDE_PROBE: u32 = 0;
pub const TGP_SIDE_BUILD: u32 = 1;

pub const TGP_MAX_FACTORS: usize = 4;
pub const TGP_MAX_AGGS: usize = 8;
pub const TGP_MAX_GROUP_KEYS: usize = 4;
pub const TGP_RESULT_ROW_OVERFLOW: u32 = 1;
pub const TGP_NOALLOC_SCRATCH_BYTES: usize = 1024 * 1024;

// ---------------------------------------------------------------------------
// Structs
// ---------------------------------------------------------------------------
/// Opaque context (`tgp_ctx`).
#[repr(C)]
pub struct tgp_ctx {
    _private: [u8; 0],
}

#[repr(C)]
#[derive(Debug, Default, Clone, Copy)]
pub struct tgp_kernel_params {
    pub target_u64: u64,
    pub low_u64: u64,
    pub high_u64: u64,
    pub max_distance: u32,
    pub _pad0: u32,
    pub cell_count: u64,
    pub target2_u64: u64,
    pub target3_u64: u64,
    pub pred1_op: u8,
    pub pred2_op: u8,
    pub pred3_op: u8,
    pub predicate_count: u8,
    pub _pad1: u32,
}

#[repr(C)]
#[derive(Debug, Default, Clone, Copy)]
pub struct tgp_kernel_result {
    pub count: u64,
    pub sum: f64,
    pub mask: u64,
}

#[repr(C)]
#[derive(Debug, Clone, Copy)]
pub struct tgp_kernel_info {
    pub op: u32,
    pub cpu: u32,
    pub tier: u32,
    pub _pad: u32,
    pub name: *const c_char,
}

#[repr(C)]
#[derive(Debug, Clone, Copy)]
pub struct tgp_column_desc {
    pub dtype: u32,
    pub coltype: u32,
    pub data: *const c_void,
}

#[repr(C)]
#[derive(Debug, Clone, Copy)]
pub struct tgp_cell_column {
    pub cells: *const u64,
    pub i32_sidecar: *const i32,
    pub coltype: u32,
    pub _pad: u32,
}

#[repr(C)]
#[derive(Debug, Default, Clone, Copy)]
pub struct tgp_pred_node {
    pub kind: u32,
    pub column: u32,
    pub cmp: u32,
    pub _pad: u32,
    pub lit: u64,
    pub lit2: u64,
}

#[repr(C)]
#[derive(Debug, Default, Clone, Copy)]
pub struct tgp_factor {
    pub column: i32,
    pub side: u32,
    pub mul: i64,
    pub add: i64,
}

#[repr(C)]
#[derive(Debug, Default, Clone, Copy)]
pub struct tgp_agg {
    pub func: u32,
    pub nfactors: u32,
    pub f: [tgp_factor; TGP_MAX_FACTORS],
}

#[repr(C)]
#[derive(Debug, Default, Clone, Copy)]
pub struct tgp_group_key {
    pub column: u32,
    pub side: u32,
}

#[repr(C)]
#[derive(Debug, Clone, Copy)]
pub struct tgp_query {
    pub table: u64,
    pub pred: *const tgp_pred_node,
    pub npred: u32,
    pub ngroup: u32,
    pub group: *const tgp_group_key,
    pub nagg: u32,
    pub _pad: u32,
    pub aggs: *const tgp_agg,
    pub join: u64,
    pub probe_key_column: u32,
    pub flags: u32,
}

#[repr(C)]
#[derive(Debug, Default, Clone, Copy)]
pub struct tgp_agg_value {
    pub lo: u64,
    pub hi: i64,
    pub count: u64,
    pub as_f64: f64,
}

#[repr(C)]
#[derive(Debug, Default, Clone, Copy)]
pub struct tgp_query_result {
    pub rows_scanned: u64,
    pub rows_selected: u64,
    pub ngroups: u64,
    pub flags: u32,
    pub _pad: u32,
}

#[repr(C)]
#[derive(Debug, Clone, Copy)]
pub struct tgp_batch_item {
    pub query: *const tgp_query,
    pub keys_out: *mut u64,
    pub vals_out: *mut tgp_agg_value,
    pub group_cap: u64,
    pub result: tgp_query_result,
    pub status: i32,
    pub _pad: u32,
}

#[repr(C)]
#[derive(Debug, Default, Clone, Copy)]
pub struct tgp_variant {
    pub threads: u32,
    pub max_stages: u32,
    pub placement: u32,
    pub presum: u32,
    pub dense: u32,
    pub shapes: u32,
    pub payload: u32,
    pub ctas_per_sm: u32,
    pub l2_ahead: u32,
    pub _pad: u32,
}

#[repr(C)]
#[derive(Debug, Default, Clone, Copy)]
pub struct tgp_tune_entry {
    pub variant: tgp_variant,
    pub ms: f64,
    pub status: i32,
    pub same_result: u32,
    pub threads_used: u32,
    pub stages_used: u32,
    pub mode_used: u32,
    pub _pad: u32,
}

#[repr(C)]
#[derive(Debug, Default, Clone, Copy)]
pub struct tgp_key_domain {
    pub column: u32,
    pub _pad: u32,
    pub min: i64,
    pub count: u64,
}

// ---------------------------------------------------------------------------
// Functions
// ---------------------------------------------------------------------------
extern "C" {
    pub fn tgp_status_string(status: c_int) -> *const c_char;
    pub fn tgp_init(out: *mut *mut tgp_ctx, device: c_int) -> c_int;
    pub fn tgp_shutdown(ctx: *mut tgp_ctx) -> c_int;
    pub fn tgp_last_error(ctx: *const tgp_ctx) -> *const c_char;
    pub fn tgp_ctx_stream(ctx: *mut tgp_ctx) -> *mut c_void;
    pub fn tgp_ctx_sm_count(ctx: *const tgp_ctx) -> c_int;
    pub fn tgp_sync(ctx: *mut tgp_ctx) -> c_int;
    pub fn tgp_profile_enable(ctx: *mut tgp_ctx, on: c_int) -> c_int;
    pub fn tgp_profile_read(ctx: *mut tgp_ctx, launches: *mut u64, total_ms: *mut f64) -> c_int;

    pub fn tgp_kernel_count() -> u32;
    pub fn tgp_kernel_info_at(i: u32, out: *mut tgp_kernel_info) -> c_int;
    pub fn tgp_kernel_execute(
        ctx: *mut tgp_ctx,
        op: u32,
        input: *const c_void,
        output: *mut c_void,
        params: *const tgp_kernel_params,
        result: *mut tgp_kernel_result,
    ) -> c_int;
    pub fn tgp_hash_table_free(ctx: *mut tgp_ctx, handle: *mut c_void) -> c_int;

    pub fn tgp_table_register(
        ctx: *mut tgp_ctx,
        cols: *const tgp_column_desc,
        ncols: u32,
        rows: u64,
        out: *mut u64,
    ) -> c_int;
    pub fn tgp_table_register_device(
        ctx: *mut tgp_ctx,
        cols: *const tgp_column_desc,
        ncols: u32,
        rows: u64,
        out: *mut u64,
    ) -> c_int;
    pub fn tgp_table_register_cells(
        ctx: *mut tgp_ctx,
        cols: *const tgp_cell_column,
        ncols: u32,
        rows: u64,
        out: *mut u64,
    ) -> c_int;
    pub fn tgp_table_column_dtype(ctx: *mut tgp_ctx, table: u64, col: u32, dtype: *mut u32) -> c_int;
    pub fn tgp_table_reload(ctx: *mut tgp_ctx, table: u64, cols: *const tgp_column_desc, ncols: u32) -> c_int;
    pub fn tgp_table_drop(ctx: *mut tgp_ctx, table: u64) -> c_int;
    pub fn tgp_table_info(ctx: *mut tgp_ctx, table: u64, rows: *mut u64, ncols: *mut u32) -> c_int;
    pub fn tgp_table_column_stats(
        ctx: *mut tgp_ctx,
        table: u64,
        col: u32,
        min_cell: *mut i64,
        max_cell: *mut i64,
    ) -> c_int;

    pub fn tgp_filter(
        ctx: *mut tgp_ctx,
        table: u64,
        pred: *const tgp_pred_node,
        npred: u32,
        bitmap_out: *mut u8,
        rowids_out: *mut u32,
        rowids_cap: u64,
        count_out: *mut u64,
    ) -> c_int;
    pub fn tgp_execute(
        ctx: *mut tgp_ctx,
        q: *const tgp_query,
        keys_out: *mut u64,
        vals_out: *mut tgp_agg_value,
        group_cap: u64,
        result: *mut tgp_query_result,
    ) -> c_int;
    pub fn tgp_execute_topn(
        ctx: *mut tgp_ctx,
        q: *const tgp_query,
        order_agg: u32,
        descending: c_int,
        limit: u64,
        keys_out: *mut u64,
        vals_out: *mut tgp_agg_value,
        result: *mut tgp_query_result,
    ) -> c_int;
    pub fn tgp_query_footprint(ctx: *mut tgp_ctx, q: *const tgp_query, device_bytes: *mut u64) -> c_int;
    pub fn tgp_count_distinct(
        ctx: *mut tgp_ctx,
        table: u64,
        column: u32,
        pred: *const tgp_pred_node,
        npred: u32,
        count: *mut u64,
        method: *mut u32,
    ) -> c_int;
    pub fn tgp_hll_estimate(regs: *const u32, out: *mut u64) -> c_int;

    pub fn tgp_join_build(
        ctx: *mut tgp_ctx,
        build_table: u64,
        key_column: u32,
        pred: *const tgp_pred_node,
        npred: u32,
        out: *mut u64,
    ) -> c_int;
    pub fn tgp_join_build_smaller(
        ctx: *mut tgp_ctx,
        table_a: u64,
        key_a: u32,
        pred_a: *const tgp_pred_node,
        npred_a: u32,
        table_b: u64,
        key_b: u32,
        pred_b: *const tgp_pred_node,
        npred_b: u32,
        out: *mut u64,
        build_is_a: *mut u32,
        rows_a: *mut u64,
        rows_b: *mut u64,
    ) -> c_int;
    pub fn tgp_join_drop(ctx: *mut tgp_ctx, join: u64) -> c_int;
    pub fn tgp_join_probe_pairs(
        ctx: *mut tgp_ctx,
        join: u64,
        probe_table: u64,
        probe_key_column: u32,
        pred: *const tgp_pred_node,
        npred: u32,
        probe_rows: *mut u32,
        build_rows: *mut u32,
        cap: u64,
        npairs: *mut u64,
    ) -> c_int;

    pub fn tgp_batch_submit(ctx: *mut tgp_ctx, items: *mut tgp_batch_item, n: u32, out: *mut u64) -> c_int;
    pub fn tgp_batch_poll(ctx: *mut tgp_ctx, batch: u64, wait: c_int) -> c_int;

    pub fn tgp_graph_capture(ctx: *mut tgp_ctx, q: *const tgp_query, out: *mut u64) -> c_int;
    pub fn tgp_graph_launch(
        ctx: *mut tgp_ctx,
        graph: u64,
        keys_out: *mut u64,
        vals_out: *mut tgp_agg_value,
        group_cap: u64,
        result: *mut tgp_query_result,
    ) -> c_int;
    pub fn tgp_graph_drop(ctx: *mut tgp_ctx, graph: u64) -> c_int;

    pub fn tgp_strings_register(
        ctx: *mut tgp_ctx,
        bytes: *const u8,
        nbytes: u64,
        offsets: *const u64,
        n: u64,
        out: *mut u64,
    ) -> c_int;
    pub fn tgp_strings_drop(ctx: *mut tgp_ctx, strings: u64) -> c_int;
    pub fn tgp_debug_fail_next_scan(ctx: *mut tgp_ctx, tile: u64, wait_ns: u64) -> c_int;
    pub fn tgp_like(
        ctx: *mut tgp_ctx,
        strings: u64,
        pattern: *const c_char,
        pattern_len: u32,
        negated: c_int,
        bitmap_out: *mut u8,
        count_out: *mut u64,
    ) -> c_int;

    pub fn tgp_set_default_variant(ctx: *mut tgp_ctx, v: *const tgp_variant) -> c_int;
    pub fn tgp_get_default_variant(ctx: *mut tgp_ctx, v: *mut tgp_variant) -> c_int;
    pub fn tgp_batch_config(ctx: *mut tgp_ctx, morsel_tiles: u32, shared_scans: c_int, share_extra_max: u64) -> c_int;
    pub fn tgp_tune_class(ctx: *mut tgp_ctx, q: *const tgp_query, key: *mut u64) -> c_int;
    pub fn tgp_tune_set(ctx: *mut tgp_ctx, key: u64, v: *const tgp_variant) -> c_int;
    pub fn tgp_tune_get(ctx: *mut tgp_ctx, key: u64, v: *mut tgp_variant, found: *mut c_int) -> c_int;
    pub fn tgp_tune_count(ctx: *mut tgp_ctx, n: *mut u32) -> c_int;
    pub fn tgp_tune_at(ctx: *mut tgp_ctx, i: u32, key: *mut u64, v: *mut tgp_variant) -> c_int;
    pub fn tgp_tune_clear(ctx: *mut tgp_ctx) -> c_int;
    pub fn tgp_autotune(
        ctx: *mut tgp_ctx,
        q: *const tgp_query,
        reps: u32,
        entries: *mut tgp_tune_entry,
        cap: u32,
        n: *mut u32,
        best: *mut u32,
        key: *mut u64,
    ) -> c_int;

    pub fn tgp_aggregate_noalloc(
        device: c_int,
        stream: *mut c_void,
        cols: *const tgp_column_desc,
        ncols: u32,
        rows: u64,
        pred: *const tgp_pred_node,
        npred: u32,
        keys: *const tgp_key_domain,
        nkeys: u32,
        aggs: *const tgp_agg,
        nagg: u32,
        vals_out: *mut tgp_agg_value,
        vals_cap: u64,
        result: *mut tgp_query_result,
        err_msg: *mut c_char,
        err_cap: usize,
    ) -> c_int;
}
