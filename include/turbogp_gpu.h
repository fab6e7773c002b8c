/*
 * turbogp_gpu.h — C ABI of the B200 (sm_100a) execution backend for turboGP's
 * data-parallel hot path: predicate scan/filter into selection bitmaps,
 * hash-join build and probe, and grouped/scalar hash aggregation.
 *
 * Every entry point is `extern "C"`, takes plain pointers, sizes and POD
 * structs, never throws, and reports failures through `tgp_status`.
 * Column and output pointers may be host memory (pageable or pinned) or device
 * memory of the context's GPU; the library detects which.
 *
 * Reference interfaces these entry points replace (paths inside pkhairkh/turboGP):
 *   - src/kernel/mod.rs:48-177    Operator / PredicateOp / KernelParams /
 *                                 KernelResult / trait Kernel::execute
 *   - src/kernel/mod.rs:188-242   KernelTable::{new, select, register, list}
 *   - src/memory/tier.rs:11-29    MemoryTier (the HBM tier the GPU kernels use)
 *   - src/exec/bitmap.rs:42-316   Bitmap (LSB-first packed selection bitmap),
 *                                 filter_* and iter_set_bits
 *   - src/engine/query_interpreter/expr.rs:419,633,1468  build_mask → bitmap
 *   - src/engine/query_interpreter/aggregate.rs:507,1270,1291  grouped/scalar agg
 *   - src/engine/query_interpreter/accum_grouped.rs:55   accumulator GROUP BY
 *   - src/engine/query_interpreter/join.rs:544           hash_join_with_keys
 *   - src/exec/join_hash_table.rs:55-212                 JoinHashTable
 */
#ifndef TURBOGP_GPU_H
#define TURBOGP_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TGP_ABI_VERSION 1u

#if defined(__GNUC__)
#define TGP_API __attribute__((visibility("default")))
#else
#define TGP_API
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */

/* The reference's Kernel trait has no error channel (src/kernel/mod.rs:158-177;
 * callers map a missing kernel to Error::Unsupported, src/engine/executor.rs:1015).
 * The C ABI returns one of these from every call instead. */
typedef enum tgp_status {
    TGP_OK = 0,
    TGP_INVALID_ARG = 1,   /* null pointer, bad index, misaligned device column, bad program */
    TGP_OOM = 2,           /* device or pinned-host allocation failed, or over the memory budget */
    TGP_UNSUPPORTED = 3,   /* query shape this backend does not execute */
    TGP_TIMEOUT = 4,       /* a bounded device wait gave up; the context stays usable */
    TGP_DEVICE_ERROR = 5,  /* CUDA runtime error */
    TGP_NOT_FOUND = 6,     /* unknown table / join / ticket id */
    TGP_CAPACITY = 7,      /* caller-provided output buffer too small; required size reported */
    TGP_PENDING = 8        /* tgp_batch_poll: the batch has not finished yet */
} tgp_status;

/* Human-readable name of a status code (static storage). */
TGP_API const char* tgp_status_string(int status);

/* ------------------------------------------------------------------------ */
/* Context                                                                   */
/* ------------------------------------------------------------------------ */

typedef struct tgp_ctx tgp_ctx;

/* Opens a context on CUDA device `device`: a stream, a device scratch arena
 * and pinned staging buffers. One context may be used from one host thread at
 * a time. */
TGP_API int tgp_init(tgp_ctx** out, int device);
TGP_API int tgp_shutdown(tgp_ctx* ctx);

/* Last error message recorded on this context (static until the next call). */
TGP_API const char* tgp_last_error(const tgp_ctx* ctx);

/* The cudaStream_t (as void*) every kernel of this context is launched on. */
TGP_API void* tgp_ctx_stream(tgp_ctx* ctx);

/* Number of streaming multiprocessors of the context's device. */
TGP_API int tgp_ctx_sm_count(const tgp_ctx* ctx);

/* Blocks until all work enqueued on the context's stream has finished. */
TGP_API int tgp_sync(tgp_ctx* ctx);

/* When enabled, the context records CUDA events on its stream around every
 * scan-kernel launch; tgp_profile_read returns the launches recorded since the
 * last read and their summed device time (ms), then resets the record.
 * on = 1: events only (a launch issued to an idle GPU also counts the host's
 * submission time). on = 2: each timed launch is queued behind a one-thread
 * device delay (50 us), so the events bracket the kernel alone. 0: off. */
TGP_API int tgp_profile_enable(tgp_ctx* ctx, int on);
TGP_API int tgp_profile_read(tgp_ctx* ctx, uint64_t* launches, double* total_ms);

/* ------------------------------------------------------------------------ */
/* Kernel table boundary (mirrors src/kernel/mod.rs)                         */
/* ------------------------------------------------------------------------ */

/* Mirrors `enum Operator` (src/kernel/mod.rs:48-74), same order. */
typedef enum tgp_operator {
    TGP_OP_SCAN_EQ_U64 = 0,
    TGP_OP_SCAN_RANGE_U64 = 1,
    TGP_OP_SCAN_MULTI_PREDICATE = 2,
    TGP_OP_HASH_BUILD = 3,
    TGP_OP_HASH_PROBE = 4,
    TGP_OP_AGGREGATE_SUM_F64 = 5,
    TGP_OP_AGGREGATE_COUNT_DISTINCT = 6,
    TGP_OP_SIMILARITY_HAMMING = 7,   /* not implemented on the GPU: TGP_UNSUPPORTED */
    TGP_OP_LEAPFROG_JOIN = 8         /* not implemented on the GPU: TGP_UNSUPPORTED */
} tgp_operator;

/* Mirrors `enum PredicateOp` (src/kernel/mod.rs:84-92). */
typedef enum tgp_predicate_op {
    TGP_PRED_EQ = 0,
    TGP_PRED_GT = 1,
    TGP_PRED_LT = 2
} tgp_predicate_op;

/* Mirrors `enum MemoryTier` (src/memory/tier.rs:11-29), same order. */
typedef enum tgp_memory_tier {
    TGP_TIER_L1L2 = 0,
    TGP_TIER_L3 = 1,
    TGP_TIER_DDR5 = 2,
    TGP_TIER_HBM = 3,
    TGP_TIER_CXL = 4,
    TGP_TIER_NVME = 5,
    TGP_TIER_NVMEOF = 6,
    TGP_TIER_NETWORK = 7
} tgp_memory_tier;

/* Mirrors `enum CpuTarget` (src/kernel/cpu.rs:31-43) plus the new GPU target
 * the B200 kernels register under. */
typedef enum tgp_cpu_target {
    TGP_CPU_SCALAR = 0,
    TGP_CPU_X86_AVX2 = 1,
    TGP_CPU_X86_AVX512 = 2,
    TGP_CPU_ARM_NEON = 3,
    TGP_CPU_ARM_SVE = 4,
    TGP_CPU_GPU_SM100A = 5
} tgp_cpu_target;

/* Field-for-field mirror of `struct KernelParams` (src/kernel/mod.rs:96-119).
 * The Rust struct has no #[repr(C)], so a Rust caller declares a #[repr(C)]
 * twin of this layout and converts field by field. */
typedef struct tgp_kernel_params {
    uint64_t target_u64;
    uint64_t low_u64;
    uint64_t high_u64;
    uint32_t max_distance;
    uint32_t _pad0;
    uint64_t cell_count;
    uint64_t target2_u64;
    uint64_t target3_u64;
    uint8_t pred1_op;          /* tgp_predicate_op */
    uint8_t pred2_op;
    uint8_t pred3_op;
    uint8_t predicate_count;   /* 0..=3 */
    uint32_t _pad1;
} tgp_kernel_params;

/* Mirror of `struct KernelResult` (src/kernel/mod.rs:140-148). */
typedef struct tgp_kernel_result {
    uint64_t count;
    double sum;
    uint64_t mask;
} tgp_kernel_result;

/* One GPU kernel as it registers into the reference's KernelTable:
 * key (operator, cpu, tier) as in src/kernel/mod.rs:39, plus its name. */
typedef struct tgp_kernel_info {
    uint32_t op;      /* tgp_operator */
    uint32_t cpu;     /* tgp_cpu_target (always TGP_CPU_GPU_SM100A) */
    uint32_t tier;    /* tgp_memory_tier (always TGP_TIER_HBM) */
    uint32_t _pad;
    const char* name; /* static storage */
} tgp_kernel_info;

/* Number of GPU kernels this library registers, and the i-th one. Replaces the
 * register_*_kernels functions of src/kernel/mod.rs:245-375 for the GPU. */
TGP_API uint32_t tgp_kernel_count(void);
TGP_API int tgp_kernel_info_at(uint32_t i, tgp_kernel_info* out);

/* Replaces `unsafe fn Kernel::execute(&self, input, output, params)`
 * (src/kernel/mod.rs:171-176) for every operator the GPU registers.
 *
 * Input layouts follow the reference exactly:
 *  - scan / sum / count-distinct: `input` = `cell_count` u64 cells
 *    (src/kernel/scan.rs:45-48, src/kernel/aggregate.rs:36-41).
 *  - HASH_BUILD: `input` = `cell_count` u64 keys; `output` receives an opaque
 *    table handle in its first 8 bytes (src/kernel/hash.rs:135-147). Free it
 *    with tgp_hash_table_free (the reference frees its Box with
 *    Box::from_raw, src/kernel/hash.rs:284).
 *  - HASH_PROBE: `input` = [handle: 8 bytes][cell_count u64 probe keys]
 *    (src/kernel/hash.rs:171-178); result.count = number of matching
 *    (probe, build) pairs.
 * `input` may be host or device memory. `output` is caller-owned host memory of
 * at least 64 bytes (callers pass `[0u8; 64]`, src/engine/executor.rs:1018),
 * or NULL for operators other than HASH_BUILD.
 * Scan kernels fill `mask` with the match bits of the first 64 cells, as the
 * scalar kernel does (src/kernel/scan.rs:50-62). */
TGP_API int tgp_kernel_execute(tgp_ctx* ctx, uint32_t op, const void* input, void* output,
                       const tgp_kernel_params* params, tgp_kernel_result* result);

/* Frees a table handle produced by TGP_OP_HASH_BUILD. */
TGP_API int tgp_hash_table_free(tgp_ctx* ctx, void* handle);

/* ------------------------------------------------------------------------ */
/* HBM-resident tables (device tier for src/datasource/table.rs:25-66)       */
/* ------------------------------------------------------------------------ */

/* Physical element type of a resident column. The reference stores every
 * value as one u64 cell (src/datasource/table.rs:27-30); a narrow column's
 * cell value is its sign-extended (I32, I64) or zero-extended (U8) value,
 * which is exactly the cell the reference would hold for the same integer. */
typedef enum tgp_dtype {
    TGP_DT_U8 = 1,
    TGP_DT_I32 = 2,
    TGP_DT_I64 = 3,
    TGP_DT_U64 = 4,  /* a raw reference cell */
    TGP_DT_F64 = 5   /* f64 stored as its bits, as the reference does */
} tgp_dtype;

/* How a column's cells compare, mirroring `ColType` (src/engine/
 * query_interpreter/types.rs:79): Int compares as signed i64, Date as
 * unsigned u64 (expr.rs:1482-1506), Float as f64. */
typedef enum tgp_coltype {
    TGP_CT_INT = 0,
    TGP_CT_DATE = 1,
    TGP_CT_FLOAT = 2
} tgp_coltype;

typedef struct tgp_column_desc {
    uint32_t dtype;     /* tgp_dtype */
    uint32_t coltype;   /* tgp_coltype used by predicates on this column */
    const void* data;   /* `rows` elements, host or device memory */
} tgp_column_desc;

typedef uint64_t tgp_table_id;

/* Copies `ncols` host (or device) columns of `rows` rows into device memory
 * owned by the context, computes per-column min/max statistics, and returns a
 * table id. */
TGP_API int tgp_table_register(tgp_ctx* ctx, const tgp_column_desc* cols, uint32_t ncols,
                       uint64_t rows, tgp_table_id* out);

/* Registers device columns without copying (the caller keeps them alive until
 * tgp_table_drop). Device column pointers must be 16-byte aligned. */
TGP_API int tgp_table_register_device(tgp_ctx* ctx, const tgp_column_desc* cols, uint32_t ncols,
                              uint64_t rows, tgp_table_id* out);

/* One column in the reference's own table layout (src/datasource/table.rs:
 * 25-66): `cells` is Table::columns[i] (one u64 cell per value) and
 * `i32_sidecar` is Table::i32_columns[i] when its loader filled one (values
 * that fit i32, table.rs:52-61), else NULL. `coltype` is the column's ColType.
 * Host or device memory. */
typedef struct tgp_cell_column {
    const uint64_t* cells;
    const int32_t* i32_sidecar;
    uint32_t coltype;          /* tgp_coltype */
    uint32_t _pad;
} tgp_cell_column;

/* Registers a table given in the reference's layout and keeps each column at
 * the narrowest width that holds every cell exactly, so scans read 1-4 bytes
 * per value instead of 8:
 *  - an i32 sidecar, when present, is taken as the column (4 bytes per value
 *    cross the link; the cells are not read);
 *  - Float columns stay f64 bits (TGP_DT_F64);
 *  - otherwise the cells are copied, their min / max taken on the device, and
 *    an Int column whose values lie in 0..255 becomes TGP_DT_U8, one within
 *    the i32 range TGP_DT_I32, else TGP_DT_I64; a Date column (unsigned cells)
 *    becomes TGP_DT_U8 up to 255, TGP_DT_I32 up to 2^31-1, else TGP_DT_U64.
 * Every narrow value widens back to its original cell, so predicates and
 * aggregates give the results the cells would. */
TGP_API int tgp_table_register_cells(tgp_ctx* ctx, const tgp_cell_column* cols, uint32_t ncols,
                                     uint64_t rows, tgp_table_id* out);

/* The stored dtype (tgp_dtype) of column `col` of a registered table. */
TGP_API int tgp_table_column_dtype(tgp_ctx* ctx, tgp_table_id table, uint32_t col, uint32_t* dtype);

/* Replaces the contents of every column of a registered (copying) table from
 * new host buffers of the same row count, reusing its device memory. */
TGP_API int tgp_table_reload(tgp_ctx* ctx, tgp_table_id table, const tgp_column_desc* cols,
                     uint32_t ncols);

TGP_API int tgp_table_drop(tgp_ctx* ctx, tgp_table_id table);

/* Row count and the device pointer of column `col` (for callers that launch
 * their own work on resident data). */
TGP_API int tgp_table_info(tgp_ctx* ctx, tgp_table_id table, uint64_t* rows, uint32_t* ncols);
TGP_API int tgp_table_column_stats(tgp_ctx* ctx, tgp_table_id table, uint32_t col, int64_t* min_cell,
                           int64_t* max_cell);

/* ------------------------------------------------------------------------ */
/* Predicate programs (WHERE → selection bitmap)                             */
/* ------------------------------------------------------------------------ */

/* Comparison of one column against literal(s). Semantics per column coltype
 * follow apply_comparison (expr.rs:1468-1530) and BETWEEN (expr.rs:687-760):
 * BETWEEN = lit <= cell AND cell <= lit2; NOT_BETWEEN = cell < lit OR cell > lit2.
 * For FLOAT, EQ is the reference's epsilon equality (|x - v| <= 1e-6*max(|v|,1),
 * bitmap.rs:505-515) and NE is its negation (bitmap.rs:498-500). */
typedef enum tgp_cmp {
    TGP_CMP_EQ = 0,
    TGP_CMP_NE = 1,
    TGP_CMP_LT = 2,
    TGP_CMP_LE = 3,
    TGP_CMP_GT = 4,
    TGP_CMP_GE = 5,
    TGP_CMP_BETWEEN = 6,
    TGP_CMP_NOT_BETWEEN = 7
} tgp_cmp;

/* Node kinds of a postfix predicate program. AND/OR pop two masks and push
 * one; NOT pops one. The program must leave exactly one mask on the stack.
 * An empty program selects every row (Bitmap::all_ones, bitmap.rs:57). */
typedef enum tgp_pred_kind {
    TGP_PN_LEAF = 0,
    TGP_PN_AND = 1,
    TGP_PN_OR = 2,
    TGP_PN_NOT = 3
} tgp_pred_kind;

#define TGP_MAX_PRED_NODES 16

typedef struct tgp_pred_node {
    uint32_t kind;    /* tgp_pred_kind */
    uint32_t column;  /* LEAF: column index in the table */
    uint32_t cmp;     /* LEAF: tgp_cmp */
    uint32_t _pad;
    uint64_t lit;     /* LEAF: literal bits (i64 for INT, u64 for DATE, f64 bits for FLOAT) */
    uint64_t lit2;    /* LEAF: upper bound for BETWEEN / NOT_BETWEEN */
} tgp_pred_node;

/* Evaluates a predicate program over a resident table.
 *  bitmap_out: NULL or ((rows + 7) / 8) bytes, LSB-first (bitmap.rs:36-40);
 *              tail bits of the last byte are zero.
 *  rowids_out: NULL or `rowids_cap` u32 entries, receives the selected row
 *              indices in ascending order (Bitmap::iter_set_bits, bitmap.rs:224).
 *  count_out:  number of selected rows (always written on TGP_OK and
 *              TGP_CAPACITY). Output pointers may be host or device memory. */
TGP_API int tgp_filter(tgp_ctx* ctx, tgp_table_id table, const tgp_pred_node* pred, uint32_t npred,
               uint8_t* bitmap_out, uint32_t* rowids_out, uint64_t rowids_cap,
               uint64_t* count_out);

/* ------------------------------------------------------------------------ */
/* Aggregation queries (scalar, grouped, and join + grouped)                 */
/* ------------------------------------------------------------------------ */

typedef enum tgp_agg_func {
    TGP_AGG_COUNT_STAR = 0,    /* COUNT(*) */
    TGP_AGG_COUNT_NONZERO = 1, /* COUNT(col): the reference counts cells != 0
                                  (aggregate.rs:1364-1367, accum_grouped.rs:243-246) */
    TGP_AGG_SUM = 2,           /* exact int128 sum of the per-row i64 argument */
    TGP_AGG_AVG = 3,           /* f64(sum) / f64(count), aggregate.rs:1416-1424 */
    TGP_AGG_MIN = 4,           /* signed i64 min of the argument, aggregate.rs:1822-1836 */
    TGP_AGG_MAX = 5
} tgp_agg_func;

/* Which table a column reference reads in a join query. */
typedef enum tgp_side {
    TGP_SIDE_PROBE = 0,  /* the query's own table (the probe side of a join) */
    TGP_SIDE_BUILD = 1   /* the joined build table */
} tgp_side;

#define TGP_MAX_FACTORS 4
#define TGP_MAX_AGGS 8
#define TGP_MAX_GROUP_KEYS 4

/* One affine factor `mul * cell + add` (wrapping i64). column = -1 means the
 * constant `add`. The per-row argument of an aggregate is the wrapping i64
 * product of its factors, which is exactly the reference's per-row
 * Int x Int evaluation (expr.rs:2063-2076) of expressions such as
 * `price`, `price * disc`, `price * (100 - disc) * (100 + tax)`. */
typedef struct tgp_factor {
    int32_t column;
    uint32_t side;   /* tgp_side */
    int64_t mul;
    int64_t add;
} tgp_factor;

typedef struct tgp_agg {
    uint32_t func;      /* tgp_agg_func */
    uint32_t nfactors;  /* 0..=TGP_MAX_FACTORS (COUNT_STAR uses 0) */
    tgp_factor f[TGP_MAX_FACTORS];
} tgp_agg;

typedef struct tgp_group_key {
    uint32_t column;
    uint32_t side;   /* tgp_side */
} tgp_group_key;

typedef uint64_t tgp_join_id;

typedef struct tgp_query {
    tgp_table_id table;              /* table scanned (probe side when join != 0) */
    const tgp_pred_node* pred;       /* WHERE program on `table` (may be NULL) */
    uint32_t npred;
    uint32_t ngroup;                 /* 0 = scalar aggregate */
    const tgp_group_key* group;
    uint32_t nagg;
    uint32_t _pad;
    const tgp_agg* aggs;
    tgp_join_id join;                /* 0 = no join */
    uint32_t probe_key_column;       /* join key column of `table` */
    uint32_t flags;                  /* reserved, 0 */
} tgp_query;

/* Value of one aggregate of one group. (lo, hi) is a two's-complement int128:
 * COUNT* → count; SUM/AVG → exact sum; MIN/MAX → value. `as_f64` is the
 * reference's f64 view (AVG result; f64(sum) for SUM). */
typedef struct tgp_agg_value {
    uint64_t lo;
    int64_t hi;
    uint64_t count;   /* rows that reached this aggregate */
    double as_f64;
} tgp_agg_value;

typedef struct tgp_query_result {
    uint64_t rows_scanned;
    uint64_t rows_selected;    /* rows passing WHERE (join: probe rows passing WHERE) */
    uint64_t ngroups;          /* groups produced (1 for a scalar aggregate) */
    uint32_t flags;            /* TGP_RESULT_* bits */
    uint32_t _pad;
} tgp_query_result;

/* Set when some per-row argument wrapped in i64, as the reference's own
 * wrapping arithmetic would (expr.rs:2063-2076). */
#define TGP_RESULT_ROW_OVERFLOW 1u

/* Executes one aggregation query.
 *  keys_out:  group_cap * ngroup u64 cells (group key values), may be NULL for
 *             a scalar query;
 *  vals_out:  group_cap * nagg values;
 * Groups are returned sorted by key tuple (ascending signed cells), so results
 * compare as multisets independent of hash order. Returns TGP_CAPACITY (with
 * result->ngroups set) when group_cap is too small. */
TGP_API int tgp_execute(tgp_ctx* ctx, const tgp_query* q, uint64_t* keys_out, tgp_agg_value* vals_out,
                uint64_t group_cap, tgp_query_result* result);

/* Executes one aggregation query with ORDER BY aggregate `order_agg`
 * (ascending, or descending when `descending` != 0) LIMIT `limit`: the
 * grouped-result ordering of apply_order_by_grouped / topn_indices
 * (src/engine/query_interpreter/expr.rs:2378-2420, 56-110). keys_out and
 * vals_out hold `limit` groups; result->ngroups is the number returned,
 * min(limit, groups). Groups are ordered by the aggregate's exact value (AVG:
 * its f64), ties in ascending key order. The reference compares the result
 * cells as f64 bit patterns, which orders non-negative integers the same way
 * and negative integer results differently. Hash-grouped results are ordered
 * on the device, and only the returned groups are formatted and copied. */
TGP_API int tgp_execute_topn(tgp_ctx* ctx, const tgp_query* q, uint32_t order_agg, int descending, uint64_t limit,
                             uint64_t* keys_out, tgp_agg_value* vals_out, tgp_query_result* result);

/* Device memory one tgp_execute of `q` holds while it runs, as its plan sizes
 * it: the result block, the group hash table with the gather and sort
 * buffers of its result (hash grouping), and a join payload array still to
 * be built; the resident tables and the join table are not counted. This is
 * the estimate that a per-query memory budget is compared against — the
 * reference's `MEMORY BUDGET <bytes>` statement extension
 * (src/sql/extensions.rs:13,58,155) — and what the serving loop admits
 * requests by. Plans only: launches nothing, allocates nothing. */
TGP_API int tgp_query_footprint(tgp_ctx* ctx, const tgp_query* q, uint64_t* device_bytes);

/* COUNT(DISTINCT column) over the rows passing `pred` (all rows when npred =
 * 0), as the reference evaluates it (aggregate.rs:1301-1325,
 * src/exec/hll.rs): with fewer than 100,000 selected rows the exact number of
 * distinct cells (*method = 0); otherwise the HyperLogLog estimate with 2^14
 * registers over xxh3_64 of each selected row's u64 cell, including its
 * small-range linear counting (*method = 1, ~0.81 % standard error). The
 * registers are exact, so the estimate equals the reference's for the same
 * cells. `method` may be NULL. */
TGP_API int tgp_count_distinct(tgp_ctx* ctx, tgp_table_id table, uint32_t column, const tgp_pred_node* pred,
                               uint32_t npred, uint64_t* count, uint32_t* method);

/* The HyperLogLog estimate tgp_count_distinct makes from 2^14 registers (the
 * reference's HyperLogLog::estimate, src/exec/hll.rs:53-76), for callers that
 * merge register sets themselves (the registers of a union are the element-wise
 * max). Host-only: needs no context or device. */
TGP_API int tgp_hll_estimate(const uint32_t* regs, uint64_t* out);

/* ------------------------------------------------------------------------ */
/* Hash join (src/engine/query_interpreter/join.rs:544-939)                  */
/* ------------------------------------------------------------------------ */

/* Builds a device hash table over the rows of `build_table` that pass `pred`
 * (the single-table build filter of join.rs:79-100), keyed by `key_column`.
 * Duplicate keys are kept (join_hash_table.rs:27-30). */
TGP_API int tgp_join_build(tgp_ctx* ctx, tgp_table_id build_table, uint32_t key_column,
                   const tgp_pred_node* pred, uint32_t npred, tgp_join_id* out);
/* An inner equi-join of two registered tables, a.key_a = b.key_b, each side
 * with its own single-table filter: counts both filtered sides on the
 * device and builds the join table on the side with fewer rows — the left
 * (a) when it has strictly fewer, else the right (b) — as the reference's
 * hash_join_with_keys picks its build side for an inner join
 * (src/engine/query_interpreter/join.rs:557-575) after
 * join_tables_greedy_core / plan_join_dp ordered a two-table join
 * (join.rs:250-333, 336-503). *build_is_a says which side was built; the
 * other side is then the probe side of tgp_execute / tgp_join_probe_pairs
 * (its filter going into the query's WHERE). *rows_a / *rows_b are the
 * filtered counts. */
TGP_API int tgp_join_build_smaller(tgp_ctx* ctx, tgp_table_id table_a, uint32_t key_a, const tgp_pred_node* pred_a,
                                   uint32_t npred_a, tgp_table_id table_b, uint32_t key_b,
                                   const tgp_pred_node* pred_b, uint32_t npred_b, tgp_join_id* out,
                                   uint32_t* build_is_a, uint64_t* rows_a, uint64_t* rows_b);
TGP_API int tgp_join_drop(tgp_ctx* ctx, tgp_join_id join);

/* Inner equi-join probe that emits the (probe_row, build_row) pairs, as the
 * reference's probe loop does (join.rs:748-790). Pairs are returned sorted by
 * (probe_row, build_row). Returns TGP_CAPACITY with *npairs set when `cap` is
 * too small. */
TGP_API int tgp_join_probe_pairs(tgp_ctx* ctx, tgp_join_id join, tgp_table_id probe_table,
                         uint32_t probe_key_column, const tgp_pred_node* pred, uint32_t npred,
                         uint32_t* probe_rows, uint32_t* build_rows, uint64_t cap,
                         uint64_t* npairs);

/* ------------------------------------------------------------------------ */
/* Batches: many queries, one persistent launch                              */
/* ------------------------------------------------------------------------ */

/* One query of a batch and its outputs (the arguments of tgp_execute). The
 * caller keeps `query` (and what it points to) and the output buffers alive
 * until tgp_batch_poll reports the batch done; `result` and `status` are
 * written then. */
typedef struct tgp_batch_item {
    const tgp_query* query;
    uint64_t* keys_out;
    tgp_agg_value* vals_out;
    uint64_t group_cap;
    tgp_query_result result;
    int32_t status;            /* tgp_status of this query */
    uint32_t _pad;
} tgp_batch_item;

typedef uint64_t tgp_batch_id;

/* Plans every query and launches them without waiting: the direct-indexed and
 * scalar aggregates run in one persistent kernel per CTA shape whose blocks
 * take (query, tile range) morsels from a device work counter, with one
 * upload of all plans and one readback of all result blocks; other queries
 * (hash grouping, ...) run one by one inside this call. This is the batched
 * counterpart of issuing tgp_execute n times. Per-query planning errors land
 * in items[i].status; the call itself fails only when nothing can run. */
TGP_API int tgp_batch_submit(tgp_ctx* ctx, tgp_batch_item* items, uint32_t n, tgp_batch_id* out);

/* Completes a batch: with wait != 0 blocks until its GPU work is done;
 * otherwise returns TGP_PENDING if it is still running. On completion fills
 * every item's result and status, releases the batch and returns TGP_OK. */
TGP_API int tgp_batch_poll(tgp_ctx* ctx, tgp_batch_id batch, int wait);

/* ------------------------------------------------------------------------ */
/* Captured queries: one CUDA graph per query template                       */
/* ------------------------------------------------------------------------ */

/* The reference plans and interprets every statement again on each call
 * (route_and_execute, src/engine/mod.rs:527-533; execute_shape,
 * src/engine/dispatch.rs:364). A captured query is planned once: its result
 * clear, scan launch and result readback are recorded as one CUDA graph that
 * tgp_graph_launch replays with one launch and one synchronisation.
 *
 * Direct-indexed and scalar aggregates only (hash grouping sizes its result
 * from the data: TGP_UNSUPPORTED). The graph reads the table's and join's
 * device memory as they were at capture: launching after the table or join was
 * dropped returns TGP_NOT_FOUND (capture again); a join keeps one payload
 * array per build-side key layout until it is dropped, so queries of other
 * layouts leave the graph valid. Reloading a table in place
 * (tgp_table_reload) keeps the graph valid, and the graph sees the new rows,
 * as long as every column's min / max stays as it was (the plan's bounds are
 * proven from them); otherwise the launch returns TGP_NOT_FOUND as well. */
typedef uint64_t tgp_graph_id;

TGP_API int tgp_graph_capture(tgp_ctx* ctx, const tgp_query* q, tgp_graph_id* out);

/* Runs a captured query on the context's stream and waits for it; outputs as
 * tgp_execute. */
TGP_API int tgp_graph_launch(tgp_ctx* ctx, tgp_graph_id graph, uint64_t* keys_out, tgp_agg_value* vals_out,
                             uint64_t group_cap, tgp_query_result* result);

TGP_API int tgp_graph_drop(tgp_ctx* ctx, tgp_graph_id graph);

/* Failure-path test hook (no counterpart in the reference): the next scan
 * launch of this context does not issue the shared-memory copy of tile
 * `tile` (of the CTA that owns it), and its bounded device waits give up
 * after `wait_ns` (1 ms to 1 s) instead of 1 s. The consumers' wait for that
 * copy runs out, the kernel raises its timeout bit and returns, and the call
 * returns TGP_TIMEOUT; the context stays usable for the next query. One-shot:
 * later launches are not affected. A wait that gives up, not a fault. While
 * it is armed, the next aggregate runs on the scan pipeline even where a
 * streaming GROUP BY kernel (which has no stage copies and no waits) would
 * otherwise take it. */
TGP_API int tgp_debug_fail_next_scan(tgp_ctx* ctx, uint64_t tile, uint64_t wait_ns);

/* ------------------------------------------------------------------------ */
/* String columns and LIKE                                                   */
/* ------------------------------------------------------------------------ */

typedef uint64_t tgp_strings_id;

/* Copies a string column into HBM in the layout of the reference's
 * StringSearchColumn flat buffer (src/exec/fm_index.rs:273-277): all strings'
 * bytes back to back (`nbytes`) and n + 1 nondecreasing offsets, string i =
 * bytes[offsets[i], offsets[i + 1]), offsets[0] = 0, offsets[n] = nbytes.
 * Host memory. The offsets are checked (TGP_INVALID_ARG otherwise). */
TGP_API int tgp_strings_register(tgp_ctx* ctx, const uint8_t* bytes, uint64_t nbytes, const uint64_t* offsets,
                                 uint64_t n, tgp_strings_id* out);
TGP_API int tgp_strings_drop(tgp_ctx* ctx, tgp_strings_id strings);

/* `column [NOT] LIKE pattern` into a selection bitmap: the reference's LIKE
 * (the interpreter's like_mask / like, src/engine/query_interpreter/expr.rs:
 * 1159-1240, 2144-2171): byte-wise, '_' matches one byte, '%' any run of
 * bytes, a pattern byte equal to the string byte matches it (also '%' or '_'),
 * no escape character; NOT LIKE is the complement. The pattern is
 * `pattern_len` bytes (at most 256), not NUL-terminated. bitmap_out: NULL or
 * (n + 7) / 8 bytes, LSB-first (bitmap.rs:36-40), host or device memory;
 * *count_out = rows selected. AND it into a WHERE bitmap as the interpreter
 * does (mask.and_inplace, expr.rs:845-848). */
TGP_API int tgp_like(tgp_ctx* ctx, tgp_strings_id strings, const char* pattern, uint32_t pattern_len, int negated,
                     uint8_t* bitmap_out, uint64_t* count_out);

/* ------------------------------------------------------------------------ */
/* Scan variants and the autotuner                                           */
/* ------------------------------------------------------------------------ */

/* The knobs of a scan launch that the planner otherwise sets by rule. The
 * reference picks a CPU kernel per (operator, CPU target, memory tier) from
 * its kernel table (src/kernel/mod.rs:209-221) and sizes its morsels by a
 * fixed 65,536-row chunk (aggregate.rs:259); here one query class can run
 * several variants of the scan kernel, and tgp_autotune measures which is
 * fastest. */
typedef struct tgp_variant {
    uint32_t threads;      /* consumer threads per CTA: 0 = the planner's rule, 256 or 512
                              (8 or 4 rows per thread of a 2,048-row tile) */
    uint32_t max_stages;   /* cap on the shared-memory pipeline stages, 1..8 */
    uint32_t placement;    /* direct groups: 0 = rule, 1 = per-thread private accumulators,
                              2 = per-CTA shared (64-bit), 3 = global, 4 = per-warp shared tables of
                              32-bit limbs with native atomics */
    uint32_t presum;       /* 1 = shared pre-aggregation of repeated keys (hash / global grouping) allowed */
    uint32_t dense;        /* 1 = dense column programs (private placement) allowed */
    uint32_t shapes;       /* 1 = ahead-of-time fixed-shape kernels allowed */
    uint32_t payload;      /* 1 = unique-key join payload arrays allowed */
    uint32_t ctas_per_sm;  /* 1 or 2 */
    uint32_t l2_ahead;     /* tiles of L2 bulk prefetch ahead of the stage copies, 0 = off */
    uint32_t _pad;
} tgp_variant;

/* The variant used for every query whose class has no tuned entry (the
 * planner's rules: threads 0, max_stages 8, placement 0, presum / dense /
 * shapes / payload 1, ctas_per_sm 1, l2_ahead 0). */
TGP_API int tgp_set_default_variant(tgp_ctx* ctx, const tgp_variant* v);
TGP_API int tgp_get_default_variant(tgp_ctx* ctx, tgp_variant* v);

/* Batch shaping: morsel length in tiles (default 16), whether same-table
 * queries of a batch share scans (default 1), and the largest per-plan
 * accumulator region that joins a shared scan (default 32 KiB). */
TGP_API int tgp_batch_config(tgp_ctx* ctx, uint32_t morsel_tiles, int shared_scans, uint64_t share_extra_max);

/* A query's class: its shape (join, number of group keys, of values and of
 * predicate leaves, direct or hash grouping) and the binary orders of
 * magnitude of its row count and of its bound on distinct groups. Tuned
 * variants are kept per class. */
TGP_API int tgp_tune_class(tgp_ctx* ctx, const tgp_query* q, uint64_t* key);
TGP_API int tgp_tune_set(tgp_ctx* ctx, uint64_t key, const tgp_variant* v);
/* *found = 0 when the class has no tuned entry (v then holds the default). */
TGP_API int tgp_tune_get(tgp_ctx* ctx, uint64_t key, tgp_variant* v, int* found);
/* The tuned entries in ascending key order (for saving them). */
TGP_API int tgp_tune_count(tgp_ctx* ctx, uint32_t* n);
TGP_API int tgp_tune_at(tgp_ctx* ctx, uint32_t i, uint64_t* key, tgp_variant* v);
TGP_API int tgp_tune_clear(tgp_ctx* ctx);

/* One measured candidate of tgp_autotune. */
typedef struct tgp_tune_entry {
    tgp_variant variant;
    double ms;              /* median scan-kernel time over `reps` runs (CUDA events, each launch
                               queued behind a short device delay) */
    int32_t status;         /* TGP_OK, or why the candidate could not run */
    uint32_t same_result;   /* 1 = its result equals the planner's rule's, bit for bit */
    uint32_t threads_used;  /* what the plan launched with */
    uint32_t stages_used;
    uint32_t mode_used;     /* accumulator placement the plan chose: 2 private, 3 shared, 4 global, 5 hash,
                               8 per-warp 32-bit limb tables */
    uint32_t _pad;
} tgp_tune_entry;

/* Measures the variants of the query's scan (threads x stage cap x
 * accumulator placement / dense programs for direct groups, or x
 * pre-aggregation for hash grouping), each first checked to return the
 * result of the planner's rule bit for bit, then timed `reps` times; installs
 * the fastest correct one for the query's class and reports every candidate
 * (the rule's first) in `entries` (*n of them; only the first `cap` are
 * written) and the index of the fastest in *best. Launch profiling must be
 * off. */
TGP_API int tgp_autotune(tgp_ctx* ctx, const tgp_query* q, uint32_t reps, tgp_tune_entry* entries, uint32_t cap,
                         uint32_t* n, uint32_t* best, uint64_t* key);

/* ------------------------------------------------------------------------ */
/* Allocation-free aggregate                                                 */
/* ------------------------------------------------------------------------ */

/* Size of the library's fixed device scratch for tgp_aggregate_noalloc. */
#define TGP_NOALLOC_SCRATCH_BYTES (1024u * 1024u)

/* One GROUP BY column of tgp_aggregate_noalloc and the values it may hold:
 * every cell lies in [min, min + count). */
typedef struct tgp_key_domain {
    uint32_t column;
    uint32_t _pad;
    int64_t min;
    uint64_t count;
} tgp_key_domain;

/* Has no counterpart in the reference: an entry point for callers that cannot
 * allocate GPU memory — an embedding engine whose own allocator reserved the
 * whole device at start-up (a cudaMalloc here would fail, or take memory the
 * allocator has promised elsewhere), a latency-bound serving thread that may
 * not take the device-wide synchronisation a cudaMalloc / cudaFree can cause,
 * or a host bound by a no-allocation-after-start-up policy. It computes the
 * same scalar or grouped aggregate as tgp_execute over caller-owned,
 * 16-byte-aligned DEVICE columns on `device`, without a context and without
 * calling cudaMalloc, cudaFree or any allocating routine: its accumulators live
 * in a fixed TGP_NOALLOC_SCRATCH_BYTES (1 MiB) device array that every GPU
 * loading the library keeps until the process exits.
 *
 *  - Groups are dense: group g enumerates the key domains with the first key
 *    most significant; vals_out (HOST memory) receives ngroups * nagg values in
 *    that order (ngroups = product of the domain counts), with count = 0 for
 *    empty groups. A key cell outside its declared domain is rejected
 *    (TGP_INVALID_ARG) before any accumulation.
 *  - Queries whose scratch exceeds TGP_NOALLOC_SCRATCH_BYTES (many groups times
 *    many aggregates) are rejected with TGP_CAPACITY and a message.
 *  - Columns that live on another GPU are rejected (TGP_INVALID_ARG).
 *  - The first call on a device looks up the array's device address (once per
 *    device, with that device current); make it before any stream capture. The
 *    address is kept for the life of the process, so a cudaDeviceReset of that
 *    device, or a non-primary context made current on it, is not supported.
 *  - All calls share the array and it keeps the last call's contents; each call
 *    clears what it accumulates into. Calls that overlap on the GPU (two
 *    streams, or two host threads) race on it: the caller serialises them.
 *  - `stream` is a cudaStream_t (NULL = the default stream); the call returns
 *    after its work on that stream has finished, with the caller's current
 *    device unchanged. Failures carry a message in err_msg (may be NULL). */
TGP_API int tgp_aggregate_noalloc(int device, void* stream, const tgp_column_desc* cols, uint32_t ncols,
                                  uint64_t rows, const tgp_pred_node* pred, uint32_t npred,
                                  const tgp_key_domain* keys, uint32_t nkeys, const tgp_agg* aggs, uint32_t nagg,
                                  tgp_agg_value* vals_out, uint64_t vals_cap, tgp_query_result* result,
                                  char* err_msg, size_t err_cap);

#ifdef __cplusplus
}
#endif

#endif /* TURBOGP_GPU_H */
