// runtime.hpp — host-side state behind the C ABI: the context, the
// HBM-resident table registry (the device tier the reference's MemoryTier::Hbm
// names, src/memory/tier.rs:20), join tables, and the scratch arena.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <map>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "plan.hpp"
#include "turbogp_gpu.h"

struct tgp_ctx;

namespace tgp {

// Launchers implemented in the .cu files.
cudaError_t launch_scan(const Plan& P, uint32_t mode, bool acc128, int grid, cudaStream_t st);

// Unfiltered GROUP BY of one key into one-word direct slots
// (groupby_direct.cu): the slot of a row is (u32)key - (u32)kmin (< 2^27);
// it receives `one` + the row's value argument (one = (1 << shift) - bias),
// or, through the shared table of `hs` slots (0 = none), the per-slot
// count << shift plus the partial sum minus count * bias.
struct DirectGroupArgs {
    const uint8_t* key;
    const uint8_t* val;            // null: COUNT(*) only
    uint64_t nrows;
    int64_t kmin;
    int64_t mul, add;              // value argument = mul * cell + add
    uint32_t ident;                // mul == 1 && add == 0
    uint32_t nz;                   // COUNT(col): the argument is (value != 0)
    uint32_t hs, hs_shift;         // shared slots (power of two) and 32 - log2(hs)
    uint32_t last;                 // the last slot
    uint32_t shift;
    unsigned long long one;
    int64_t bias;
    unsigned long long* slots;
    uint32_t* err;
    unsigned long long* counters;  // [0] += nrows (every row is selected)
};
// The TPC-H Q1 shape (groupby_direct.cu): GROUP BY two u8 keys under at
// most four int32 predicate leaves (x - lo <= span, negated per bit of
// leaf_neg); COUNT(*) and sum(mul0 * c0 + add0), sum(c1), sum(c1 * (mul1 *
// c2 + add1)), sum(c1 * (mul1 * c2 + add1) * (mul2 * c3 + add2)) with c0, c2,
// c3 int32 (non-negative factors) and c1 int64; accumulators [g][5][2]
// receive int64 partials in their low limbs.
struct Q1Args {
    const uint8_t* leaf_col[4];
    uint32_t leaf_lo[4], leaf_sp[4];
    uint32_t leaf_neg, nleaf;
    const uint8_t* key0;
    const uint8_t* key1;
    uint32_t kmin0, kmin1, kstride0, kstride1;
    const uint8_t* col[4];
    uint32_t mul[3], add[3];
    uint32_t ngroups, _pad;
    uint64_t nrows;
    unsigned long long* acc;
    unsigned long long* counters;
};
size_t q1_group_smem(uint32_t ngroups);
int q1_group_ctas_per_sm(uint32_t ngroups);
cudaError_t launch_q1_group(const Q1Args& A, int grid, cudaStream_t st);
bool direct_group_supported(uint32_t kdt, uint32_t vdt);
int direct_group_ctas_per_sm(uint32_t hs, bool hasv);
cudaError_t launch_direct_group(const DirectGroupArgs& A, uint32_t kdt, uint32_t vdt, int grid, cudaStream_t st);
int scan_occupancy(uint32_t mode, bool acc128, int nt, size_t dyn_smem, uint32_t shape = 0, bool pair = false);
// Index (>= 1) of the ahead-of-time dense kernel matching the plan's key
// dtypes and value program, or 0 (the interpreted dense program runs).
uint32_t dense_shape_of(const Plan& P);
// The shape whose value program (steps only, keys aside) a plan's dense
// program matches, for the limb-table kernels; 0 = none.
uint32_t value_shape_of(const Plan& P);
// kShapeScalar when the plan is a scalar aggregate the register fast path
// takes (one or two SUMs of one or two staged factors, bounded), else 0.
uint32_t scalar_shape_of(const Plan& P);
// Fills P.rb (the register images the kernels load) from the rest of the plan;
// every launch path calls it once the plan is final.
void fill_reg_block(Plan& P);
size_t scan_kernel_static_smem();
size_t batch_kernel_static_smem();
int batch_occupancy(bool acc128, int nt, size_t dyn_smem);
cudaError_t launch_batch(const BatchDesc& B, bool acc128, int nt, int grid, size_t dyn_smem, cudaStream_t st);
cudaError_t launch_column_minmax(const uint8_t* col, uint32_t dtype, uint64_t n, long long* out,
                                 int sms, cudaStream_t st);
// dst[i] = src[i] narrowed to DT_U8 or DT_I32 (the caller proved every value fits).
// src 16-byte aligned; dst 16-byte aligned for DT_I32, 4-byte for DT_U8.
cudaError_t launch_narrow_cells(const long long* src, uint64_t n, uint8_t* dst, uint32_t dtype, int sms,
                                cudaStream_t st);
cudaError_t tile_prefix(const uint32_t* counts, unsigned long long* out, uint64_t n, void* tmp,
                        size_t* tmp_bytes, cudaStream_t st);
cudaError_t launch_compact(const uint32_t* bitmap, uint64_t nwords, uint64_t ntiles,
                           const unsigned long long* tile_base, uint32_t* rowids, uint64_t cap,
                           cudaStream_t st);
cudaError_t launch_sum_f64(const double* x, uint64_t n, double* out, int blocks, cudaStream_t st);
// Exact distinct count / HyperLogLog registers (2^14 u32, zeroed by the
// caller) of the cells of a resident column, rows filtered by an optional
// selection bitmap.
cudaError_t launch_distinct_cells(const uint8_t* col, uint32_t dtype, uint64_t n, const uint32_t* bitmap,
                                  unsigned long long* set, uint64_t mask, uint32_t log2cap,
                                  unsigned long long* counters, uint32_t* err, int sms, cudaStream_t st);
// HyperLogLog: `partial` holds hll_blocks(n, sms) rows of 2^14 bytes (one per
// CTA, 16-byte aligned); regs gets their max (every register written).
int hll_blocks(uint64_t n, int sms);
cudaError_t launch_hll(const uint8_t* col, uint32_t dtype, uint64_t n, const uint32_t* bitmap, uint8_t* partial,
                       uint32_t* regs, int sms, cudaStream_t st);
cudaError_t launch_count_distinct(const unsigned long long* x, uint64_t n, unsigned long long* set,
                                  uint64_t mask, uint32_t log2cap, unsigned long long* counters,
                                  uint32_t* err, int blocks, cudaStream_t st);
cudaError_t sort_pairs(const unsigned long long* in, unsigned long long* out, uint64_t n, void* tmp,
                       size_t* tmp_bytes, cudaStream_t st);
cudaError_t launch_split_pairs(const unsigned long long* pairs, uint64_t n, uint32_t* probe,
                               uint32_t* build, int sms, cudaStream_t st);
cudaError_t launch_fill_u64(unsigned long long* p, uint64_t n, unsigned long long v, int sms,
                            cudaStream_t st);
cudaError_t launch_join_pay(const unsigned long long* tab, uint64_t cap, const PayKeys& K, uint32_t* pay,
                            uint32_t width, uint64_t pay_entries, int sms, cudaStream_t st);
cudaError_t format_hash_groups(const unsigned long long* packed, uint64_t n, const HashFormat& F, uint32_t key_bits,
                               void* scratch, size_t scratch_bytes, uint64_t* keys_out, tgp_agg_value* vals_out,
                               int sms, cudaStream_t st);
size_t format_hash_groups_scratch(uint64_t n, uint32_t key_bits);
// Directly indexed group tables (Plan::hdirect): count_direct_groups writes
// the number of occupied slots to the device word `total` (scratch:
// direct_groups_scratch bytes, kept for format_direct_groups), then
// format_direct_groups writes the groups in slot (= key) order, at most cap.
size_t direct_groups_scratch(uint64_t nslots);
cudaError_t count_direct_groups(const unsigned long long* htab, uint64_t nslots, uint32_t stride, void* scratch,
                                size_t scratch_bytes, unsigned long long* total, cudaStream_t st);
cudaError_t format_direct_groups(const unsigned long long* htab, uint64_t nslots, const void* scratch, uint64_t cap,
                                 const HashFormat& F, uint64_t* keys_out, tgp_agg_value* vals_out, cudaStream_t st);
// The first min(limit, n) gathered groups in the order of one aggregate
// (ties in ascending key order), formatted like format_hash_groups.
// Scratch: format_hash_groups_scratch(n, 64) bytes.
cudaError_t topn_hash_groups(const unsigned long long* packed, uint64_t n, const HashFormat& F, uint32_t key_bits,
                             const TopNSpec& S, uint64_t limit, void* scratch, size_t scratch_bytes,
                             uint64_t* keys_out, tgp_agg_value* vals_out, int sms, cudaStream_t st);
// One thread that spins on %globaltimer for `ns` nanoseconds (at most 1 ms).
cudaError_t launch_delay(uint64_t ns, cudaStream_t st);
// Device-to-host copy by a kernel into page-locked (mapped) host memory; both
// addresses and the size 16-byte aligned.
cudaError_t launch_copy_to_host(void* host_dst, const void* dev_src, size_t bytes, cudaStream_t st);
cudaError_t launch_like(const uint8_t* bytes, const unsigned long long* offs, uint64_t n, const LikePattern& P,
                        bool negated, uint32_t* bitmap, unsigned long long* count, uint32_t* err, int sms,
                        cudaStream_t st);
cudaError_t launch_fill_slots(unsigned long long* p, uint64_t nslots, const SlotImage& img, int sms, cudaStream_t st);
cudaError_t launch_gather_groups(const unsigned long long* htab, uint64_t nslots, uint32_t stride,
                                 unsigned long long* out, uint64_t cap, unsigned long long* counter,
                                 int sms, cudaStream_t st, bool direct = false);

struct Column;
// Lowers one predicate leaf over column `c` staged in `slot` (capi.cu).
// `ctx` may be null (no error message is recorded then).
int lower_leaf(tgp_ctx* ctx, const Column& c, const tgp_pred_node& n, uint8_t slot, Leaf& lf);

struct Column {
    uint32_t dtype = 0;
    uint32_t coltype = 0;
    uint32_t width = 0;
    uint8_t* dptr = nullptr;
    bool owned = false;
    int64_t min = 0;
    int64_t max = 0;
};

struct Table {
    uint64_t rows = 0;
    std::vector<Column> cols;
};

// Device join hash table over the selected rows of a build table.
struct JoinTable {
    tgp_table_id build_table = 0;
    uint32_t key_col = 0;
    unsigned long long* tab = nullptr;  // packed u64 slots or wide [key_rel, row+1] pairs
    uint64_t cap = 0;                   // slots (power of two)
    uint32_t log2 = 0;
    bool wide = false;
    int64_t kmin = 0;
    uint64_t krange = 0;
    uint64_t entries = 0;               // build rows inserted
    bool empty_range = false;           // no build key statistics (empty build side)
    bool unique = false;                // no two build rows share a key (packed tables only)
    // Payload arrays, one per build-side group-key layout (see PayKeys;
    // keyed by (column, min, stride) per build-side key, then the entry
    // width), each kept until the join is dropped: a plan reads its layout's
    // array for as long as its launches run, so no array is rebuilt in place
    // under a plan of another layout.
    struct Payload {
        uint32_t* ptr = nullptr;
        uint32_t width = 4;
    };
    std::map<std::vector<uint64_t>, Payload> pays;
};

// Scan variant knobs. The planner's rules fill them by default; the
// autotuner (tgp_autotune) measures alternatives per query class and keeps
// the fastest (tgp_variant in the C ABI is their external form).
struct Knobs {
    int threads = 0;          // consumer threads per CTA: 0 = the planner's rule, else 256 or 512
    int max_stages = kMaxStages;
    int placement = 0;        // direct groups: 0 = rule, 1 = per-thread private, 2 = per-CTA shared, 3 = global,
                              // 4 = per-warp shared tables of 32-bit limbs (native atomics)
    bool presum = true;       // shared pre-aggregation for hash / global grouping (when provably exact)
    bool dense = true;        // dense column programs for private placement
    bool shapes = true;       // ahead-of-time fixed-shape kernels
    bool payload = true;      // unique-key join payload arrays
    int ctas_per_sm = 1;
    int l2_ahead = 0;         // L2 bulk prefetch distance in tiles (0 = off)
};

// A string column resident in HBM: all strings' bytes back to back and n + 1
// offsets (string i = bytes[offs[i], offs[i + 1])).
struct StringColumn {
    uint8_t* bytes = nullptr;
    unsigned long long* offs = nullptr;
    uint64_t n = 0;
    uint64_t nbytes = 0;
};

// Grow-only device scratch carved per call.
struct Arena {
    uint8_t* base = nullptr;
    size_t cap = 0;
    size_t used = 0;
};

}  // namespace tgp

struct tgp_ctx {
    int device = 0;
    int sms = 0;
    size_t max_dyn_smem = 0;
    cudaStream_t stream = nullptr;
    // This context's stream-ordered pool (its memory is never handed to another
    // context's stream, so no cross-stream reuse dependency can chain two
    // contexts' work); null: the device's default pool.
    cudaMemPool_t pool = nullptr;
    std::string err;
    std::unordered_map<uint64_t, tgp::Table> tables;
    std::unordered_map<uint64_t, tgp::JoinTable> joins;
    std::unordered_map<uint64_t, tgp::StringColumn> strings;
    uint64_t next_id = 1;
    tgp::Arena arena;
    // Pinned host staging for small readbacks.
    uint8_t* hpin = nullptr;
    size_t hpin_cap = 0;
    // Device staging of kernel-table inputs (kept apart from the arena so
    // scans that grow the arena never move a staged input).
    uint8_t* kin = nullptr;
    size_t kin_cap = 0;
    // Pinned host buffers kept for reuse (batch staging and readback).
    struct PinnedBuf {
        uint8_t* p;
        size_t cap;
        bool busy;
    };
    std::vector<PinnedBuf> pinned_pool;
    // Batches submitted and not yet polled (opaque records owned by capi.cu).
    std::unordered_map<uint64_t, void*> batches;
    // Captured queries (opaque records owned by capi.cu).
    std::unordered_map<uint64_t, void*> graphs;
    // Live HashBuild handles (opaque pointers handed to callers).
    std::unordered_set<void*> hash_handles;
    // Launch profiling: event pairs around scan-kernel launches.
    bool profile = false;
    bool profile_gate = false;  // queue a device delay before each timed launch
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
    size_t prof_used = 0;
    // The scan variant used when no tuned entry matches a query's class.
    tgp::Knobs knobs;
    // Tuned variants by query class (tgp_autotune / tgp_tune_set).
    std::unordered_map<uint64_t, tgp::Knobs> tuned;
    // Failure-path test hook (tgp_debug_fail_next_scan): armed for one launch.
    uint64_t dbg_skip_tile1 = 0;
    uint64_t dbg_wait_ns = 0;
    // While the autotuner measures a candidate: the knobs every plan takes.
    const tgp::Knobs* force_knobs = nullptr;
    // Batch shaping (tgp_batch_config).
    int morsel_tiles = 16;           // batch morsel length in tiles
    bool shared_scans = true;        // batches merge same-table queries into shared scans
    size_t share_extra_max = 32768;  // largest accumulator region of a plan that joins a shared scan
};
