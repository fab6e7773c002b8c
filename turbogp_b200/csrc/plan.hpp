// plan.hpp — the lowered form of one scan over one resident table, shared by
// the host planner (capi.cpp) and the device kernels (scan_engine.cu).
//
// A plan is a POD passed by value as a __grid_constant__ kernel parameter, so
// launching a query needs no descriptor copy. Host code lowers the C-ABI
// query (predicate program, aggregates, group keys, join) into it.
#pragma once

#include <cstdint>

namespace tgp {

// A tile is kTileRows consecutive rows; a CTA of NT threads (256 or 512, a
// template parameter of the scan kernel) gives each thread kTileRows / NT
// consecutive rows of it.
constexpr int kTileRows = 2048;
constexpr int kMaxSlots = 8;       // distinct columns staged per scan
constexpr int kMaxLeaves = 16;     // predicate leaves
constexpr int kMaxPredOps = 32;    // postfix program length
constexpr int kMaxVals = 8;        // value accumulators per group
constexpr int kMaxFactors = 4;
constexpr int kMaxGroupKeys = 4;
constexpr int kMaxStages = 8;
constexpr int kBarrierBytes = 128; // shared bytes for the stage mbarriers (full[8], empty[8])

// Error bits a kernel raises in its plan's error word (never __trap()).
enum : uint32_t {
    kErrWaitTimeout = 1u,   // an mbarrier wait gave up
    kErrHashFull = 2u,      // a hash table ran out of slots
    kErrOutputFull = 4u,    // an output buffer reservation ran past its capacity
    kErrRowOverflow = 8u    // a per-row i64 argument wrapped (informational)
};

// Physical column types (values match tgp_dtype).
enum : uint32_t { DT_U8 = 1, DT_I32 = 2, DT_I64 = 3, DT_U64 = 4, DT_F64 = 5 };

// Scan modes (one kernel instantiation each).
enum : uint32_t {
    MODE_FILTER = 0,         // count selected rows; write bitmap words; per-tile counts
    MODE_SCALAR = 1,         // scalar aggregate (host: MODE_GROUP_PRIVATE with one group)
    MODE_GROUP_PRIVATE = 2,  // direct-indexed groups, per-thread shared accumulators
    MODE_GROUP_SHARED = 3,   // direct-indexed groups, per-CTA shared table with atomics
    MODE_GROUP_GLOBAL = 4,   // direct-indexed groups, global int128 atomics
    MODE_GROUP_HASH = 5,     // open-addressing global hash table of groups
    MODE_JOIN_BUILD = 6,     // insert selected rows into a join hash table
    MODE_JOIN_PAIRS = 7,     // probe and emit (probe_row, build_row) pairs
    MODE_GROUP_SHARED32 = 8  // direct-indexed groups, per-warp shared tables of 32-bit limbs, native atomics
};

// A staged column.
struct SlotDesc {
    const uint8_t* ptr;   // device column base (16-byte aligned)
    uint32_t width;       // bytes per row: 1, 4 or 8
    uint32_t dtype;       // DT_*
    uint32_t smem_off;    // offset of this column's tile inside a stage
    uint32_t _pad;
};

// Leaf kinds after lowering. Integer leaves test (x - lo) <= span as unsigned
// integers on the raw stored word x (u8 zero-extended, i32 as u32, 64-bit as
// u64): lo is pre-biased so that this equals testing key - lo' with
// key = x ^ xor, which maps the column's comparison order onto unsigned
// order (xor with the sign bit = adding it). `negate` flips the result.
enum : uint8_t { LK_U8 = 0, LK_I32 = 1, LK_64 = 2, LK_F64 = 3, LK_CONST = 4 };
enum : uint8_t { FOP_EQ_EPS = 0, FOP_NE = 1, FOP_LT = 2, FOP_LE = 3, FOP_GT = 4, FOP_GE = 5,
                 FOP_BETWEEN = 6, FOP_NOT_BETWEEN = 7 };

struct Leaf {
    uint8_t slot;
    uint8_t kind;     // LK_*
    uint8_t negate;   // 0 or 1 (LK_CONST: the constant value)
    uint8_t fop;      // FOP_* for LK_F64
    uint32_t xor32;
    uint32_t lo32;
    uint32_t span32;
    uint64_t xor64;
    union {
        struct {
            uint64_t lo64;
            uint64_t span64;
        };
        struct {
            double f1;  // LK_F64 literal / lower bound / epsilon target
            double f2;  // LK_F64 upper bound or epsilon
        };
    };
};

// Plan::shape of scalar aggregates on the register fast path.
constexpr uint32_t kShapeScalar = 0xffffu;

// Postfix program opcodes: values < kMaxLeaves push leaf i.
enum : uint8_t { OP_AND = 0x80, OP_OR = 0x81, OP_NOT = 0x82 };

// Value accumulator kinds.
enum : uint8_t { VK_SUM = 0, VK_MIN = 1, VK_MAX = 2, VK_COUNT_NZ = 3 };

struct Factor {
    int8_t slot;          // staged column slot, or -1 for a constant
    uint8_t build_side;   // 1: gather from a build-side column at the matched build row
    uint8_t dtype;        // dtype of the staged or build-side column
    uint8_t _pad;
    uint32_t soff;        // staged: the slot's offset inside a stage
    const uint8_t* bptr;  // build-side column (device)
    int64_t mul;
    int64_t add;
};

struct ValDesc {
    uint8_t kind;   // VK_*
    uint8_t nf;     // number of factors
    uint8_t _pad[6];
    Factor f[kMaxFactors];
};

// One step of a dense value program (MODE_GROUP_PRIVATE, int64 partials).
// Values that extend the previous value's factor list share its running
// product: sum(p), sum(p * (100 - d)), sum(p * (100 - d) * (100 + t)) run as
// three steps, not six factor evaluations.
constexpr int kMaxSteps = 8;
enum : uint8_t {
    CS_COL = 1,     // factor reads a staged column (else the constant `add`)
    CS_CHAIN = 2,   // multiply into the running product (else start a new one)
    CS_NARROW = 4,  // mul * x + add fits int32 for every cell: 32-bit arithmetic
    CS_IDENT = 8,   // mul == 1 and add == 0: the factor is the cell itself
    CS_NONNEG = 16  // CS_NARROW and mul * x + add >= 0 for every cell
};
struct ChainStep {
    uint32_t soff;   // staged column offset inside a stage
    uint8_t dtype;   // staged column dtype
    uint8_t flags;   // CS_*
    uint8_t acc;     // value slot (1..nval) the running product goes to; 0 = none
    uint8_t kind;    // VK_* of that value
    int32_t mul32, add32;
    int64_t mul, add;
};
struct ChainProg {
    uint32_t nsteps;
    uint32_t _pad;
    ChainStep s[kMaxSteps];
};

struct GKey {
    int8_t slot;          // staged slot (probe/own side)
    uint8_t build_side;   // 1: key column lives on the build side
    uint8_t dtype;        // dtype of the staged or build-side column
    uint8_t shift;        // MODE_GROUP_HASH: bit position in the packed key
    uint32_t soff;        // staged: the slot's offset inside a stage
    const uint8_t* bptr;
    int64_t min;          // key cell minimum (from column statistics)
    uint64_t stride;      // direct modes: multiplier of (cell - min) in the group index
    const uint8_t* lut;   // bucket key: digit = lut[cell - min] (u8 per cell of [min, max]); null = cell - min
};

// Register images the scan kernel loads once per plan (host-computed, so a
// load is a few independent reads instead of dependent field walks): a
// conjunction of up to four int32 leaves, and the scalar fast path's values
// (one or two SUMs of one or two staged affine factors).
constexpr int kRegLeaves = 4;
struct alignas(16) RegBlock {
    uint32_t leaf_n;                // 0 = the register leaves do not apply
    uint32_t leaf_neg;              // bit i: leaf i negated
    uint32_t leaf_soff[kRegLeaves];
    uint32_t leaf_lo[kRegLeaves];
    uint32_t leaf_sp[kRegLeaves];
    uint32_t vals_on;               // scalar fast path applies (MODE_GROUP_PRIVATE, int64)
    uint32_t vals_nv;
    uint32_t vals_nf[2];
    uint32_t vals_soff[2][2];
    uint32_t vals_dt[2][2];
    uint32_t _pad[2];
    int64_t vals_mul[2][2];
    int64_t vals_add[2][2];
};

struct alignas(16) Plan {
    uint64_t nrows;
    uint32_t nslots;
    uint32_t stage_bytes;   // bytes of one stage (all slots of one tile)
    uint32_t nstages;
    uint32_t extra_off;     // shared offset of per-mode scratch (accumulators)
    uint32_t smem_bytes;    // total dynamic shared memory
    uint32_t bitmap_words;  // MODE_FILTER: bitmap words written (0 = none)
    uint32_t nthreads;      // CTA size the plan's shared memory was sized for (256 or 512)
    uint32_t l2_ahead;      // tiles a CTA prefetches into L2 ahead of its next stage copy (0 = none)
    SlotDesc slot[kMaxSlots];

    // WHERE program
    uint32_t nleaf;
    uint32_t nops;
    uint32_t all_and;       // program is a conjunction of all leaves
    // For conjunctions the host orders leaves by kind: [0, kend[0]) LK_I32,
    // [kend[0], kend[1]) LK_U8, [kend[1], kend[2]) LK_64, the rest any kind.
    uint8_t kend[4];
    Leaf leaf[kMaxLeaves];
    uint8_t ops[kMaxPredOps];

    // Values (per group: slot 0 = row count, slots 1..nval = values)
    uint32_t nval;
    uint32_t check_ovf;     // per-row overflow detection needed
    uint32_t count_by_tile; // MODE_GROUP_PRIVATE, one group, no join: row count = popcount per tile
    uint32_t dense_vec;     // MODE_GROUP_PRIVATE int64: `chain` holds the dense value program
    uint32_t shape;         // ahead-of-time kernel for `chain` (0 = interpreted; kShapeScalar: scalar fast path)
    uint32_t stage_off;     // batch launches: shared offset of the stage ring (plans precede it)
    uint64_t flush_limit;   // MODE_GROUP_PRIVATE int64: per-thread updates between flushes
    ValDesc val[kMaxVals];

    ChainProg chain;

    // Group keys
    uint32_t ngkey;
    uint32_t ngroups;       // direct modes: number of group indices
    GKey gkey[kMaxGroupKeys];

    // Group hash table (MODE_GROUP_HASH): slot = [key][count][v0 lo][v0 hi]...
    unsigned long long* htab;
    uint64_t hmask;
    uint32_t hlog2;
    uint32_t hstride;       // u64 words per slot
    uint32_t hsm_slots;     // per-CTA shared pre-aggregation slots (power of two; 0 = none):
                            // [keys][counts u32][value partials i32 x nval], SUM / COUNT_NZ only
    uint32_t hsm_log2;
    uint32_t hsm_key32;     // its keys are u32 (every key below 2^32 - 1), else u64

    // Join table (probe side: MODE_GROUP_* / MODE_SCALAR with join, MODE_JOIN_PAIRS;
    // build side: MODE_JOIN_BUILD). Packed slots: (key_rel << 32) | build_row.
    // Wide slots: [key_rel][build_row + 1].
    unsigned long long* jtab;
    uint64_t jmask;
    uint32_t jlog2;
    uint32_t jwide;
    int32_t jslot;          // staged slot of the join key (-1 = no join)
    uint32_t sum64;         // global / hash sums fit int64 (host-proven): plain atomic adds, lo limb only
    int64_t jkmin;
    uint64_t jkrange;       // kmax - kmin (unsigned)
    const uint32_t* jpay;   // unique build keys: per-key payload (build-side group index part), or null;
                            // entries of jpay_w bytes (1, 2 or 4), all ones = no match

    // Outputs
    unsigned long long* acc;        // direct/scalar accumulators [g][1 + nval][2]
    uint32_t* bitmap;               // MODE_FILTER bitmap words
    uint32_t* tile_counts;          // MODE_FILTER per-tile selected counts
    unsigned long long* counters;   // [0] selected rows [1] pairs reserved [2] matches
    uint32_t* err;                  // kErr* bits
    unsigned long long* out_pairs;  // MODE_JOIN_PAIRS: (probe_row << 32) | build_row
    uint64_t out_cap;
    uint32_t hash_fast;             // global / hash grouping by one staged key, values SUM / COUNT(col)
                                    // of one staged factor each (at most two): the column path
    uint32_t group_fast;            // batch launches: every plan of this plan's morsel group is a scalar
                                    // fast-path plan with the same register leaf columns and values
    // MODE_GROUP_SHARED32: tables of s32_words u32 words per group ([count]
    // [lo, hi] per value), one per s32_copies groups of warps (warp w uses
    // table w % s32_copies).
    uint32_t s32_copies;
    uint32_t s32_words;
    // Failure-path test hook (tgp_debug_fail_next_scan): tile + 1 whose stage
    // copy the producer skips (0 = none), and the bounded waits' limit in ns
    // (0 = kWaitLimitNs).
    uint64_t skip_tile1;
    uint64_t wait_ns;
    // MODE_GROUP_HASH, one key over a moderate range: the slot of a key is
    // the key itself (relative to its minimum; hmask = the last slot), so a
    // row's update needs no probe, no compare and no claim; a slot whose
    // count is not zero is occupied (its key word stays empty).
    uint32_t hdirect;
    // One-word direct slots (MODE_GROUP_HASH, hdirect, hstride = 1): a slot
    // holds (row count << hpack_shift) + the sum of (value - hpack_bias) over
    // its rows, both fields proven by the host never to carry into the other
    // (rows < 2^(64 - hpack_shift), rows x value range < 2^hpack_shift), so a
    // row is one non-returning 64-bit add and the table is a quarter of the
    // [key][count][lo][hi] layout's size. 0 = that layout.
    uint32_t hpack;
    uint32_t hpack_shift;
    int64_t hpack_bias;
    uint32_t jpay_w;
    uint32_t two_ctas;      // launch the register budget of two CTAs per SM (join-payload limb-table shapes)
    RegBlock rb;                    // filled by fill_reg_block before every launch
};

// Build-side group keys folded into a join payload array.
struct PayKeys {
    uint32_t n;
    uint32_t dtype[kMaxGroupKeys];
    const uint8_t* ptr[kMaxGroupKeys];
    int64_t min[kMaxGroupKeys];
    uint64_t stride[kMaxGroupKeys];
};

#if defined(__CUDACC__)
#define TGP_HD __host__ __device__
#else
#define TGP_HD
#endif

// The int128 (hi:lo two's complement) nearest to a double, round to nearest
// even: the same value on host and device.
TGP_HD inline double i128_to_f64_rn(uint64_t lo, int64_t hi) {
    const bool neg = hi < 0;
    unsigned __int128 m = (static_cast<unsigned __int128>(static_cast<uint64_t>(hi)) << 64) | lo;
    if (neg) m = ~m + 1;
    const uint64_t mhi = static_cast<uint64_t>(m >> 64), mlo = static_cast<uint64_t>(m);
    double d;
    if (mhi == 0 && (mlo >> 53) == 0) {
        d = static_cast<double>(mlo);  // exact
    } else {
#if defined(__CUDA_ARCH__)
        const int msb = mhi ? 127 - __clzll(static_cast<long long>(mhi)) : 63 - __clzll(static_cast<long long>(mlo));
#else
        const int msb = mhi ? 127 - __builtin_clzll(mhi) : 63 - __builtin_clzll(mlo);
#endif
        int shift = msb - 52;
        unsigned __int128 mant = m >> shift;
        const unsigned __int128 rem = m & ((static_cast<unsigned __int128>(1) << shift) - 1);
        const unsigned __int128 half = static_cast<unsigned __int128>(1) << (shift - 1);
        if (rem > half || (rem == half && (mant & 1))) {
            mant += 1;
            if (mant >> 53) {
                mant >>= 1;
                shift += 1;
            }
        }
        const uint64_t bits = (static_cast<uint64_t>(shift + 52 + 1023) << 52) |
                              (static_cast<uint64_t>(mant) & ((1ull << 52) - 1));
#if defined(__CUDA_ARCH__)
        d = __longlong_as_double(static_cast<long long>(bits));
#else
        __builtin_memcpy(&d, &bits, 8);
#endif
    }
    return neg ? -d : d;
}

// MODE_GROUP_PRIVATE with int64 partials keeps, per consumer thread, u32 row
// counts [group][thread] followed (16-byte aligned) by int64 values
// [group][value][thread]. Bytes of the count array:
TGP_HD inline uint32_t priv_count_bytes(uint32_t ngroups, uint32_t nt) {
    return (ngroups * nt * 4u + 15u) & ~15u;
}

// The initial contents of one group hash table slot (at most 2 + 2 * kMaxVals words).
struct SlotImage {
    uint32_t stride;
    uint32_t _pad;
    unsigned long long w[2 + 2 * kMaxVals];
};

// Output layout of hash-grouped results (tgp_execute with hash grouping).
constexpr int kMaxFormatAggs = 32;
struct HashFormat {
    uint32_t nkey, nagg, hstride, sum64;  // sum64: value limbs hold int64 sums (hi = sign of lo)
    uint32_t hpack, hpack_shift;          // one-word direct slots (Plan::hpack)
    int64_t hpack_bias;
    uint32_t key_shift[kMaxGroupKeys];
    uint64_t key_mask[kMaxGroupKeys];
    int64_t key_min[kMaxGroupKeys];
    uint8_t func[kMaxFormatAggs];   // tgp_agg_func
    int8_t val[kMaxFormatAggs];     // value index, -1 = COUNT(*)
    uint8_t kind[kMaxFormatAggs];   // VK_* of that value
};

// ORDER BY one aggregate of a hash-grouped result (top-N): which slot holds
// the ordering value and how it compares.
struct TopNSpec {
    int32_t val;      // value index, -1 = the row count (COUNT(*))
    uint8_t kind;     // VK_* of that value
    uint8_t func;     // tgp_agg_func of the ordering aggregate (AVG orders by its f64)
    uint8_t desc;     // 1 = descending
    uint8_t sum64;    // value limbs hold int64 sums (hi = sign of lo)
};

static_assert(sizeof(Plan) % 16 == 0, "plans are copied in 16-byte words");

// A range of tiles of one table, processed by one CTA of a batch launch for
// `count` consecutive plans starting at `first` (a shared scan when count > 1:
// the plans share one stage layout and have disjoint accumulator regions).
constexpr int kMaxShare = 16;
struct Morsel {
    uint32_t first;
    uint32_t count;
    uint64_t tile_begin;
    uint64_t tile_end;
};

// A persistent batch launch: the plans of its queries (each with its own
// result pointers), the morsels and the device work counter.
struct BatchDesc {
    const Plan* plans;
    const Morsel* morsels;
    uint32_t nmorsels;
    uint32_t _pad;
    unsigned int* next;
};

// Multiplicative hash of a relative key into a power-of-two table.
#if defined(__CUDACC__)
__host__ __device__
#endif
inline uint64_t hash_slot(uint64_t key_rel, uint32_t log2cap) {
    return (key_rel * 0x9E3779B97F4A7C15ull) >> (64u - log2cap);
}

// LIKE pattern bytes, passed by value to the LIKE kernel.
constexpr uint32_t kLikeMaxPattern = 256;
struct LikePattern {
    uint32_t len;
    uint8_t b[kLikeMaxPattern];
};

}  // namespace tgp
