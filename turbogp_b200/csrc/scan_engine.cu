// scan_engine.cu — the persistent, TMA-staged scan kernel behind every
// filter / aggregate / join entry point of the C ABI.
//
// One CTA per SM slot walks tiles of kTileRows rows (tile = blockIdx.x +
// k * gridDim.x). Thread 0 streams the referenced columns of upcoming tiles
// into a ring of shared-memory stages with 1-D bulk copies
// (cp.async.bulk ... mbarrier::complete_tx). Each of the NT threads owns
// R = kTileRows / NT consecutive rows of the current stage: it reads them with
// 128-bit shared loads (chunk order rotated per thread so a quarter-warp never
// hits the same banks twice), evaluates the lowered WHERE program into an
// R-bit mask with one subtract and one unsigned compare per row and leaf, and
// feeds the selected rows to the mode's sink (bitmap words, per-thread or
// per-CTA group accumulators, global group / join hash tables, join pairs).
// The final partial tile is read straight from global memory with bounds
// checks.
//
// Reference semantics each piece restates:
//   predicate leaves  — apply_comparison (src/engine/query_interpreter/expr.rs:1468-1530),
//                       BETWEEN (expr.rs:687-760), filter_* (src/exec/bitmap.rs:321-590)
//   AND / OR / NOT    — eval_bool_mask_vec (expr.rs:633-679), Bitmap::not (bitmap.rs:120)
//   bitmap layout     — Bitmap, LSB-first (bitmap.rs:36-40)
//   per-row argument  — binop Int x Int wrapping i64 (expr.rs:2063-2076)
//   group keys        — exact key tuples (the reference hashes them, aggregate.rs:603)
//   join              — hash_join_with_keys inner equi-join (join.rs:544-794)
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <type_traits>
#include <utility>

#include "device_common.cuh"
#include "plan.hpp"

namespace tgp {

constexpr unsigned kFull = 0xffffffffu;
constexpr unsigned long long kEmpty = ~0ull;

// ---------------------------------------------------------------------------
// Cell access. `base` points at row 0 of the tile (shared stage or global).
// ---------------------------------------------------------------------------
template <bool TAIL>
__device__ __forceinline__ const uint8_t* slot_base(const Plan& P, const uint8_t* stage, int s,
                                                    uint64_t r0) {
    if (TAIL) return P.slot[s].ptr + r0 * P.slot[s].width;
    return stage + P.slot[s].smem_off;
}

__device__ __forceinline__ int64_t load_cell(const uint8_t* base, uint32_t dtype, uint32_t row) {
    if (dtype == DT_U8) return static_cast<int64_t>(base[row]);
    if (dtype == DT_I32) return static_cast<int64_t>(reinterpret_cast<const int32_t*>(base)[row]);
    return reinterpret_cast<const int64_t*>(base)[row];
}

__device__ __forceinline__ int64_t load_cell_ro(const uint8_t* base, uint32_t dtype, uint64_t row) {
    if (dtype == DT_U8) return static_cast<int64_t>(__ldg(base + row));
    if (dtype == DT_I32) return static_cast<int64_t>(__ldg(reinterpret_cast<const int32_t*>(base) + row));
    return static_cast<int64_t>(__ldg(reinterpret_cast<const long long*>(base) + row));
}

// ---------------------------------------------------------------------------
// Predicate evaluation: thread t owns rows R*t .. R*t+R-1 of the tile; the
// result is an R-bit mask (bit j = row R*t + j).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool f64_leaf(uint8_t fop, double x, double a, double b) {
    switch (fop) {
        case FOP_EQ_EPS: return fabs(x - a) <= b;          // bitmap.rs:505-515
        case FOP_NE: return !(fabs(x - a) <= b);            // bitmap.rs:498-500
        case FOP_LT: return x < a;
        case FOP_LE: return x <= a;
        case FOP_GT: return x > a;
        case FOP_GE: return x >= a;
        case FOP_BETWEEN: return x >= a && x <= b;
        default: return x < a || x > b;                     // FOP_NOT_BETWEEN
    }
}

__device__ __forceinline__ uint32_t in32(uint32_t x, uint32_t lo, uint32_t sp) {
    return (x - lo) <= sp ? 1u : 0u;
}

__device__ __forceinline__ uint32_t in64(uint64_t x, uint64_t lo, uint64_t sp) {
    return (x - lo) <= sp ? 1u : 0u;
}

// Loads the C 16-byte chunks of thread t's span (C * 16 bytes at base + C*16*t)
// in rotated order and calls f(chunk_index, value). Rotating by t / (8 / C)
// makes the 8 threads of a shared-memory phase touch 8 different 16-byte bank
// groups, so every load is conflict-free.
template <int C, typename F>
__device__ __forceinline__ void for_chunks(const uint8_t* base, uint32_t t, F&& f) {
    const uint4* p = reinterpret_cast<const uint4*>(base) + static_cast<size_t>(C) * t;
    const uint32_t rot = (C == 1) ? 0u : (t / (8 / C)) & (C - 1);
#pragma unroll
    for (int k = 0; k < C; ++k) {
        const uint32_t q = (k + rot) & (C - 1);
        f(q, p[q]);
    }
}

template <int R>
__device__ __forceinline__ uint32_t leaf_smem(const Leaf& L, const uint8_t* base, uint32_t t) {
    uint32_t m = 0;
    switch (L.kind) {
        case LK_U8: {
            const uint32_t lo = L.lo32, sp = L.span32;
            if (R == 4) {
                const uint32_t w = reinterpret_cast<const uint32_t*>(base)[t];
#pragma unroll
                for (int e = 0; e < 4; ++e) m |= in32((w >> (8 * e)) & 0xffu, lo, sp) << e;
            } else {
                const uint2 w = reinterpret_cast<const uint2*>(base)[t];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    m |= in32((w.x >> (8 * e)) & 0xffu, lo, sp) << e;
                    m |= in32((w.y >> (8 * e)) & 0xffu, lo, sp) << (e + 4);
                }
            }
            break;
        }
        case LK_I32: {
            const uint32_t lo = L.lo32, sp = L.span32;
            for_chunks<R / 4>(base, t, [&](uint32_t q, const uint4& v) {
                const uint32_t b = in32(v.x, lo, sp) | (in32(v.y, lo, sp) << 1) | (in32(v.z, lo, sp) << 2) |
                                   (in32(v.w, lo, sp) << 3);
                m |= b << (4 * q);
            });
            break;
        }
        case LK_64: {
            const uint64_t lo = L.lo64, sp = L.span64;
            for_chunks<R / 2>(base, t, [&](uint32_t q, const uint4& v) {
                const uint64_t a = (static_cast<uint64_t>(v.y) << 32) | v.x;
                const uint64_t b = (static_cast<uint64_t>(v.w) << 32) | v.z;
                m |= (in64(a, lo, sp) | (in64(b, lo, sp) << 1)) << (2 * q);
            });
            break;
        }
        case LK_F64: {
            for_chunks<R / 2>(base, t, [&](uint32_t q, const uint4& v) {
                const double a = __longlong_as_double(static_cast<long long>((static_cast<uint64_t>(v.y) << 32) | v.x));
                const double b = __longlong_as_double(static_cast<long long>((static_cast<uint64_t>(v.w) << 32) | v.z));
                const uint32_t r = (f64_leaf(L.fop, a, L.f1, L.f2) ? 1u : 0u) |
                                   ((f64_leaf(L.fop, b, L.f1, L.f2) ? 1u : 0u) << 1);
                m |= r << (2 * q);
            });
            break;
        }
        default:
            return L.negate ? 0xffffffffu : 0u;  // LK_CONST
    }
    return L.negate ? ~m : m;
}

// Tail tile: global memory, rows past nrem are never read.
template <int R>
__device__ __forceinline__ uint32_t leaf_global(const Leaf& L, const uint8_t* base, uint32_t t,
                                                uint32_t nrem, uint32_t dtype) {
    if (L.kind == LK_CONST) return L.negate ? 0xffffffffu : 0u;
    uint32_t m = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
        const uint32_t r = R * t + j;
        if (r >= nrem) break;
        uint32_t c;
        if (L.kind == LK_F64) {
            c = f64_leaf(L.fop, reinterpret_cast<const double*>(base)[r], L.f1, L.f2) ? 1u : 0u;
        } else if (L.kind == LK_64) {
            c = in64(reinterpret_cast<const uint64_t*>(base)[r], L.lo64, L.span64);
        } else {
            const uint32_t x = dtype == DT_U8 ? static_cast<uint32_t>(base[r]) : reinterpret_cast<const uint32_t*>(base)[r];
            c = in32(x, L.lo32, L.span32);
        }
        m |= c << j;
    }
    return L.negate ? ~m : m;
}

template <int R, bool TAIL>
__device__ __forceinline__ uint32_t eval_leaf(const Plan& P, const Leaf& L, const uint8_t* stage, uint64_t r0,
                                              uint32_t t, uint32_t nrem) {
    const uint8_t* base = slot_base<TAIL>(P, stage, L.slot, r0);
    if (TAIL) return leaf_global<R>(L, base, t, nrem, P.slot[L.slot].dtype);
    return leaf_smem<R>(L, base, t);
}

template <int R>
__device__ __forceinline__ uint32_t leaf_i32(const Leaf& L, const uint8_t* stage, const Plan& P, uint32_t t) {
    const uint8_t* base = stage + P.slot[L.slot].smem_off;
    const uint32_t lo = L.lo32, sp = L.span32;
    uint32_t m = 0;
    for_chunks<R / 4>(base, t, [&](uint32_t q, const uint4& v) {
        const uint32_t b = in32(v.x, lo, sp) | (in32(v.y, lo, sp) << 1) | (in32(v.z, lo, sp) << 2) |
                           (in32(v.w, lo, sp) << 3);
        m |= b << (4 * q);
    });
    return L.negate ? ~m : m;
}

// A conjunction of at most kRegLeaves I32 leaves, kept in registers for the
// whole kernel (no constant-bank loads per tile).
struct RegLeaves {
    uint32_t n;       // 0 = not applicable
    uint32_t neg;     // bit i: leaf i negated
    uint32_t soff[kRegLeaves];
    uint32_t lo[kRegLeaves];
    uint32_t sp[kRegLeaves];
};

__device__ __forceinline__ void load_reg_leaves(const Plan& P, RegLeaves& L) {
    L.n = P.rb.leaf_n;
    L.neg = P.rb.leaf_neg;
#pragma unroll
    for (int i = 0; i < kRegLeaves; ++i) {
        L.soff[i] = P.rb.leaf_soff[i];
        L.lo[i] = P.rb.leaf_lo[i];
        L.sp[i] = P.rb.leaf_sp[i];
    }
}

template <int R, int N>
__device__ __forceinline__ uint32_t eval_reg_leaves_n(const RegLeaves& L, const uint8_t* stage, uint32_t t) {
    uint32_t m = 0xffffffffu;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const uint32_t lo = L.lo[i], sp = L.sp[i];
        uint32_t b = 0;
        for_chunks<R / 4>(stage + L.soff[i], t, [&](uint32_t q, const uint4& v) {
            const uint32_t c = in32(v.x, lo, sp) | (in32(v.y, lo, sp) << 1) | (in32(v.z, lo, sp) << 2) |
                               (in32(v.w, lo, sp) << 3);
            b |= c << (4 * q);
        });
        m &= ((L.neg >> i) & 1u) ? ~b : b;
    }
    return m & ((1u << R) - 1u);
}

// Straight-line code per leaf count, so loads of all leaves can be in flight
// together.
template <int R>
__device__ __forceinline__ uint32_t eval_reg_leaves(const RegLeaves& L, const uint8_t* stage, uint32_t t) {
    switch (L.n) {
        case 1: return eval_reg_leaves_n<R, 1>(L, stage, t);
        case 2: return eval_reg_leaves_n<R, 2>(L, stage, t);
        case 3: return eval_reg_leaves_n<R, 3>(L, stage, t);
        default: return eval_reg_leaves_n<R, 4>(L, stage, t);
    }
}

template <int R, bool TAIL>
__device__ __forceinline__ uint32_t eval_pred(const Plan& P, const uint8_t* stage, uint64_t r0, uint32_t t,
                                              uint32_t nrem) {
    constexpr uint32_t kAll = (R == 32) ? 0xffffffffu : ((1u << R) - 1u);
    uint32_t valid = kAll;
    if (TAIL) {
        const uint32_t first = R * t;
        valid = first >= nrem ? 0u : (nrem - first >= static_cast<uint32_t>(R) ? kAll : ((1u << (nrem - first)) - 1u));
    }
    if (P.nleaf == 0) return valid;
    if (P.all_and) {
        uint32_t m = valid;
        uint32_t i = 0;
        if (!TAIL) {
            // Leaves grouped by kind: branch-free loop bodies for the common kinds.
            for (; i < P.kend[0]; ++i) m &= leaf_i32<R>(P.leaf[i], stage, P, t);
            for (; i < P.kend[2]; ++i) m &= leaf_smem<R>(P.leaf[i], stage + P.slot[P.leaf[i].slot].smem_off, t);
        }
        for (; i < P.nleaf; ++i) m &= eval_leaf<R, TAIL>(P, P.leaf[i], stage, r0, t, nrem);
        return m;
    }
    // General postfix program on an 8-deep register stack (depth checked on host).
    uint32_t s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0, s6 = 0, s7 = 0;
    for (uint32_t i = 0; i < P.nops; ++i) {
        const uint8_t op = P.ops[i];
        if (op < kMaxLeaves) {
            const uint32_t v = eval_leaf<R, TAIL>(P, P.leaf[op], stage, r0, t, nrem);
            s7 = s6; s6 = s5; s5 = s4; s4 = s3; s3 = s2; s2 = s1; s1 = s0; s0 = v;
        } else if (op == OP_NOT) {
            s0 = ~s0;
        } else {
            s0 = (op == OP_AND) ? (s0 & s1) : (s0 | s1);
            s1 = s2; s2 = s3; s3 = s4; s4 = s5; s5 = s6; s6 = s7; s7 = 0;
        }
    }
    return s0 & valid;
}

// ---------------------------------------------------------------------------
// Per-row argument of a value accumulator: wrapping i64 product of affine
// factors (mul * cell + add). `brow` is the matched build row for factors that
// read the build side of a join. Loops stay rolled: the code runs only for
// selected rows, and a small body keeps the hot loop in the instruction cache.
// ---------------------------------------------------------------------------
template <bool TAIL>
__device__ __forceinline__ int64_t eval_val(const Plan& P, const ValDesc& V, const uint8_t* stage, uint64_t r0,
                                            uint32_t rl, uint32_t brow, uint32_t& ovf) {
    int64_t acc = 1;
#pragma unroll 1
    for (int f = 0; f < V.nf; ++f) {
        const Factor& F = V.f[f];
        int64_t x = 0;
        if (F.slot >= 0) {
            x = load_cell(TAIL ? slot_base<true>(P, stage, F.slot, r0) : stage + F.soff, F.dtype, rl);
        } else if (F.build_side) {
            x = load_cell_ro(F.bptr, F.dtype, brow);
        }
        int64_t t;
        if (P.check_ovf) {
            t = add_wrap_checked(mul_wrap_checked(F.mul, x, ovf), F.add, ovf);
            acc = (f == 0) ? t : mul_wrap_checked(acc, t, ovf);
        } else {
            t = static_cast<int64_t>(static_cast<uint64_t>(F.mul) * static_cast<uint64_t>(x) +
                                     static_cast<uint64_t>(F.add));
            acc = (f == 0) ? t : static_cast<int64_t>(static_cast<uint64_t>(acc) * static_cast<uint64_t>(t));
        }
    }
    return acc;
}

template <bool TAIL>
__device__ __forceinline__ int64_t key_cell(const Plan& P, const GKey& K, const uint8_t* stage, uint64_t r0,
                                            uint32_t rl, uint32_t brow) {
    if (K.build_side) return load_cell_ro(K.bptr, K.dtype, brow);
    return load_cell(TAIL ? slot_base<true>(P, stage, K.slot, r0) : stage + K.soff, K.dtype, rl);
}

// Direct group index: sum over keys of (cell - min) * stride.
// With a join payload (gpay != kNoPay), the build-side keys' part of the
// index is gpay and only probe-side keys are read.
constexpr uint32_t kNoPay = 0xffffffffu;
template <bool TAIL>
__device__ __forceinline__ uint32_t group_index(const Plan& P, const uint8_t* stage, uint64_t r0, uint32_t rl,
                                                uint32_t brow, uint32_t gpay = kNoPay) {
    uint64_t g = gpay != kNoPay ? gpay : 0u;
#pragma unroll 1
    for (uint32_t k = 0; k < P.ngkey; ++k) {
        const GKey& K = P.gkey[k];
        if (gpay != kNoPay && K.build_side) continue;
        const int64_t c = key_cell<TAIL>(P, K, stage, r0, rl, brow);
        const uint64_t rel = static_cast<uint64_t>(c) - static_cast<uint64_t>(K.min);
        // A bucket key maps the cell to its bucket through a per-cell table.
        g += (K.lut ? static_cast<uint64_t>(__ldg(K.lut + rel)) : rel) * K.stride;
    }
    return static_cast<uint32_t>(g);
}

// Packed exact key for MODE_GROUP_HASH.
template <bool TAIL>
__device__ __forceinline__ uint64_t group_hash_key(const Plan& P, const uint8_t* stage, uint64_t r0, uint32_t rl,
                                                   uint32_t brow) {
    uint64_t key = 0;
#pragma unroll 1
    for (uint32_t k = 0; k < P.ngkey; ++k) {
        const GKey& K = P.gkey[k];
        const int64_t c = key_cell<TAIL>(P, K, stage, r0, rl, brow);
        key |= (static_cast<uint64_t>(c) - static_cast<uint64_t>(K.min)) << K.shift;
    }
    return key;
}

// ---------------------------------------------------------------------------
// Join table probing (read-only during the probe kernel).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool join_rel(const Plan& P, int64_t cell, uint64_t& rel) {
    rel = static_cast<uint64_t>(cell) - static_cast<uint64_t>(P.jkmin);
    return rel <= P.jkrange;
}

template <typename F>
__device__ __forceinline__ void join_foreach(const Plan& P, uint64_t rel, F&& f) {
    uint64_t h = hash_slot(rel, P.jlog2);
    const unsigned long long* t = P.jtab;
    for (uint64_t n = 0; n <= P.jmask; ++n) {
        if (!P.jwide) {
            const unsigned long long e = __ldg(t + h);
            if (e == kEmpty) break;
            if ((e >> 32) == rel) f(static_cast<uint32_t>(e & 0xffffffffull));
        } else {
            const unsigned long long br = __ldg(t + 2 * h + 1);
            if (br == 0) break;
            if (__ldg(t + 2 * h) == rel) f(static_cast<uint32_t>(br - 1));
        }
        h = (h + 1) & P.jmask;
    }
}

// ---------------------------------------------------------------------------
// Accumulator helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint8_t slot_kind(const Plan& P, uint32_t v) {
    return v == 0 ? VK_SUM : P.val[v - 1].kind;  // value slot 0 is the row count
}

__device__ __forceinline__ long long kind_identity(uint8_t kind) {
    return kind == VK_MIN ? 0x7fffffffffffffffll
                          : kind == VK_MAX ? static_cast<long long>(0x8000000000000000ull) : 0ll;
}

__device__ __forceinline__ void acc_init(I128& a, uint8_t kind) {
    a.lo = static_cast<uint64_t>(kind_identity(kind));
    a.hi = 0;
}

__device__ __forceinline__ void acc_update(I128& a, uint8_t kind, int64_t v) {
    if (kind == VK_SUM) {
        i128_add_i64(a, v);
    } else if (kind == VK_COUNT_NZ) {
        i128_add_i64(a, v != 0 ? 1 : 0);
    } else if (kind == VK_MIN) {
        a.lo = static_cast<uint64_t>(min(static_cast<long long>(a.lo), static_cast<long long>(v)));
    } else {
        a.lo = static_cast<uint64_t>(max(static_cast<long long>(a.lo), static_cast<long long>(v)));
    }
}

__device__ __forceinline__ void acc_combine(I128& a, uint8_t kind, const I128& b) {
    if (kind == VK_MIN) {
        a.lo = static_cast<uint64_t>(min(static_cast<long long>(a.lo), static_cast<long long>(b.lo)));
    } else if (kind == VK_MAX) {
        a.lo = static_cast<uint64_t>(max(static_cast<long long>(a.lo), static_cast<long long>(b.lo)));
    } else {
        i128_add(a, b);
    }
}

__device__ __forceinline__ bool acc_untouched(const I128& a, uint8_t kind) {
    return a.lo == static_cast<uint64_t>(kind_identity(kind)) && a.hi == 0;
}

// Global accumulator pair (lo at slot[0], hi at slot[1]).
__device__ __forceinline__ void acc_global(unsigned long long* slot, uint8_t kind, const I128& v) {
    if (kind == VK_MIN) {
        atomicMin(reinterpret_cast<long long*>(slot), static_cast<long long>(v.lo));
    } else if (kind == VK_MAX) {
        atomicMax(reinterpret_cast<long long*>(slot), static_cast<long long>(v.lo));
    } else {
        atomic_add_i128(slot, v);
    }
}

__device__ __forceinline__ void acc_global_i64(unsigned long long* slot, uint8_t kind, int64_t v) {
    I128 x;
    if (kind == VK_COUNT_NZ) {
        x.lo = v != 0 ? 1 : 0;
        x.hi = 0;
    } else {
        x.lo = static_cast<uint64_t>(v);
        x.hi = v >> 63;
    }
    acc_global(slot, kind, x);
}

// With sum64 (every group's sum provably fits int64) SUM / COUNT(col) add
// to the low limb with a non-returning atomic; the high limb stays 0 and the
// host sign-extends the low one.
__device__ __forceinline__ void acc_global_i64(unsigned long long* slot, uint8_t kind, int64_t v, bool sum64) {
    if (sum64 && (kind == VK_SUM || kind == VK_COUNT_NZ)) {
        const unsigned long long add = kind == VK_SUM ? static_cast<unsigned long long>(v) : (v != 0 ? 1ull : 0ull);
        if (add) atomicAdd(slot, add);
        return;
    }
    acc_global_i64(slot, kind, v);
}

// acc_global with the sum64 form: SUM / COUNT partials add to the low limb
// without waiting for the old value.
__device__ __forceinline__ void acc_global_s(unsigned long long* slot, uint8_t kind, const I128& v, bool sum64) {
    if (sum64 && kind != VK_MIN && kind != VK_MAX) {
        if (v.lo) atomicAdd(slot, static_cast<unsigned long long>(v.lo));
        return;
    }
    acc_global(slot, kind, v);
}

// ---------------------------------------------------------------------------
// Sinks. Shared-memory scratch layouts (nv1 = 1 + nval; value slot 0 is the
// group's row count):
//   MODE_GROUP_PRIVATE, int64 partials:  u32 counts [g * NT + t], then (at
//                                        priv_count_bytes) int64 values
//                                        [(g * nval + v - 1) * NT + t]
//   MODE_GROUP_PRIVATE, int128 partials: words ((g * nv1 + v) * 2 + limb) * NT + t
//   MODE_GROUP_SHARED:                   words (g * nv1 + v) * 2 + limb (carry atomics)
// MODE_SCALAR runs as MODE_GROUP_PRIVATE with a single group.
// ---------------------------------------------------------------------------
// Barrier 1 over the NT consumer threads only (the producer warp never joins).
template <int NT>
__device__ __forceinline__ void consumer_sync() {
    asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
}

__device__ __forceinline__ uint32_t* priv_counts(uint8_t* extra) { return reinterpret_cast<uint32_t*>(extra); }
template <int NT>
__device__ __forceinline__ long long* priv_values(const Plan& P, uint8_t* extra) {
    return reinterpret_cast<long long*>(extra + priv_count_bytes(P.ngroups, NT));
}

// Slot of `key` in the global group hash table (inserted if absent), or null
// with kErrHashFull raised.
constexpr uint32_t kSmemProbes = 2;
__device__ __forceinline__ unsigned long long* hash_group_slot(const Plan& P, uint64_t key) {
    if (P.hdirect) {
        // The slot is the key; its count marks it occupied (the key word is
        // not written).
        if (key > P.hmask) {
            atomicOr(P.err, kErrHashFull);
            return nullptr;
        }
        return P.htab + key * P.hstride;
    }
    uint64_t h = hash_slot(key, P.hlog2);
    for (uint64_t n = 0; n <= P.hmask; ++n) {
        unsigned long long* s = P.htab + h * P.hstride;
        unsigned long long k = *reinterpret_cast<volatile unsigned long long*>(s);
        if (k == kEmpty) k = atomicCAS(s, kEmpty, key);
        if (k == kEmpty || k == key) return s;
        h = (h + 1) & P.hmask;
    }
    atomicOr(P.err, kErrHashFull);
    return nullptr;
}

// Adds `cnt` rows whose value arguments sum to `xsum` to the one-word direct
// slot of `key` (P.hpack): one non-returning 64-bit add of
// (cnt << shift) + (xsum - cnt * bias).
__device__ __forceinline__ void hpack_add(const Plan& P, uint64_t key, uint64_t cnt, int64_t xsum) {
    if (key > P.hmask) {
        atomicOr(P.err, kErrHashFull);
        return;
    }
    atomicAdd(P.htab + key, (cnt << P.hpack_shift) +
                                (static_cast<unsigned long long>(xsum) - cnt * static_cast<uint64_t>(P.hpack_bias)));
}

// This CTA's shared pre-aggregation table (P.hsm_slots slots: keys, u32
// counts, i32 partials per value) absorbs repeated (hot) keys with native
// 32-bit shared atomics. Keys are u32 when every key is below 2^32 - 1
// (P.hsm_key32: 32-bit hash, compares and claims, and less shared memory),
// else u64; the empty key is all ones.
template <typename KT>
struct PresumTab {
    KT* keys;
    uint32_t* cnt;
    int32_t* sums;
    __device__ __forceinline__ PresumTab(uint8_t* extra, uint32_t HS)
        : keys(reinterpret_cast<KT*>(extra)),
          cnt(reinterpret_cast<uint32_t*>(reinterpret_cast<KT*>(extra) + HS)),
          sums(reinterpret_cast<int32_t*>(reinterpret_cast<uint32_t*>(reinterpret_cast<KT*>(extra) + HS) + HS)) {}
    static constexpr KT kEmptyKey = static_cast<KT>(~0ull);
    __device__ __forceinline__ static uint32_t slot(KT key, uint32_t log2) {
        if constexpr (sizeof(KT) == 4) return (static_cast<uint32_t>(key) * 0x9E3779B1u) >> (32u - log2);
        else return static_cast<uint32_t>(hash_slot(key, log2));
    }
};

// Runs f(PresumTab<KT>) with the plan's key width.
template <typename F>
__device__ __forceinline__ void with_presum(const Plan& P, uint8_t* extra, F&& f) {
    if (P.hsm_key32) f(PresumTab<uint32_t>(extra, P.hsm_slots));
    else f(PresumTab<unsigned long long>(extra, P.hsm_slots));
}

// Adds a row to its key's slot; false when the key found no slot within
// kSmemProbes probes (the caller updates the global table instead). The host
// proves that no partial can pass 2^31 in magnitude.
template <bool TAIL>
__device__ __forceinline__ bool presum_add(const Plan& P, uint8_t* extra, uint64_t key, const uint8_t* stage,
                                           uint64_t r0, uint32_t rl, uint32_t brow, uint32_t& ovf) {
    const uint32_t HS = P.hsm_slots;
    bool done = false;
    with_presum(P, extra, [&](auto T) {
        using KT = std::remove_pointer_t<decltype(T.keys)>;
        const KT k0 = static_cast<KT>(key);
        uint32_t h = T.slot(k0, P.hsm_log2);
#pragma unroll 1
        for (uint32_t n = 0; n < kSmemProbes; ++n) {
            KT k = *reinterpret_cast<volatile KT*>(&T.keys[h]);
            if (k == T.kEmptyKey) k = atomicCAS(&T.keys[h], T.kEmptyKey, k0);
            if (k == T.kEmptyKey || k == k0) {
                atomicAdd(&T.cnt[h], 1u);
#pragma unroll 1
                for (uint32_t v = 0; v < P.nval; ++v) {
                    const ValDesc& V = P.val[v];
                    const int64_t x = eval_val<TAIL>(P, V, stage, r0, rl, brow, ovf);
                    atomicAdd(&T.sums[v * HS + h], static_cast<int32_t>(V.kind == VK_COUNT_NZ ? (x != 0) : x));
                }
                done = true;
                return;
            }
            h = (h + 1) & (HS - 1);
        }
    });
    return done;
}

template <uint32_t MODE, bool ACC128, int NT>
struct Sink {
    uint32_t ovf;
    uint64_t upd;  // MODE_GROUP_PRIVATE int64: updates since the last flush

    __device__ __forceinline__ void init(const Plan& P, uint8_t* extra, uint32_t t) {
        ovf = 0;
        upd = 0;
        const uint32_t nv1 = P.nval + 1;
        long long* w = reinterpret_cast<long long*>(extra);
        if (MODE == MODE_GROUP_PRIVATE && ACC128) {
            for (uint32_t i = 0; i < P.ngroups * nv1; ++i) {
                w[(i * 2 + 0) * NT + t] = kind_identity(slot_kind(P, i % nv1));
                w[(i * 2 + 1) * NT + t] = 0;
            }
        } else if (MODE == MODE_GROUP_PRIVATE) {
            uint32_t* cnt = priv_counts(extra);
            long long* val = priv_values<NT>(P, extra);
            for (uint32_t g = 0; g < P.ngroups; ++g) cnt[g * NT + t] = 0;
            for (uint32_t i = 0; i < P.ngroups * P.nval; ++i) val[i * NT + t] = kind_identity(P.val[i % P.nval].kind);
        } else if (MODE == MODE_GROUP_SHARED) {
            for (uint32_t i = t; i < P.ngroups * nv1; i += NT) {
                w[2 * i] = kind_identity(slot_kind(P, i % nv1));
                w[2 * i + 1] = 0;
            }
        } else if (MODE == MODE_GROUP_SHARED32) {
            uint32_t* tab = reinterpret_cast<uint32_t*>(extra);
            for (uint32_t i = t; i < P.s32_copies * P.ngroups * P.s32_words; i += NT) tab[i] = 0;
        } else if ((MODE == MODE_GROUP_HASH || MODE == MODE_GROUP_GLOBAL) && P.hsm_slots) {
            const uint32_t HS = P.hsm_slots;
            with_presum(P, extra, [&](auto T) {
                for (uint32_t i = t; i < HS; i += NT) {
                    T.keys[i] = T.kEmptyKey;
                    T.cnt[i] = 0;
                    for (uint32_t v = 0; v < P.nval; ++v) T.sums[v * HS + i] = 0;
                }
            });
        }
    }

    // Moves this thread's int64 private partials into the global int128
    // accumulators and resets them.
    __device__ __noinline__ void flush_private_thread(const Plan& P, uint8_t* extra, uint32_t t) {
        const uint32_t nv1 = P.nval + 1;
        uint32_t* cnt = priv_counts(extra);
        long long* val = priv_values<NT>(P, extra);
        for (uint32_t g = 0; g < P.ngroups; ++g) {
            uint32_t& c = cnt[g * NT + t];
            if (c != 0) {
                acc_global_s(P.acc + 2ull * g * nv1, VK_SUM, I128{c, 0}, P.sum64 != 0);
                c = 0;
            }
        }
        for (uint32_t i = 0; i < P.ngroups * P.nval; ++i) {
            const uint32_t g = i / P.nval, v = i % P.nval;
            const uint8_t kind = P.val[v].kind;
            if (kind == VK_MIN || kind == VK_MAX) continue;
            long long& a = val[i * NT + t];
            if (a != 0) {
                I128 x;
                x.lo = static_cast<uint64_t>(a);
                x.hi = a >> 63;
                acc_global_s(P.acc + 2ull * (g * nv1 + 1 + v), VK_SUM, x, P.sum64 != 0);
                a = 0;
            }
        }
    }

    // One selected (row[, build row]) pair.
    template <bool TAIL>
    __device__ __forceinline__ void row(const Plan& P, uint8_t* extra, const uint8_t* stage, uint64_t r0,
                                        uint32_t rl, uint32_t brow, uint32_t t, uint32_t gpay = kNoPay) {
        const uint32_t nv1 = P.nval + 1;
        if (MODE == MODE_GROUP_PRIVATE) {
            const uint32_t g = group_index<TAIL>(P, stage, r0, rl, brow, gpay);
            long long* w = reinterpret_cast<long long*>(extra);
            if (ACC128) {
                if (!P.count_by_tile) {
                    uint64_t* lo = reinterpret_cast<uint64_t*>(&w[((g * nv1) * 2 + 0) * NT + t]);
                    long long* hi = &w[((g * nv1) * 2 + 1) * NT + t];
                    const uint64_t nl = *lo + 1;
                    *hi += (nl == 0) ? 1 : 0;
                    *lo = nl;
                }
#pragma unroll 1
                for (uint32_t v = 1; v < nv1; ++v) {
                    const ValDesc& V = P.val[v - 1];
                    const int64_t x = eval_val<TAIL>(P, V, stage, r0, rl, brow, ovf);
                    uint64_t* plo = reinterpret_cast<uint64_t*>(&w[((g * nv1 + v) * 2 + 0) * NT + t]);
                    long long* phi = &w[((g * nv1 + v) * 2 + 1) * NT + t];
                    I128 a{*plo, *phi};
                    acc_update(a, V.kind, x);
                    *plo = a.lo;
                    *phi = a.hi;
                }
            } else {
                if (!P.count_by_tile) priv_counts(extra)[g * NT + t] += 1;
                long long* val = priv_values<NT>(P, extra);
#pragma unroll 1
                for (uint32_t v = 1; v < nv1; ++v) {
                    const ValDesc& V = P.val[v - 1];
                    const int64_t x = eval_val<TAIL>(P, V, stage, r0, rl, brow, ovf);
                    long long& a = val[(g * P.nval + v - 1) * NT + t];
                    if (V.kind == VK_SUM) a = static_cast<long long>(static_cast<uint64_t>(a) + static_cast<uint64_t>(x));
                    else if (V.kind == VK_COUNT_NZ) a += (x != 0);
                    else if (V.kind == VK_MIN) a = min(a, static_cast<long long>(x));
                    else a = max(a, static_cast<long long>(x));
                }
                // |x| <= bound for every value, so after flush_limit updates an
                // int64 partial could be one update away from wrapping: move
                // this thread's partials into the global int128 accumulators.
                if (++upd >= P.flush_limit) {
                    flush_private_thread(P, extra, t);
                    upd = 0;
                }
            }
        } else if (MODE == MODE_GROUP_SHARED) {
            const uint32_t g = group_index<TAIL>(P, stage, r0, rl, brow, gpay);
            unsigned long long* w = reinterpret_cast<unsigned long long*>(extra);
            atomicAdd(&w[(g * nv1) * 2], 1ull);
#pragma unroll 1
            for (uint32_t v = 1; v < nv1; ++v) {
                const ValDesc& V = P.val[v - 1];
                const int64_t x = eval_val<TAIL>(P, V, stage, r0, rl, brow, ovf);
                unsigned long long* s = &w[(g * nv1 + v) * 2];
                if (V.kind == VK_SUM || V.kind == VK_COUNT_NZ) {
                    const unsigned long long add =
                        V.kind == VK_SUM ? static_cast<unsigned long long>(x) : (x != 0 ? 1ull : 0ull);
                    if (add) {
                        const unsigned long long old = atomicAdd(s, add);
                        const unsigned long long hadd =
                            (V.kind == VK_SUM ? static_cast<unsigned long long>(x >> 63) : 0ull) +
                            ((old + add < old) ? 1ull : 0ull);
                        if (hadd) atomicAdd(s + 1, hadd);
                    }
                } else if (V.kind == VK_MIN) {
                    atomicMin(reinterpret_cast<long long*>(s), static_cast<long long>(x));
                } else {
                    atomicMax(reinterpret_cast<long long*>(s), static_cast<long long>(x));
                }
            }
        } else if (MODE == MODE_GROUP_SHARED32) {
            // Native 32-bit shared atomics on this warp group's table: the row
            // count, and per value the low 32 bits (the returned old value
            // gives the carry) and the signed high 32 bits. The host proved
            // every table's sums stay below 2^63 in magnitude, so the limbs
            // recombine exactly.
            const uint32_t g = group_index<TAIL>(P, stage, r0, rl, brow, gpay);
            uint32_t* tab = reinterpret_cast<uint32_t*>(extra) +
                            (static_cast<size_t>((t >> 5) & (P.s32_copies - 1u)) * P.ngroups + g) * P.s32_words;
            atomicAdd(&tab[0], 1u);
#pragma unroll 1
            for (uint32_t v = 0; v < P.nval; ++v) {
                const ValDesc& V = P.val[v];
                int64_t x = eval_val<TAIL>(P, V, stage, r0, rl, brow, ovf);
                if (V.kind == VK_COUNT_NZ) x = x != 0 ? 1 : 0;
                const uint32_t xl = static_cast<uint32_t>(x);
                const uint32_t old = atomicAdd(&tab[1 + 2 * v], xl);
                const int32_t add = static_cast<int32_t>(x >> 32) + ((old + xl < old) ? 1 : 0);
                if (add) atomicAdd(reinterpret_cast<int*>(&tab[2 + 2 * v]), add);
            }
        } else if (MODE == MODE_GROUP_GLOBAL) {
            const uint32_t g = group_index<TAIL>(P, stage, r0, rl, brow, gpay);
            if (P.hsm_slots && presum_add<TAIL>(P, extra, g, stage, r0, rl, brow, ovf)) return;
            unsigned long long* a = P.acc + static_cast<uint64_t>(g) * nv1 * 2;
            atomicAdd(a, 1ull);
#pragma unroll 1
            for (uint32_t v = 1; v < nv1; ++v) {
                const ValDesc& V = P.val[v - 1];
                acc_global_i64(a + 2 * v, V.kind, eval_val<TAIL>(P, V, stage, r0, rl, brow, ovf), P.sum64 != 0);
            }
        } else if (MODE == MODE_GROUP_HASH) {
            const uint64_t key = group_hash_key<TAIL>(P, stage, r0, rl, brow);
            if (P.hsm_slots && presum_add<TAIL>(P, extra, key, stage, r0, rl, brow, ovf)) return;
            if (P.hpack) {
                int64_t x = P.nval ? eval_val<TAIL>(P, P.val[0], stage, r0, rl, brow, ovf) : 0;
                if (P.nval && P.val[0].kind == VK_COUNT_NZ) x = x != 0 ? 1 : 0;
                hpack_add(P, key, 1, x);
                return;
            }
            unsigned long long* slot = hash_group_slot(P, key);
            if (slot == nullptr) return;
            atomicAdd(slot + 1, 1ull);
#pragma unroll 1
            for (uint32_t v = 0; v < P.nval; ++v) {
                const ValDesc& V = P.val[v];
                acc_global_i64(slot + 2 + 2 * v, V.kind, eval_val<TAIL>(P, V, stage, r0, rl, brow, ovf), P.sum64 != 0);
            }
        } else if (MODE == MODE_JOIN_BUILD) {
            // Scanned table is the build side; P.jslot is its key column.
            const int64_t c = load_cell(slot_base<TAIL>(P, stage, P.jslot, r0), P.slot[P.jslot].dtype, rl);
            const uint64_t rel = static_cast<uint64_t>(c) - static_cast<uint64_t>(P.jkmin);
            const uint32_t row = static_cast<uint32_t>(r0 + rl);
            uint64_t h = hash_slot(rel, P.jlog2);
            bool done = false;
            for (uint64_t n = 0; n <= P.jmask && !done; ++n) {
                if (!P.jwide) {
                    // A failed CAS returns the slot's entry: an equal key there
                    // means the build side has duplicate keys (counter word 3).
                    const unsigned long long old = atomicCAS(P.jtab + h, kEmpty, (rel << 32) | row);
                    done = old == kEmpty;
                    if (!done && (old >> 32) == rel) atomicAdd(P.counters + 3, 1ull);
                } else if (atomicCAS(P.jtab + 2 * h + 1, 0ull, static_cast<unsigned long long>(row) + 1) == 0ull) {
                    P.jtab[2 * h] = rel;
                    done = true;
                }
                h = (h + 1) & P.jmask;
            }
            if (!done) atomicOr(P.err, kErrHashFull);
        }
    }

    // End of kernel: merge partials into global results.
    __device__ __forceinline__ void flush(const Plan& P, uint8_t* extra, uint32_t t) {
        const uint32_t lane = t & 31u, warp = t >> 5;
        const uint32_t nv1 = P.nval + 1;
        if (MODE == MODE_GROUP_PRIVATE) {
            consumer_sync<NT>();
            const long long* w = reinterpret_cast<const long long*>(extra);
            for (uint32_t idx = warp; idx < P.ngroups * nv1; idx += NT / 32) {
                const uint8_t kind = slot_kind(P, idx % nv1);
                I128 a;
                acc_init(a, kind);
                for (uint32_t u = lane; u < static_cast<uint32_t>(NT); u += 32) {
                    I128 b;
                    if (ACC128) {
                        b.lo = static_cast<uint64_t>(w[(idx * 2 + 0) * NT + u]);
                        b.hi = w[(idx * 2 + 1) * NT + u];
                    } else if (idx % nv1 == 0) {
                        b.lo = priv_counts(extra)[(idx / nv1) * NT + u];
                        b.hi = 0;
                    } else {
                        const long long x =
                            priv_values<NT>(P, extra)[((idx / nv1) * P.nval + idx % nv1 - 1) * NT + u];
                        b.lo = static_cast<uint64_t>(x);
                        b.hi = (kind == VK_MIN || kind == VK_MAX) ? 0 : (x >> 63);
                    }
                    acc_combine(a, kind, b);
                }
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) acc_combine(a, kind, shfl_down_i128(a, d));
                if (lane == 0 && !acc_untouched(a, kind)) acc_global_s(P.acc + 2ull * idx, kind, a, P.sum64 != 0);
            }
        } else if (MODE == MODE_GROUP_SHARED) {
            consumer_sync<NT>();
            const long long* w = reinterpret_cast<const long long*>(extra);
            for (uint32_t idx = t; idx < P.ngroups * nv1; idx += NT) {
                const uint8_t kind = slot_kind(P, idx % nv1);
                I128 a;
                a.lo = static_cast<uint64_t>(w[2 * idx]);
                a.hi = w[2 * idx + 1];
                if (!acc_untouched(a, kind)) acc_global_s(P.acc + 2ull * idx, kind, a, P.sum64 != 0);
            }
        } else if (MODE == MODE_GROUP_SHARED32) {
            consumer_sync<NT>();
            const uint32_t* tab = reinterpret_cast<const uint32_t*>(extra);
            const uint32_t W = P.s32_words, G = P.ngroups;
            for (uint32_t idx = t; idx < G * nv1; idx += NT) {
                const uint32_t g = idx / nv1, v = idx % nv1;
                // Sum the copies' limbs: counts as u64; a value as the exact
                // int64 (hi << 32) + lo of each copy.
                int64_t sum = 0;
                for (uint32_t c = 0; c < P.s32_copies; ++c) {
                    const uint32_t* e = tab + (static_cast<size_t>(c) * G + g) * W;
                    if (v == 0) {
                        sum += static_cast<int64_t>(e[0]);
                    } else {
                        const uint64_t hi = static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(e[2 * v])));
                        sum = static_cast<int64_t>(static_cast<uint64_t>(sum) + ((hi << 32) | e[2 * v - 1]));
                    }
                }
                if (sum == 0) continue;
                I128 a;
                a.lo = static_cast<uint64_t>(sum);
                a.hi = sum >> 63;
                acc_global_s(P.acc + 2ull * idx, VK_SUM, a, P.sum64 != 0);
            }
        } else if ((MODE == MODE_GROUP_HASH || MODE == MODE_GROUP_GLOBAL) && P.hsm_slots) {
            consumer_sync<NT>();
            const uint32_t HS = P.hsm_slots;
            with_presum(P, extra, [&](auto T) {
            const uint32_t* cnt = T.cnt;
            const int32_t* sums = T.sums;
            for (uint32_t i = t; i < HS; i += NT) {
                if (T.keys[i] == T.kEmptyKey) continue;
                const unsigned long long key = static_cast<unsigned long long>(T.keys[i]);
                // Hash slots are [key][count][v0 lo][v0 hi]...; direct
                // accumulators are [count lo][count hi][v0 lo][v0 hi]...
                if (MODE == MODE_GROUP_HASH && P.hpack) {
                    hpack_add(P, key, cnt[i], P.nval ? static_cast<int64_t>(sums[i]) : 0);
                    continue;
                }
                unsigned long long* base;
                uint32_t vofs;
                if (MODE == MODE_GROUP_HASH) {
                    unsigned long long* slot = hash_group_slot(P, key);
                    if (slot == nullptr) continue;
                    base = slot + 1;
                    vofs = 1;
                } else {
                    base = P.acc + key * (P.nval + 1) * 2;
                    vofs = 2;
                }
                atomicAdd(base, static_cast<unsigned long long>(cnt[i]));
                for (uint32_t v = 0; v < P.nval; ++v) {
                    const int64_t x = sums[v * HS + i];
                    if (P.sum64) {
                        if (x) atomicAdd(base + vofs + 2 * v, static_cast<unsigned long long>(x));
                        continue;
                    }
                    I128 a;
                    a.lo = static_cast<uint64_t>(x);
                    a.hi = x >> 63;
                    atomic_add_i128(base + vofs + 2 * v, a);
                }
            }
            });
        }
        if (ovf) atomicOr(P.err, kErrRowOverflow);
    }
};

// ---------------------------------------------------------------------------
// Register-resident value descriptors for the scalar fast path: up to two
// SUM values, each a product of up to two staged affine factors, int64
// private partials, no per-row overflow checks (the host proved the bound).
// ---------------------------------------------------------------------------
struct RegVals {
    uint32_t on;        // fast path applies
    uint32_t nv;        // 1 or 2
    uint32_t nf[2];     // 1 or 2
    uint32_t soff[2][2];
    uint32_t dt[2][2];
    int64_t mul[2][2];
    int64_t add[2][2];
};

template <uint32_t MODE, bool ACC128>
__device__ __forceinline__ void load_reg_vals(const Plan& P, RegVals& V) {
    const RegBlock& B = P.rb;
    V.on = (MODE == MODE_GROUP_PRIVATE && !ACC128) ? B.vals_on : 0u;
    V.nv = B.vals_nv;
#pragma unroll
    for (int v = 0; v < 2; ++v) {
        V.nf[v] = B.vals_nf[v];
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            V.soff[v][f] = B.vals_soff[v][f];
            V.dt[v][f] = B.vals_dt[v][f];
            V.mul[v][f] = B.vals_mul[v][f];
            V.add[v][f] = B.vals_add[v][f];
        }
    }
}

__device__ __forceinline__ int64_t fast_factor(const uint8_t* stage, uint32_t soff, uint32_t dt, int64_t mul,
                                               int64_t add, uint32_t rl) {
    const int64_t x = load_cell(stage + soff, dt, rl);
    return static_cast<int64_t>(static_cast<uint64_t>(mul) * static_cast<uint64_t>(x) + static_cast<uint64_t>(add));
}

template <int NT>
__device__ __forceinline__ void fast_row(const Plan& P, const RegVals& V, uint8_t* extra, const uint8_t* stage,
                                         uint32_t rl, uint32_t t, uint64_t& upd, Sink<MODE_GROUP_PRIVATE, false, NT>& sink) {
    long long* w = priv_values<NT>(P, extra);
#pragma unroll
    for (int v = 0; v < 2; ++v) {
        if (static_cast<uint32_t>(v) < V.nv) {
            const int64_t a = fast_factor(stage, V.soff[v][0], V.dt[v][0], V.mul[v][0], V.add[v][0], rl);
            const int64_t b = V.nf[v] > 1 ? fast_factor(stage, V.soff[v][1], V.dt[v][1], V.mul[v][1], V.add[v][1], rl)
                                          : int64_t{1};
            const uint64_t x = static_cast<uint64_t>(a) * static_cast<uint64_t>(b);
            long long& s = w[v * NT + t];  // group 0, value v
            s = static_cast<long long>(static_cast<uint64_t>(s) + x);
        }
    }
    if (++upd >= P.flush_limit) {
        sink.flush_private_thread(P, extra, t);
        upd = 0;
    }
}

// ---------------------------------------------------------------------------
// Dense tiles of MODE_GROUP_PRIVATE with int64 partials (no join, staged keys
// and factors): the thread's R rows are processed column by column in
// straight-line code. Unselected rows add 0 (MIN / MAX skip them), so the
// per-row loop has no data-dependent branch; every step of the host's value
// program (ChainProg) is uniform across the CTA.
// ---------------------------------------------------------------------------
// The R cells of thread t (rows R*t .. R*t+R-1) as 64-bit integers.
template <int R>
__device__ __forceinline__ void load_cells64(const uint8_t* base, uint32_t dtype, uint32_t t, int64_t (&x)[R]) {
    if (dtype == DT_U8) {
        if constexpr (R == 4) {
            const uint32_t w = reinterpret_cast<const uint32_t*>(base)[t];
#pragma unroll
            for (int e = 0; e < 4; ++e) x[e] = (w >> (8 * e)) & 0xffu;
        } else {
            const uint2 w = reinterpret_cast<const uint2*>(base)[t];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                x[e] = (w.x >> (8 * e)) & 0xffu;
                x[e + 4] = (w.y >> (8 * e)) & 0xffu;
            }
        }
    } else if (dtype == DT_I32) {
        const uint4* p = reinterpret_cast<const uint4*>(base) + (R / 4) * t;
#pragma unroll
        for (int c = 0; c < R / 4; ++c) {
            const uint4 v = p[c];
            x[4 * c + 0] = static_cast<int32_t>(v.x);
            x[4 * c + 1] = static_cast<int32_t>(v.y);
            x[4 * c + 2] = static_cast<int32_t>(v.z);
            x[4 * c + 3] = static_cast<int32_t>(v.w);
        }
    } else {
        const uint4* p = reinterpret_cast<const uint4*>(base) + (R / 2) * t;
#pragma unroll
        for (int c = 0; c < R / 2; ++c) {
            const uint4 v = p[c];
            x[2 * c + 0] = static_cast<int64_t>((static_cast<uint64_t>(v.y) << 32) | v.x);
            x[2 * c + 1] = static_cast<int64_t>((static_cast<uint64_t>(v.w) << 32) | v.z);
        }
    }
}

// The low 32 bits of the same cells (u8 zero-extended, i32 as stored).
template <int R>
__device__ __forceinline__ void load_cells32(const uint8_t* base, uint32_t dtype, uint32_t t, uint32_t (&x)[R]) {
    if (dtype == DT_U8) {
        if constexpr (R == 4) {
            const uint32_t w = reinterpret_cast<const uint32_t*>(base)[t];
#pragma unroll
            for (int e = 0; e < 4; ++e) x[e] = (w >> (8 * e)) & 0xffu;
        } else {
            const uint2 w = reinterpret_cast<const uint2*>(base)[t];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                x[e] = (w.x >> (8 * e)) & 0xffu;
                x[e + 4] = (w.y >> (8 * e)) & 0xffu;
            }
        }
    } else if (dtype == DT_I32) {
        const uint4* p = reinterpret_cast<const uint4*>(base) + (R / 4) * t;
#pragma unroll
        for (int c = 0; c < R / 4; ++c) {
            const uint4 v = p[c];
            x[4 * c + 0] = v.x;
            x[4 * c + 1] = v.y;
            x[4 * c + 2] = v.z;
            x[4 * c + 3] = v.w;
        }
    } else {
        const uint4* p = reinterpret_cast<const uint4*>(base) + (R / 2) * t;
#pragma unroll
        for (int c = 0; c < R / 2; ++c) {
            const uint4 v = p[c];
            x[2 * c + 0] = v.x;
            x[2 * c + 1] = v.z;
        }
    }
}

template <int NT>
__device__ __forceinline__ void chain_private_tile(const Plan& P, uint8_t* extra, const uint8_t* stage, uint32_t t,
                                                   uint32_t m, Sink<MODE_GROUP_PRIVATE, false, NT>& sink,
                                                   const uint32_t* gin = nullptr) {
    constexpr int R = kTileRows / NT;
    unsigned long long* w = reinterpret_cast<unsigned long long*>(extra);
    // The int64 partials stay below 2^63 in magnitude: flush before this
    // tile's updates could pass the host's bound.
    const uint32_t nsel = __popc(m);
    if (sink.upd + nsel > P.flush_limit) {
        sink.flush_private_thread(P, extra, t);
        sink.upd = 0;
    }
    sink.upd += nsel;

    // Direct group index of each row: sum over keys of (cell - min) * stride,
    // exact in 32 bits because the group count is below 2^31.
    // With a join payload, gin holds the build-side keys' part for the rows
    // in m. Every other row adds 0 to group 0, an in-range slot (its gin is
    // the no-match sentinel, which must never become an address).
    uint32_t g[R];
#pragma unroll
    for (int r = 0; r < R; ++r) g[r] = (gin && ((m >> r) & 1u)) ? gin[r] : 0u;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        if (static_cast<uint32_t>(k) < P.ngkey && !P.gkey[k].build_side) {
            const GKey& K = P.gkey[k];
            uint32_t x[R];
            load_cells32<R>(stage + K.soff, K.dtype, t, x);
            const uint32_t mn = static_cast<uint32_t>(K.min), st = static_cast<uint32_t>(K.stride);
#pragma unroll
            for (int r = 0; r < R; ++r) g[r] += (gin && !((m >> r) & 1u)) ? 0u : (x[r] - mn) * st;
        }
    }
    uint32_t* cnt = priv_counts(extra);
    w = reinterpret_cast<unsigned long long*>(priv_values<NT>(P, extra));
    const uint32_t gstride = P.nval * static_cast<uint32_t>(NT);
    uint32_t base[R];  // value word of row r's group; value v (1-based) is at base + (v - 1) * NT
#pragma unroll
    for (int r = 0; r < R; ++r) base[r] = g[r] * gstride + t;
    // The slots are private to this thread, so plain read-modify-writes in
    // program order are exact (64-bit shared atomics would run as CAS loops).
    if (!P.count_by_tile) {
#pragma unroll
        for (int r = 0; r < R; ++r) cnt[g[r] * NT + t] += (m >> r) & 1u;
    }

    int64_t cur[R];
#pragma unroll
    for (int r = 0; r < R; ++r) cur[r] = 0;
#pragma unroll
    for (int s = 0; s < kMaxSteps; ++s) {
        if (static_cast<uint32_t>(s) >= P.chain.nsteps) break;
        const ChainStep& S = P.chain.s[s];
        int64_t f[R];
        if (S.flags & CS_COL) {
            if (S.flags & CS_NARROW) {
                uint32_t x[R];
                load_cells32<R>(stage + S.soff, S.dtype, t, x);
#pragma unroll
                for (int r = 0; r < R; ++r)
                    f[r] = static_cast<int32_t>(static_cast<uint32_t>(S.mul32) * x[r] + static_cast<uint32_t>(S.add32));
            } else {
                int64_t x[R];
                load_cells64<R>(stage + S.soff, S.dtype, t, x);
                if (S.flags & CS_IDENT) {
#pragma unroll
                    for (int r = 0; r < R; ++r) f[r] = x[r];
                } else {
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        f[r] = static_cast<int64_t>(static_cast<uint64_t>(S.mul) * static_cast<uint64_t>(x[r]) +
                                                    static_cast<uint64_t>(S.add));
                }
            }
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) f[r] = S.add;
        }
        if (S.flags & CS_CHAIN) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                cur[r] = static_cast<int64_t>(static_cast<uint64_t>(cur[r]) * static_cast<uint64_t>(f[r]));
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) cur[r] = f[r];
        }
        if (S.acc) {
            const uint32_t off = (S.acc - 1u) * static_cast<uint32_t>(NT);
            if (S.kind == VK_SUM) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    w[base[r] + off] += ((m >> r) & 1u) ? static_cast<unsigned long long>(cur[r]) : 0ull;
            } else if (S.kind == VK_COUNT_NZ) {
#pragma unroll
                for (int r = 0; r < R; ++r) w[base[r] + off] += (((m >> r) & 1u) && cur[r] != 0) ? 1ull : 0ull;
            } else {
                long long* a = reinterpret_cast<long long*>(w);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (!((m >> r) & 1u)) continue;
                    long long& x = a[base[r] + off];
                    x = S.kind == VK_MIN ? min(x, static_cast<long long>(cur[r])) : max(x, static_cast<long long>(cur[r]));
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Dense tiles of MODE_GROUP_SHARED32: each row's group index (staged keys,
// bucket tables, the join payload's build-side part) and the value program's
// steps are computed for the thread's R rows column by column, then the
// selected rows add to this warp group's table with native 32-bit shared
// atomics: the row count, and per value the low limb (its returned old value
// gives the carry) and the signed high limb.
// ---------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ void chain_s32_tile(const Plan& P, uint8_t* extra, const uint8_t* stage, uint32_t t,
                                               uint32_t m, const uint32_t* gin = nullptr) {
    constexpr int R = kTileRows / NT;
    uint32_t g[R];
#pragma unroll
    for (int r = 0; r < R; ++r) g[r] = (gin && ((m >> r) & 1u)) ? gin[r] : 0u;
#pragma unroll 1
    for (uint32_t k = 0; k < P.ngkey; ++k) {
        const GKey& K = P.gkey[k];
        if (K.build_side) continue;   // its part comes with the payload
        uint32_t x[R];
        load_cells32<R>(stage + K.soff, K.dtype, t, x);
        const uint32_t mn = static_cast<uint32_t>(K.min), st = static_cast<uint32_t>(K.stride);
        if (K.lut) {
#pragma unroll
            for (int r = 0; r < R; ++r) g[r] += static_cast<uint32_t>(__ldg(K.lut + (x[r] - mn))) * st;
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) g[r] += (x[r] - mn) * st;
        }
    }
    const uint32_t W = P.s32_words;
    // (s32_copies is a power of two.)
    uint32_t* tab = reinterpret_cast<uint32_t*>(extra) + static_cast<size_t>((t >> 5) & (P.s32_copies - 1u)) * P.ngroups * W;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if ((m >> r) & 1u) atomicAdd(&tab[g[r] * W], 1u);
    int64_t cur[R];
#pragma unroll
    for (int r = 0; r < R; ++r) cur[r] = 0;
#pragma unroll 1
    for (uint32_t s = 0; s < P.chain.nsteps; ++s) {
        const ChainStep& S = P.chain.s[s];
        int64_t f[R];
        if (S.flags & CS_COL) {
            if (S.flags & CS_NARROW) {
                uint32_t x[R];
                load_cells32<R>(stage + S.soff, S.dtype, t, x);
#pragma unroll
                for (int r = 0; r < R; ++r)
                    f[r] = static_cast<int32_t>(static_cast<uint32_t>(S.mul32) * x[r] + static_cast<uint32_t>(S.add32));
            } else {
                int64_t x[R];
                load_cells64<R>(stage + S.soff, S.dtype, t, x);
#pragma unroll
                for (int r = 0; r < R; ++r)
                    f[r] = (S.flags & CS_IDENT) ? x[r]
                                                : static_cast<int64_t>(static_cast<uint64_t>(S.mul) * static_cast<uint64_t>(x[r]) +
                                                                       static_cast<uint64_t>(S.add));
            }
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) f[r] = S.add;
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
            cur[r] = (S.flags & CS_CHAIN) ? static_cast<int64_t>(static_cast<uint64_t>(cur[r]) * static_cast<uint64_t>(f[r]))
                                          : f[r];
        if (S.acc) {
            // (Issuing all R low-limb adds before reading any returned value
            // measured slower: more instructions, no latency gained.)
            const uint32_t w0 = 1u + 2u * (S.acc - 1u);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (!((m >> r) & 1u)) continue;
                const int64_t x = S.kind == VK_COUNT_NZ ? (cur[r] != 0 ? 1 : 0) : cur[r];
                uint32_t* e = &tab[g[r] * W + w0];
                const uint32_t xl = static_cast<uint32_t>(x);
                const uint32_t old = atomicAdd(e, xl);
                const int32_t add = static_cast<int32_t>(x >> 32) + ((old + xl < old) ? 1 : 0);
                if (add) atomicAdd(reinterpret_cast<int*>(e + 1), add);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Dense value programs of a fixed shape. The key dtypes and every step's
// dtype / flags / kind / value slot are template constants (literals and
// column offsets still come from the plan), so a tile runs as one
// straight-line block: all shared-memory loads first, then the arithmetic,
// then one batch of read-modify-writes per row.
// Step code: dtype | flags << 4 | kind << 10 | value slot << 13.
// ---------------------------------------------------------------------------
constexpr uint32_t step_code(uint32_t dt, uint32_t fl, uint32_t kind, uint32_t acc) {
    return dt | (fl << 4) | (kind << 10) | (acc << 13);
}

// Kernel tag: scalar aggregates on the register fast path (RegVals).
struct ScalarTag {};



template <uint32_t NKEY, uint32_t KDT0, uint32_t KDT1, uint32_t... STEPS>
struct DenseShape {
    static constexpr uint32_t nkey = NKEY;
    static constexpr uint32_t kdt0 = KDT0;
    static constexpr uint32_t kdt1 = KDT1;
    static constexpr uint32_t nsteps = sizeof...(STEPS);
    static constexpr uint32_t step[sizeof...(STEPS)] = {STEPS...};
    __host__ __device__ static constexpr uint32_t max_acc() {
        uint32_t m = 0;
        for (uint32_t i = 0; i < sizeof...(STEPS); ++i) m = ((step[i] >> 13) > m) ? (step[i] >> 13) : m;
        return m;
    }
    static constexpr uint32_t nv1 = max_acc() + 1;  // value slots per group (slot 0 = row count)
    static constexpr bool dense_shape = true;
    __host__ __device__ static constexpr uint32_t kind_of(uint32_t v) {  // VK_* accumulated into value slot v
        uint32_t k = VK_SUM;
        for (uint32_t i = 0; i < sizeof...(STEPS); ++i)
            if ((step[i] >> 13) == v) k = (step[i] >> 10) & 7u;
        return k;
    }
};

// A fixed-shape kernel tag (DenseShape) as opposed to void or ScalarTag.
template <class T, class = void>
struct IsDenseShape : std::false_type {};
template <class T>
struct IsDenseShape<T, std::void_t<decltype(T::dense_shape)>> : std::true_type {};

template <int... I, typename F>
__device__ __forceinline__ void static_for_impl(std::integer_sequence<int, I...>, F&& f) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
    static_for_impl(std::make_integer_sequence<int, N>{}, f);
}

// Thread t's R cells of a staged column at shared address `a` (low 32 bits).
template <int R, uint32_t DT>
__device__ __forceinline__ void lds_cells32(uint32_t a, uint32_t t, uint32_t (&x)[R]) {
    if constexpr (DT == DT_U8) {
        if constexpr (R == 4) {
            const uint32_t w = lds_u32(a + 4u * t);
#pragma unroll
            for (int e = 0; e < 4; ++e) x[e] = (w >> (8 * e)) & 0xffu;
        } else {
            const uint2 w = lds_v2(a + 8u * t);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                x[e] = (w.x >> (8 * e)) & 0xffu;
                x[e + 4] = (w.y >> (8 * e)) & 0xffu;
            }
        }
    } else if constexpr (DT == DT_I32) {
#pragma unroll
        for (int c = 0; c < R / 4; ++c) {
            const uint4 v = lds_v4(a + 16u * ((R / 4) * t + c));
            x[4 * c + 0] = v.x;
            x[4 * c + 1] = v.y;
            x[4 * c + 2] = v.z;
            x[4 * c + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int c = 0; c < R / 2; ++c) {
            const uint4 v = lds_v4(a + 16u * ((R / 2) * t + c));
            x[2 * c + 0] = v.x;
            x[2 * c + 1] = v.z;
        }
    }
}

template <int R, uint32_t DT>
__device__ __forceinline__ void lds_cells64(uint32_t a, uint32_t t, uint64_t (&x)[R]) {
    if constexpr (DT == DT_I64 || DT == DT_U64) {
#pragma unroll
        for (int c = 0; c < R / 2; ++c) {
            const uint4 v = lds_v4(a + 16u * ((R / 2) * t + c));
            x[2 * c + 0] = (static_cast<uint64_t>(v.y) << 32) | v.x;
            x[2 * c + 1] = (static_cast<uint64_t>(v.w) << 32) | v.z;
        }
    } else {
        uint32_t y[R];
        lds_cells32<R, DT>(a, t, y);
#pragma unroll
        for (int r = 0; r < R; ++r)
            x[r] = DT == DT_I32 ? static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(y[r]))) : y[r];
    }
}

template <int NT, class SH>
__device__ __forceinline__ void chain_tile_static(const Plan& P, uint8_t* extra, const uint8_t* stage, uint32_t t,
                                                  uint32_t m, Sink<MODE_GROUP_PRIVATE, false, NT>& sink,
                                                  const uint32_t* gin = nullptr) {
    constexpr int R = kTileRows / NT;
    constexpr int NS = static_cast<int>(SH::nsteps);
    constexpr uint32_t NV1 = SH::nv1;
    const uint32_t sa = smem_addr(stage);

    // Shared-memory loads of every referenced column, issued back to back.
    uint32_t kx0[R], kx1[R];
    if constexpr (SH::nkey >= 1) lds_cells32<R, SH::kdt0>(sa + P.gkey[0].soff, t, kx0);
    if constexpr (SH::nkey >= 2) lds_cells32<R, SH::kdt1>(sa + P.gkey[1].soff, t, kx1);
    uint32_t c32[NS][R];
    uint64_t c64[NS][R];
    static_for<NS>([&](auto I) {
        constexpr uint32_t c = SH::step[I.value];
        constexpr uint32_t dt = c & 15u, fl = (c >> 4) & 63u;
        if constexpr ((fl & CS_COL) != 0) {
            if constexpr ((fl & CS_NARROW) != 0) lds_cells32<R, dt>(sa + P.chain.s[I.value].soff, t, c32[I.value]);
            else lds_cells64<R, dt>(sa + P.chain.s[I.value].soff, t, c64[I.value]);
        }
    });

    const uint32_t nsel = __popc(m);
    if (sink.upd + nsel > P.flush_limit) {
        sink.flush_private_thread(P, extra, t);
        sink.upd = 0;
    }
    sink.upd += nsel;

    uint32_t sm[R];  // all ones for a selected row, else 0
#pragma unroll
    for (int r = 0; r < R; ++r) sm[r] = 0u - ((m >> r) & 1u);

    // Values. A product starts from its first factor masked by the selection,
    // so unselected rows carry 0 through every chained step.
    uint64_t val[NV1][R];
    uint64_t cur[R];
    static_for<NS>([&](auto I) {
        constexpr int s = I.value;
        constexpr uint32_t c = SH::step[s];
        constexpr uint32_t fl = (c >> 4) & 63u, acc = c >> 13;
        constexpr bool chain = (fl & CS_CHAIN) != 0;
        const ChainStep& S = P.chain.s[s];
        if constexpr ((fl & CS_COL) != 0 && (fl & CS_NARROW) != 0) {
            const uint32_t mu = static_cast<uint32_t>(S.mul32), ad = static_cast<uint32_t>(S.add32);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                uint32_t f = mu * c32[s][r] + ad;
                if constexpr (!chain) f &= sm[r];
                const uint64_t fw = (fl & CS_NONNEG) ? static_cast<uint64_t>(f)
                                                     : static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(f)));
                cur[r] = chain ? cur[r] * fw : fw;
            }
        } else if constexpr ((fl & CS_COL) != 0) {
            const uint64_t mu = static_cast<uint64_t>(S.mul), ad = static_cast<uint64_t>(S.add);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                uint64_t f = (fl & CS_IDENT) ? c64[s][r] : mu * c64[s][r] + ad;
                if constexpr (!chain) f &= static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(sm[r])));
                cur[r] = chain ? cur[r] * f : f;
            }
        } else {
            const uint64_t k = static_cast<uint64_t>(S.add);
#pragma unroll
            for (int r = 0; r < R; ++r)
                cur[r] = chain ? cur[r] * k : (k & static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(sm[r]))));
        }
        if constexpr (acc != 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) val[acc][r] = cur[r];
        }
    });

    // Read-modify-writes of the thread's private slots, row by row (rows of
    // one group share slots, so each row reads what the previous one wrote).
    constexpr uint32_t kGroupBytes = (NV1 - 1) * NT * 8u;
    const uint32_t ca0 = smem_addr(extra) + 4u * t;
    const uint32_t wa = smem_addr(extra) + priv_count_bytes(P.ngroups, NT) + 8u * t;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        // With a join payload, gin holds the (build-side) group index of the
        // rows in m; every other row adds 0 to group 0.
        uint32_t g = (gin && ((m >> r) & 1u)) ? gin[r] : 0u;
        if constexpr (SH::nkey >= 1)
            g += (kx0[r] - static_cast<uint32_t>(P.gkey[0].min)) * static_cast<uint32_t>(P.gkey[0].stride);
        if constexpr (SH::nkey >= 2)
            g += (kx1[r] - static_cast<uint32_t>(P.gkey[1].min)) * static_cast<uint32_t>(P.gkey[1].stride);
        const uint32_t a = wa + g * kGroupBytes;
        const uint32_t ca = ca0 + g * static_cast<uint32_t>(NT) * 4u;
        unsigned long long old[NV1];
        uint32_t oldc = 0;
        // The row count (a scalar aggregate counts by popcount per tile).
        const bool count_rows = SH::nkey > 0 || !P.count_by_tile;
        if (count_rows) oldc = lds_u32(ca);
        static_for<NV1>([&](auto V) {
            constexpr uint32_t v = V.value;
            if constexpr (v > 0) old[v] = lds_u64<(v - 1) * NT * 8u>(a);
        });
        if (count_rows) sts_u32(ca, oldc + (sm[r] & 1u));
        static_for<NV1>([&](auto V) {
            constexpr uint32_t v = V.value;
            if constexpr (v > 0) {
                constexpr uint32_t kind = SH::kind_of(v);
                unsigned long long nw;
                const long long x = static_cast<long long>(val[v][r]);
                if constexpr (kind == VK_SUM) nw = old[v] + val[v][r];
                else if constexpr (kind == VK_COUNT_NZ) nw = old[v] + (val[v][r] != 0 ? 1ull : 0ull);
                else if constexpr (kind == VK_MIN) nw = sm[r] ? static_cast<unsigned long long>(min(static_cast<long long>(old[v]), x)) : old[v];
                else nw = sm[r] ? static_cast<unsigned long long>(max(static_cast<long long>(old[v]), x)) : old[v];
                sts_u64<(v - 1) * NT * 8u>(a, nw);
            }
        });
    }
}

// ---------------------------------------------------------------------------
// Fixed-shape value programs on the 32-bit limb tables (MODE_GROUP_SHARED32,
// merged scans of the serving templates): the keys come from the runtime
// loop of chain_s32_tile (bucket tables, staged keys, the payload's part);
// the value program's steps, their dtypes and value slots are template
// constants, so a tile runs the shared loads, the arithmetic and the limb
// atomics as straight-line code instead of a loop over plan steps.
// SUM / COUNT(col) values only (the limb tables' kinds).
// ---------------------------------------------------------------------------
template <int NT, class SH>
__device__ __forceinline__ void chain_s32_tile_static(const Plan& P, uint8_t* extra, const uint8_t* stage, uint32_t t,
                                                      uint32_t m, const uint32_t* gin = nullptr) {
    constexpr int R = kTileRows / NT;
    constexpr int NS = static_cast<int>(SH::nsteps);
    const uint32_t sa = smem_addr(stage);
    // Shared-memory loads of the value program's columns, issued first.
    uint32_t c32[NS][R];
    uint64_t c64[NS][R];
    static_for<NS>([&](auto I) {
        constexpr uint32_t c = SH::step[I.value];
        constexpr uint32_t dt = c & 15u, fl = (c >> 4) & 63u;
        if constexpr ((fl & CS_COL) != 0) {
            if constexpr ((fl & CS_NARROW) != 0) lds_cells32<R, dt>(sa + P.chain.s[I.value].soff, t, c32[I.value]);
            else lds_cells64<R, dt>(sa + P.chain.s[I.value].soff, t, c64[I.value]);
        }
    });
    uint32_t g[R];
#pragma unroll
    for (int r = 0; r < R; ++r) g[r] = (gin && ((m >> r) & 1u)) ? gin[r] : 0u;
#pragma unroll 1
    for (uint32_t k = 0; k < P.ngkey; ++k) {
        const GKey& K = P.gkey[k];
        if (K.build_side) continue;   // its part comes with the payload
        uint32_t x[R];
        load_cells32<R>(stage + K.soff, K.dtype, t, x);
        const uint32_t mn = static_cast<uint32_t>(K.min), st = static_cast<uint32_t>(K.stride);
        if (K.lut) {
#pragma unroll
            for (int r = 0; r < R; ++r) g[r] += static_cast<uint32_t>(__ldg(K.lut + (x[r] - mn))) * st;
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) g[r] += (x[r] - mn) * st;
        }
    }
    const uint32_t W = P.s32_words;
    // (s32_copies is a power of two.)
    uint32_t* tab = reinterpret_cast<uint32_t*>(extra) + static_cast<size_t>((t >> 5) & (P.s32_copies - 1u)) * P.ngroups * W;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if ((m >> r) & 1u) atomicAdd(&tab[g[r] * W], 1u);
    uint64_t cur[R];
    static_for<NS>([&](auto I) {
        constexpr int s = I.value;
        constexpr uint32_t c = SH::step[s];
        constexpr uint32_t fl = (c >> 4) & 63u, kind = (c >> 10) & 7u, acc = c >> 13;
        constexpr bool chain = (fl & CS_CHAIN) != 0;
        const ChainStep& S = P.chain.s[s];
        if constexpr ((fl & CS_COL) != 0 && (fl & CS_NARROW) != 0) {
            const uint32_t mu = static_cast<uint32_t>(S.mul32), ad = static_cast<uint32_t>(S.add32);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t f = mu * c32[s][r] + ad;
                const uint64_t fw = (fl & CS_NONNEG) ? static_cast<uint64_t>(f)
                                                     : static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(f)));
                cur[r] = chain ? cur[r] * fw : fw;
            }
        } else if constexpr ((fl & CS_COL) != 0) {
            const uint64_t mu = static_cast<uint64_t>(S.mul), ad = static_cast<uint64_t>(S.add);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint64_t f = (fl & CS_IDENT) ? c64[s][r] : mu * c64[s][r] + ad;
                cur[r] = chain ? cur[r] * f : f;
            }
        } else {
            const uint64_t k = static_cast<uint64_t>(S.add);
#pragma unroll
            for (int r = 0; r < R; ++r) cur[r] = chain ? cur[r] * k : k;
        }
        if constexpr (acc != 0) {
            static_assert(kind == VK_SUM || kind == VK_COUNT_NZ, "limb tables hold SUM / COUNT(col) values");
            constexpr uint32_t w0 = 1u + 2u * (acc - 1u);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (!((m >> r) & 1u)) continue;
                const int64_t x = kind == VK_COUNT_NZ ? (cur[r] != 0 ? 1 : 0) : static_cast<int64_t>(cur[r]);
                uint32_t* e = &tab[g[r] * W + w0];
                const uint32_t xl = static_cast<uint32_t>(x);
                const uint32_t old = atomicAdd(e, xl);
                const int32_t add = static_cast<int32_t>(x >> 32) + ((old + xl < old) ? 1 : 0);
                if (add) atomicAdd(reinterpret_cast<int*>(e + 1), add);
            }
        }
    });
}

// ---------------------------------------------------------------------------
// Join probe through the payload array (unique build keys, dense key range):
// pay[key - kmin] is the build-side part of the group index of the one
// matching build row, or kNoPay. The R lookups of a thread are independent
// loads, so they are all in flight at once.
// ---------------------------------------------------------------------------
// Payload entry `rel` (P.jpay_w bytes; all ones = kNoPay).
__device__ __forceinline__ uint32_t pay_load(const Plan& P, uint64_t rel) {
    if (P.jpay_w == 1) {
        const uint32_t v = __ldg(reinterpret_cast<const uint8_t*>(P.jpay) + rel);
        return v == 0xffu ? kNoPay : v;
    }
    if (P.jpay_w == 2) {
        const uint32_t v = __ldg(reinterpret_cast<const uint16_t*>(P.jpay) + rel);
        return v == 0xffffu ? kNoPay : v;
    }
    return __ldg(P.jpay + rel);
}

template <int R, typename E>
__device__ __forceinline__ void pay_lookups(const Plan& P, const int64_t (&cell)[R], uint32_t m, uint32_t (&g)[R]) {
    const E* pay = reinterpret_cast<const E*>(P.jpay);
    constexpr E kNone = static_cast<E>(~0u);
    E v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint64_t rel = static_cast<uint64_t>(cell[r]) - static_cast<uint64_t>(P.jkmin);
        const bool probe = ((m >> r) & 1u) && rel <= P.jkrange;
        v[r] = probe ? __ldg(pay + rel) : kNone;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) g[r] = v[r] == kNone ? kNoPay : static_cast<uint32_t>(v[r]);
}

template <int R>
__device__ __forceinline__ uint32_t join_pay_probe(const Plan& P, const uint8_t* stage, uint32_t t, uint32_t m,
                                                   uint32_t (&g)[R]) {
    const uint8_t* kb = stage + P.slot[P.jslot].smem_off;
    const uint32_t kdt = P.slot[P.jslot].dtype;
    int64_t cell[R];
    load_cells64<R>(kb, kdt, t, cell);
    if (P.jpay_w == 1) pay_lookups<R, uint8_t>(P, cell, m, g);
    else if (P.jpay_w == 2) pay_lookups<R, uint16_t>(P, cell, m, g);
    else pay_lookups<R, uint32_t>(P, cell, m, g);
    uint32_t hit = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) hit |= (g[r] != kNoPay ? 1u : 0u) << r;
    return hit;
}

// ---------------------------------------------------------------------------
// Global / hash grouping by one staged key with one or two values, each a
// SUM or COUNT(col) of one staged affine factor (P.hash_fast): the thread's R
// key and value cells are loaded column by column, then each selected row
// goes to the shared pre-aggregation table or, failing that, the global one.
// COUNT(col) arguments arrive already reduced to 0 / 1.
// ---------------------------------------------------------------------------
template <uint32_t MODE, int R>
__device__ __forceinline__ void hash_fast_tile(const Plan& P, uint8_t* extra, const uint8_t* stage, uint32_t t,
                                               uint32_t m) {
    const GKey& K = P.gkey[0];
    int64_t kc[R], vc[2][R];
    load_cells64<R>(stage + K.soff, K.dtype, t, kc);
#pragma unroll
    for (int v = 0; v < 2; ++v)
        if (static_cast<uint32_t>(v) < P.nval) load_cells64<R>(stage + P.val[v].f[0].soff, P.val[v].f[0].dtype, t, vc[v]);
    const uint32_t nv1 = P.nval + 1;
    // Keys and value arguments of the thread's R rows.
    uint64_t key[R];
    int64_t x[R][2];
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            if (static_cast<uint32_t>(v) >= P.nval) continue;
            const Factor& F = P.val[v].f[0];
            const int64_t a = static_cast<int64_t>(static_cast<uint64_t>(F.mul) * static_cast<uint64_t>(vc[v][r]) +
                                                   static_cast<uint64_t>(F.add));
            x[r][v] = P.val[v].kind == VK_COUNT_NZ ? (a != 0 ? 1 : 0) : a;
        }
        const uint64_t rel = static_cast<uint64_t>(kc[r]) - static_cast<uint64_t>(K.min);
        key[r] = MODE == MODE_GROUP_HASH ? (rel << K.shift) : rel * K.stride;
    }
    // Shared pre-aggregation: the first probe's key loads of all R rows are
    // issued together, then each row either adds to its slot (the common
    // case once the table holds the hot keys), claims an empty one, tries
    // the second probe, or falls through to the global table.
    uint32_t pend = m;
    if (P.hsm_slots) {
        const uint32_t HS = P.hsm_slots;
        with_presum(P, extra, [&](auto T) {
            using KT = std::remove_pointer_t<decltype(T.keys)>;
            uint32_t h[R];
            KT kr[R], k0[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                kr[r] = static_cast<KT>(key[r]);
                h[r] = T.slot(kr[r], P.hsm_log2);
                k0[r] = ((m >> r) & 1u) ? *reinterpret_cast<volatile KT*>(&T.keys[h[r]]) : KT{0};
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (!((m >> r) & 1u)) continue;
                uint32_t hs = h[r];
                KT k = k0[r];
#pragma unroll
                for (uint32_t n = 0; n < kSmemProbes; ++n) {
                    if (n) {
                        hs = (hs + 1) & (HS - 1);
                        k = *reinterpret_cast<volatile KT*>(&T.keys[hs]);
                    }
                    if (k == T.kEmptyKey) k = atomicCAS(&T.keys[hs], T.kEmptyKey, kr[r]);
                    if (k == T.kEmptyKey || k == kr[r]) {
                        atomicAdd(&T.cnt[hs], 1u);
#pragma unroll
                        for (int v = 0; v < 2; ++v)
                            if (static_cast<uint32_t>(v) < P.nval)
                                atomicAdd(&T.sums[v * HS + hs], static_cast<int32_t>(x[r][v]));
                        pend &= ~(1u << r);
                        break;
                    }
                }
            }
        });
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        if (!((pend >> r) & 1u)) continue;
        unsigned long long* base;
        if (MODE == MODE_GROUP_HASH) {
            unsigned long long* slot = hash_group_slot(P, key[r]);
            if (slot == nullptr) continue;
            base = slot + 1;   // [key][count][v0 lo][v0 hi]...
        } else {
            base = P.acc + key[r] * nv1 * 2;   // [count lo][count hi][v0 lo][v0 hi]...
        }
        atomicAdd(base, 1ull);
#pragma unroll
        for (int v = 0; v < 2; ++v)
            if (static_cast<uint32_t>(v) < P.nval)
                acc_global_i64(base + (MODE == MODE_GROUP_HASH ? 1 : 2) + 2 * v, VK_SUM, x[r][v], P.sum64 != 0);
    }
}

// ---------------------------------------------------------------------------
// The column path on one-word direct slots (P.hpack; one key, COUNT(*) and
// at most one SUM / COUNT(col)). A direct slot index is below 2^27, so keys,
// the shared table's hash and its compares run in 32 bits; a row that finds
// no shared slot is one non-returning 64-bit add of (1 << shift) +
// (value - bias) to its key's word.
// ---------------------------------------------------------------------------
template <int R>
__device__ __forceinline__ void hpack_tile(const Plan& P, uint8_t* extra, const uint8_t* stage, uint32_t t,
                                           uint32_t m) {
    const GKey& K = P.gkey[0];
    const ValDesc& V = P.val[0];
    const bool hasv = P.nval != 0;
    int64_t kc[R], vc[R];
    load_cells64<R>(stage + K.soff, K.dtype, t, kc);
    if (hasv) load_cells64<R>(stage + V.f[0].soff, V.f[0].dtype, t, vc);
    const uint32_t kmin = static_cast<uint32_t>(K.min);
    const uint64_t mul = static_cast<uint64_t>(V.f[0].mul), add = static_cast<uint64_t>(V.f[0].add);
    const bool ident = mul == 1 && add == 0, nz = V.kind == VK_COUNT_NZ;
    uint32_t key[R];
    int64_t x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        // The cell lies in [min, min + 2^27): its slot is the low word's difference.
        key[r] = static_cast<uint32_t>(kc[r]) - kmin;
        int64_t a = 0;
        if (hasv) a = ident ? vc[r] : static_cast<int64_t>(mul * static_cast<uint64_t>(vc[r]) + add);
        x[r] = nz ? (a != 0 ? 1 : 0) : a;
    }
    uint32_t pend = m;
    if (P.hsm_slots) {
        PresumTab<uint32_t> T(extra, P.hsm_slots);
        const uint32_t HS = P.hsm_slots;
        uint32_t h[R], k0[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            h[r] = PresumTab<uint32_t>::slot(key[r], P.hsm_log2);
            k0[r] = ((m >> r) & 1u) ? *reinterpret_cast<volatile uint32_t*>(&T.keys[h[r]]) : 0u;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (!((m >> r) & 1u)) continue;
            uint32_t hs = h[r], k = k0[r];
#pragma unroll
            for (uint32_t n = 0; n < kSmemProbes; ++n) {
                if (n) {
                    hs = (hs + 1) & (HS - 1);
                    k = *reinterpret_cast<volatile uint32_t*>(&T.keys[hs]);
                }
                if (k == T.kEmptyKey) k = atomicCAS(&T.keys[hs], T.kEmptyKey, key[r]);
                if (k == T.kEmptyKey || k == key[r]) {
                    atomicAdd(&T.cnt[hs], 1u);
                    if (hasv) atomicAdd(&T.sums[hs], static_cast<int32_t>(x[r]));
                    pend &= ~(1u << r);
                    break;
                }
            }
        }
    }
    const unsigned long long one = (1ull << P.hpack_shift) - static_cast<uint64_t>(P.hpack_bias);
    const uint32_t last = static_cast<uint32_t>(P.hmask);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        if (!((pend >> r) & 1u)) continue;
        if (key[r] > last) {
            atomicOr(P.err, kErrHashFull);
            continue;
        }
        atomicAdd(P.htab + key[r], one + static_cast<unsigned long long>(x[r]));
    }
}

// ---------------------------------------------------------------------------
// Tile processing (consumer threads)
// ---------------------------------------------------------------------------
template <uint32_t MODE, bool ACC128, int NT, bool TAIL, class SH>
__device__ __forceinline__ void process_tile(const Plan& P, Sink<MODE, ACC128, NT>& sink, uint8_t* extra,
                                             const uint8_t* stage, uint64_t tile, uint32_t t,
                                             unsigned long long& selected, const RegLeaves& RL,
                                             const RegVals& RV) {
    constexpr int R = kTileRows / NT;
    const uint64_t r0 = tile * kTileRows;
    const uint32_t nrem = TAIL ? static_cast<uint32_t>(P.nrows - r0) : static_cast<uint32_t>(kTileRows);
    const uint32_t m = (!TAIL && RL.n) ? eval_reg_leaves<R>(RL, stage, t) : eval_pred<R, TAIL>(P, stage, r0, t, nrem);
    const uint32_t lane = t & 31u;
    selected += __popc(m);
    if (MODE == MODE_GROUP_PRIVATE && P.count_by_tile) {
        // Scalar aggregate: the group's row count is the number of selected rows.
        long long* w = reinterpret_cast<long long*>(extra);
        if (ACC128) {
            uint64_t* lo = reinterpret_cast<uint64_t*>(&w[t]);
            const uint64_t nl = *lo + __popc(m);
            w[NT + t] += (nl < *lo) ? 1 : 0;
            *lo = nl;
        } else {
            priv_counts(extra)[t] += __popc(m);
        }
    }

    if (MODE == MODE_FILTER) {
        // 32 / R consecutive lanes hold the bits of one 32-row bitmap word.
        constexpr uint32_t G = 32 / R;
        uint32_t v = m << (R * (lane % G));
#pragma unroll
        for (uint32_t d = 1; d < G; d <<= 1) v |= __shfl_xor_sync(kFull, v, d);
        if (lane % G == 0) {
            const uint64_t wi = (r0 + static_cast<uint64_t>(R) * t) / 32;
            if (wi < P.bitmap_words) P.bitmap[wi] = v;
        }
        if (P.tile_counts) {
            unsigned c = __popc(m);
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(kFull, c, d);
            if (lane == 0 && c) atomicAdd(P.tile_counts + tile, c);
        }
        return;
    }

    if (MODE == MODE_JOIN_PAIRS) {
        const uint8_t* kb = slot_base<TAIL>(P, stage, P.jslot, r0);
        const uint32_t kdt = P.slot[P.jslot].dtype;
        uint32_t nmatch = 0;
        for (uint32_t sel = m; sel; sel &= sel - 1) {
            uint64_t rel;
            if (join_rel(P, load_cell(kb, kdt, R * t + __ffs(sel) - 1), rel))
                join_foreach(P, rel, [&](uint32_t) { ++nmatch; });
        }
        // Warp-aggregated reservation of this warp's output pairs.
        uint32_t incl = nmatch;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, d);
            if (lane >= static_cast<uint32_t>(d)) incl += y;
        }
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        unsigned long long base = 0;
        if (lane == 31 && total) base = atomicAdd(P.counters + 1, static_cast<unsigned long long>(total));
        base = __shfl_sync(kFull, base, 31);
        unsigned long long o = base + incl - nmatch;
        for (uint32_t sel = nmatch ? m : 0u; sel; sel &= sel - 1) {
            const uint32_t rl = R * t + __ffs(sel) - 1;
            uint64_t rel;
            if (!join_rel(P, load_cell(kb, kdt, rl), rel)) continue;
            const unsigned long long prow = static_cast<unsigned long long>(r0 + rl) << 32;
            join_foreach(P, rel, [&](uint32_t b) {
                if (o < P.out_cap) P.out_pairs[o] = prow | b;
                ++o;
            });
        }
        return;
    }

    // Grouped / scalar aggregates, join build, and joined aggregates.
    auto one_row = [&](uint32_t rl) {
        if (P.jslot >= 0 && MODE != MODE_JOIN_BUILD) {
            const int64_t c = load_cell(slot_base<TAIL>(P, stage, P.jslot, r0), P.slot[P.jslot].dtype, rl);
            uint64_t rel;
            if (join_rel(P, c, rel))
                join_foreach(P, rel, [&](uint32_t b) { sink.template row<TAIL>(P, extra, stage, r0, rl, b, t); });
        } else {
            sink.template row<TAIL>(P, extra, stage, r0, rl, 0, t);
        }
    };
    // The scalar kernel (SH = ScalarTag) carries only the register fast path
    // and the generic row loop.
    constexpr bool kScalar = std::is_same<SH, ScalarTag>::value;
    if constexpr (!kScalar && (MODE == MODE_GROUP_PRIVATE || MODE == MODE_GROUP_SHARED || MODE == MODE_GROUP_GLOBAL ||
                               MODE == MODE_GROUP_SHARED32)) {
        if (!TAIL && P.jpay) {
            uint32_t g[R];
            const uint32_t hit = join_pay_probe<R>(P, stage, t, m, g);
            if constexpr (MODE == MODE_GROUP_SHARED32) {
                if (P.dense_vec) {
                    if constexpr (IsDenseShape<SH>::value) chain_s32_tile_static<NT, SH>(P, extra, stage, t, hit, g);
                    else chain_s32_tile<NT>(P, extra, stage, t, hit, g);
                    return;
                }
            }
            if constexpr (MODE == MODE_GROUP_PRIVATE && !ACC128) {
                if (P.dense_vec && __reduce_add_sync(kFull, __popc(hit)) >= 8u * R) {
                    if constexpr (!std::is_void<SH>::value && !kScalar) {
                        if (P.shape) chain_tile_static<NT, SH>(P, extra, stage, t, hit, sink, g);
                        else chain_private_tile<NT>(P, extra, stage, t, hit, sink, g);
                    } else {
                        chain_private_tile<NT>(P, extra, stage, t, hit, sink, g);
                    }
                    return;
                }
            }
            const uint8_t* kb = stage + P.slot[P.jslot].smem_off;
            const uint32_t kdt = P.slot[P.jslot].dtype;
            for (uint32_t sel = hit; sel; sel &= sel - 1) {
                const uint32_t rl = R * t + __ffs(sel) - 1;
                const uint64_t rel = static_cast<uint64_t>(load_cell(kb, kdt, rl)) - static_cast<uint64_t>(P.jkmin);
                sink.template row<TAIL>(P, extra, stage, r0, rl, 0, t, pay_load(P, rel));
            }
            return;
        }
    }
    // Each iteration handles the next selected row of every lane at once, so a
    // sparse selection costs max(rows per lane) iterations, not the total.
    if constexpr (MODE == MODE_GROUP_PRIVATE && !ACC128) {
        if (!TAIL && RV.on) {
            for (uint32_t sel = m; sel; sel &= sel - 1) fast_row<NT>(P, RV, extra, stage, R * t + __ffs(sel) - 1, t, sink.upd, sink);
            return;
        }
        // A warp whose rows are at least a quarter selected runs the dense
        // column program; sparser warps loop over their selected rows only.
        if (!kScalar && !TAIL && P.dense_vec && __reduce_add_sync(kFull, __popc(m)) >= 8u * R) {
            if constexpr (kScalar) {
            } else if constexpr (std::is_void<SH>::value) {
                chain_private_tile<NT>(P, extra, stage, t, m, sink);
            } else {
                if (P.shape) chain_tile_static<NT, SH>(P, extra, stage, t, m, sink);
                else chain_private_tile<NT>(P, extra, stage, t, m, sink);
            }
            return;
        }
    }
    if constexpr (MODE == MODE_GROUP_SHARED32) {
        if (!TAIL && P.dense_vec) {
            if constexpr (IsDenseShape<SH>::value) chain_s32_tile_static<NT, SH>(P, extra, stage, t, m);
            else chain_s32_tile<NT>(P, extra, stage, t, m);
            return;
        }
    }
    if constexpr (MODE == MODE_GROUP_HASH || MODE == MODE_GROUP_GLOBAL) {
        if (!TAIL && P.hash_fast) {
            if constexpr (MODE == MODE_GROUP_HASH) {
                if (P.hpack) {
                    hpack_tile<R>(P, extra, stage, t, m);
                    return;
                }
            }
            hash_fast_tile<MODE, R>(P, extra, stage, t, m);
            return;
        }
    }
    for (uint32_t sel = m; sel; sel &= sel - 1) one_row(R * t + __ffs(sel) - 1);
}

// ---------------------------------------------------------------------------
// The tile pipeline: NT consumer threads + one producer warp.
//
// Stage s has two mbarriers: full[s] (producer arrive + TMA transaction bytes)
// and empty[s] (one arrive per consumer warp once it has read the stage). The
// producer waits on empty[s] before refilling stage s; consumers wait on
// full[s]. No CTA-wide barrier runs per tile. Every wait is bounded; a wait
// that gives up raises kErrWaitTimeout and sets the CTA's abort flag.
//
// A CTA walks the tiles first + k * stride (k < count). The full tiles
// (tile < nfull) go through the stages; the final partial tile is read from
// global memory. (s, phase, issued) carry over between calls on the same
// barriers.
// ---------------------------------------------------------------------------
struct PipeState {
    uint32_t s = 0;      // stage of the next full tile
    uint32_t phase = 0;  // its mbarrier phase
    uint64_t n = 0;      // full tiles handled so far on these barriers
};

__device__ __forceinline__ void pipe_produce(const Plan& P, uint64_t* full, uint64_t* empty, uint8_t* stages,
                                             uint64_t first, uint64_t stride, uint64_t count, PipeState& st,
                                             uint32_t* abort_flag) {
    const uint64_t nfull = P.nrows / kTileRows;
    const uint32_t S = P.nstages;
    const uint64_t policy = l2_policy_evict_first();
    // Tile j is prefetched into L2 when tile j - l2_ahead is copied into its
    // stage, so a stage copy reads L2 instead of waiting out the HBM latency.
    const uint32_t D = P.l2_ahead;
    auto prefetch = [&](uint64_t j) {
        if (j >= count) return;
        const uint64_t tj = first + j * stride;
        if (tj >= nfull) return;
        for (uint32_t c = 0; c < P.nslots; ++c) {
            const uint32_t bytes = kTileRows * P.slot[c].width;
            bulk_prefetch_l2(P.slot[c].ptr + tj * bytes, bytes);
        }
    };
    for (uint64_t j = S; j < D; ++j) prefetch(j);
    for (uint64_t k = 0; k < count; ++k) {
        const uint64_t tl = first + k * stride;
        if (tl >= nfull) break;
        if (D && k + D >= S) prefetch(k + D);
        if (st.n >= S) {
            // Wait until every consumer warp has released the previous use of
            // stage s (one phase earlier).
            if (!mbar_wait_bounded(&empty[st.s], st.phase ^ 1u, P.wait_ns)) {
                atomicOr(P.err, kErrWaitTimeout);
                atomicExch(abort_flag, 1u);
                break;
            }
        }
        if (*reinterpret_cast<volatile uint32_t*>(abort_flag)) break;
        if (P.skip_tile1 == tl + 1) {
            // Test hook: this stage's copy is never issued, so the consumers'
            // bounded wait for it runs out (kErrWaitTimeout), as would a copy
            // that never lands.
            ++st.n;
            if (++st.s == S) {
                st.s = 0;
                st.phase ^= 1u;
            }
            continue;
        }
        uint8_t* dst = stages + static_cast<size_t>(st.s) * P.stage_bytes;
        mbar_arrive_expect_tx(&full[st.s], P.stage_bytes);
        for (uint32_t c = 0; c < P.nslots; ++c) {
            const uint32_t bytes = kTileRows * P.slot[c].width;
            bulk_g2s(dst + P.slot[c].smem_off, P.slot[c].ptr + tl * bytes, bytes, &full[st.s], policy);
        }
        ++st.n;
        if (++st.s == S) {
            st.s = 0;
            st.phase ^= 1u;
        }
    }
}

// Consumers: returns false after a timeout or abort.
template <uint32_t MODE, bool ACC128, int NT, class SH>
__device__ __forceinline__ bool pipe_consume(const Plan& P, Sink<MODE, ACC128, NT>& sink, uint8_t* extra,
                                             uint64_t* full, uint64_t* empty, uint8_t* stages, uint64_t first,
                                             uint64_t stride, uint64_t count, PipeState& st, uint32_t* abort_flag,
                                             const RegLeaves& RL, const RegVals& RV, unsigned long long& selected) {
    const uint32_t t = threadIdx.x, lane = t & 31u;
    const uint64_t ntiles = (P.nrows + kTileRows - 1) / kTileRows;
    const uint64_t nfull = P.nrows / kTileRows;
    const uint32_t S = P.nstages;
    // Waits (bounded) until stage s of phase ph has landed; false after a
    // timeout or an abort (which it records).
    auto land = [&](uint32_t s, uint32_t ph) -> bool {
        bool landed = false;
        if (lane == 0) landed = mbar_wait_bounded(&full[s], ph, P.wait_ns);
        landed = __shfl_sync(kFull, landed ? 1 : 0, 0) != 0;
        if (!landed || *reinterpret_cast<volatile uint32_t*>(abort_flag)) {
            if (lane == 0) {
                atomicOr(P.err, kErrWaitTimeout);
                atomicExch(abort_flag, 1u);
            }
            return false;
        }
        // Lanes other than 0 observe the completed phase through a cheap
        // try_wait so their shared-memory reads are ordered after the copy.
        mbar_try_wait(&full[s], ph);
        return true;
    };
    for (uint64_t k = 0; k < count; ++k) {
        const uint64_t tl = first + k * stride;
        if (tl >= ntiles) break;
        if (tl < nfull) {
            if (!land(st.s, st.phase)) return false;
            process_tile<MODE, ACC128, NT, false, SH>(P, sink, extra, stages + static_cast<size_t>(st.s) * P.stage_bytes,
                                                      tl, t, selected, RL, RV);
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[st.s]);
            ++st.n;
            if (++st.s == S) {
                st.s = 0;
                st.phase ^= 1u;
            }
        } else {
            process_tile<MODE, ACC128, NT, true, SH>(P, sink, extra, nullptr, tl, t, selected, RL, RV);
        }
    }
    return true;
}

__device__ __forceinline__ void pipe_init_barriers(uint64_t* full, uint64_t* empty, uint32_t S, uint32_t consumer_warps) {
    for (uint32_t s = 0; s < S; ++s) {
        mbar_init(&full[s], 1);
        mbar_init(&empty[s], consumer_warps);
    }
    fence_barrier_init();
}

// Register-held predicate leaves and fast-path value descriptors of a plan.
template <uint32_t MODE, bool ACC128, class SH, bool MIXED = false>
__device__ __forceinline__ void load_regs(const Plan& P, RegLeaves& RL, RegVals& RV) {
    load_reg_leaves(P, RL);
    // A fixed-shape kernel of one query never takes the scalar fast path; a
    // batch kernel (MIXED) serves both kinds of plan.
    if constexpr (std::is_void<SH>::value || MIXED || std::is_same<SH, ScalarTag>::value)
        load_reg_vals<MODE, ACC128>(P, RV);
    else RV.on = 0;
}

template <int NT>
__device__ __forceinline__ void count_selected(const Plan& P, unsigned long long selected) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) selected += __shfl_down_sync(kFull, selected, d);
    if ((threadIdx.x & 31u) == 0 && selected) atomicAdd(P.counters, selected);
}

// One query: CTA b walks tiles b, b + gridDim.x, ...
// MINB: CTAs per SM the register budget is set for (2 for the join-payload
// limb-table shapes, which run two CTAs of two stages each).
template <uint32_t MODE, bool ACC128, int NT, class SH = void, int MINB = 1>
__global__ void __launch_bounds__(NT + 32, MINB) scan_kernel(const __grid_constant__ Plan P) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + kMaxStages;
    uint8_t* stages = smem + kBarrierBytes;
    uint8_t* extra = smem + P.extra_off;
    __shared__ uint32_t abort_flag;

    const uint32_t t = threadIdx.x;
    const uint64_t ntiles = (P.nrows + kTileRows - 1) / kTileRows;
    const uint64_t G = gridDim.x;
    const uint64_t count = ntiles > blockIdx.x ? (ntiles - blockIdx.x + G - 1) / G : 0;

    Sink<MODE, ACC128, NT> sink;
    if (t < static_cast<uint32_t>(NT)) sink.init(P, extra, t);
    if (t == static_cast<uint32_t>(NT)) {
        pipe_init_barriers(full, empty, P.nstages, NT / 32);
        abort_flag = 0;
    }
    __syncthreads();
    PipeState st;
    if (t >= static_cast<uint32_t>(NT)) {
        if (t != static_cast<uint32_t>(NT)) return;
        pipe_produce(P, full, empty, stages, blockIdx.x, G, count, st, &abort_flag);
        // Drain: the last min(S, n) copies have landed before this thread
        // exits (earlier ones were waited for through empty[]).
        const uint32_t S = P.nstages;
        const uint64_t first = st.n > S ? st.n - S : 0;
        for (uint64_t i = first; i < st.n; ++i)
            if (!mbar_wait_bounded(&full[i % S], static_cast<uint32_t>((i / S) & 1u), P.wait_ns))
                atomicOr(P.err, kErrWaitTimeout);
        return;
    }
    RegLeaves RL;
    RegVals RV;
    load_regs<MODE, ACC128, SH>(P, RL, RV);
    unsigned long long selected = 0;
    pipe_consume<MODE, ACC128, NT, SH>(P, sink, extra, full, empty, stages, blockIdx.x, G, count, st, &abort_flag, RL,
                                       RV, selected);
    count_selected<NT>(P, selected);
    // Every consumer reaches the flush, also after a timeout (the host then
    // discards the result), so the consumer barrier inside it always completes.
    sink.flush(P, extra, t);
}

// ---------------------------------------------------------------------------
// Many queries in one persistent launch. The host splits the work into
// morsels: a group of plans over the same table that share one stage layout
// (the union of their columns; each plan has its own accumulator region) and
// a range of tiles. CTAs take morsels from a device counter until none is
// left. Per morsel the CTA re-initializes its stage barriers for the group's
// layout, streams each tile once and runs every plan of the group on it (a
// shared scan), then merges each plan's partial aggregates into that query's
// accumulators. Plans are read from global memory (L1-resident, uniform).
// ---------------------------------------------------------------------------
// A shared scan whose plans are all scalar fast-path plans over the same
// register leaf columns and the same values (the same statement with other
// literals): the tile's leaf cells are loaded once into registers, then each
// plan only reads its own bounds and tests them. Selected rows (rare for a
// selective scan) go through the plan's register value path.
template <int NT>
__device__ __forceinline__ void fast_group_tile(const Plan* plans, uint32_t np, Sink<MODE_GROUP_PRIVATE, false, NT>* sinks,
                                                uint8_t* smem, const uint8_t* stage, uint32_t t,
                                                unsigned long long* selected) {
    constexpr int R = kTileRows / NT;
    const Plan& P0 = plans[0];
    const uint32_t nl = P0.rb.leaf_n;
    uint32_t x[kRegLeaves][R];
#pragma unroll
    for (int i = 0; i < kRegLeaves; ++i) {
        if (static_cast<uint32_t>(i) >= nl) break;
        for_chunks<R / 4>(stage + P0.rb.leaf_soff[i], t, [&](uint32_t q, const uint4& v) {
            x[i][4 * q + 0] = v.x;
            x[i][4 * q + 1] = v.y;
            x[i][4 * q + 2] = v.z;
            x[i][4 * q + 3] = v.w;
        });
    }
    RegVals RV;
    load_reg_vals<MODE_GROUP_PRIVATE, false>(P0, RV);
#pragma unroll 1
    for (uint32_t q = 0; q < np; ++q) {
        const Plan& P = plans[q];
        const uint32_t neg = P.rb.leaf_neg;
        uint32_t m = (R == 32) ? 0xffffffffu : ((1u << R) - 1u);
#pragma unroll
        for (int i = 0; i < kRegLeaves; ++i) {
            if (static_cast<uint32_t>(i) >= nl) break;
            const uint32_t lo = P.rb.leaf_lo[i], sp = P.rb.leaf_sp[i];
            uint32_t b = 0;
#pragma unroll
            for (int r = 0; r < R; ++r) b |= in32(x[i][r], lo, sp) << r;
            m &= ((neg >> i) & 1u) ? ~b : b;
        }
        uint8_t* extra = smem + P.extra_off;
        const uint32_t c = __popc(m);
        selected[q] += c;
        priv_counts(extra)[t] += c;   // a scalar aggregate counts rows by popcount
        for (uint32_t sel = m; sel; sel &= sel - 1)
            fast_row<NT>(P, RV, extra, stage, R * t + __ffs(sel) - 1, t, sinks[q].upd, sinks[q]);
    }
}

template <uint32_t MODE, bool ACC128, int NT, class SH>
__device__ __forceinline__ void consume_group(const Plan* plans, uint32_t np, Sink<MODE, ACC128, NT>* sinks,
                                              uint8_t* smem, uint64_t* full, uint64_t* empty, uint8_t* stages,
                                              uint64_t first, uint64_t count, PipeState& st, uint32_t* abort_flag,
                                              unsigned long long* selected) {
    const Plan& P0 = plans[0];
    const uint32_t t = threadIdx.x, lane = t & 31u;
    const uint64_t ntiles = (P0.nrows + kTileRows - 1) / kTileRows;
    const uint64_t nfull = P0.nrows / kTileRows;
    const uint32_t S = P0.nstages;
    for (uint64_t k = 0; k < count; ++k) {
        const uint64_t tl = first + k;
        if (tl >= ntiles) break;
        const bool staged = tl < nfull;
        uint8_t* stage = nullptr;
        if (staged) {
            bool landed = false;
            if (lane == 0) landed = mbar_wait_bounded(&full[st.s], st.phase, P0.wait_ns);
            landed = __shfl_sync(kFull, landed ? 1 : 0, 0) != 0;
            if (!landed || *reinterpret_cast<volatile uint32_t*>(abort_flag)) {
                if (lane == 0) {
                    atomicOr(P0.err, kErrWaitTimeout);
                    atomicExch(abort_flag, 1u);
                }
                return;
            }
            mbar_try_wait(&full[st.s], st.phase);
            stage = stages + static_cast<size_t>(st.s) * P0.stage_bytes;
        }
        if constexpr (MODE == MODE_GROUP_PRIVATE && !ACC128) {
            if (staged && P0.group_fast) {
                fast_group_tile<NT>(plans, np, sinks, smem, stage, t, selected);
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[st.s]);
                ++st.n;
                if (++st.s == S) {
                    st.s = 0;
                    st.phase ^= 1u;
                }
                continue;
            }
        }
#pragma unroll 1
        for (uint32_t q = 0; q < np; ++q) {
            const Plan& P = plans[q];
            RegLeaves RL;
            RegVals RV;
            load_regs<MODE, ACC128, SH, true>(P, RL, RV);
            if (staged)
                process_tile<MODE, ACC128, NT, false, SH>(P, sinks[q], smem + P.extra_off, stage, tl, t, selected[q],
                                                          RL, RV);
            else
                process_tile<MODE, ACC128, NT, true, SH>(P, sinks[q], smem + P.extra_off, nullptr, tl, t,
                                                         selected[q], RL, RV);
        }
        if (staged) {
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[st.s]);
            ++st.n;
            if (++st.s == S) {
                st.s = 0;
                st.phase ^= 1u;
            }
        }
    }
}

template <uint32_t MODE, bool ACC128, int NT, class SH>
__global__ void __launch_bounds__(NT + 32, 1) batch_kernel(const __grid_constant__ BatchDesc B) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + kMaxStages;
    __shared__ uint32_t abort_flag, s_morsel;
    const uint32_t t = threadIdx.x;
    if (t == 0) abort_flag = 0;
    for (;;) {
        if (t == 0) s_morsel = atomicAdd(B.next, 1u);
        __syncthreads();
        const uint32_t mi = s_morsel;
        if (mi >= B.nmorsels || *reinterpret_cast<volatile uint32_t*>(&abort_flag)) break;
        const Morsel M = B.morsels[mi];
        const uint32_t np = M.count;
        // The group's plans go to shared memory (after the barriers, before
        // the stage ring at plans[0].stage_off).
        {
            const uint4* src = reinterpret_cast<const uint4*>(B.plans + M.first);
            uint4* dst = reinterpret_cast<uint4*>(smem + kBarrierBytes);
            const uint32_t words = np * static_cast<uint32_t>(sizeof(Plan) / 16);
            for (uint32_t i = t; i < words; i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
        const Plan* plans = reinterpret_cast<const Plan*>(smem + kBarrierBytes);
        const Plan& P0 = plans[0];
        uint8_t* stages = smem + P0.stage_off;
        Sink<MODE, ACC128, NT> sinks[kMaxShare];
        if (t < static_cast<uint32_t>(NT))
            for (uint32_t q = 0; q < np; ++q) sinks[q].init(plans[q], smem + plans[q].extra_off, t);
        if (t == static_cast<uint32_t>(NT)) pipe_init_barriers(full, empty, P0.nstages, NT / 32);
        __syncthreads();
        PipeState st;
        const uint64_t count = M.tile_end - M.tile_begin;
        if (t == static_cast<uint32_t>(NT)) {
            pipe_produce(P0, full, empty, stages, M.tile_begin, 1, count, st, &abort_flag);
            // Drain (a no-op unless the consumers gave up): no copy may still
            // be in flight when the barriers are invalidated.
            const uint32_t S = P0.nstages;
            for (uint64_t i = st.n > S ? st.n - S : 0; i < st.n; ++i)
                if (!mbar_wait_bounded(&full[i % S], static_cast<uint32_t>((i / S) & 1u), P0.wait_ns))
                    atomicOr(P0.err, kErrWaitTimeout);
        } else if (t < static_cast<uint32_t>(NT)) {
            unsigned long long selected[kMaxShare];
            for (uint32_t q = 0; q < np; ++q) selected[q] = 0;
            consume_group<MODE, ACC128, NT, SH>(plans, np, sinks, smem, full, empty, stages, M.tile_begin, count, st,
                                                &abort_flag, selected);
            for (uint32_t q = 0; q < np; ++q) {
                count_selected<NT>(plans[q], selected[q]);
                sinks[q].flush(plans[q], smem + plans[q].extra_off, t);
            }
        }
        // Every stage copy of this morsel was consumed: the barriers can be
        // re-initialized for the next morsel's layout.
        __syncthreads();
        if (t == static_cast<uint32_t>(NT))
            for (uint32_t s = 0; s < P0.nstages; ++s) {
                mbar_inval(&full[s]);
                mbar_inval(&empty[s]);
            }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
template <uint32_t MODE, bool ACC128, int NT>
static const void* kernel_ptr() {
    return reinterpret_cast<const void*>(scan_kernel<MODE, ACC128, NT>);
}

template <int NT>
static const void* select_kernel(uint32_t mode, bool acc128) {
    switch (mode) {
        case MODE_FILTER: return kernel_ptr<MODE_FILTER, false, NT>();
        case MODE_SCALAR:
        case MODE_GROUP_PRIVATE:
            return acc128 ? kernel_ptr<MODE_GROUP_PRIVATE, true, NT>() : kernel_ptr<MODE_GROUP_PRIVATE, false, NT>();
        case MODE_GROUP_SHARED: return kernel_ptr<MODE_GROUP_SHARED, false, NT>();
        case MODE_GROUP_SHARED32: return kernel_ptr<MODE_GROUP_SHARED32, false, NT>();
        case MODE_GROUP_GLOBAL: return kernel_ptr<MODE_GROUP_GLOBAL, false, NT>();
        case MODE_GROUP_HASH: return kernel_ptr<MODE_GROUP_HASH, false, NT>();
        case MODE_JOIN_BUILD: return kernel_ptr<MODE_JOIN_BUILD, false, NT>();
        case MODE_JOIN_PAIRS: return kernel_ptr<MODE_JOIN_PAIRS, false, NT>();
        default: return nullptr;
    }
}

// Dense value-program shapes compiled ahead of time (index = Plan::shape).
// The TPC-H Q1 shape: GROUP BY two u8 flags; sum(i32), sum(i64),
// sum(i64 * (k - i32)), sum(i64 * (k - i32) * (k + i32)).
constexpr uint32_t kNarrowPos = CS_COL | CS_NARROW | CS_NONNEG;
using ShapeQ1 = DenseShape<2, DT_U8, DT_U8, step_code(DT_I32, kNarrowPos, VK_SUM, 1),
                           step_code(DT_I64, CS_COL | CS_IDENT, VK_SUM, 2),
                           step_code(DT_I32, kNarrowPos | CS_CHAIN, VK_SUM, 3),
                           step_code(DT_I32, kNarrowPos | CS_CHAIN, VK_SUM, 4)>;

// The join + grouped aggregate shape: groups from the join payload, no staged
// key; sum(i64 * (k - i32)).
using ShapeJoin = DenseShape<0, 0, 0, step_code(DT_I64, CS_COL | CS_IDENT, VK_SUM, 0),
                             step_code(DT_I32, kNarrowPos | CS_CHAIN, VK_SUM, 1)>;

struct ShapeEntry {
    uint32_t nkey, kdt0, kdt1, nsteps;
    uint32_t code[kMaxSteps];
    const void* k256;
    const void* k512;
    const void* s32_256;   // the same value program on the limb tables (keys at run time)
    const void* s32_512;
    const void* s32_512_pair;  // registers for two CTAs per SM (Plan::two_ctas)
};

template <class SH>
static ShapeEntry shape_entry() {
    ShapeEntry e{};
    e.nkey = SH::nkey;
    e.kdt0 = SH::nkey >= 1 ? SH::kdt0 : 0u;
    e.kdt1 = SH::nkey >= 2 ? SH::kdt1 : 0u;
    e.nsteps = SH::nsteps;
    for (uint32_t i = 0; i < SH::nsteps; ++i) e.code[i] = SH::step[i];
    e.k256 = reinterpret_cast<const void*>(scan_kernel<MODE_GROUP_PRIVATE, false, 256, SH>);
    e.k512 = reinterpret_cast<const void*>(scan_kernel<MODE_GROUP_PRIVATE, false, 512, SH>);
    e.s32_256 = reinterpret_cast<const void*>(scan_kernel<MODE_GROUP_SHARED32, false, 256, SH>);
    e.s32_512 = reinterpret_cast<const void*>(scan_kernel<MODE_GROUP_SHARED32, false, 512, SH>);
    e.s32_512_pair = reinterpret_cast<const void*>(scan_kernel<MODE_GROUP_SHARED32, false, 512, SH, 2>);
    return e;
}

static const ShapeEntry* shape_table(uint32_t* n) {
    static const ShapeEntry table[] = {shape_entry<ShapeQ1>(), shape_entry<ShapeJoin>()};
    *n = sizeof(table) / sizeof(table[0]);
    return table;
}

void fill_reg_block(Plan& P) {
    RegBlock& B = P.rb;
    B = RegBlock{};
    B.leaf_n = (P.all_and && P.nleaf <= kRegLeaves && P.kend[0] == P.nleaf) ? P.nleaf : 0u;
    for (uint32_t i = 0; i < B.leaf_n; ++i) {
        B.leaf_soff[i] = P.slot[P.leaf[i].slot].smem_off;
        B.leaf_lo[i] = P.leaf[i].lo32;
        B.leaf_sp[i] = P.leaf[i].span32;
        if (P.leaf[i].negate) B.leaf_neg |= 1u << i;
    }
    bool on = P.count_by_tile && !P.check_ovf && P.jslot < 0 && P.ngkey == 0 && P.nval >= 1 && P.nval <= 2;
    B.vals_nv = P.nval;
    for (int v = 0; v < 2; ++v) {
        const bool use = static_cast<uint32_t>(v) < P.nval;
        const ValDesc& D = P.val[use ? v : 0];
        if (use && (D.kind != VK_SUM || D.nf < 1 || D.nf > 2)) on = false;
        B.vals_nf[v] = use ? D.nf : 0u;
        for (int f = 0; f < 2; ++f) {
            const bool uf = use && static_cast<uint32_t>(f) < D.nf;
            const Factor& F = D.f[uf ? f : 0];
            if (uf && F.slot < 0) on = false;
            B.vals_soff[v][f] = uf ? F.soff : 0u;
            B.vals_dt[v][f] = uf ? F.dtype : static_cast<uint32_t>(DT_I64);
            B.vals_mul[v][f] = uf ? F.mul : 0;
            B.vals_add[v][f] = uf ? F.add : 1;  // an absent factor multiplies by 1
        }
    }
    B.vals_on = on ? 1u : 0u;
}

uint32_t scalar_shape_of(const Plan& P) {
    if (!(P.count_by_tile && !P.check_ovf && P.jslot < 0 && P.ngkey == 0 && P.nval >= 1 && P.nval <= 2)) return 0;
    for (uint32_t v = 0; v < P.nval; ++v) {
        const ValDesc& D = P.val[v];
        if (D.kind != VK_SUM || D.nf < 1 || D.nf > 2) return 0;
        for (uint32_t f = 0; f < D.nf; ++f)
            if (D.f[f].slot < 0) return 0;
    }
    return kShapeScalar;
}

uint32_t value_shape_of(const Plan& P) {
    if (!P.dense_vec || P.chain.nsteps == 0) return 0;
    uint32_t n = 0;
    const ShapeEntry* tab = shape_table(&n);
    for (uint32_t j = 0; j < n; ++j) {
        const ShapeEntry& e = tab[j];
        if (e.nsteps != P.chain.nsteps) continue;
        bool same = true;
        for (uint32_t i = 0; i < e.nsteps; ++i) {
            const ChainStep& S = P.chain.s[i];
            same = same && e.code[i] == step_code((S.flags & CS_COL) ? S.dtype : 0u, S.flags, S.kind, S.acc);
        }
        if (same) return j + 1;
    }
    return 0;
}

uint32_t dense_shape_of(const Plan& P) {
    if (!P.dense_vec || P.chain.nsteps == 0) return 0;
    uint32_t code[kMaxSteps] = {};
    for (uint32_t i = 0; i < P.chain.nsteps; ++i) {
        const ChainStep& S = P.chain.s[i];
        code[i] = step_code((S.flags & CS_COL) ? S.dtype : 0u, S.flags, S.kind, S.acc);
    }
    uint32_t n = 0;
    const ShapeEntry* tab = shape_table(&n);
    for (uint32_t j = 0; j < n; ++j) {
        const ShapeEntry& e = tab[j];
        // Build-side keys come from the join payload; a shape's keys are the
        // staged ones, and the two kinds do not mix.
        uint32_t staged = 0, build = 0;
        for (uint32_t k = 0; k < P.ngkey; ++k) (P.gkey[k].build_side ? build : staged) += 1;
        if (build && staged) continue;
        if (e.nkey != staged || e.nsteps != P.chain.nsteps) continue;
        if (e.nkey >= 1 && e.kdt0 != P.gkey[0].dtype) continue;
        if (e.nkey >= 2 && e.kdt1 != P.gkey[1].dtype) continue;
        bool same = true;
        for (uint32_t i = 0; i < e.nsteps; ++i) same = same && e.code[i] == code[i];
        if (same) return j + 1;
    }
    return 0;
}

static const void* select_kernel(uint32_t mode, bool acc128, int nt, uint32_t shape = 0, bool pair = false) {
    if (shape == kShapeScalar && mode == MODE_GROUP_PRIVATE && !acc128) {
        return nt == 512 ? reinterpret_cast<const void*>(scan_kernel<MODE_GROUP_PRIVATE, false, 512, ScalarTag>)
             : nt == 256 ? reinterpret_cast<const void*>(scan_kernel<MODE_GROUP_PRIVATE, false, 256, ScalarTag>)
                         : nullptr;
    }
    if (shape && mode == MODE_GROUP_PRIVATE && !acc128) {
        uint32_t n = 0;
        const ShapeEntry* tab = shape_table(&n);
        if (shape <= n) return nt == 512 ? tab[shape - 1].k512 : nt == 256 ? tab[shape - 1].k256 : nullptr;
        return nullptr;
    }
    if (shape && mode == MODE_GROUP_SHARED32) {
        uint32_t n = 0;
        const ShapeEntry* tab = shape_table(&n);
        if (shape <= n)
            return nt == 512 ? (pair ? tab[shape - 1].s32_512_pair : tab[shape - 1].s32_512)
                 : nt == 256 ? tab[shape - 1].s32_256 : nullptr;
        return nullptr;
    }
    return nt == 512 ? select_kernel<512>(mode, acc128) : nt == 256 ? select_kernel<256>(mode, acc128) : nullptr;
}

// Launches with blockDim = nthreads consumers + one producer warp.
// Per (device, kernel): the dynamic shared-memory limit already raised, and
// occupancies already queried, so a launch costs one cudaLaunchKernel.
struct KernelCacheEntry {
    int device;
    const void* f;
    int smem_limit;
    size_t occ_smem[4];
    int occ[4];
    int nocc;
};

static std::mutex g_kcache_mu;
static KernelCacheEntry g_kcache[128];
static int g_kcache_n = 0;

static KernelCacheEntry* kernel_entry(const void* f) {
    int dev = 0;
    cudaGetDevice(&dev);
    for (int i = 0; i < g_kcache_n; ++i)
        if (g_kcache[i].f == f && g_kcache[i].device == dev) return &g_kcache[i];
    if (g_kcache_n == static_cast<int>(sizeof(g_kcache) / sizeof(g_kcache[0]))) return nullptr;
    KernelCacheEntry& e = g_kcache[g_kcache_n++];
    e.device = dev;
    e.f = f;
    e.smem_limit = 0;
    e.nocc = 0;
    return &e;
}

static cudaError_t ensure_smem_limit(KernelCacheEntry* e, const void* f, int smem) {
    if (e && e->smem_limit >= smem) return cudaSuccess;
    const cudaError_t r = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (r == cudaSuccess && e) e->smem_limit = smem;
    return r;
}

// Launches with blockDim = nthreads consumers + one producer warp.
cudaError_t launch_scan(const Plan& P, uint32_t mode, bool acc128, int grid, cudaStream_t st) {
    const void* f = select_kernel(mode, acc128, static_cast<int>(P.nthreads), P.shape, P.two_ctas != 0);
    if (!f) return cudaErrorInvalidValue;
    {
        std::lock_guard<std::mutex> lock(g_kcache_mu);
        const cudaError_t e = ensure_smem_limit(kernel_entry(f), f, static_cast<int>(P.smem_bytes));
        if (e != cudaSuccess) return e;
    }
    // The register images are derived here, once the plan is final.
    Plan L = P;
    fill_reg_block(L);
    void* args[] = {&L};
    return cudaLaunchKernel(f, dim3(grid), dim3(L.nthreads + 32), args, L.smem_bytes, st);
}

int scan_occupancy(uint32_t mode, bool acc128, int nt, size_t dyn_smem, uint32_t shape, bool pair) {
    const void* f = select_kernel(mode, acc128, nt, shape, pair);
    if (!f) return 0;
    std::lock_guard<std::mutex> lock(g_kcache_mu);
    KernelCacheEntry* e = kernel_entry(f);
    if (e)
        for (int i = 0; i < e->nocc; ++i)
            if (e->occ_smem[i] == dyn_smem) return e->occ[i];
    if (ensure_smem_limit(e, f, static_cast<int>(dyn_smem)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, nt + 32, dyn_smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (e) {
        const int slot = e->nocc < 4 ? e->nocc++ : 0;
        e->occ_smem[slot] = dyn_smem;
        e->occ[slot] = n;
    }
    return n;
}

// Static shared memory used by scan_kernel besides the dynamic stages.
size_t scan_kernel_static_smem() { return 128; }

// Batch launches (MODE_GROUP_PRIVATE plans): one persistent kernel per
// (acc128, NT) class.
size_t batch_kernel_static_smem() { return 16; }

// The int64 kernels carry the fixed-shape dense path (plans with shape 1);
// every other plan runs the interpreted paths.
static const void* batch_kernel_ptr(bool acc128, int nt) {
    if (nt == 512)
        return acc128 ? reinterpret_cast<const void*>(batch_kernel<MODE_GROUP_PRIVATE, true, 512, void>)
                      : reinterpret_cast<const void*>(batch_kernel<MODE_GROUP_PRIVATE, false, 512, ShapeQ1>);
    if (nt == 256)
        return acc128 ? reinterpret_cast<const void*>(batch_kernel<MODE_GROUP_PRIVATE, true, 256, void>)
                      : reinterpret_cast<const void*>(batch_kernel<MODE_GROUP_PRIVATE, false, 256, ShapeQ1>);
    return nullptr;
}

int batch_occupancy(bool acc128, int nt, size_t dyn_smem) {
    const void* f = batch_kernel_ptr(acc128, nt);
    if (!f) return 0;
    std::lock_guard<std::mutex> lock(g_kcache_mu);
    KernelCacheEntry* e = kernel_entry(f);
    if (ensure_smem_limit(e, f, static_cast<int>(dyn_smem)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, nt + 32, dyn_smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

cudaError_t launch_batch(const BatchDesc& B, bool acc128, int nt, int grid, size_t dyn_smem, cudaStream_t st) {
    const void* f = batch_kernel_ptr(acc128, nt);
    if (!f) return cudaErrorInvalidValue;
    {
        std::lock_guard<std::mutex> lock(g_kcache_mu);
        const cudaError_t e = ensure_smem_limit(kernel_entry(f), f, static_cast<int>(dyn_smem));
        if (e != cudaSuccess) return e;
    }
    void* args[] = {const_cast<BatchDesc*>(&B)};
    return cudaLaunchKernel(f, dim3(grid), dim3(nt + 32), args, dyn_smem, st);
}

}  // namespace tgp
