// scan_engine.cu — the persistent, TMA-staged scan kernel behind every
// filter / aggregate / join entry point of the C ABI.
//
// One CTA per SM slot walks tiles of kTileRows rows (tile = blockIdx.x +
// k * gridDim.x). Thread 0 streams the referenced columns of upcoming tiles
// into a ring of shared-memory stages with 1-D bulk copies
// (cp.async.bulk ... mbarrier::complete_tx); every thread evaluates the
// lowered WHERE program on its 8 rows of the current stage into an 8-bit
// mask, then feeds the selected rows to the mode's sink (bitmap words, scalar
// int128 registers, per-thread or per-CTA group accumulators, global hash
// groups, join build / probe). The final partial tile is read straight from
// global memory with bounds checks.
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

__device__ __forceinline__ uint32_t valid_bits(uint32_t tid, uint32_t nrem) {
    uint32_t v = 0;
#pragma unroll
    for (int j = 0; j < kRowsPerThread; ++j) v |= (j * kThreads + tid < nrem ? 1u : 0u) << j;
    return v;
}

// ---------------------------------------------------------------------------
// Predicate evaluation: 8 rows (j * kThreads + tid) per call → 8-bit mask.
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

template <bool TAIL>
__device__ __forceinline__ uint32_t eval_leaf(const Leaf& L, const uint8_t* base, uint32_t tid,
                                              uint32_t nrem) {
    uint32_t m = 0;
    switch (L.kind) {
        case LK_U8: {
            const uint32_t x = L.xor32, lo = L.lo32, sp = L.span32;
#pragma unroll
            for (int j = 0; j < kRowsPerThread; ++j) {
                const uint32_t r = j * kThreads + tid;
                if (!TAIL || r < nrem) {
                    const uint32_t k = static_cast<uint32_t>(base[r]) ^ x;
                    m |= ((k - lo) <= sp ? 1u : 0u) << j;
                }
            }
            break;
        }
        case LK_I32: {
            const uint32_t* c = reinterpret_cast<const uint32_t*>(base);
            const uint32_t x = L.xor32, lo = L.lo32, sp = L.span32;
#pragma unroll
            for (int j = 0; j < kRowsPerThread; ++j) {
                const uint32_t r = j * kThreads + tid;
                if (!TAIL || r < nrem) {
                    const uint32_t k = c[r] ^ x;
                    m |= ((k - lo) <= sp ? 1u : 0u) << j;
                }
            }
            break;
        }
        case LK_64: {
            const uint64_t* c = reinterpret_cast<const uint64_t*>(base);
            const uint64_t x = L.xor64, lo = L.lo64, sp = L.span64;
#pragma unroll
            for (int j = 0; j < kRowsPerThread; ++j) {
                const uint32_t r = j * kThreads + tid;
                if (!TAIL || r < nrem) {
                    const uint64_t k = c[r] ^ x;
                    m |= ((k - lo) <= sp ? 1u : 0u) << j;
                }
            }
            break;
        }
        case LK_F64: {
            const double* c = reinterpret_cast<const double*>(base);
#pragma unroll
            for (int j = 0; j < kRowsPerThread; ++j) {
                const uint32_t r = j * kThreads + tid;
                if (!TAIL || r < nrem) m |= (f64_leaf(L.fop, c[r], L.f1, L.f2) ? 1u : 0u) << j;
            }
            break;
        }
        default:
            return L.negate ? 0xFFu : 0u;  // LK_CONST
    }
    return L.negate ? (m ^ 0xFFu) : m;
}

template <bool TAIL>
__device__ __forceinline__ uint32_t eval_pred(const Plan& P, const uint8_t* stage, uint64_t r0,
                                              uint32_t tid, uint32_t nrem) {
    const uint32_t valid = TAIL ? valid_bits(tid, nrem) : 0xFFu;
    if (P.nleaf == 0) return valid;
    if (P.all_and) {
        uint32_t m = valid;
        for (uint32_t i = 0; i < P.nleaf; ++i) {
            const Leaf& L = P.leaf[i];
            m &= eval_leaf<TAIL>(L, slot_base<TAIL>(P, stage, L.slot, r0), tid, nrem);
        }
        return m;
    }
    // General postfix program on an 8-deep register stack (depth checked on host).
    uint32_t s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0, s6 = 0, s7 = 0;
    for (uint32_t i = 0; i < P.nops; ++i) {
        const uint8_t op = P.ops[i];
        if (op < kMaxLeaves) {
            const Leaf& L = P.leaf[op];
            const uint32_t v = eval_leaf<TAIL>(L, slot_base<TAIL>(P, stage, L.slot, r0), tid, nrem);
            s7 = s6; s6 = s5; s5 = s4; s4 = s3; s3 = s2; s2 = s1; s1 = s0; s0 = v;
        } else if (op == OP_NOT) {
            s0 = s0 ^ 0xFFu;
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
// read the build side of a join.
// ---------------------------------------------------------------------------
template <bool TAIL>
__device__ __forceinline__ int64_t eval_val(const Plan& P, const ValDesc& V, const uint8_t* stage,
                                            uint64_t r0, uint32_t rl, uint32_t brow,
                                            uint32_t& ovf) {
    int64_t acc = 1;
#pragma unroll
    for (int f = 0; f < kMaxFactors; ++f) {
        if (f < V.nf) {
            const Factor& F = V.f[f];
            int64_t x = 0;
            if (F.slot >= 0) {
                x = load_cell(slot_base<TAIL>(P, stage, F.slot, r0), P.slot[F.slot].dtype, rl);
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
                acc = (f == 0) ? t
                               : static_cast<int64_t>(static_cast<uint64_t>(acc) *
                                                      static_cast<uint64_t>(t));
            }
        }
    }
    return acc;
}

template <bool TAIL>
__device__ __forceinline__ int64_t key_cell(const Plan& P, const GKey& K, const uint8_t* stage,
                                            uint64_t r0, uint32_t rl, uint32_t brow) {
    if (K.build_side) return load_cell_ro(K.bptr, K.dtype, brow);
    return load_cell(slot_base<TAIL>(P, stage, K.slot, r0), P.slot[K.slot].dtype, rl);
}

// Direct group index: sum over keys of (cell - min) * stride.
template <bool TAIL>
__device__ __forceinline__ uint32_t group_index(const Plan& P, const uint8_t* stage, uint64_t r0,
                                                uint32_t rl, uint32_t brow) {
    uint64_t g = 0;
    for (uint32_t k = 0; k < P.ngkey; ++k) {
        const GKey& K = P.gkey[k];
        const int64_t c = key_cell<TAIL>(P, K, stage, r0, rl, brow);
        g += (static_cast<uint64_t>(c) - static_cast<uint64_t>(K.min)) * K.stride;
    }
    return static_cast<uint32_t>(g);
}

// Packed exact key for MODE_GROUP_HASH.
template <bool TAIL>
__device__ __forceinline__ uint64_t group_hash_key(const Plan& P, const uint8_t* stage,
                                                   uint64_t r0, uint32_t rl, uint32_t brow) {
    uint64_t key = 0;
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
__device__ __forceinline__ void acc_init(I128& a, uint8_t kind) {
    a.lo = (kind == VK_MIN) ? 0x7fffffffffffffffull : (kind == VK_MAX ? 0x8000000000000000ull : 0ull);
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

// Global accumulator pair at word index `w` (lo at w, hi at w + 1).
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

// ---------------------------------------------------------------------------
// Shared-memory layout of per-mode scratch
// ---------------------------------------------------------------------------
// MODE_GROUP_PRIVATE, int64 partials: word ((g * nv1 + v) * kThreads + tid)
// MODE_GROUP_PRIVATE, int128 partials: words ((g * nv1 + v) * 2 + limb) * kThreads + tid
// MODE_GROUP_SHARED: words (g * nv1 + v) * 2 + limb (int128 via carry atomics)
// (nv1 = 1 + nval; value slot 0 is the group's row count.)

template <uint32_t MODE, bool ACC128>
struct Sink {
    // Scalar-mode registers.
    I128 acc[kMaxVals];
    unsigned long long count;
    uint32_t ovf;
    uint64_t upd;   // MODE_GROUP_PRIVATE int64: updates since the last flush

    // Moves this thread's int64 private partials into the global int128
    // accumulators and resets them.
    __device__ __forceinline__ void flush_private_thread(const Plan& P, uint8_t* extra, uint32_t tid) {
        const uint32_t nv1 = P.nval + 1;
        long long* w = reinterpret_cast<long long*>(extra);
        for (uint32_t i = 0; i < P.ngroups * nv1; ++i) {
            const uint32_t v = i % nv1;
            const uint8_t kind = v == 0 ? VK_SUM : P.val[v - 1].kind;
            if (kind == VK_MIN || kind == VK_MAX) continue;
            long long& a = w[i * kThreads + tid];
            if (a != 0) {
                I128 x;
                x.lo = static_cast<uint64_t>(a);
                x.hi = a >> 63;
                atomic_add_i128(P.acc + 2ull * i, x);
                a = 0;
            }
        }
    }

    __device__ __forceinline__ void init(const Plan& P, uint8_t* extra, uint32_t tid) {
        count = 0;
        ovf = 0;
        upd = 0;
#pragma unroll
        for (int v = 0; v < kMaxVals; ++v) acc_init(acc[v], v < (int)P.nval ? P.val[v].kind : VK_SUM);
        if (MODE == MODE_GROUP_PRIVATE) {
            const uint32_t nv1 = P.nval + 1;
            long long* w = reinterpret_cast<long long*>(extra);
            for (uint32_t g = 0; g < P.ngroups; ++g) {
                for (uint32_t v = 0; v < nv1; ++v) {
                    const uint8_t kind = v == 0 ? VK_SUM : P.val[v - 1].kind;
                    const long long init = kind == VK_MIN ? 0x7fffffffffffffffll
                                           : kind == VK_MAX ? static_cast<long long>(0x8000000000000000ull) : 0ll;
                    if (ACC128) {
                        w[((g * nv1 + v) * 2 + 0) * kThreads + tid] = init;
                        w[((g * nv1 + v) * 2 + 1) * kThreads + tid] = 0;
                    } else {
                        w[(g * nv1 + v) * kThreads + tid] = init;
                    }
                }
            }
        } else if (MODE == MODE_GROUP_SHARED) {
            const uint32_t nv1 = P.nval + 1;
            long long* w = reinterpret_cast<long long*>(extra);
            for (uint32_t i = tid; i < P.ngroups * nv1; i += kThreads) {
                const uint32_t v = i % nv1;
                const uint8_t kind = v == 0 ? VK_SUM : P.val[v - 1].kind;
                w[2 * i] = kind == VK_MIN ? 0x7fffffffffffffffll
                           : kind == VK_MAX ? static_cast<long long>(0x8000000000000000ull) : 0ll;
                w[2 * i + 1] = 0;
            }
        }
    }

    // One selected (row[, build row]) pair.
    template <bool TAIL>
    __device__ __forceinline__ void row(const Plan& P, uint8_t* extra, const uint8_t* stage,
                                        uint64_t r0, uint32_t rl, uint32_t brow, uint32_t tid) {
        if (MODE == MODE_SCALAR) {
            count += 1;
#pragma unroll
            for (int v = 0; v < kMaxVals; ++v) {
                if (v < (int)P.nval) {
                    const int64_t x = eval_val<TAIL>(P, P.val[v], stage, r0, rl, brow, ovf);
                    acc_update(acc[v], P.val[v].kind, x);
                }
            }
        } else if (MODE == MODE_GROUP_PRIVATE) {
            const uint32_t nv1 = P.nval + 1;
            const uint32_t g = group_index<TAIL>(P, stage, r0, rl, brow);
            long long* w = reinterpret_cast<long long*>(extra);
            if (ACC128) {
                uint64_t* lo = reinterpret_cast<uint64_t*>(&w[((g * nv1) * 2 + 0) * kThreads + tid]);
                long long* hi = &w[((g * nv1) * 2 + 1) * kThreads + tid];
                const uint64_t nl = *lo + 1;
                *hi += (nl == 0) ? 1 : 0;
                *lo = nl;
                for (uint32_t v = 1; v < nv1; ++v) {
                    const ValDesc& V = P.val[v - 1];
                    const int64_t x = eval_val<TAIL>(P, V, stage, r0, rl, brow, ovf);
                    uint64_t* plo = reinterpret_cast<uint64_t*>(&w[((g * nv1 + v) * 2 + 0) * kThreads + tid]);
                    long long* phi = &w[((g * nv1 + v) * 2 + 1) * kThreads + tid];
                    I128 a{*plo, *phi};
                    acc_update(a, V.kind, x);
                    *plo = a.lo;
                    *phi = a.hi;
                }
            } else {
                w[(g * nv1) * kThreads + tid] += 1;
                for (uint32_t v = 1; v < nv1; ++v) {
                    const ValDesc& V = P.val[v - 1];
                    const int64_t x = eval_val<TAIL>(P, V, stage, r0, rl, brow, ovf);
                    long long& a = w[(g * nv1 + v) * kThreads + tid];
                    if (V.kind == VK_SUM) a = static_cast<long long>(static_cast<uint64_t>(a) + static_cast<uint64_t>(x));
                    else if (V.kind == VK_COUNT_NZ) a += (x != 0);
                    else if (V.kind == VK_MIN) a = min(a, static_cast<long long>(x));
                    else a = max(a, static_cast<long long>(x));
                }
                // |x| <= bound for every value, so after flush_limit updates an
                // int64 partial could be one update away from wrapping: move
                // this thread's partials into the global int128 accumulators.
                if (++upd >= P.flush_limit) {
                    flush_private_thread(P, extra, tid);
                    upd = 0;
                }
            }
        } else if (MODE == MODE_GROUP_SHARED) {
            // Per-CTA int128 table: word pair ((g * nv1 + v) * 2, +1).
            const uint32_t nv1 = P.nval + 1;
            const uint32_t g = group_index<TAIL>(P, stage, r0, rl, brow);
            unsigned long long* w = reinterpret_cast<unsigned long long*>(extra);
            atomicAdd(&w[(g * nv1) * 2], 1ull);
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
        } else if (MODE == MODE_GROUP_GLOBAL) {
            const uint32_t nv1 = P.nval + 1;
            const uint32_t g = group_index<TAIL>(P, stage, r0, rl, brow);
            unsigned long long* a = P.acc + static_cast<uint64_t>(g) * nv1 * 2;
            atomicAdd(a, 1ull);
            for (uint32_t v = 1; v < nv1; ++v) {
                const ValDesc& V = P.val[v - 1];
                const int64_t x = eval_val<TAIL>(P, V, stage, r0, rl, brow, ovf);
                acc_global_i64(a + 2 * v, V.kind, x);
            }
        } else if (MODE == MODE_GROUP_HASH) {
            const uint64_t key = group_hash_key<TAIL>(P, stage, r0, rl, brow);
            uint64_t h = hash_slot(key, P.hlog2);
            unsigned long long* slot = nullptr;
            for (uint64_t n = 0; n <= P.hmask; ++n) {
                unsigned long long* s = P.htab + h * P.hstride;
                unsigned long long k = *reinterpret_cast<volatile unsigned long long*>(s);
                if (k == kEmpty) k = atomicCAS(s, kEmpty, key);
                if (k == kEmpty || k == key) {
                    slot = s;
                    break;
                }
                h = (h + 1) & P.hmask;
            }
            if (slot == nullptr) {
                atomicOr(P.err, kErrHashFull);
                return;
            }
            atomicAdd(slot + 1, 1ull);
            for (uint32_t v = 0; v < P.nval; ++v) {
                const ValDesc& V = P.val[v];
                const int64_t x = eval_val<TAIL>(P, V, stage, r0, rl, brow, ovf);
                acc_global_i64(slot + 2 + 2 * v, V.kind, x);
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
                    const unsigned long long e = (rel << 32) | row;
                    done = atomicCAS(P.jtab + h, kEmpty, e) == kEmpty;
                } else {
                    if (atomicCAS(P.jtab + 2 * h + 1, 0ull, static_cast<unsigned long long>(row) + 1) == 0ull) {
                        P.jtab[2 * h] = rel;
                        done = true;
                    }
                }
                h = (h + 1) & P.jmask;
            }
            if (!done) atomicOr(P.err, kErrHashFull);
        }
    }

    // End of kernel: merge partials into global results.
    __device__ __forceinline__ void flush(const Plan& P, uint8_t* extra, uint32_t tid,
                                          I128* red /* shared: 8 warps x kMaxVals */,
                                          unsigned long long* redc) {
        const uint32_t lane = tid & 31u, warp = tid >> 5;
        if (MODE == MODE_SCALAR) {
            unsigned long long c = count;
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(kFull, c, d);
            if (lane == 0) redc[warp] = c;
#pragma unroll
            for (int v = 0; v < kMaxVals; ++v) {
                if (v < (int)P.nval) {
                    I128 a = acc[v];
                    const uint8_t kind = P.val[v].kind;
#pragma unroll
                    for (int d = 16; d > 0; d >>= 1) acc_combine(a, kind, shfl_down_i128(a, d));
                    if (lane == 0) red[warp * kMaxVals + v] = a;
                }
            }
            __syncthreads();
            if (tid == 0) {
                unsigned long long tc = 0;
                for (int w = 0; w < kThreads / 32; ++w) tc += redc[w];
                if (tc) atomicAdd(P.acc, tc);
                for (uint32_t v = 0; v < P.nval; ++v) {
                    I128 a = red[v];
                    for (int w = 1; w < kThreads / 32; ++w) acc_combine(a, P.val[v].kind, red[w * kMaxVals + v]);
                    acc_global(P.acc + 2 * (v + 1), P.val[v].kind, a);
                }
            }
        } else if (MODE == MODE_GROUP_PRIVATE) {
            __syncthreads();
            const uint32_t nv1 = P.nval + 1;
            const long long* w = reinterpret_cast<const long long*>(extra);
            for (uint32_t idx = warp; idx < P.ngroups * nv1; idx += kThreads / 32) {
                const uint32_t v = idx % nv1;
                const uint8_t kind = v == 0 ? VK_SUM : P.val[v - 1].kind;
                I128 a;
                acc_init(a, kind);
                for (uint32_t t = lane; t < kThreads; t += 32) {
                    I128 b;
                    if (ACC128) {
                        b.lo = static_cast<uint64_t>(w[(idx * 2 + 0) * kThreads + t]);
                        b.hi = w[(idx * 2 + 1) * kThreads + t];
                    } else {
                        const long long x = w[idx * kThreads + t];
                        b.lo = static_cast<uint64_t>(x);
                        b.hi = (kind == VK_MIN || kind == VK_MAX) ? 0 : (x >> 63);
                    }
                    acc_combine(a, kind, b);
                }
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) acc_combine(a, kind, shfl_down_i128(a, d));
                if (lane == 0) {
                    const bool untouched = (kind == VK_MIN) ? (a.lo == 0x7fffffffffffffffull)
                                           : (kind == VK_MAX) ? (a.lo == 0x8000000000000000ull)
                                                              : (a.lo == 0 && a.hi == 0);
                    if (!untouched) acc_global(P.acc + 2ull * idx, kind, a);
                }
            }
        } else if (MODE == MODE_GROUP_SHARED) {
            __syncthreads();
            const uint32_t nv1 = P.nval + 1;
            const long long* w = reinterpret_cast<const long long*>(extra);
            for (uint32_t idx = tid; idx < P.ngroups * nv1; idx += kThreads) {
                const uint32_t v = idx % nv1;
                const uint8_t kind = v == 0 ? VK_SUM : P.val[v - 1].kind;
                I128 a;
                a.lo = static_cast<uint64_t>(w[2 * idx]);
                a.hi = w[2 * idx + 1];
                const bool untouched = (kind == VK_MIN) ? (a.lo == 0x7fffffffffffffffull)
                                       : (kind == VK_MAX) ? (a.lo == 0x8000000000000000ull)
                                                          : (a.lo == 0 && a.hi == 0);
                if (!untouched) acc_global(P.acc + 2ull * idx, kind, a);
            }
        }
        if (ovf) atomicOr(P.err, kErrRowOverflow);
    }
};

// ---------------------------------------------------------------------------
// Tile processing
// ---------------------------------------------------------------------------
template <uint32_t MODE, bool ACC128, bool TAIL>
__device__ __forceinline__ void process_tile(const Plan& P, Sink<MODE, ACC128>& sink,
                                             uint8_t* extra, const uint8_t* stage, uint64_t tile,
                                             uint32_t tid, unsigned long long* tile_sel) {
    const uint64_t r0 = tile * kTileRows;
    const uint32_t nrem = TAIL ? static_cast<uint32_t>(P.nrows - r0) : kTileRows;
    const uint32_t m = eval_pred<TAIL>(P, stage, r0, tid, nrem);
    const uint32_t lane = tid & 31u, warp = tid >> 5;

    if (MODE == MODE_FILTER) {
        const uint64_t w0 = r0 / 32;
#pragma unroll
        for (int j = 0; j < kRowsPerThread; ++j) {
            const uint32_t word = __ballot_sync(kFull, (m >> j) & 1u);
            const uint64_t wi = w0 + j * (kThreads / 32) + warp;
            if (lane == 0 && wi < P.bitmap_words) P.bitmap[wi] = word;
        }
        unsigned c = __popc(m);
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(kFull, c, d);
        if (lane == 0 && c) atomicAdd(tile_sel, static_cast<unsigned long long>(c));
        return;
    }

    unsigned csel = __popc(m);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) csel += __shfl_down_sync(kFull, csel, d);
    if (lane == 0 && csel) atomicAdd(tile_sel, static_cast<unsigned long long>(csel));

    if (MODE == MODE_SCALAR && P.jslot < 0) {
        sink.count += __popc(m);
        if (P.nval == 0) return;
#pragma unroll
        for (int j = 0; j < kRowsPerThread; ++j) {
            const bool take = (m >> j) & 1u;
            if (__any_sync(kFull, take) && take) {
                const uint32_t rl = j * kThreads + tid;
#pragma unroll
                for (int v = 0; v < kMaxVals; ++v) {
                    if (v < (int)P.nval) {
                        const int64_t x = eval_val<TAIL>(P, P.val[v], stage, r0, rl, 0, sink.ovf);
                        acc_update(sink.acc[v], P.val[v].kind, x);
                    }
                }
            }
        }
        return;
    }

    if (MODE == MODE_JOIN_PAIRS) {
#pragma unroll 1
        for (int j = 0; j < kRowsPerThread; ++j) {
            const bool take = (m >> j) & 1u;
            if (!__any_sync(kFull, take)) continue;
            const uint32_t rl = j * kThreads + tid;
            uint64_t rel = 0;
            uint32_t nmatch = 0;
            bool probe = false;
            if (take) {
                const int64_t c = load_cell(slot_base<TAIL>(P, stage, P.jslot, r0), P.slot[P.jslot].dtype, rl);
                probe = join_rel(P, c, rel);
                if (probe) join_foreach(P, rel, [&](uint32_t) { ++nmatch; });
            }
            // Warp-aggregated reservation of nmatch output pairs.
            uint32_t incl = nmatch;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(kFull, incl, d);
                if (lane >= (uint32_t)d) incl += y;
            }
            const uint32_t total = __shfl_sync(kFull, incl, 31);
            unsigned long long base = 0;
            if (lane == 31 && total) base = atomicAdd(P.counters + 1, static_cast<unsigned long long>(total));
            base = __shfl_sync(kFull, base, 31);
            if (nmatch) {
                unsigned long long o = base + incl - nmatch;
                const uint32_t prow = static_cast<uint32_t>(r0 + rl);
                unsigned long long* out = P.out_pairs;
                join_foreach(P, rel, [&](uint32_t b) {
                    if (o < P.out_cap) out[o] = (static_cast<unsigned long long>(prow) << 32) | b;
                    ++o;
                });
            }
        }
        return;
    }

    // Generic sink path: grouped modes, join build, and joined aggregates.
#pragma unroll 1
    for (int j = 0; j < kRowsPerThread; ++j) {
        const bool take = (m >> j) & 1u;
        if (!__any_sync(kFull, take) || !take) continue;
        const uint32_t rl = j * kThreads + tid;
        if (P.jslot >= 0 && MODE != MODE_JOIN_BUILD) {
            const int64_t c = load_cell(slot_base<TAIL>(P, stage, P.jslot, r0), P.slot[P.jslot].dtype, rl);
            uint64_t rel;
            if (join_rel(P, c, rel)) {
                join_foreach(P, rel, [&](uint32_t b) { sink.template row<TAIL>(P, extra, stage, r0, rl, b, tid); });
            }
        } else {
            sink.template row<TAIL>(P, extra, stage, r0, rl, 0, tid);
        }
    }
}

// ---------------------------------------------------------------------------
// The persistent kernel
// ---------------------------------------------------------------------------
template <uint32_t MODE, bool ACC128>
__global__ void __launch_bounds__(kThreads, 1) scan_kernel(const __grid_constant__ Plan P) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint8_t* stages = smem + kBarrierBytes;
    uint8_t* extra = smem + P.extra_off;
    __shared__ I128 red[(kThreads / 32) * kMaxVals];
    __shared__ unsigned long long redc[kThreads / 32];
    __shared__ unsigned long long tile_sel;

    const uint32_t tid = threadIdx.x;
    const uint64_t ntiles = (P.nrows + kTileRows - 1) / kTileRows;
    const uint64_t nfull = P.nrows / kTileRows;
    const uint32_t S = P.nstages;
    const uint64_t G = gridDim.x;

    Sink<MODE, ACC128> sink;
    sink.init(P, extra, tid);

    uint64_t policy = 0;
    if (tid == 0) {
        for (uint32_t s = 0; s < S; ++s) mbar_init(&full[s], 1);
        fence_barrier_init();
        policy = l2_policy_evict_first();
    }
    if (tid == 0) tile_sel = 0;
    __syncthreads();

    auto issue = [&](uint64_t tile, uint32_t s) {
        uint8_t* dst = stages + static_cast<size_t>(s) * P.stage_bytes;
        mbar_arrive_expect_tx(&full[s], P.stage_bytes);
        for (uint32_t c = 0; c < P.nslots; ++c) {
            const uint32_t bytes = kTileRows * P.slot[c].width;
            bulk_g2s(dst + P.slot[c].smem_off, P.slot[c].ptr + tile * bytes, bytes, &full[s], policy);
        }
    };

    if (tid == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            const uint64_t t = blockIdx.x + s * G;
            if (t < nfull) issue(t, s);
        }
    }

    bool timed_out = false;
    uint64_t k = 0;
    for (;; ++k) {
        const uint64_t t = blockIdx.x + k * G;
        if (t >= ntiles) break;
        if (t < nfull) {
            const uint32_t s = static_cast<uint32_t>(k % S);
            const uint32_t parity = static_cast<uint32_t>((k / S) & 1u);
            const bool ok = mbar_wait_bounded(&full[s], parity);
            if (__syncthreads_or(!ok)) {
                timed_out = true;
                break;
            }
            process_tile<MODE, ACC128, false>(P, sink, extra, stages + static_cast<size_t>(s) * P.stage_bytes,
                                              t, tid, &tile_sel);
            __syncthreads();
            if (tid == 0) {
                if (MODE == MODE_FILTER && P.tile_counts) P.tile_counts[t] = static_cast<uint32_t>(tile_sel);
                if (tile_sel) atomicAdd(P.counters, tile_sel);
                tile_sel = 0;
                const uint64_t tn = t + S * G;
                if (tn < nfull) issue(tn, s);
            }
        } else {
            process_tile<MODE, ACC128, true>(P, sink, extra, nullptr, t, tid, &tile_sel);
            __syncthreads();
            if (tid == 0) {
                if (MODE == MODE_FILTER && P.tile_counts) P.tile_counts[t] = static_cast<uint32_t>(tile_sel);
                if (tile_sel) atomicAdd(P.counters, tile_sel);
                tile_sel = 0;
            }
        }
        __syncthreads();
    }

    if (timed_out) {
        // Let every copy this CTA issued land (bounded) before the CTA exits.
        if (tid == 0) {
            atomicOr(P.err, kErrWaitTimeout);
            for (uint64_t i = k; i < k + S; ++i) {
                const uint64_t t = blockIdx.x + i * G;
                if (t >= nfull) break;
                mbar_wait_bounded(&full[i % S], static_cast<uint32_t>((i / S) & 1u));
            }
        }
        __syncthreads();
        return;
    }
    sink.flush(P, extra, tid, red, redc);
}

// ---------------------------------------------------------------------------
// Host launcher
// ---------------------------------------------------------------------------
template <uint32_t MODE, bool ACC128>
static cudaError_t launch_mode(const Plan& P, int grid, cudaStream_t st) {
    auto kern = scan_kernel<MODE, ACC128>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(P.smem_bytes));
    if (e != cudaSuccess) return e;
    kern<<<grid, kThreads, P.smem_bytes, st>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_scan(const Plan& P, uint32_t mode, bool acc128, int grid, cudaStream_t st) {
    switch (mode) {
        case MODE_FILTER: return launch_mode<MODE_FILTER, false>(P, grid, st);
        case MODE_SCALAR: return launch_mode<MODE_SCALAR, false>(P, grid, st);
        case MODE_GROUP_PRIVATE:
            return acc128 ? launch_mode<MODE_GROUP_PRIVATE, true>(P, grid, st)
                          : launch_mode<MODE_GROUP_PRIVATE, false>(P, grid, st);
        case MODE_GROUP_SHARED: return launch_mode<MODE_GROUP_SHARED, false>(P, grid, st);
        case MODE_GROUP_GLOBAL: return launch_mode<MODE_GROUP_GLOBAL, false>(P, grid, st);
        case MODE_GROUP_HASH: return launch_mode<MODE_GROUP_HASH, false>(P, grid, st);
        case MODE_JOIN_BUILD: return launch_mode<MODE_JOIN_BUILD, false>(P, grid, st);
        case MODE_JOIN_PAIRS: return launch_mode<MODE_JOIN_PAIRS, false>(P, grid, st);
        default: return cudaErrorInvalidValue;
    }
}

int scan_occupancy(uint32_t mode, bool acc128, size_t dyn_smem) {
    int n = 0;
    const void* f = nullptr;
    switch (mode) {
        case MODE_FILTER: f = (const void*)scan_kernel<MODE_FILTER, false>; break;
        case MODE_SCALAR: f = (const void*)scan_kernel<MODE_SCALAR, false>; break;
        case MODE_GROUP_PRIVATE:
            f = acc128 ? (const void*)scan_kernel<MODE_GROUP_PRIVATE, true>
                       : (const void*)scan_kernel<MODE_GROUP_PRIVATE, false>;
            break;
        case MODE_GROUP_SHARED: f = (const void*)scan_kernel<MODE_GROUP_SHARED, false>; break;
        case MODE_GROUP_GLOBAL: f = (const void*)scan_kernel<MODE_GROUP_GLOBAL, false>; break;
        case MODE_GROUP_HASH: f = (const void*)scan_kernel<MODE_GROUP_HASH, false>; break;
        case MODE_JOIN_BUILD: f = (const void*)scan_kernel<MODE_JOIN_BUILD, false>; break;
        case MODE_JOIN_PAIRS: f = (const void*)scan_kernel<MODE_JOIN_PAIRS, false>; break;
        default: return 0;
    }
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dyn_smem)) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, kThreads, dyn_smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// Static shared memory used by scan_kernel besides the dynamic stages.
size_t scan_kernel_static_smem() {
    return sizeof(I128) * (kThreads / 32) * kMaxVals + sizeof(unsigned long long) * (kThreads / 32 + 1);
}

}  // namespace tgp
