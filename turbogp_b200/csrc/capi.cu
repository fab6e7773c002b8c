// capi.cu — implementation of the C ABI declared in include/turbogp_gpu.h:
// context, resident tables, the query planner that lowers C-ABI descriptors
// into a Plan, launches, and result decoding. Host code only; kernels live in
// scan_engine.cu and aux_kernels.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <memory>
#include <unordered_map>
#include <vector>

#include "runtime.hpp"

using namespace tgp;

namespace {

constexpr unsigned long long kEmptySlot = ~0ull;
constexpr uint64_t kDirectMaxGroups = 1ull << 22;
constexpr uint64_t kHashDirectMax = 1ull << 27;   // key values of a directly indexed group table
constexpr size_t kJoinSmemCap = 144u << 10;        // shared memory per CTA of a payload-join scan (see size_smem)

int fail(tgp_ctx* ctx, int st, const std::string& m) {
    if (ctx) ctx->err = m;
    return st;
}

#define TGP_CUDA(call)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(ctx, TGP_DEVICE_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define TGP_TRY(expr)              \
    do {                           \
        int st_ = (expr);          \
        if (st_ != TGP_OK) return st_; \
    } while (0)

uint32_t dtype_width(uint32_t dt) {
    switch (dt) {
        case DT_U8: return 1;
        case DT_I32: return 4;
        case DT_I64:
        case DT_U64:
        case DT_F64: return 8;
        default: return 0;
    }
}

bool is_device_ptr(const void* p) {
    if (p == nullptr) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

uint64_t next_pow2(uint64_t x) {
    uint64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

uint32_t log2u(uint64_t p) {
    uint32_t l = 0;
    while ((1ull << l) < p) ++l;
    return l;
}

// --------------------------------------------------------------------------
// Scratch arena: one grow-only device buffer carved per call.
// --------------------------------------------------------------------------
struct Carve {
    uint8_t* base;
    size_t off = 0;
    size_t cap;
    template <typename T>
    T* take(size_t count) {
        off = (off + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + off);
        off += count * sizeof(T);
        return p;
    }
};

// Per-call device buffers (join tables, payloads, gathered groups) come from
// the stream-ordered pool, which keeps freed memory for the next call.
int dev_alloc(tgp_ctx* ctx, void** p, size_t bytes, const char* what) {
    *p = nullptr;
    const size_t n = std::max<size_t>(bytes, 256);
    const cudaError_t e = ctx->pool ? cudaMallocFromPoolAsync(p, n, ctx->pool, ctx->stream)
                                    : cudaMallocAsync(p, n, ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(ctx, TGP_OOM, what);
    }
    return TGP_OK;
}

void dev_free(tgp_ctx* ctx, void* p) {
    if (p) cudaFreeAsync(p, ctx->stream);
}

int arena_reserve(tgp_ctx* ctx, size_t bytes, Carve* out) {
    bytes = bytes + 4096;
    if (bytes > ctx->arena.cap) {
        TGP_CUDA(cudaStreamSynchronize(ctx->stream));
        const size_t want = std::max(bytes, ctx->arena.cap * 2);
        if (ctx->arena.base) cudaFree(ctx->arena.base);
        ctx->arena.base = nullptr;
        ctx->arena.cap = 0;
        if (cudaMalloc(&ctx->arena.base, want) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, TGP_OOM, "device scratch allocation failed");
        }
        ctx->arena.cap = want;
    }
    out->base = ctx->arena.base;
    out->off = 0;
    out->cap = ctx->arena.cap;
    return TGP_OK;
}

int pinned_reserve(tgp_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->hpin_cap) return TGP_OK;
    if (ctx->hpin) cudaFreeHost(ctx->hpin);
    ctx->hpin = nullptr;
    ctx->hpin_cap = 0;
    size_t want = std::max<size_t>(bytes, 1 << 16);
    if (cudaMallocHost(&ctx->hpin, want) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, TGP_OOM, "pinned host allocation failed");
    }
    ctx->hpin_cap = want;
    return TGP_OK;
}

// Copies `bytes` from device memory to `dst` (host or device).
int copy_out(tgp_ctx* ctx, void* dst, const void* src_dev, size_t bytes) {
    if (bytes == 0) return TGP_OK;
    TGP_CUDA(cudaMemcpyAsync(dst, src_dev, bytes, cudaMemcpyDefault, ctx->stream));
    return TGP_OK;
}

// Reads the device error word and maps kernel error bits to a status.
int check_kernel_err(tgp_ctx* ctx, uint32_t err) {
    if (err & kErrWaitTimeout) return fail(ctx, TGP_TIMEOUT, "a bounded device wait gave up");
    if (err & kErrHashFull) return fail(ctx, TGP_DEVICE_ERROR, "device hash table overflowed");
    return TGP_OK;
}

}  // namespace

// The predicate lowering below is shared with the allocation-free entry point
// (noalloc.cu), so it lives in namespace tgp rather than in this file's
// anonymous namespace.
namespace tgp {

// --------------------------------------------------------------------------
// Predicate lowering
// --------------------------------------------------------------------------
// Interval [a, b] over order keys (signed order: key = cell ^ 2^63, unsigned:
// key = cell), optionally negated, or a constant.
struct Interval {
    bool is_const = false;
    bool value = false;
    uint64_t a = 0, b = 0;
    bool negate = false;
};

Interval cmp_interval(uint32_t cmp, uint64_t L, uint64_t L2) {
    Interval iv;
    const uint64_t MAX = ~0ull;
    switch (cmp) {
        case 0: iv.a = L; iv.b = L; break;                                   // EQ
        case 1: iv.a = L; iv.b = L; iv.negate = true; break;                 // NE
        case 2:                                                              // LT
            if (L == 0) { iv.is_const = true; iv.value = false; }
            else { iv.a = 0; iv.b = L - 1; }
            break;
        case 3: iv.a = 0; iv.b = L; break;                                   // LE
        case 4:                                                              // GT
            if (L == MAX) { iv.is_const = true; iv.value = false; }
            else { iv.a = L + 1; iv.b = MAX; }
            break;
        case 5: iv.a = L; iv.b = MAX; break;                                 // GE
        case 6:                                                              // BETWEEN
            if (L > L2) { iv.is_const = true; iv.value = false; }
            else { iv.a = L; iv.b = L2; }
            break;
        default:                                                             // NOT_BETWEEN
            if (L > L2) { iv.is_const = true; iv.value = true; }
            else { iv.a = L; iv.b = L2; iv.negate = true; }
            break;
    }
    return iv;
}

void set_const(Leaf& lf, bool v) {
    lf.kind = LK_CONST;
    lf.negate = v ? 1 : 0;
}

int lower_leaf(tgp_ctx* ctx, const Column& c, const tgp_pred_node& n, uint8_t slot, Leaf& lf) {
    std::memset(&lf, 0, sizeof(lf));
    lf.slot = slot;
    if (n.cmp > TGP_CMP_NOT_BETWEEN) return fail(ctx, TGP_INVALID_ARG, "bad comparison code");
    if (c.coltype == TGP_CT_FLOAT) {
        if (c.dtype != DT_F64) return fail(ctx, TGP_INVALID_ARG, "FLOAT comparison on a non-f64 column");
        double v, v2;
        std::memcpy(&v, &n.lit, 8);
        std::memcpy(&v2, &n.lit2, 8);
        lf.kind = LK_F64;
        lf.f1 = v;
        lf.f2 = v2;
        static const uint8_t fmap[8] = {FOP_EQ_EPS, FOP_NE, FOP_LT, FOP_LE, FOP_GT, FOP_GE, FOP_BETWEEN,
                                        FOP_NOT_BETWEEN};
        lf.fop = fmap[n.cmp];
        if (n.cmp == TGP_CMP_EQ || n.cmp == TGP_CMP_NE) lf.f2 = 1e-6 * std::max(std::fabs(v), 1.0);
        return TGP_OK;
    }
    const bool sgn = c.coltype == TGP_CT_INT;
    const uint64_t flip = sgn ? (1ull << 63) : 0ull;
    Interval iv = cmp_interval(n.cmp, n.lit ^ flip, n.lit2 ^ flip);
    if (iv.is_const) {
        set_const(lf, iv.value);
        return TGP_OK;
    }
    lf.negate = iv.negate ? 1 : 0;
    if (c.width == 8) {
        lf.kind = LK_64;
        lf.xor64 = flip;
        lf.lo64 = iv.a;
        lf.span64 = iv.b - iv.a;
        return TGP_OK;
    }
    // Narrow columns: map the order-key interval onto the 32-bit physical key.
    uint64_t a = iv.a, b = iv.b;
    uint32_t lo32 = 0, hi32 = 0;
    bool empty = false;
    if (c.dtype == DT_U8) {
        const uint64_t base = sgn ? (1ull << 63) : 0ull;  // order key of cell 0
        const uint64_t ka = std::max(a, base), kb = std::min(b, base + 255);
        if (ka > kb) empty = true;
        else { lo32 = static_cast<uint32_t>(ka - base); hi32 = static_cast<uint32_t>(kb - base); }
        lf.kind = LK_U8;
        lf.xor32 = 0;
    } else {  // DT_I32
        lf.kind = LK_I32;
        if (sgn) {
            const uint64_t base = (1ull << 63) - (1ull << 31);  // order key of INT32_MIN
            const uint64_t top = (1ull << 63) + (1ull << 31) - 1;
            const uint64_t ka = std::max(a, base), kb = std::min(b, top);
            if (ka > kb) empty = true;
            else { lo32 = static_cast<uint32_t>(ka - base); hi32 = static_cast<uint32_t>(kb - base); }
            lf.xor32 = 0x80000000u;
        } else {
            // cells: [0, 2^31-1] (v >= 0) and [2^64-2^31, 2^64-1] (v < 0); key32 = (u32)v.
            const uint64_t neg0 = ~0ull - (1ull << 31) + 1;  // 2^64 - 2^31
            const uint64_t shift = ~0ull - (1ull << 32) + 1;  // 2^64 - 2^32
            uint64_t ca, cb;
            if (a <= 0x7fffffffull) ca = a;
            else if (a <= neg0) ca = 0x80000000ull;
            else ca = a - shift;
            if (b >= neg0) cb = b - shift;
            else if (b >= 0x7fffffffull) cb = 0x7fffffffull;
            else cb = b;
            if (ca > cb) empty = true;
            else { lo32 = static_cast<uint32_t>(ca); hi32 = static_cast<uint32_t>(cb); }
            lf.xor32 = 0;
        }
    }
    if (empty) {
        set_const(lf, iv.negate);
        return TGP_OK;
    }
    lf.lo32 = lo32;
    lf.span32 = hi32 - lo32;
    return TGP_OK;
}

}  // namespace tgp

namespace {

// --------------------------------------------------------------------------
// Query builder
// --------------------------------------------------------------------------
struct Bound {  // |value| bound; exact in 128-bit
    __int128 lo, hi;
};

__int128 abs128(__int128 x) { return x < 0 ? -x : x; }

struct Builder {
    tgp_ctx* ctx;
    const Table* T;
    const Table* B = nullptr;       // build table of a join
    const JoinTable* J = nullptr;
    Plan P;
    std::vector<int> col2slot;
    uint64_t max_abs_val = 0;       // max |per-row value| over all values (saturating)
    // Per value: the range of its per-row argument (valid when !val_big).
    __int128 val_lo[kMaxVals] = {}, val_hi[kMaxVals] = {};
    bool val_big[kMaxVals] = {};
    bool unbounded = false;         // some value may exceed 2^62 in magnitude
    size_t static_smem = 0;         // static shared bytes of the kernel the plan is sized for

    Builder(tgp_ctx* c, const Table* t) : ctx(c), T(t), static_smem(scan_kernel_static_smem()) {
        std::memset(&P, 0, sizeof(P));
        col2slot.assign(t->cols.size(), -1);
        P.nrows = t->rows;
        P.nthreads = 512;  // private placement picks its own; a variant may ask for 256
        P.jslot = -1;
        P.flush_limit = ~0ull;
    }

    int slot_of(uint32_t col, int* out) {
        if (col >= T->cols.size()) return fail(ctx, TGP_INVALID_ARG, "column index out of range");
        if (col2slot[col] < 0) {
            if (P.nslots >= static_cast<uint32_t>(kMaxSlots))
                return fail(ctx, TGP_UNSUPPORTED, "query references more than 8 columns");
            const Column& c = T->cols[col];
            SlotDesc& s = P.slot[P.nslots];
            s.ptr = c.dptr;
            s.width = c.width;
            s.dtype = c.dtype;
            s.smem_off = P.stage_bytes;
            P.stage_bytes += kTileRows * c.width;
            col2slot[col] = static_cast<int>(P.nslots++);
        }
        *out = col2slot[col];
        return TGP_OK;
    }

    int add_pred(const tgp_pred_node* pred, uint32_t npred) {
        if (npred == 0) return TGP_OK;
        if (pred == nullptr) return fail(ctx, TGP_INVALID_ARG, "null predicate program");
        if (npred > static_cast<uint32_t>(kMaxPredOps)) return fail(ctx, TGP_UNSUPPORTED, "predicate program too long");
        int depth = 0, maxdepth = 0;
        uint32_t nand = 0;
        bool only_and = true;
        for (uint32_t i = 0; i < npred; ++i) {
            const tgp_pred_node& n = pred[i];
            switch (n.kind) {
                case TGP_PN_LEAF: {
                    if (P.nleaf >= static_cast<uint32_t>(kMaxLeaves))
                        return fail(ctx, TGP_UNSUPPORTED, "more than 16 predicate leaves");
                    int slot;
                    TGP_TRY(slot_of(n.column, &slot));
                    TGP_TRY(lower_leaf(ctx, T->cols[n.column], n, static_cast<uint8_t>(slot), P.leaf[P.nleaf]));
                    P.ops[i] = static_cast<uint8_t>(P.nleaf++);
                    ++depth;
                    break;
                }
                case TGP_PN_AND:
                case TGP_PN_OR:
                    if (depth < 2) return fail(ctx, TGP_INVALID_ARG, "AND/OR needs two operands");
                    --depth;
                    P.ops[i] = n.kind == TGP_PN_AND ? OP_AND : OP_OR;
                    if (n.kind == TGP_PN_AND) ++nand; else only_and = false;
                    break;
                case TGP_PN_NOT:
                    if (depth < 1) return fail(ctx, TGP_INVALID_ARG, "NOT needs one operand");
                    P.ops[i] = OP_NOT;
                    only_and = false;
                    break;
                default:
                    return fail(ctx, TGP_INVALID_ARG, "bad predicate node kind");
            }
            maxdepth = std::max(maxdepth, depth);
        }
        if (depth != 1) return fail(ctx, TGP_INVALID_ARG, "predicate program must leave one value");
        if (maxdepth > 8) return fail(ctx, TGP_UNSUPPORTED, "predicate program deeper than 8");
        P.nops = npred;
        P.all_and = (only_and && nand + 1 == P.nleaf) ? 1u : 0u;
        if (P.all_and) merge_conjuncts();
        bias_leaves();
        return TGP_OK;
    }

    // In a pure conjunction, leaves on the same column intersect into one
    // interval test (e.g. ship_day >= a AND ship_day < b), so the column is
    // read once per row. Intervals are still in unbiased key space here.
    void merge_conjuncts() {
        uint32_t n = 0;
        for (uint32_t i = 0; i < P.nleaf; ++i) {
            Leaf cur = P.leaf[i];
            bool merged = false;
            const bool mergeable = cur.negate == 0 && (cur.kind == LK_U8 || cur.kind == LK_I32 || cur.kind == LK_64);
            for (uint32_t j = 0; mergeable && j < n; ++j) {
                Leaf& L = P.leaf[j];
                if (L.slot != cur.slot || L.kind != cur.kind || L.negate != 0) continue;
                if (cur.kind == LK_64) {
                    const uint64_t lo = std::max(L.lo64, cur.lo64);
                    const uint64_t hi = std::min(L.lo64 + L.span64, cur.lo64 + cur.span64);
                    if (lo > hi) set_const(L, false);
                    else { L.lo64 = lo; L.span64 = hi - lo; }
                } else {
                    const uint32_t lo = std::max(L.lo32, cur.lo32);
                    const uint32_t hi = std::min(L.lo32 + L.span32, cur.lo32 + cur.span32);
                    if (lo > hi) set_const(L, false);
                    else { L.lo32 = lo; L.span32 = hi - lo; }
                }
                merged = true;
                break;
            }
            if (!merged) P.leaf[n++] = cur;
        }
        // Order by kind so the device runs one branch-free loop per kind.
        auto rank = [](uint8_t k) { return k == LK_I32 ? 0 : k == LK_U8 ? 1 : k == LK_64 ? 2 : 3; };
        std::stable_sort(P.leaf, P.leaf + n, [&](const Leaf& x, const Leaf& y) { return rank(x.kind) < rank(y.kind); });
        for (uint32_t r = 0; r < 3; ++r) {
            uint32_t e = 0;
            while (e < n && rank(P.leaf[e].kind) <= static_cast<int>(r)) ++e;
            P.kend[r] = static_cast<uint8_t>(e);
        }
        P.kend[3] = static_cast<uint8_t>(n);
        P.nleaf = n;
        P.nops = 0;
        for (uint32_t i = 0; i < n; ++i) {
            P.ops[P.nops++] = static_cast<uint8_t>(i);
            if (i > 0) P.ops[P.nops++] = OP_AND;
        }
    }

    // The device tests (x - lo) <= span on the stored word x; key = x ^ xor
    // equals x + xor modulo 2^bits, so key - lo = x - (lo - xor).
    void bias_leaves() {
        for (uint32_t i = 0; i < P.nleaf; ++i) {
            Leaf& L = P.leaf[i];
            if (L.kind == LK_64) L.lo64 -= L.xor64;
            else if (L.kind == LK_U8 || L.kind == LK_I32) L.lo32 -= L.xor32;
        }
    }

    int lower_factor(const tgp_factor& f, Factor& out, __int128* blo, __int128* bhi) {
        std::memset(&out, 0, sizeof(out));
        out.mul = f.mul;
        out.add = f.add;
        out.slot = -1;
        if (f.column < 0) {
            *blo = *bhi = static_cast<__int128>(f.add);
            return TGP_OK;
        }
        const Table* S = T;
        if (f.side == TGP_SIDE_BUILD) {
            if (!B) return fail(ctx, TGP_INVALID_ARG, "build-side column without a join");
            S = B;
        } else if (f.side != TGP_SIDE_PROBE) {
            return fail(ctx, TGP_INVALID_ARG, "bad side");
        }
        if (static_cast<uint32_t>(f.column) >= S->cols.size()) return fail(ctx, TGP_INVALID_ARG, "factor column out of range");
        const Column& c = S->cols[f.column];
        if (c.coltype == TGP_CT_FLOAT) return fail(ctx, TGP_UNSUPPORTED, "aggregate arguments over FLOAT columns");
        if (f.side == TGP_SIDE_BUILD) {
            out.build_side = 1;
            out.dtype = static_cast<uint8_t>(c.dtype);
            out.bptr = c.dptr;
        } else {
            int slot;
            TGP_TRY(slot_of(static_cast<uint32_t>(f.column), &slot));
            out.slot = static_cast<int8_t>(slot);
            out.dtype = static_cast<uint8_t>(P.slot[slot].dtype);
            out.soff = P.slot[slot].smem_off;
        }
        const __int128 m = f.mul, a = f.add;
        const __int128 x0 = m * c.min + a, x1 = m * c.max + a;
        *blo = std::min(x0, x1);
        *bhi = std::max(x0, x1);
        return TGP_OK;
    }

    // Returns the value index for (kind, factors), deduplicating.
    int add_value(uint8_t kind, const tgp_agg& a, int* idx) {
        if (a.nfactors > static_cast<uint32_t>(kMaxFactors)) return fail(ctx, TGP_UNSUPPORTED, "more than 4 factors");
        ValDesc v;
        std::memset(&v, 0, sizeof(v));
        v.kind = kind;
        v.nf = static_cast<uint8_t>(a.nfactors);
        __int128 lo = 1, hi = 1;
        bool big = false;
        const __int128 lim = static_cast<__int128>(1) << 63;
        for (uint32_t f = 0; f < a.nfactors; ++f) {
            __int128 flo, fhi;
            TGP_TRY(lower_factor(a.f[f], v.f[f], &flo, &fhi));
            if (abs128(flo) >= lim || abs128(fhi) >= lim) big = true;
            if (f == 0) {
                lo = flo;
                hi = fhi;
            } else if (!big) {
                const __int128 c[4] = {lo * flo, lo * fhi, hi * flo, hi * fhi};
                lo = *std::min_element(c, c + 4);
                hi = *std::max_element(c, c + 4);
                if (abs128(lo) >= lim || abs128(hi) >= lim) big = true;
            }
        }
        if (big) {
            P.check_ovf = 1;
            unbounded = true;
        } else {
            const __int128 m = std::max(abs128(lo), abs128(hi));
            if (kind == VK_SUM && m > (static_cast<__int128>(1) << 62)) unbounded = true;
            if (kind == VK_SUM || kind == VK_COUNT_NZ) {
                const uint64_t mm = kind == VK_COUNT_NZ ? 1ull : static_cast<uint64_t>(m);
                max_abs_val = std::max(max_abs_val, mm);
            }
        }
        for (uint32_t i = 0; i < P.nval; ++i) {
            if (std::memcmp(&P.val[i], &v, sizeof(v)) == 0) {
                *idx = static_cast<int>(i);
                return TGP_OK;
            }
        }
        if (P.nval >= static_cast<uint32_t>(kMaxVals)) return fail(ctx, TGP_UNSUPPORTED, "more than 8 distinct aggregates");
        val_lo[P.nval] = kind == VK_COUNT_NZ ? 0 : lo;
        val_hi[P.nval] = kind == VK_COUNT_NZ ? 1 : hi;
        val_big[P.nval] = big;
        P.val[P.nval] = v;
        *idx = static_cast<int>(P.nval++);
        return TGP_OK;
    }
};

// Lowers the values of a MODE_GROUP_PRIVATE int64 plan into the dense step
// program (ChainProg). A value whose factor list extends the previous value's
// continues its running product; any other value starts a new one. Returns
// false (dense path off) when a factor or key is not staged, more than two
// keys group, or the program needs more than kMaxSteps steps.
bool compile_chain(Builder& b, bool build_keys_in_payload, uint32_t max_keys = 2) {
    Plan& P = b.P;
    if (P.ngkey > max_keys) return false;
    for (uint32_t k = 0; k < P.ngkey; ++k) {
        if (P.gkey[k].build_side && build_keys_in_payload) continue;
        if (P.gkey[k].slot < 0 || P.gkey[k].build_side) return false;
    }
    std::vector<int> slot2col(P.nslots, -1);
    for (size_t c = 0; c < b.col2slot.size(); ++c)
        if (b.col2slot[c] >= 0) slot2col[b.col2slot[c]] = static_cast<int>(c);
    ChainProg C;
    std::memset(&C, 0, sizeof(C));
    const ValDesc* prev = nullptr;
    for (uint32_t v = 0; v < P.nval; ++v) {
        const ValDesc& V = P.val[v];
        for (uint32_t f = 0; f < V.nf; ++f)
            if (V.f[f].build_side || (V.f[f].slot < 0 && V.f[f].bptr != nullptr)) return false;
        // Shared prefix with the previous value's whole factor list.
        uint32_t start = 0;
        if (prev && prev->nf >= 1 && prev->nf <= V.nf &&
            std::memcmp(prev->f, V.f, sizeof(Factor) * prev->nf) == 0)
            start = prev->nf;
        if (V.nf == 0) {
            // A value of no factors is the constant 1.
            if (C.nsteps >= static_cast<uint32_t>(kMaxSteps)) return false;
            ChainStep& S = C.s[C.nsteps++];
            S.add = 1;
            S.add32 = 1;
        }
        for (uint32_t f = start; f < V.nf; ++f) {
            if (C.nsteps >= static_cast<uint32_t>(kMaxSteps)) return false;
            const Factor& F = V.f[f];
            ChainStep& S = C.s[C.nsteps++];
            S.mul = F.mul;
            S.add = F.add;
            S.flags = f > 0 ? CS_CHAIN : 0;
            if (F.slot >= 0) {
                S.flags |= CS_COL;
                S.soff = F.soff;
                S.dtype = F.dtype;
                const Column& c = b.T->cols[slot2col[F.slot]];
                const __int128 x0 = static_cast<__int128>(F.mul) * c.min + F.add;
                const __int128 x1 = static_cast<__int128>(F.mul) * c.max + F.add;
                const __int128 lim = static_cast<__int128>(1) << 31;
                const bool small = F.mul >= INT32_MIN && F.mul <= INT32_MAX && F.add >= INT32_MIN && F.add <= INT32_MAX;
                if (F.dtype != DT_F64 && small && std::min(x0, x1) >= -lim && std::max(x0, x1) < lim &&
                    (F.dtype == DT_U8 || F.dtype == DT_I32)) {
                    S.flags |= CS_NARROW;
                    if (std::min(x0, x1) >= 0) S.flags |= CS_NONNEG;
                    S.mul32 = static_cast<int32_t>(F.mul);
                    S.add32 = static_cast<int32_t>(F.add);
                } else if (F.mul == 1 && F.add == 0) {
                    S.flags |= CS_IDENT;
                }
            }
        }
        if (C.nsteps == 0 || (start == V.nf && V.nf > 0 && C.s[C.nsteps - 1].acc != 0)) {
            // Same factor list as the previous value (a different kind): one
            // step that re-multiplies by 1 and accumulates.
            if (C.nsteps >= static_cast<uint32_t>(kMaxSteps)) return false;
            ChainStep& S = C.s[C.nsteps++];
            S.flags = CS_CHAIN;
            S.add = 1;
            S.add32 = 1;
        }
        C.s[C.nsteps - 1].acc = static_cast<uint8_t>(v + 1);
        C.s[C.nsteps - 1].kind = V.kind;
        prev = &V;
    }
    P.chain = C;
    return true;
}

// Per-aggregate mapping to accumulator slots.
struct AggMap {
    uint32_t func;
    int val;  // value index, -1 for COUNT_STAR
};

int lower_aggs(Builder& b, const tgp_agg* aggs, uint32_t nagg, std::vector<AggMap>* map) {
    if (nagg > 0 && aggs == nullptr) return fail(b.ctx, TGP_INVALID_ARG, "null aggregate list");
    map->clear();
    for (uint32_t i = 0; i < nagg; ++i) {
        const tgp_agg& a = aggs[i];
        AggMap m{a.func, -1};
        switch (a.func) {
            case TGP_AGG_COUNT_STAR: break;
            case TGP_AGG_COUNT_NONZERO: TGP_TRY(b.add_value(VK_COUNT_NZ, a, &m.val)); break;
            case TGP_AGG_SUM:
            case TGP_AGG_AVG: TGP_TRY(b.add_value(VK_SUM, a, &m.val)); break;
            case TGP_AGG_MIN: TGP_TRY(b.add_value(VK_MIN, a, &m.val)); break;
            case TGP_AGG_MAX: TGP_TRY(b.add_value(VK_MAX, a, &m.val)); break;
            default: return fail(b.ctx, TGP_INVALID_ARG, "bad aggregate function");
        }
        map->push_back(m);
    }
    return TGP_OK;
}

double i128_to_f64(uint64_t lo, int64_t hi) {
    const __int128 v = (static_cast<__int128>(hi) << 64) | static_cast<__int128>(lo);
    return static_cast<double>(v);
}

void fill_value(const AggMap& m, const unsigned long long* slot /* [nv1][2] */, const Plan& P,
                tgp_agg_value* out) {
    const uint64_t cnt = slot[0];
    out->count = cnt;
    if (m.val < 0) {
        out->lo = cnt;
        out->hi = 0;
        out->as_f64 = static_cast<double>(cnt);
        return;
    }
    const unsigned long long* s = slot + 2 * (m.val + 1);
    const uint8_t kind = P.val[m.val].kind;
    if (kind == VK_MIN || kind == VK_MAX) {
        const int64_t v = static_cast<int64_t>(s[0]);
        out->lo = static_cast<uint64_t>(v);
        out->hi = v < 0 ? -1 : 0;
        out->as_f64 = static_cast<double>(v);
        return;
    }
    out->lo = s[0];
    out->hi = P.sum64 ? (static_cast<int64_t>(s[0]) >> 63) : static_cast<int64_t>(s[1]);
    const double f = i128_to_f64(out->lo, out->hi);
    if (m.func == TGP_AGG_AVG) out->as_f64 = cnt ? f / static_cast<double>(cnt) : 0.0;
    else out->as_f64 = f;
}

// Chooses shared-memory stages for a plan given per-mode scratch bytes.
int size_smem(tgp_ctx* ctx, Plan& P, size_t extra_bytes, size_t static_smem = scan_kernel_static_smem(),
              const Knobs* kn = nullptr) {
    const Knobs& K = kn ? *kn : ctx->knobs;
    const size_t budget = ctx->max_dyn_smem > static_smem ? ctx->max_dyn_smem - static_smem : 0;
    size_t stage = P.stage_bytes;
    if (stage == 0) {
        // Nothing to stage (e.g. COUNT(*) without WHERE): stage one tiny dummy.
        stage = 0;
    }
    const size_t per_cta = budget / static_cast<size_t>(std::max(1, K.ctas_per_sm));
    size_t avail = per_cta > kBarrierBytes + extra_bytes ? per_cta - kBarrierBytes - extra_bytes : 0;
    // Joins through a payload array keep the CTA's shared memory to at most
    // 144 KB (at least two stages) unless a variant asks for fewer stages
    // than the maximum, so that the rest of the SM's combined L1 / shared
    // memory caches the payload lookups of hot keys: with private
    // accumulators (77 KB) the 60M x 1.5M join probe ran 0.516 ms with four
    // stages and 0.373 ms with two (L1 hit rate 8.8 -> 17.5 %), merged join
    // batches 0.85 -> 0.77 ms; the limb tables' few KB leave room for four.
    int max_st = K.max_stages;
    // Joins through a payload array on the limb tables with a fixed-shape
    // value program run two CTAs of 512 threads and two stages per SM (34
    // warps instead of 17 to hide the payload lookups; 60M x 1.5M probe
    // 0.164 -> 0.140 ms at 30M probe rows), unless a variant caps the stages
    // and keeps one CTA.
    P.two_ctas = (P.jpay != nullptr && P.s32_copies != 0 && P.shape != 0 && P.nthreads == 512 && stage &&
                  (K.ctas_per_sm == 2 || K.max_stages >= kMaxStages)) ? 1u : 0u;
    if (P.two_ctas) {
        avail = budget / 2 > kBarrierBytes + extra_bytes ? budget / 2 - kBarrierBytes - extra_bytes : 0;
        max_st = 2;
    } else if (P.jpay != nullptr && K.max_stages >= kMaxStages && stage) {
        const size_t room = kJoinSmemCap > kBarrierBytes + extra_bytes ? kJoinSmemCap - kBarrierBytes - extra_bytes : 0;
        max_st = static_cast<int>(std::max<size_t>(2, room / stage));
    }
    const size_t cap = static_cast<size_t>(std::max(1, std::min(max_st, kMaxStages)));
    uint32_t S = stage ? static_cast<uint32_t>(std::min<size_t>(avail / stage, cap)) : 1;
    if (S == 0) {
        // Fall back to a single CTA per SM.
        P.two_ctas = 0;
        avail = budget > kBarrierBytes + extra_bytes ? budget - kBarrierBytes - extra_bytes : 0;
        S = stage ? static_cast<uint32_t>(std::min<size_t>(avail / stage, cap)) : 1;
        if (S == 0) return fail(ctx, TGP_UNSUPPORTED, "query does not fit in shared memory");
    }
    P.nstages = S;
    // L2 prefetch ahead of the stage copies measured neutral on the scan and
    // grouped-aggregate workloads, so it is off unless a variant asks for it.
    P.l2_ahead = static_cast<uint32_t>(std::max(0, K.l2_ahead));
    P.extra_off = static_cast<uint32_t>(kBarrierBytes + static_cast<size_t>(S) * stage);
    P.extra_off = (P.extra_off + 127u) & ~127u;
    P.smem_bytes = static_cast<uint32_t>(P.extra_off + extra_bytes);
    return TGP_OK;
}

// With profiling on, takes the next pair of timing events and records the
// first on the context's stream (after a bounded device delay when gated);
// *ev stays null otherwise.
int profile_begin(tgp_ctx* ctx, std::pair<cudaEvent_t, cudaEvent_t>** ev) {
    *ev = nullptr;
    if (!ctx->profile) return TGP_OK;
    if (ctx->prof_used == ctx->prof_events.size()) {
        std::pair<cudaEvent_t, cudaEvent_t> p;
        TGP_CUDA(cudaEventCreate(&p.first));
        TGP_CUDA(cudaEventCreate(&p.second));
        ctx->prof_events.push_back(p);
    }
    *ev = &ctx->prof_events[ctx->prof_used++];
    // Gated timing: the GPU is busy with the delay while the host submits
    // the launch, so the start event is stamped right before the kernel.
    if (ctx->profile_gate) TGP_CUDA(launch_delay(50000, ctx->stream));
    TGP_CUDA(cudaEventRecord((*ev)->first, ctx->stream));
    return TGP_OK;
}

int launch(tgp_ctx* ctx, const Plan& P0, uint32_t mode, bool acc128) {
    // An armed failure-path hook (tgp_debug_fail_next_scan) applies to this
    // launch only.
    Plan armed;
    const Plan* pp = &P0;
    if (ctx->dbg_skip_tile1) {
        armed = P0;
        armed.skip_tile1 = ctx->dbg_skip_tile1;
        armed.wait_ns = ctx->dbg_wait_ns;
        ctx->dbg_skip_tile1 = 0;
        pp = &armed;
    }
    const Plan& P = *pp;
    const uint64_t ntiles = (P.nrows + kTileRows - 1) / kTileRows;
    if (ntiles == 0) return TGP_OK;
    int occ = scan_occupancy(mode, acc128, static_cast<int>(P.nthreads), P.smem_bytes, P.shape, P.two_ctas != 0);
    if (occ <= 0) return fail(ctx, TGP_DEVICE_ERROR, "scan kernel cannot be resident with this shared memory");
    const uint64_t grid = std::min<uint64_t>(ntiles, static_cast<uint64_t>(ctx->sms) * occ);
    std::pair<cudaEvent_t, cudaEvent_t>* ev = nullptr;
    TGP_TRY(profile_begin(ctx, &ev));
    cudaError_t e = launch_scan(P, mode, acc128, static_cast<int>(grid), ctx->stream);
    if (e != cudaSuccess) return fail(ctx, TGP_DEVICE_ERROR, std::string("scan launch: ") + cudaGetErrorString(e));
    if (ev) TGP_CUDA(cudaEventRecord(ev->second, ctx->stream));
    return TGP_OK;
}

// Unfiltered GROUP BY of one key into one-word direct slots: the streaming
// kernel of groupby_direct.cu in place of the scan pipeline. Its per-CTA
// shared table is kept only when no CTA's rows can take a 32-bit partial to
// 2^31 in magnitude.
// Shared slots of the direct-group kernel's table (96 KB with a value, two
// CTAs per SM): 8,192 measured faster than 4,096 (more hot keys held, fewer
// global adds) and than 16,384 (one CTA per SM).
constexpr uint32_t kDirectGroupSlots = 8192;

int launch_direct_groups(tgp_ctx* ctx, const Plan& P, uint64_t max_abs_val) {
    const bool hasv = P.nval != 0;
    uint32_t hs = P.hsm_slots ? kDirectGroupSlots : 0u;
    const int occ = std::max(1, direct_group_ctas_per_sm(hs, hasv));
    const uint64_t chunks = (P.nrows + 127) / 128;
    const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>((chunks + 15) / 16, static_cast<uint64_t>(ctx->sms) * occ));
    if (hs) {
        // A CTA's 16 warps take at most ceil(chunks / warps) chunks of 128
        // rows each, and one warp the partial last chunk.
        const uint64_t nwarps = grid * 16;
        const unsigned __int128 rows_cta = static_cast<unsigned __int128>((chunks + nwarps - 1) / nwarps) * 128 * 16 + 128;
        if (rows_cta * std::max<uint64_t>(max_abs_val, 1) >= (static_cast<unsigned __int128>(1) << 31)) hs = 0;
    }
    DirectGroupArgs A;
    std::memset(&A, 0, sizeof(A));
    A.key = P.slot[P.gkey[0].slot].ptr;
    A.val = hasv ? P.slot[P.val[0].f[0].slot].ptr : nullptr;
    A.nrows = P.nrows;
    A.kmin = P.gkey[0].min;
    A.mul = hasv ? P.val[0].f[0].mul : 1;
    A.add = hasv ? P.val[0].f[0].add : 0;
    A.ident = A.mul == 1 && A.add == 0;
    A.nz = hasv && P.val[0].kind == VK_COUNT_NZ;
    A.hs = hs;
    A.hs_shift = hs ? 32u - log2u(hs) : 0u;
    A.last = static_cast<uint32_t>(P.hmask);
    A.shift = P.hpack_shift;
    A.bias = P.hpack_bias;
    A.one = (1ull << P.hpack_shift) - static_cast<uint64_t>(P.hpack_bias);
    A.slots = P.htab;
    A.err = P.err;
    A.counters = P.counters;
    const uint32_t kdt = P.slot[P.gkey[0].slot].dtype, vdt = hasv ? P.slot[P.val[0].f[0].slot].dtype : 0u;
    std::pair<cudaEvent_t, cudaEvent_t>* ev = nullptr;
    TGP_TRY(profile_begin(ctx, &ev));
    cudaError_t e = launch_direct_group(A, kdt, vdt, static_cast<int>(grid), ctx->stream);
    if (e != cudaSuccess) return fail(ctx, TGP_DEVICE_ERROR, std::string("group launch: ") + cudaGetErrorString(e));
    if (ev) TGP_CUDA(cudaEventRecord(ev->second, ctx->stream));
    return TGP_OK;
}

// The TPC-H Q1 shape (two u8 keys, the fixed value program ShapeQ1) under at
// most four int32 predicate leaves and no join: the streaming kernel of
// groupby_direct.cu in place of the scan pipeline when every global sum and
// every thread's partial provably fits int64 and two CTAs' private partials
// fit an SM (else false, nothing launched).
int try_launch_q1(tgp_ctx* ctx, const Plan& P, uint32_t mode, bool acc128, uint64_t ngroups, uint64_t max_abs_val,
                  bool* done) {
    *done = false;
    // An armed failure-path hook (tgp_debug_fail_next_scan) targets the scan
    // pipeline's stage copies; this kernel has no stage ring and no waits.
    if (ctx->dbg_skip_tile1) return TGP_OK;
    if (mode != MODE_GROUP_PRIVATE || acc128 || P.shape != 1 || !P.dense_vec || P.jslot >= 0 || P.ngkey != 2 ||
        !P.sum64 || P.check_ovf || P.nval != 4 || P.chain.nsteps != 4 || ngroups == 0 || ngroups > 0xffffffffull)
        return TGP_OK;
    if (P.nleaf > 4 || (P.nleaf && !(P.all_and && P.kend[0] == P.nleaf))) return TGP_OK;
    if (P.gkey[0].lut || P.gkey[1].lut || P.gkey[0].build_side || P.gkey[1].build_side) return TGP_OK;
    if (q1_group_ctas_per_sm(static_cast<uint32_t>(ngroups)) < 2) return TGP_OK;
    auto slot_ptr = [&](uint32_t soff) -> const uint8_t* {
        for (uint32_t k = 0; k < P.nslots; ++k)
            if (P.slot[k].smem_off == soff) return P.slot[k].ptr;
        return nullptr;
    };
    Q1Args A;
    std::memset(&A, 0, sizeof(A));
    for (uint32_t i = 0; i < P.nleaf; ++i) {
        A.leaf_col[i] = P.slot[P.leaf[i].slot].ptr;
        A.leaf_lo[i] = P.leaf[i].lo32;
        A.leaf_sp[i] = P.leaf[i].span32;
        if (P.leaf[i].negate) A.leaf_neg |= 1u << i;
    }
    A.nleaf = P.nleaf;
    A.key0 = P.slot[P.gkey[0].slot].ptr;
    A.key1 = P.slot[P.gkey[1].slot].ptr;
    A.kmin0 = static_cast<uint32_t>(P.gkey[0].min);
    A.kmin1 = static_cast<uint32_t>(P.gkey[1].min);
    A.kstride0 = static_cast<uint32_t>(P.gkey[0].stride);
    A.kstride1 = static_cast<uint32_t>(P.gkey[1].stride);
    for (uint32_t s = 0; s < 4; ++s) {
        const ChainStep& S = P.chain.s[s];
        if (S.acc != s + 1) return TGP_OK;
        A.col[s] = slot_ptr(S.soff);
        if (!A.col[s]) return TGP_OK;
    }
    const int ms[3] = {0, 2, 3};
    for (int i = 0; i < 3; ++i) {
        A.mul[i] = static_cast<uint32_t>(P.chain.s[ms[i]].mul32);
        A.add[i] = static_cast<uint32_t>(P.chain.s[ms[i]].add32);
    }
    A.ngroups = static_cast<uint32_t>(ngroups);
    A.nrows = P.nrows;
    A.acc = P.acc;
    A.counters = P.counters;
    const uint64_t chunks = P.nrows / 128;
    const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>((chunks + 15) / 16, static_cast<uint64_t>(ctx->sms) * 2));
    // A thread adds at most ceil(chunks / warps) chunks of four rows and four
    // rows of the partial last chunk: its int64 partials must not wrap.
    const uint64_t nwarps = grid * 16;
    const unsigned __int128 rows_thread = static_cast<unsigned __int128>((chunks + nwarps - 1) / nwarps + 1) * 4;
    if (rows_thread * std::max<uint64_t>(max_abs_val, 1) >= (static_cast<unsigned __int128>(1) << 63)) return TGP_OK;
    std::pair<cudaEvent_t, cudaEvent_t>* ev = nullptr;
    TGP_TRY(profile_begin(ctx, &ev));
    const cudaError_t e = launch_q1_group(A, static_cast<int>(grid), ctx->stream);
    if (e != cudaSuccess) return fail(ctx, TGP_DEVICE_ERROR, std::string("grouped launch: ") + cudaGetErrorString(e));
    if (ev) TGP_CUDA(cudaEventRecord(ev->second, ctx->stream));
    *done = true;
    return TGP_OK;
}

int get_table(tgp_ctx* ctx, tgp_table_id id, const Table** out) {
    auto it = ctx->tables.find(id);
    if (it == ctx->tables.end()) return fail(ctx, TGP_NOT_FOUND, "unknown table id");
    *out = &it->second;
    return TGP_OK;
}

// Device buffers every scan call needs: accumulators, counters, error word.
struct ScanScratch {
    unsigned long long* acc = nullptr;
    unsigned long long* counters = nullptr;
    uint32_t* err = nullptr;
};

// Initial accumulator image: per group [count][v lo][v hi]...; MIN/MAX start
// at the identity of their operation.
void init_acc_image(const Plan& P, uint64_t ngroups, std::vector<unsigned long long>* img) {
    const uint32_t nv1 = P.nval + 1;
    img->assign(ngroups * nv1 * 2, 0ull);
    for (uint32_t v = 0; v < P.nval; ++v) {
        unsigned long long init = 0;
        if (P.val[v].kind == VK_MIN) init = 0x7fffffffffffffffull;
        else if (P.val[v].kind == VK_MAX) init = 0x8000000000000000ull;
        if (!init) continue;
        for (uint64_t g = 0; g < ngroups; ++g) (*img)[(g * nv1 + v + 1) * 2] = init;
    }
}

int upload(tgp_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return TGP_OK;
    TGP_TRY(pinned_reserve(ctx, bytes));
    std::memcpy(ctx->hpin, src, bytes);
    TGP_CUDA(cudaMemcpyAsync(dst, ctx->hpin, bytes, cudaMemcpyHostToDevice, ctx->stream));
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    return TGP_OK;
}

void free_join(tgp_ctx* ctx, JoinTable& J) {
    dev_free(ctx, J.tab);
    J.tab = nullptr;
    for (auto& kv : J.pays) dev_free(ctx, kv.second.ptr);
    J.pays.clear();
}

}  // namespace

// Releases a batch record (defined with the batch entry points).
extern "C" void tgp_batch_free_rec(tgp_ctx* ctx, void* rec);
// Releases a captured-query record (defined with the graph entry points).
extern "C" void tgp_graph_free_rec(void* rec);

// ==========================================================================
// C ABI
// ==========================================================================
extern "C" {

const char* tgp_status_string(int s) {
    switch (s) {
        case TGP_OK: return "OK";
        case TGP_INVALID_ARG: return "INVALID_ARG";
        case TGP_OOM: return "OOM";
        case TGP_UNSUPPORTED: return "UNSUPPORTED";
        case TGP_TIMEOUT: return "TIMEOUT";
        case TGP_DEVICE_ERROR: return "DEVICE_ERROR";
        case TGP_NOT_FOUND: return "NOT_FOUND";
        case TGP_CAPACITY: return "CAPACITY";
        case TGP_PENDING: return "PENDING";
        default: return "UNKNOWN";
    }
}

int tgp_init(tgp_ctx** out, int device) {
    if (!out) return TGP_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return TGP_DEVICE_ERROR;
    }
    tgp_ctx* ctx = new (std::nothrow) tgp_ctx();
    if (!ctx) return TGP_OOM;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete ctx;
        return TGP_DEVICE_ERROR;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete ctx;
        return TGP_DEVICE_ERROR;
    }
    if (prop.major < 10) {
        delete ctx;
        return TGP_UNSUPPORTED;  // built for sm_100a only
    }
    ctx->sms = prop.multiProcessorCount;
    ctx->max_dyn_smem = prop.sharedMemPerBlockOptin;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return TGP_DEVICE_ERROR;
    }
    // A stream-ordered pool of this context's own, which keeps freed memory
    // for the next call. Two contexts sharing the device's default pool could
    // each reuse memory the other freed, and the pool then makes the reusing
    // stream wait for the other stream's work. The device's default pool
    // (same release setting) serves if a pool cannot be created.
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    uint64_t keep = ~0ull;
    if (cudaMemPoolCreate(&ctx->pool, &props) == cudaSuccess) {
        cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    } else {
        ctx->pool = nullptr;
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess)
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    *out = ctx;
    return TGP_OK;
}

int tgp_shutdown(tgp_ctx* ctx) {
    if (!ctx) return TGP_INVALID_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->tables)
        for (auto& c : kv.second.cols)
            if (c.owned && c.dptr) cudaFree(c.dptr);
    for (auto& kv : ctx->joins) free_join(ctx, kv.second);
    for (auto& kv : ctx->strings) {
        dev_free(ctx, kv.second.offs);
        dev_free(ctx, kv.second.bytes);
    }
    ctx->strings.clear();
    for (void* h : ctx->hash_handles) {
        JoinTable* J = static_cast<JoinTable*>(h);
        free_join(ctx, *J);
        delete J;
    }
    for (auto& kv : ctx->batches) tgp_batch_free_rec(ctx, kv.second);
    ctx->batches.clear();
    for (auto& kv : ctx->graphs) tgp_graph_free_rec(kv.second);
    ctx->graphs.clear();
    cudaStreamSynchronize(ctx->stream);
    for (auto& pb : ctx->pinned_pool) cudaFreeHost(pb.p);
    ctx->pinned_pool.clear();
    if (ctx->arena.base) cudaFree(ctx->arena.base);
    if (ctx->kin) cudaFree(ctx->kin);
    if (ctx->hpin) cudaFreeHost(ctx->hpin);
    for (auto& p : ctx->prof_events) {
        cudaEventDestroy(p.first);
        cudaEventDestroy(p.second);
    }
    cudaStreamDestroy(ctx->stream);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
    return TGP_OK;
}

const char* tgp_last_error(const tgp_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void* tgp_ctx_stream(tgp_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int tgp_ctx_sm_count(const tgp_ctx* ctx) { return ctx ? ctx->sms : 0; }

int tgp_sync(tgp_ctx* ctx) {
    if (!ctx) return TGP_INVALID_ARG;
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    return TGP_OK;
}

int tgp_profile_enable(tgp_ctx* ctx, int on) {
    if (!ctx) return TGP_INVALID_ARG;
    ctx->profile = on != 0;
    ctx->profile_gate = on == 2;
    ctx->prof_used = 0;
    return TGP_OK;
}

int tgp_profile_read(tgp_ctx* ctx, uint64_t* launches, double* total_ms) {
    if (!ctx || !launches || !total_ms) return fail(ctx, TGP_INVALID_ARG, "null argument");
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    double t = 0.0;
    for (size_t i = 0; i < ctx->prof_used; ++i) {
        float ms = 0.f;
        TGP_CUDA(cudaEventElapsedTime(&ms, ctx->prof_events[i].first, ctx->prof_events[i].second));
        t += ms;
    }
    *launches = ctx->prof_used;
    *total_ms = t;
    ctx->prof_used = 0;
    return TGP_OK;
}

// --------------------------------------------------------------------------
// Tables
// --------------------------------------------------------------------------
static int compute_stats(tgp_ctx* ctx, Table& t) {
    if (t.cols.empty()) return TGP_OK;
    Carve cv;
    TGP_TRY(arena_reserve(ctx, t.cols.size() * 16, &cv));
    long long* mm = cv.take<long long>(2 * t.cols.size());
    std::vector<long long> init(2 * t.cols.size());
    for (size_t i = 0; i < t.cols.size(); ++i) {
        init[2 * i] = 0x7fffffffffffffffll;
        init[2 * i + 1] = static_cast<long long>(0x8000000000000000ull);
    }
    TGP_TRY(upload(ctx, mm, init.data(), init.size() * 8));
    for (size_t i = 0; i < t.cols.size(); ++i) {
        TGP_CUDA(launch_column_minmax(t.cols[i].dptr, t.cols[i].dtype, t.rows, mm + 2 * i, ctx->sms, ctx->stream));
    }
    std::vector<long long> res(2 * t.cols.size());
    TGP_CUDA(cudaMemcpyAsync(res.data(), mm, res.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < t.cols.size(); ++i) {
        t.cols[i].min = res[2 * i];
        t.cols[i].max = res[2 * i + 1];
        if (t.rows == 0) {
            t.cols[i].min = 0;
            t.cols[i].max = 0;
        }
    }
    return TGP_OK;
}

static int register_impl(tgp_ctx* ctx, const tgp_column_desc* cols, uint32_t ncols, uint64_t rows,
                         bool copy, tgp_table_id* out) {
    if (!ctx || !out || (ncols && !cols)) return fail(ctx, TGP_INVALID_ARG, "null argument");
    if (rows >= (1ull << 32)) return fail(ctx, TGP_UNSUPPORTED, "tables hold fewer than 2^32 rows (u32 row ids)");
    TGP_CUDA(cudaSetDevice(ctx->device));
    Table t;
    t.rows = rows;
    for (uint32_t i = 0; i < ncols; ++i) {
        Column c;
        c.dtype = cols[i].dtype;
        c.coltype = cols[i].coltype;
        c.width = dtype_width(c.dtype);
        if (c.width == 0) return fail(ctx, TGP_INVALID_ARG, "bad column dtype");
        if (c.coltype > TGP_CT_FLOAT) return fail(ctx, TGP_INVALID_ARG, "bad column coltype");
        if (rows && !cols[i].data) return fail(ctx, TGP_INVALID_ARG, "null column data");
        const size_t bytes = rows * c.width;
        if (copy) {
            // Pad to whole tiles so bulk copies of the last full tile stay in bounds.
            const size_t alloc = std::max<size_t>(16, ((bytes + 255) / 256) * 256);
            if (cudaMalloc(&c.dptr, alloc) != cudaSuccess) {
                cudaGetLastError();
                for (auto& p : t.cols) cudaFree(p.dptr);
                return fail(ctx, TGP_OOM, "column allocation failed");
            }
            c.owned = true;
            if (bytes) {
                cudaError_t e = cudaMemcpyAsync(c.dptr, cols[i].data, bytes, cudaMemcpyDefault, ctx->stream);
                if (e != cudaSuccess) {
                    for (auto& p : t.cols) cudaFree(p.dptr);
                    cudaFree(c.dptr);
                    return fail(ctx, TGP_DEVICE_ERROR, cudaGetErrorString(e));
                }
            }
        } else {
            if (rows && !is_device_ptr(cols[i].data)) return fail(ctx, TGP_INVALID_ARG, "column is not device memory");
            if (reinterpret_cast<uintptr_t>(cols[i].data) % 16 != 0)
                return fail(ctx, TGP_INVALID_ARG, "device column not 16-byte aligned");
            c.dptr = static_cast<uint8_t*>(const_cast<void*>(cols[i].data));
        }
        t.cols.push_back(c);
    }
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    int st = compute_stats(ctx, t);
    if (st != TGP_OK) {
        for (auto& c : t.cols)
            if (c.owned) cudaFree(c.dptr);
        return st;
    }
    const uint64_t id = ctx->next_id++;
    ctx->tables.emplace(id, std::move(t));
    *out = id;
    return TGP_OK;
}

int tgp_table_register(tgp_ctx* ctx, const tgp_column_desc* cols, uint32_t ncols, uint64_t rows,
                       tgp_table_id* out) {
    return register_impl(ctx, cols, ncols, rows, true, out);
}

int tgp_table_register_device(tgp_ctx* ctx, const tgp_column_desc* cols, uint32_t ncols, uint64_t rows,
                              tgp_table_id* out) {
    return register_impl(ctx, cols, ncols, rows, false, out);
}

int tgp_table_register_cells(tgp_ctx* ctx, const tgp_cell_column* cols, uint32_t ncols, uint64_t rows,
                             tgp_table_id* out) {
    if (!ctx || !out || (ncols && !cols)) return fail(ctx, TGP_INVALID_ARG, "null argument");
    if (rows >= (1ull << 32)) return fail(ctx, TGP_UNSUPPORTED, "tables hold fewer than 2^32 rows (u32 row ids)");
    TGP_CUDA(cudaSetDevice(ctx->device));
    Table t;
    t.rows = rows;
    uint8_t* cells = nullptr;  // device copy of the current column's cells
    auto give_up = [&](int st, const std::string& m) {
        cudaStreamSynchronize(ctx->stream);
        if (cells) cudaFree(cells);
        for (auto& c : t.cols) cudaFree(c.dptr);
        return fail(ctx, st, m);
    };
    // Whole 256-byte blocks, as tgp_table_register pads, so bulk copies of
    // the last tile stay in bounds.
    auto alloc = [&](uint8_t** p, size_t bytes) {
        if (cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(16, ((bytes + 255) / 256) * 256)) == cudaSuccess)
            return true;
        cudaGetLastError();
        *p = nullptr;
        return false;
    };
    Carve cv;
    TGP_TRY(arena_reserve(ctx, 16, &cv));
    long long* mm = cv.take<long long>(2);
    for (uint32_t i = 0; i < ncols; ++i) {
        const tgp_cell_column& in = cols[i];
        if (in.coltype > TGP_CT_FLOAT) return give_up(TGP_INVALID_ARG, "bad column coltype");
        Column c;
        c.coltype = in.coltype;
        c.owned = true;
        if (in.i32_sidecar) {
            c.dtype = DT_I32;
            c.width = 4;
            if (!alloc(&c.dptr, rows * 4)) return give_up(TGP_OOM, "column allocation failed");
            t.cols.push_back(c);
            if (rows && cudaMemcpyAsync(c.dptr, in.i32_sidecar, rows * 4, cudaMemcpyDefault, ctx->stream) != cudaSuccess)
                return give_up(TGP_DEVICE_ERROR, "sidecar copy failed");
            continue;
        }
        if (rows && !in.cells) return give_up(TGP_INVALID_ARG, "null column cells");
        if (!alloc(&cells, rows * 8)) return give_up(TGP_OOM, "column allocation failed");
        if (rows && cudaMemcpyAsync(cells, in.cells, rows * 8, cudaMemcpyDefault, ctx->stream) != cudaSuccess)
            return give_up(TGP_DEVICE_ERROR, "cell copy failed");
        uint32_t dt = in.coltype == TGP_CT_FLOAT ? DT_F64 : in.coltype == TGP_CT_DATE ? DT_U64 : DT_I64;
        if (in.coltype != TGP_CT_FLOAT && rows) {
            // Signed min / max of the cells; a Date column narrows only when
            // every cell is below 2^63 (signed and unsigned order agree).
            const long long init[2] = {0x7fffffffffffffffll, static_cast<long long>(0x8000000000000000ull)};
            if (upload(ctx, mm, init, 16) != TGP_OK) return give_up(TGP_DEVICE_ERROR, "statistics upload failed");
            long long r[2];
            if (launch_column_minmax(cells, DT_I64, rows, mm, ctx->sms, ctx->stream) != cudaSuccess ||
                cudaMemcpyAsync(r, mm, 16, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
                cudaStreamSynchronize(ctx->stream) != cudaSuccess)
                return give_up(TGP_DEVICE_ERROR, "column statistics failed");
            const long long lo = r[0], hi = r[1];
            if (lo >= 0 && hi <= 255) dt = DT_U8;
            else if (in.coltype == TGP_CT_INT ? (lo >= INT32_MIN && hi <= INT32_MAX) : (lo >= 0 && hi <= INT32_MAX))
                dt = DT_I32;
        }
        c.dtype = dt;
        c.width = dtype_width(dt);
        if (c.width == 8) {
            c.dptr = cells;
            cells = nullptr;
        } else {
            if (!alloc(&c.dptr, rows * c.width)) return give_up(TGP_OOM, "column allocation failed");
            t.cols.push_back(c);
            if (launch_narrow_cells(reinterpret_cast<const long long*>(cells), rows, c.dptr, dt, ctx->sms,
                                    ctx->stream) != cudaSuccess ||
                cudaStreamSynchronize(ctx->stream) != cudaSuccess)
                return give_up(TGP_DEVICE_ERROR, "cell narrowing failed");
            cudaFree(cells);
            cells = nullptr;
            continue;
        }
        t.cols.push_back(c);
    }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return give_up(TGP_DEVICE_ERROR, "column copy failed");
    if (int st = compute_stats(ctx, t)) {
        for (auto& c : t.cols) cudaFree(c.dptr);
        return st;
    }
    const uint64_t id = ctx->next_id++;
    ctx->tables.emplace(id, std::move(t));
    *out = id;
    return TGP_OK;
}

int tgp_table_column_dtype(tgp_ctx* ctx, tgp_table_id id, uint32_t col, uint32_t* dtype) {
    if (!ctx || !dtype) return fail(ctx, TGP_INVALID_ARG, "null argument");
    auto it = ctx->tables.find(id);
    if (it == ctx->tables.end()) return fail(ctx, TGP_NOT_FOUND, "unknown table id");
    if (col >= it->second.cols.size()) return fail(ctx, TGP_INVALID_ARG, "column index out of range");
    *dtype = it->second.cols[col].dtype;
    return TGP_OK;
}

int tgp_table_reload(tgp_ctx* ctx, tgp_table_id id, const tgp_column_desc* cols, uint32_t ncols) {
    if (!ctx || (ncols && !cols)) return fail(ctx, TGP_INVALID_ARG, "null argument");
    auto it = ctx->tables.find(id);
    if (it == ctx->tables.end()) return fail(ctx, TGP_NOT_FOUND, "unknown table id");
    Table& t = it->second;
    if (ncols != t.cols.size()) return fail(ctx, TGP_INVALID_ARG, "column count differs");
    for (uint32_t i = 0; i < ncols; ++i) {
        if (!t.cols[i].owned) return fail(ctx, TGP_INVALID_ARG, "reload of a borrowed device table");
        if (cols[i].dtype != t.cols[i].dtype) return fail(ctx, TGP_INVALID_ARG, "column dtype differs");
        if (t.rows)
            TGP_CUDA(cudaMemcpyAsync(t.cols[i].dptr, cols[i].data, t.rows * t.cols[i].width, cudaMemcpyDefault,
                                     ctx->stream));
    }
    return compute_stats(ctx, t);
}

int tgp_table_drop(tgp_ctx* ctx, tgp_table_id id) {
    if (!ctx) return TGP_INVALID_ARG;
    auto it = ctx->tables.find(id);
    if (it == ctx->tables.end()) return fail(ctx, TGP_NOT_FOUND, "unknown table id");
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    for (auto& c : it->second.cols)
        if (c.owned) cudaFree(c.dptr);
    ctx->tables.erase(it);
    return TGP_OK;
}

int tgp_table_info(tgp_ctx* ctx, tgp_table_id id, uint64_t* rows, uint32_t* ncols) {
    const Table* t;
    TGP_TRY(get_table(ctx, id, &t));
    if (rows) *rows = t->rows;
    if (ncols) *ncols = static_cast<uint32_t>(t->cols.size());
    return TGP_OK;
}

int tgp_table_column_stats(tgp_ctx* ctx, tgp_table_id id, uint32_t col, int64_t* mn, int64_t* mx) {
    const Table* t;
    TGP_TRY(get_table(ctx, id, &t));
    if (col >= t->cols.size()) return fail(ctx, TGP_INVALID_ARG, "column index out of range");
    if (mn) *mn = t->cols[col].min;
    if (mx) *mx = t->cols[col].max;
    return TGP_OK;
}

// --------------------------------------------------------------------------
// Filter → bitmap / row ids
// --------------------------------------------------------------------------
static int filter_impl(tgp_ctx* ctx, const Table* T, const tgp_pred_node* pred, uint32_t npred,
                       uint8_t* bitmap_out, uint32_t* rowids_out, uint64_t rowids_cap, uint64_t* count_out,
                       uint32_t first_words /* >0: only first words into bitmap_out (kernel table) */) {
    Builder b(ctx, T);
    TGP_TRY(b.add_pred(pred, npred));
    const uint64_t ntiles = (T->rows + kTileRows - 1) / kTileRows;
    const uint64_t nwords = (T->rows + 31) / 32;
    const bool need_words = bitmap_out || rowids_out || first_words;
    const uint64_t words = first_words ? std::min<uint64_t>(first_words, nwords) : (need_words ? nwords : 0);
    size_t cub_bytes = 0;
    if (rowids_out && ntiles) tile_prefix(nullptr, nullptr, ntiles, nullptr, &cub_bytes, ctx->stream);
    const bool host_rowids = rowids_out && !is_device_ptr(rowids_out);
    // Host row-id output is compacted into scratch first (worst case: all rows).
    const uint64_t rowid_scratch = host_rowids ? std::min<uint64_t>(T->rows, rowids_cap) : 0;
    Carve cv;
    TGP_TRY(arena_reserve(ctx, 64 + words * 4 + ntiles * 12 + cub_bytes + rowid_scratch * 4 + 2048, &cv));
    ScanScratch ss;
    ss.counters = cv.take<unsigned long long>(4);
    ss.err = cv.take<uint32_t>(4);
    uint32_t* bm = cv.take<uint32_t>(std::max<uint64_t>(words, 1));
    uint32_t* tc = cv.take<uint32_t>(std::max<uint64_t>(ntiles, 1));
    unsigned long long* tb = cv.take<unsigned long long>(std::max<uint64_t>(ntiles, 1));
    void* cub_tmp = cv.take<uint8_t>(cub_bytes + 16);
    uint32_t* rid_tmp = cv.take<uint32_t>(std::max<uint64_t>(rowid_scratch, 1));
    TGP_CUDA(cudaMemsetAsync(ss.counters, 0, 32, ctx->stream));
    TGP_CUDA(cudaMemsetAsync(ss.err, 0, 16, ctx->stream));
    if (words) TGP_CUDA(cudaMemsetAsync(bm, 0, words * 4, ctx->stream));
    if (rowids_out && ntiles) TGP_CUDA(cudaMemsetAsync(tc, 0, ntiles * 4, ctx->stream));
    Plan& P = b.P;
    P.bitmap = bm;
    P.bitmap_words = static_cast<uint32_t>(std::min<uint64_t>(words, 0xffffffffull));
    P.tile_counts = rowids_out ? tc : nullptr;
    P.counters = ss.counters;
    P.err = ss.err;
    TGP_TRY(size_smem(ctx, P, 0));
    TGP_TRY(launch(ctx, P, MODE_FILTER, false));
    unsigned long long cnt = 0;
    uint32_t err = 0;
    TGP_CUDA(cudaMemcpyAsync(&cnt, ss.counters, 8, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaMemcpyAsync(&err, ss.err, 4, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    TGP_TRY(check_kernel_err(ctx, err));
    if (count_out) *count_out = cnt;
    if (first_words) {
        TGP_TRY(copy_out(ctx, bitmap_out, bm, words * 4));
        TGP_CUDA(cudaStreamSynchronize(ctx->stream));
        return TGP_OK;
    }
    if (bitmap_out) TGP_TRY(copy_out(ctx, bitmap_out, bm, (T->rows + 7) / 8));
    if (rowids_out) {
        if (cnt > rowids_cap) {
            TGP_CUDA(cudaStreamSynchronize(ctx->stream));
            return fail(ctx, TGP_CAPACITY, "row-id buffer too small");
        }
        if (ntiles && cnt) {
            TGP_CUDA(tile_prefix(tc, tb, ntiles, cub_tmp, &cub_bytes, ctx->stream));
            if (!host_rowids) {
                TGP_CUDA(launch_compact(bm, nwords, ntiles, tb, rowids_out, rowids_cap, ctx->stream));
            } else {
                TGP_CUDA(launch_compact(bm, nwords, ntiles, tb, rid_tmp, cnt, ctx->stream));
                TGP_TRY(copy_out(ctx, rowids_out, rid_tmp, cnt * 4));
            }
        }
    }
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    return TGP_OK;
}

int tgp_filter(tgp_ctx* ctx, tgp_table_id table, const tgp_pred_node* pred, uint32_t npred, uint8_t* bitmap_out,
               uint32_t* rowids_out, uint64_t rowids_cap, uint64_t* count_out) {
    if (!ctx) return TGP_INVALID_ARG;
    const Table* T;
    TGP_TRY(get_table(ctx, table, &T));
    return filter_impl(ctx, T, pred, npred, bitmap_out, rowids_out, rowids_cap, count_out, 0);
}

// HyperLogLog estimate from 2^14 registers, in the reference's arithmetic
// (exec/hll.rs:53-76): sequential f64 sum of 2^-r in register order, raw =
// alpha * m^2 / sum, linear counting m * ln(m / zeros) when raw <= 2.5 m and
// some register is zero, truncated to u64.
static uint64_t hll_estimate(const std::vector<uint32_t>& regs) {
    constexpr double m = 16384.0;
    constexpr double alpha = 0.7213 / (1.0 + 1.079 / m);
    double sum = 0.0;
    uint64_t zeros = 0;
    for (uint32_t r : regs) {
        sum += std::ldexp(1.0, -static_cast<int>(r));
        zeros += r == 0;
    }
    const double raw = alpha * m * m / sum;
    const double est = (raw <= 2.5 * m && zeros > 0) ? m * std::log(m / static_cast<double>(zeros)) : raw;
    return static_cast<uint64_t>(est);
}

int tgp_hll_estimate(const uint32_t* regs, uint64_t* out) {
    if (!regs || !out) return TGP_INVALID_ARG;
    *out = hll_estimate(std::vector<uint32_t>(regs, regs + 16384));
    return TGP_OK;
}

int tgp_count_distinct(tgp_ctx* ctx, tgp_table_id table, uint32_t column, const tgp_pred_node* pred, uint32_t npred,
                       uint64_t* count, uint32_t* method) {
    if (!ctx || !count) return fail(ctx, TGP_INVALID_ARG, "null argument");
    *count = 0;
    if (method) *method = 0;
    const Table* T;
    TGP_TRY(get_table(ctx, table, &T));
    if (column >= T->cols.size()) return fail(ctx, TGP_INVALID_ARG, "column index out of range");
    const Column& c = T->cols[column];
    const uint64_t n = T->rows;
    // Selection: all rows, or the WHERE bitmap.
    uint32_t* bm = nullptr;
    uint64_t nsel = n;
    if (npred) {
        const uint64_t words = std::max<uint64_t>(1, (n + 31) / 32);
        TGP_TRY(dev_alloc(ctx, reinterpret_cast<void**>(&bm), words * 4, "selection bitmap allocation failed"));
        int st = TGP_OK;
        if (cudaMemsetAsync(bm, 0, words * 4, ctx->stream) != cudaSuccess) st = fail(ctx, TGP_DEVICE_ERROR, "memset");
        if (st == TGP_OK) st = filter_impl(ctx, T, pred, npred, reinterpret_cast<uint8_t*>(bm), nullptr, 0, &nsel, 0);
        if (st != TGP_OK) {
            dev_free(ctx, bm);
            return st;
        }
    }
    int st = TGP_OK;
    // The reference counts exactly below 100,000 selected rows and with a
    // HyperLogLog from there on (aggregate.rs:1308-1325, hll.rs:103-109).
    if (nsel < 100000) {
        const uint64_t cap = next_pow2(std::max<uint64_t>(16, 2 * nsel));
        Carve cv;
        st = arena_reserve(ctx, cap * 8 + 256, &cv);
        if (st == TGP_OK && nsel) {
            unsigned long long* set = cv.take<unsigned long long>(cap);
            unsigned long long* counters = cv.take<unsigned long long>(2);
            uint32_t* err = cv.take<uint32_t>(4);
            unsigned long long hc[2] = {0, 0};
            uint32_t herr = 0;
            cudaError_t e = cudaMemsetAsync(set, 0xff, cap * 8, ctx->stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, 16, ctx->stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, 16, ctx->stream);
            if (e == cudaSuccess)
                e = launch_distinct_cells(c.dptr, c.dtype, n, bm, set, cap - 1, log2u(cap), counters, err, ctx->sms,
                                          ctx->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(hc, counters, 16, cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) st = fail(ctx, TGP_DEVICE_ERROR, std::string("distinct: ") + cudaGetErrorString(e));
            if (st == TGP_OK) st = check_kernel_err(ctx, herr);
            if (st == TGP_OK) *count = hc[0] + (hc[1] ? 1 : 0);
        }
    } else {
        Carve cv;
        const uint64_t prow = static_cast<uint64_t>(hll_blocks(n, ctx->sms));
        st = arena_reserve(ctx, 16384 * 4 + prow * 16384 + 512, &cv);
        if (st == TGP_OK) {
            uint32_t* regs = cv.take<uint32_t>(16384);
            uint8_t* partial = cv.take<uint8_t>(std::max<uint64_t>(prow, 1) * 16384);
            std::vector<uint32_t> h(16384);
            cudaError_t e = launch_hll(c.dptr, c.dtype, n, bm, partial, regs, ctx->sms, ctx->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), regs, 16384 * 4, cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) st = fail(ctx, TGP_DEVICE_ERROR, std::string("hyperloglog: ") + cudaGetErrorString(e));
            if (st == TGP_OK) {
                *count = hll_estimate(h);
                if (method) *method = 1;
            }
        }
    }
    if (bm) {
        cudaStreamSynchronize(ctx->stream);
        dev_free(ctx, bm);
    }
    return st;
}

// --------------------------------------------------------------------------
// Aggregation queries
// --------------------------------------------------------------------------
static int join_lookup(tgp_ctx* ctx, tgp_join_id id, JoinTable** out) {
    auto it = ctx->joins.find(id);
    if (it == ctx->joins.end()) return fail(ctx, TGP_NOT_FOUND, "unknown join id");
    *out = &it->second;
    return TGP_OK;
}

static void attach_join(Plan& P, const JoinTable& J, int key_slot) {
    P.jtab = J.tab;
    P.jmask = J.cap - 1;
    P.jlog2 = J.log2;
    P.jwide = J.wide ? 1u : 0u;
    P.jslot = key_slot;
    P.jkmin = J.kmin;
    // An empty build side matches nothing: make every key fall out of range.
    P.jkrange = J.empty_range ? 0 : J.krange;
    if (J.empty_range) P.jkmin = 0;
}

// The class a query's scan variant is tuned for: its shape (join, number of
// group keys, values and predicate leaves, direct or hash grouping) and the
// binary orders of magnitude of its row count and of its group count bound.
static uint64_t tune_key_of(const tgp_query* q, const Plan& P, uint64_t rows, unsigned __int128 D) {
    auto log2ceil = [](unsigned __int128 x) -> uint64_t {
        uint64_t b = 0;
        while (b < 127 && (static_cast<unsigned __int128>(1) << b) < x) ++b;
        return b;
    };
    const unsigned __int128 groups = std::min<unsigned __int128>(D, std::max<uint64_t>(rows, 1));
    const uint64_t shape = (q->join ? 1ull : 0ull) | (static_cast<uint64_t>(std::min<uint32_t>(q->ngroup, 7)) << 1) |
                           (static_cast<uint64_t>(std::min<uint32_t>(P.nval, 15)) << 4) |
                           ((D > kDirectMaxGroups ? 1ull : 0ull) << 8) |
                           (static_cast<uint64_t>(std::min<uint32_t>(P.nleaf, 15)) << 9);
    return shape | (log2ceil(std::max<uint64_t>(rows, 1)) << 16) | (log2ceil(groups) << 24);
}

// A planned query: the lowered plan and what decoding its result block needs.
struct QueryState {
    const tgp_query* q = nullptr;
    const Table* T = nullptr;
    JoinTable* J = nullptr;
    std::vector<uint64_t> pay_sig;  // layout of the join payload the plan reads (JoinTable::pays key)
    std::unique_ptr<Builder> b;
    std::vector<AggMap> amap;
    uint32_t nv1 = 1;
    std::vector<uint64_t> dom;
    std::vector<int64_t> kmin;
    std::vector<uint32_t> bits;
    unsigned __int128 D = 1;
    uint32_t total_bits = 0;
    uint32_t mode = MODE_GROUP_PRIVATE;
    bool acc128 = false;
    uint64_t ngroups_direct = 1;
    size_t extra = 0;     // per-mode shared scratch bytes
    uint64_t hcap = 0;    // hash table slots (MODE_GROUP_HASH)
    uint64_t pending_dev_bytes = 0;  // device memory a dry plan would still allocate (join payload)
    Knobs kn;             // the scan variant this plan was made with
    uint64_t tune_key = 0;  // the query class the variant was looked up under
    uint64_t acc_words() const { return mode == MODE_GROUP_HASH ? 0 : ngroups_direct * nv1 * 2; }
    uint64_t block_words() const { return 6 + acc_words(); }  // [counters 4][error 2][accumulators]
    bool has_minmax() const {
        for (uint32_t v = 0; v < b->P.nval; ++v)
            if (b->P.val[v].kind == VK_MIN || b->P.val[v].kind == VK_MAX) return true;
        return false;
    }
};

// Lowers a query (predicate, aggregates, keys, join payload) and chooses its
// mode and shared-memory layout for a kernel with `static_smem` static bytes.
// `preseed` (optional) lists columns to stage first, in that order.
// Result pointers (counters, err, acc, htab) are left for the caller.
// Bucket keys (merged batch queries): group keys 0 .. nkeys-1 of the query
// are columns whose cells map to nbuckets[k] buckets through lut[k] (device,
// one u8 per cell of the column's [min, max]).
struct BucketSpec {
    uint32_t nkeys;
    const uint8_t* lut[kMaxGroupKeys];
    uint32_t nbuckets[kMaxGroupKeys];
};

static int plan_query(tgp_ctx* ctx, const tgp_query* q, QueryState& qs, size_t static_smem,
                      const std::vector<uint32_t>* preseed = nullptr, bool dry = false,
                      const BucketSpec* bucket = nullptr) {
    if (!ctx || !q) return fail(ctx, TGP_INVALID_ARG, "null argument");
    qs.q = q;
    TGP_TRY(get_table(ctx, q->table, &qs.T));
    const Table* T = qs.T;
    qs.b.reset(new Builder(ctx, T));
    Builder& b = *qs.b;
    b.static_smem = static_smem;
    // A shared scan stages the union of its queries' columns in one order.
    if (preseed)
        for (uint32_t c : *preseed) {
            int slot;
            TGP_TRY(b.slot_of(c, &slot));
        }
    JoinTable*& J = qs.J;
    J = nullptr;
    if (q->join) {
        TGP_TRY(join_lookup(ctx, q->join, &J));
        TGP_TRY(get_table(ctx, J->build_table, &b.B));
        b.J = J;
    }
    TGP_TRY(b.add_pred(q->pred, q->npred));
    if (J) {
        if (q->probe_key_column >= T->cols.size()) return fail(ctx, TGP_INVALID_ARG, "probe key column out of range");
        if (T->cols[q->probe_key_column].coltype == TGP_CT_FLOAT)
            return fail(ctx, TGP_UNSUPPORTED, "FLOAT join keys");
        int ks;
        TGP_TRY(b.slot_of(q->probe_key_column, &ks));
        attach_join(b.P, *J, ks);
    }
    std::vector<AggMap>& amap = qs.amap;
    TGP_TRY(lower_aggs(b, q->aggs, q->nagg, &amap));
    Plan& P = b.P;
    const uint32_t nv1 = qs.nv1 = P.nval + 1;

    // Group keys.
    if (q->ngroup > static_cast<uint32_t>(kMaxGroupKeys)) return fail(ctx, TGP_UNSUPPORTED, "more than 4 group keys");
    if (q->ngroup && !q->group) return fail(ctx, TGP_INVALID_ARG, "null group key list");
    std::vector<uint64_t>& dom = qs.dom;
    std::vector<int64_t>& kmin = qs.kmin;
    std::vector<uint32_t>& bits = qs.bits;
    dom.assign(q->ngroup, 0);
    kmin.assign(q->ngroup, 0);
    bits.assign(q->ngroup, 0);
    unsigned __int128& D = qs.D;
    D = 1;
    uint32_t& total_bits = qs.total_bits;
    total_bits = 0;
    for (uint32_t k = 0; k < q->ngroup; ++k) {
        const tgp_group_key& gk = q->group[k];
        const Table* S = gk.side == TGP_SIDE_BUILD ? b.B : T;
        if (!S) return fail(ctx, TGP_INVALID_ARG, "build-side group key without a join");
        if (gk.column >= S->cols.size()) return fail(ctx, TGP_INVALID_ARG, "group column out of range");
        const Column& c = S->cols[gk.column];
        GKey& K = P.gkey[k];
        std::memset(&K, 0, sizeof(K));
        if (gk.side == TGP_SIDE_BUILD) {
            K.build_side = 1;
            K.dtype = static_cast<uint8_t>(c.dtype);
            K.bptr = c.dptr;
            K.slot = -1;
        } else {
            int s;
            TGP_TRY(b.slot_of(gk.column, &s));
            K.slot = static_cast<int8_t>(s);
            K.dtype = static_cast<uint8_t>(b.P.slot[s].dtype);
            K.soff = b.P.slot[s].smem_off;
        }
        K.min = c.min;
        kmin[k] = c.min;
        uint64_t range = static_cast<uint64_t>(c.max) - static_cast<uint64_t>(c.min);
        if (bucket && k < bucket->nkeys) {
            K.lut = bucket->lut[k];
            range = bucket->nbuckets[k] - 1;
        }
        dom[k] = range == ~0ull ? 0 : range + 1;  // 0 = full 64-bit domain
        D = dom[k] ? D * dom[k] : (static_cast<unsigned __int128>(1) << 64) * D;
        uint32_t bw = 0;
        while (bw < 64 && (range >> bw) != 0) ++bw;
        bits[k] = bw;
        total_bits += bw;
    }
    P.ngkey = q->ngroup;
    if (bucket && D > kDirectMaxGroups) return fail(ctx, TGP_UNSUPPORTED, "bucketed groups beyond the direct limit");

    // The query's class and the scan variant for it: a tuned entry if the
    // autotuner measured this class, else the context's default (the
    // planner's rules).
    qs.tune_key = tune_key_of(q, P, T->rows, D);
    if (ctx->force_knobs) {
        qs.kn = *ctx->force_knobs;
    } else {
        auto it = ctx->tuned.find(qs.tune_key);
        qs.kn = it != ctx->tuned.end() ? it->second : ctx->knobs;
    }
    const Knobs& kn = qs.kn;

    // Join payload: with unique build keys over a dense key range, and no
    // build-side aggregate arguments, a probe row needs one lookup,
    // pay[key - kmin] = the build-side part of its group index.
    bool pay_ok = J && J->unique && !J->empty_range && kn.payload &&
                  J->krange + 1 <= std::min<uint64_t>(1ull << 28, std::max<uint64_t>(1ull << 22, 8 * J->entries));
    for (uint32_t v = 0; pay_ok && v < P.nval; ++v)
        for (uint32_t f = 0; f < P.val[v].nf; ++f) pay_ok = pay_ok && !P.val[v].f[f].build_side;

    uint32_t& mode = qs.mode;
    bool& acc128 = qs.acc128;
    acc128 = false;
    uint64_t& ngroups_direct = qs.ngroups_direct;
    ngroups_direct = 1;
    size_t& extra = qs.extra;
    extra = 0;
    const bool join = J != nullptr;
    // A scalar aggregate is the direct-indexed case with one group (D = 1).
    if (D <= kDirectMaxGroups) {
        ngroups_direct = static_cast<uint64_t>(D);
        P.ngroups = static_cast<uint32_t>(ngroups_direct);
        uint64_t stride = 1;
        for (int k = static_cast<int>(q->ngroup) - 1; k >= 0; --k) {
            P.gkey[k].stride = stride;
            stride *= dom[k];
        }
        acc128 = b.unbounded;
        // Per-thread private accumulators: int128 partials, or u32 row counts
        // and int64 values.
        auto private_bytes = [&](uint32_t nt) -> size_t {
            if (acc128) return static_cast<size_t>(ngroups_direct) * nv1 * 16 * nt;
            return priv_count_bytes(static_cast<uint32_t>(ngroups_direct), nt) +
                   static_cast<size_t>(ngroups_direct) * P.nval * 8 * nt;
        };
        const size_t shared_tab = static_cast<size_t>(ngroups_direct) * nv1 * 16;
        const size_t budget = ctx->max_dyn_smem - static_smem - kBarrierBytes;
        // 512 threads when two stages still fit beside them, else 256 threads
        // (twice the rows per thread).
        uint32_t nt = 0;
        const uint32_t first = kn.threads == 256 ? 256u : 512u;
        if (kn.placement <= 1 && ngroups_direct * static_cast<uint64_t>(nv1) * 512 < (1ull << 31))
            for (uint32_t cand : {first, 256u}) {
                if (private_bytes(cand) + 2 * static_cast<size_t>(P.stage_bytes) <= budget) {
                    nt = cand;
                    break;
                }
            }
        // When 512 threads' accumulators leave room for only two stages (one
        // tile in flight while the other is consumed) and 256 threads leave
        // room for four or more, the deeper pipeline wins: 60M-row join probe
        // with 25 groups 0.50 -> 0.46 ms. With three stages at 256 threads the
        // halved warp count loses (6M-row grouped aggregate 0.054 -> 0.068 ms).
        if (nt == 512 && P.stage_bytes && kn.threads == 0) {
            const size_t st = P.stage_bytes;
            const size_t s512 = budget > private_bytes(512) ? (budget - private_bytes(512)) / st : 0;
            const size_t s256 = budget > private_bytes(256) ? (budget - private_bytes(256)) / st : 0;
            if (s512 == 2 && std::min<size_t>(s256, static_cast<size_t>(kn.max_stages)) >= 4) nt = 256;
        }
        // Per-warp shared tables of 32-bit limbs with native shared atomics
        // (SUM / COUNT(col) values only): exact when every table's sums stay
        // below 2^63 in magnitude, which rows x max|value| < 2^63 proves (at
        // most one build match per probe row). Taken when the private
        // accumulators do not fit (or a variant asks for it).
        const uint32_t s32_words = 1 + 2 * P.nval;
        const uint32_t s32_nt = kn.threads == 256 ? 256u : 512u;
        // Bucketed (merged) plans take the limb tables whenever they are
        // exact: the private placement has no dense path for bucket keys
        // (a 2-member merged scan: 1.02 ms private, 0.51 ms limb tables).
        // So do joins through a payload array whose value program is one of
        // the fixed shapes: the 60M x 1.5M join probe ran 0.332 ms on the
        // limb tables (512 threads, four stages) against 0.374-0.387 ms with
        // private accumulators (autotuner, gated CUDA events).
        bool join_s32 = false;
        if (J && pay_ok && kn.placement == 0 && kn.dense && kn.shapes && !P.check_ovf &&
            compile_chain(b, pay_ok, static_cast<uint32_t>(kMaxGroupKeys))) {
            const uint32_t dv = P.dense_vec;
            P.dense_vec = 1;
            join_s32 = value_shape_of(P) != 0;
            P.dense_vec = dv;
        }
        const bool prefer_s32 = kn.placement == 4 || (bucket != nullptr && kn.placement == 0) || join_s32;
        auto s32_bytes = [&](uint32_t copies) -> size_t {
            return static_cast<size_t>(copies) * ngroups_direct * s32_words * 4;
        };
        uint32_t s32_copies = 0;
        {
            bool ok = !b.unbounded && (!J || J->unique) && kn.placement != 2 && kn.placement != 3 &&
                      (nt == 0 || prefer_s32);
            for (uint32_t v = 0; ok && v < P.nval; ++v)
                ok = P.val[v].kind == VK_SUM || P.val[v].kind == VK_COUNT_NZ;
            const unsigned __int128 bound = static_cast<unsigned __int128>(std::max<uint64_t>(T->rows, 1)) *
                                            std::max<uint64_t>(b.max_abs_val, 1);
            ok = ok && bound < (static_cast<unsigned __int128>(1) << 63);
            if (ok) {
                const size_t st = P.stage_bytes;
                uint32_t copies = s32_nt / 32;
                while (copies > 1 && s32_bytes(copies) + 3 * st > budget) copies >>= 1;
                if (s32_bytes(copies) + 2 * st <= budget) s32_copies = copies;
            }
        }
        if (nt && !(prefer_s32 && s32_copies)) {
            mode = MODE_GROUP_PRIVATE;
            P.nthreads = nt;
            P.count_by_tile = (q->ngroup == 0 && !J) ? 1u : 0u;
            extra = private_bytes(nt);
            if (!acc128) {
                // Flush before an int64 value partial could wrap or a u32 row
                // count could pass 2^32.
                const uint64_t lim = b.max_abs_val ? (0x7fffffffffffffffull / b.max_abs_val) : ~0ull;
                P.flush_limit = std::min<uint64_t>(std::max<uint64_t>(1, lim), 0xffffffffull);
            }
            // Dense column program: int64 partials, no join, no per-row
            // overflow checks.
            if (!acc128 && (!J || pay_ok) && !P.check_ovf && kn.dense && !bucket)
                P.dense_vec = compile_chain(b, pay_ok) ? 1u : 0u;
            // Scalar aggregates prefer the register fast path; a join's dense
            // program implies its payload path.
            if (!acc128) P.shape = scalar_shape_of(P);
            if (!P.shape && P.dense_vec && kn.shapes && (!J || pay_ok)) P.shape = dense_shape_of(P);
        } else if (s32_copies) {
            mode = MODE_GROUP_SHARED32;
            acc128 = false;
            P.nthreads = s32_nt;
            P.s32_copies = s32_copies;
            P.s32_words = s32_words;
            extra = s32_bytes(s32_copies);
            // Dense column program (keys of any count, bucket tables, the
            // join payload's build-side part), compiled ahead of time when
            // its value steps are one of the fixed shapes.
            if ((!J || pay_ok) && !P.check_ovf && kn.dense)
                P.dense_vec = compile_chain(b, pay_ok, static_cast<uint32_t>(kMaxGroupKeys)) ? 1u : 0u;
            if (P.dense_vec && kn.shapes) P.shape = value_shape_of(P);
        } else if (kn.placement != 3 && shared_tab + 2 * static_cast<size_t>(P.stage_bytes) <= budget) {
            mode = MODE_GROUP_SHARED;
            extra = shared_tab;
            acc128 = false;
            if (kn.threads == 256) P.nthreads = 256;
        } else {
            mode = MODE_GROUP_GLOBAL;
            acc128 = false;
            if (kn.threads == 256) P.nthreads = 256;
        }
    } else {
        mode = MODE_GROUP_HASH;
        if (kn.threads == 256) P.nthreads = 256;
        if (total_bits > 64 || (q->ngroup > 1 && total_bits > 63))
            return fail(ctx, TGP_UNSUPPORTED, "group key tuple wider than 63 bits");
        uint32_t shift = 0;
        for (int k = static_cast<int>(q->ngroup) - 1; k >= 0; --k) {
            P.gkey[k].shift = static_cast<uint8_t>(shift);
            shift += bits[k];
        }
        if (q->ngroup == 1 && bits[0] == 64 && dom[0] == 0)
            return fail(ctx, TGP_UNSUPPORTED, "group key spans all 2^64 values");
    }

    if (pay_ok && mode != MODE_GROUP_HASH) {
        PayKeys K;
        std::memset(&K, 0, sizeof(K));
        std::vector<uint64_t> sig;
        unsigned __int128 vmax = 0;  // the layout's largest payload value
        for (uint32_t k = 0; k < P.ngkey; ++k) {
            if (!P.gkey[k].build_side) continue;
            const Column& bc = b.B->cols[q->group[k].column];
            vmax += static_cast<unsigned __int128>(static_cast<uint64_t>(bc.max) - static_cast<uint64_t>(P.gkey[k].min)) *
                    P.gkey[k].stride;
            K.ptr[K.n] = P.gkey[k].bptr;
            K.dtype[K.n] = P.gkey[k].dtype;
            K.min[K.n] = P.gkey[k].min;
            K.stride[K.n] = P.gkey[k].stride;
            ++K.n;
            sig.insert(sig.end(), {q->group[k].column, static_cast<uint64_t>(P.gkey[k].min), P.gkey[k].stride});
        }
        // Payload entries as narrow as the layout's largest value allows (u8
        // below 255, u16 below 65,535; all ones = no match): the array is
        // read once per probe row, and a narrow one stays in L1 and L2. The
        // width follows from the layout alone, so every plan of one layout
        // reads the same array the same way.
        const uint32_t pw = vmax < 255 ? 1u : (vmax < 65535 ? 2u : 4u);
        sig.push_back(pw);
        const uint64_t entries = J->krange + 1;
        auto pt = J->pays.find(sig);
        if (dry) {
            // Sizing only (tgp_query_footprint): a payload still to be built
            // counts as memory the query needs; nothing is launched.
            if (pt == J->pays.end()) qs.pending_dev_bytes += entries * pw;
            P.jpay = pt != J->pays.end() ? pt->second.ptr : (J->pays.empty() ? nullptr : J->pays.begin()->second.ptr);
        } else {
            if (pt == J->pays.end()) {
                JoinTable::Payload np;
                np.width = pw;
                TGP_TRY(dev_alloc(ctx, reinterpret_cast<void**>(&np.ptr), std::max<uint64_t>(entries * pw, 16),
                                  "join payload allocation failed"));
                const cudaError_t e = launch_join_pay(J->tab, J->cap, K, np.ptr, pw, entries, ctx->sms, ctx->stream);
                if (e != cudaSuccess) {
                    dev_free(ctx, np.ptr);
                    return fail(ctx, TGP_DEVICE_ERROR, std::string("join payload: ") + cudaGetErrorString(e));
                }
                pt = J->pays.emplace(sig, np).first;
            }
            P.jpay = pt->second.ptr;
        }
        qs.pay_sig = sig;
        P.jpay_w = pw;
    }

    // Hash table sizing: 1.25x the bound on distinct groups, to a power of two.
    uint64_t& hcap = qs.hcap;
    hcap = 0;
    if (mode == MODE_GROUP_HASH) {
        const unsigned __int128 est = std::min<unsigned __int128>(D, static_cast<unsigned __int128>(std::max<uint64_t>(T->rows, 1)) *
                                                                          (join ? 4 : 1));
        P.hstride = 2 + 2 * P.nval;
        if (q->ngroup == 1 && !P.gkey[0].build_side && D <= kHashDirectMax && D <= 2 * static_cast<unsigned __int128>(std::max<uint64_t>(T->rows, 1))) {
            // One key over at most 2^27 values, no more than twice the rows:
            // a slot per key value, indexed by the key (no hashing, probing
            // or claiming), no larger than the hashed table would be.
            hcap = std::max<uint64_t>(16, static_cast<uint64_t>(D));
            P.hdirect = 1;
            P.hlog2 = log2u(next_pow2(hcap));
            P.hmask = hcap - 1;
        } else {
            // Distinct groups never exceed `est`: a load factor of at most 0.8
            // keeps linear probes short and the table (and its misses) small.
            hcap = next_pow2(std::max<uint64_t>(16, static_cast<uint64_t>(est) + static_cast<uint64_t>(est) / 4));
            P.hlog2 = log2u(hcap);
            P.hmask = hcap - 1;
        }
    }
    // One staged key and at most two SUM / COUNT(col) values of one staged
    // factor each: the column path of global / hash grouping.
    if ((mode == MODE_GROUP_HASH || mode == MODE_GROUP_GLOBAL) && !join && !P.check_ovf && P.ngkey == 1 && !bucket &&
        !P.gkey[0].build_side && P.gkey[0].slot >= 0 && P.nval <= 2) {
        bool ok = true;
        for (uint32_t v = 0; v < P.nval; ++v)
            ok = ok && (P.val[v].kind == VK_SUM || P.val[v].kind == VK_COUNT_NZ) && P.val[v].nf == 1 &&
                 P.val[v].f[0].slot >= 0;
        P.hash_fast = ok ? 1u : 0u;
    }
    // Sums that provably fit int64 (no per-row overflow, at most one build
    // match per row, rows x max|value| < 2^63) accumulate in the low limb with
    // non-returning adds; the high limb is the low one's sign.
    if ((!join || J->unique) && !P.check_ovf && !b.unbounded && !acc128) {
        const unsigned __int128 bound = static_cast<unsigned __int128>(std::max<uint64_t>(T->rows, 1)) *
                                        std::max<uint64_t>(b.max_abs_val, 1);
        if (bound < (static_cast<unsigned __int128>(1) << 63)) P.sum64 = 1;
    }
    // Shared pre-aggregation of repeated keys (hash and global direct
    // grouping): SUM / COUNT(col) values, no join, no per-row overflow checks;
    // its i32 partials are bounded once the launch grid is known.
    if (mode == MODE_GROUP_HASH || mode == MODE_GROUP_GLOBAL) {
        bool presum = kn.presum && !join && !P.check_ovf && !acc128;
        for (uint32_t v = 0; presum && v < P.nval; ++v)
            presum = P.val[v].kind == VK_SUM || P.val[v].kind == VK_COUNT_NZ;
        // u32 keys when every key is below 2^32 - 1 (the empty key): a packed
        // hash key of at most 31 bits, or a direct group index.
        const bool key32 = mode == MODE_GROUP_GLOBAL || total_bits <= 31;
        const uint32_t HS = 4096;
        const size_t bytes = static_cast<size_t>(HS) * ((key32 ? 8 : 12) + 4 * P.nval);
        const size_t budget = ctx->max_dyn_smem - static_smem - kBarrierBytes;
        if (presum && bytes + 2 * static_cast<size_t>(P.stage_bytes) <= budget) {
            P.hsm_slots = HS;
            P.hsm_log2 = log2u(HS);
            P.hsm_key32 = key32 ? 1u : 0u;
            extra = bytes;
        }
    }

    return TGP_OK;
}

// Keeps the shared pre-aggregation only when, at the grid launch() uses, no
// CTA scans enough rows for an i32 partial to reach 2^31 in magnitude.
static void bound_presum(tgp_ctx* ctx, QueryState& qs) {
    Plan& P = qs.b->P;
    if (!P.hsm_slots) return;
    const uint64_t ntiles = (P.nrows + kTileRows - 1) / kTileRows;
    const int occ = scan_occupancy(qs.mode, qs.acc128, static_cast<int>(P.nthreads), P.smem_bytes, P.shape);
    const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>(ntiles, static_cast<uint64_t>(ctx->sms) * std::max(occ, 1)));
    const unsigned __int128 rows_cta = static_cast<unsigned __int128>((ntiles + grid - 1) / grid) * kTileRows;
    const unsigned __int128 bound = rows_cta * std::max<uint64_t>(qs.b->max_abs_val, 1);
    if (bound >= (static_cast<unsigned __int128>(1) << 31)) P.hsm_slots = 0;
}

// A directly indexed table of COUNT(*) and at most one SUM / COUNT(col)
// whose fields provably never meet takes one-word slots (Plan::hpack): the
// count in the top bits (enough for every row), the sum of (value - its
// minimum) below. Groups formatted straight from the table only (no top-N,
// at most kMaxFormatAggs aggregates).
static void plan_one_word_slots(QueryState& qs, const tgp_query* q, bool topn) {
    Plan& P = qs.b->P;
    const Builder& b = *qs.b;
    if (!(qs.mode == MODE_GROUP_HASH && P.hdirect && P.hash_fast && P.nval <= 1 && !topn &&
          q->nagg <= static_cast<uint32_t>(kMaxFormatAggs) && P.ngkey == 1 && P.gkey[0].shift == 0 &&
          (!P.hsm_slots || P.hsm_key32) && (P.nval == 0 || !b.val_big[0])))
        return;
    const uint64_t rows = std::max<uint64_t>(qs.T->rows, 1);
    const uint32_t cbits = 64u - static_cast<uint32_t>(__builtin_clzll(rows));  // count <= rows < 2^cbits
    const uint32_t shift = P.nval ? 64u - cbits : 0u;
    const __int128 span = P.nval ? b.val_hi[0] - b.val_lo[0] : 0;
    const bool fits = P.nval == 0 || (shift < 64 && static_cast<unsigned __int128>(span) * rows <
                                                       (static_cast<unsigned __int128>(1) << shift));
    if (fits && (P.nval == 0 || (b.val_lo[0] >= INT64_MIN && b.val_lo[0] <= INT64_MAX))) {
        P.hpack = 1;
        P.hpack_shift = shift;
        P.hpack_bias = P.nval ? static_cast<int64_t>(b.val_lo[0]) : 0;
        P.hstride = 1;
    }
}

// Fills the caller's outputs of a direct-indexed / scalar query from a host
// copy of its result block.
static int decode_direct(tgp_ctx* ctx, const QueryState& qs, const unsigned long long* hb, uint64_t* keys_out,
                         tgp_agg_value* vals_out, uint64_t group_cap, tgp_query_result* result) {
    const tgp_query* q = qs.q;
    const Plan& P = qs.b->P;
    const uint32_t nv1 = qs.nv1;
    const uint64_t ngroups_direct = qs.ngroups_direct;
    const std::vector<uint64_t>& dom = qs.dom;
    const std::vector<int64_t>& kmin = qs.kmin;
    const std::vector<AggMap>& amap = qs.amap;
    const uint32_t nagg = q->nagg;
    const uint32_t err = static_cast<uint32_t>(hb[4] & 0xffffffffull);
    TGP_TRY(check_kernel_err(ctx, err));
    result->rows_scanned = qs.T->rows;
    result->rows_selected = hb[0];
    result->flags = (err & kErrRowOverflow) ? TGP_RESULT_ROW_OVERFLOW : 0u;
    const unsigned long long* accv = hb + 6;
        // Direct / scalar: emit groups with a nonzero row count in index order
        // (index order is ascending lexicographic key order).
        std::vector<uint64_t> present;
        if (q->ngroup == 0) {
            present.push_back(0);
        } else {
            for (uint64_t g = 0; g < ngroups_direct; ++g)
                if (accv[g * nv1 * 2] != 0) present.push_back(g);
        }
        result->ngroups = present.size();
        if (present.size() > group_cap) return fail(ctx, TGP_CAPACITY, "group buffer too small");
        for (size_t i = 0; i < present.size(); ++i) {
            const uint64_t g = present[i];
            if (keys_out) {
                for (uint32_t k = 0; k < q->ngroup; ++k) {
                    const uint64_t digit = (g / P.gkey[k].stride) % dom[k];
                    keys_out[i * q->ngroup + k] = static_cast<uint64_t>(kmin[k]) + digit;
                }
            }
            if (vals_out)
                for (uint32_t a = 0; a < nagg; ++a) fill_value(amap[a], accv + g * nv1 * 2, P, &vals_out[i * nagg + a]);
        }
        return TGP_OK;
    }

// ORDER BY one aggregate, LIMIT n (tgp_execute_topn).
struct TopNReq {
    uint32_t agg;
    bool desc;
    uint64_t limit;
};

// Keeps the first min(limit, n) of n decoded groups in the order of one
// aggregate's exact value (AVG: its f64), ties in the given (key) order.
static void host_topn(const TopNReq& tn, uint32_t nkey, uint32_t nagg, const std::vector<uint64_t>& keys,
                      const std::vector<tgp_agg_value>& vals, uint64_t n, uint32_t func, uint64_t* keys_out,
                      tgp_agg_value* vals_out, tgp_query_result* result) {
    std::vector<uint64_t> order(n);
    for (uint64_t i = 0; i < n; ++i) order[i] = i;
    auto less = [&](uint64_t x, uint64_t y) {
        const tgp_agg_value& a = vals[x * nagg + tn.agg];
        const tgp_agg_value& b = vals[y * nagg + tn.agg];
        if (func == TGP_AGG_AVG) return tn.desc ? a.as_f64 > b.as_f64 : a.as_f64 < b.as_f64;
        const __int128 va = (static_cast<__int128>(a.hi) << 64) | static_cast<__int128>(a.lo);
        const __int128 vb = (static_cast<__int128>(b.hi) << 64) | static_cast<__int128>(b.lo);
        return tn.desc ? va > vb : va < vb;
    };
    std::stable_sort(order.begin(), order.end(), less);
    const uint64_t m = std::min<uint64_t>(tn.limit, n);
    for (uint64_t i = 0; i < m; ++i) {
        if (keys_out)
            for (uint32_t k = 0; k < nkey; ++k) keys_out[i * nkey + k] = keys[order[i] * nkey + k];
        if (vals_out)
            for (uint32_t a = 0; a < nagg; ++a) vals_out[i * nagg + a] = vals[order[i] * nagg + a];
    }
    result->ngroups = m;
}

static int execute_impl(tgp_ctx* ctx, const tgp_query* q, uint64_t* keys_out, tgp_agg_value* vals_out,
                        uint64_t group_cap, tgp_query_result* result, const TopNReq* tn) {
    if (!ctx || !q || !result) return fail(ctx, TGP_INVALID_ARG, "null argument");
    std::memset(result, 0, sizeof(*result));
    if (tn && tn->agg >= q->nagg) return fail(ctx, TGP_INVALID_ARG, "ORDER BY aggregate index out of range");
    QueryState qs;
    TGP_TRY(plan_query(ctx, q, qs, scan_kernel_static_smem()));
    Builder& b = *qs.b;
    Plan& P = b.P;
    const Table* T = qs.T;
    const uint32_t mode = qs.mode;
    const bool acc128 = qs.acc128;
    const uint64_t ngroups_direct = qs.ngroups_direct;
    const size_t extra = qs.extra;
    const uint64_t hcap = qs.hcap;
    const uint32_t nv1 = qs.nv1;
    const std::vector<uint32_t>& bits = qs.bits;
    const std::vector<int64_t>& kmin = qs.kmin;
    const std::vector<AggMap>& amap = qs.amap;
    const unsigned __int128 D = qs.D;
    const uint32_t total_bits = qs.total_bits;
    (void)nv1;

    plan_one_word_slots(qs, q, tn != nullptr);

    // Scratch: accumulators (direct/scalar) or hash table, counters, error word.
    const uint64_t acc_words = qs.acc_words();
    const uint64_t htab_words = hcap * P.hstride;
    Carve cv;
    TGP_TRY(arena_reserve(ctx, acc_words * 8 + htab_words * 8 + 1024, &cv));
    // One result block [counters: 4 words][error word: 2 words][accumulators],
    // cleared with one memset and read back with one copy.
    const uint64_t block_words = qs.block_words();
    unsigned long long* block = cv.take<unsigned long long>(block_words);
    P.counters = block;
    P.err = reinterpret_cast<uint32_t*>(block + 4);
    P.acc = acc_words ? block + 6 : cv.take<unsigned long long>(2);
    P.htab = mode == MODE_GROUP_HASH ? cv.take<unsigned long long>(htab_words) : nullptr;
    bool has_minmax = false;
    for (uint32_t v = 0; v < P.nval; ++v) has_minmax |= (P.val[v].kind == VK_MIN || P.val[v].kind == VK_MAX);
    if (acc_words && has_minmax) {
        TGP_CUDA(cudaMemsetAsync(block, 0, 48, ctx->stream));
        std::vector<unsigned long long> img;
        init_acc_image(P, ngroups_direct, &img);
        TGP_TRY(upload(ctx, P.acc, img.data(), img.size() * 8));
    } else {
        TGP_CUDA(cudaMemsetAsync(block, 0, block_words * 8, ctx->stream));
    }
    if (mode == MODE_GROUP_HASH && P.hpack) {
        TGP_CUDA(cudaMemsetAsync(P.htab, 0, hcap * 8, ctx->stream));
    } else if (mode == MODE_GROUP_HASH) {
        // Keys EMPTY, counters 0, value limbs: MIN/MAX identity or 0 (one pass).
        SlotImage img;
        std::memset(&img, 0, sizeof(img));
        img.stride = P.hstride;
        img.w[0] = kEmptySlot;
        for (uint32_t v = 0; v < P.nval; ++v) {
            if (P.val[v].kind == VK_MIN) img.w[2 + 2 * v] = 0x7fffffffffffffffull;
            if (P.val[v].kind == VK_MAX) img.w[2 + 2 * v] = 0x8000000000000000ull;
        }
        TGP_CUDA(launch_fill_slots(P.htab, hcap, img, ctx->sms, ctx->stream));
    }
    TGP_TRY(size_smem(ctx, P, extra, scan_kernel_static_smem(), &qs.kn));
    bound_presum(ctx, qs);
    if (P.hpack && P.nleaf == 0 && P.hash_fast && !ctx->dbg_skip_tile1 &&
        direct_group_supported(P.slot[P.gkey[0].slot].dtype, P.nval ? P.slot[P.val[0].f[0].slot].dtype : 0u)) {
        TGP_TRY(launch_direct_groups(ctx, P, b.max_abs_val));
    } else {
        bool done = false;
        TGP_TRY(try_launch_q1(ctx, P, mode, acc128, ngroups_direct, b.max_abs_val, &done));
        if (!done) TGP_TRY(launch(ctx, P, mode, acc128));
    }

    TGP_TRY(pinned_reserve(ctx, block_words * 8));
    TGP_CUDA(cudaMemcpyAsync(ctx->hpin, block, block_words * 8, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    const unsigned long long* hb = reinterpret_cast<const unsigned long long*>(ctx->hpin);
    unsigned long long counters[4] = {hb[0], hb[1], hb[2], hb[3]};
    const uint32_t err = static_cast<uint32_t>(hb[4] & 0xffffffffull);
    TGP_TRY(check_kernel_err(ctx, err));

    result->rows_scanned = T->rows;
    result->rows_selected = counters[0];
    result->flags = (err & kErrRowOverflow) ? TGP_RESULT_ROW_OVERFLOW : 0u;
    const uint32_t nagg = q->nagg;

    if (mode != MODE_GROUP_HASH) {
        if (!tn) return decode_direct(ctx, qs, hb, keys_out, vals_out, group_cap, result);
        std::vector<uint64_t> ak(std::max<uint64_t>(1, ngroups_direct * q->ngroup));
        std::vector<tgp_agg_value> av(std::max<uint64_t>(1, ngroups_direct * q->nagg));
        TGP_TRY(decode_direct(ctx, qs, hb, ak.data(), av.data(), ngroups_direct, result));
        host_topn(*tn, q->ngroup, q->nagg, ak, av, result->ngroups, amap[tn->agg].func, keys_out, vals_out, result);
        return TGP_OK;
    }

    auto hash_format = [&]() {
        HashFormat F;
        std::memset(&F, 0, sizeof(F));
        F.nkey = q->ngroup;
        F.nagg = nagg;
        F.hstride = P.hstride;
        F.sum64 = P.sum64;
        F.hpack = P.hpack;
        F.hpack_shift = P.hpack_shift;
        F.hpack_bias = P.hpack_bias;
        for (uint32_t k = 0; k < q->ngroup; ++k) {
            F.key_shift[k] = P.gkey[k].shift;
            F.key_mask[k] = bits[k] >= 64 ? ~0ull : ((1ull << bits[k]) - 1);
            F.key_min[k] = kmin[k];
        }
        for (uint32_t a = 0; a < nagg; ++a) {
            F.func[a] = static_cast<uint8_t>(amap[a].func);
            F.val[a] = static_cast<int8_t>(amap[a].val);
            F.kind[a] = amap[a].val >= 0 ? P.val[amap[a].val].kind : VK_SUM;
        }
        return F;
    };
    // Hash groups: gather occupied slots, sort by key on the host.
    // Counter word 2 counts the gathered slots.
    TGP_CUDA(cudaMemsetAsync(P.counters + 2, 0, 8, ctx->stream));
    if (P.hdirect && !tn && nagg <= static_cast<uint32_t>(kMaxFormatAggs)) {
        // A directly indexed table holds the groups in key order already:
        // count the occupied slots, then format them in place of a gather
        // and a sort.
        const size_t sb = direct_groups_scratch(hcap);
        uint8_t* scr = nullptr;
        TGP_TRY(dev_alloc(ctx, reinterpret_cast<void**>(&scr), sb, "group count allocation failed"));
        unsigned long long ng = 0;
        cudaError_t e = count_direct_groups(P.htab, hcap, P.hstride, scr, sb, P.counters + 2, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&ng, P.counters + 2, 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            dev_free(ctx, scr);
            return fail(ctx, TGP_DEVICE_ERROR, std::string("group count: ") + cudaGetErrorString(e));
        }
        result->ngroups = ng;
        if (ng > group_cap) {
            dev_free(ctx, scr);
            return fail(ctx, TGP_CAPACITY, "group buffer too small");
        }
        const HashFormat F = hash_format();
        const size_t kbytes = (keys_out ? ng * q->ngroup * 8 : 0), vbytes = (vals_out ? ng * nagg * sizeof(tgp_agg_value) : 0);
        uint8_t* buf = nullptr;
        const size_t vofs = (kbytes + 255) & ~size_t{255};
        if (int st = dev_alloc(ctx, reinterpret_cast<void**>(&buf), std::max<size_t>(vofs + vbytes, 256),
                               "group format allocation failed")) {
            dev_free(ctx, scr);
            return st;
        }
        uint64_t* dkeys = kbytes ? reinterpret_cast<uint64_t*>(buf) : nullptr;
        tgp_agg_value* dvals = vbytes ? reinterpret_cast<tgp_agg_value*>(buf + vofs) : nullptr;
        e = format_direct_groups(P.htab, hcap, scr, ng, F, dkeys, dvals, ctx->stream);
        if (e == cudaSuccess && kbytes) e = cudaMemcpyAsync(keys_out, dkeys, kbytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess && vbytes) e = cudaMemcpyAsync(vals_out, dvals, vbytes, cudaMemcpyDeviceToHost, ctx->stream);
        dev_free(ctx, buf);
        dev_free(ctx, scr);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return fail(ctx, TGP_DEVICE_ERROR, std::string("group format: ") + cudaGetErrorString(e));
        return TGP_OK;
    }
    unsigned long long* packed = nullptr;
    const uint64_t max_groups = std::min<uint64_t>(hcap, static_cast<uint64_t>(std::min<unsigned __int128>(D, hcap)));
    TGP_TRY(dev_alloc(ctx, reinterpret_cast<void**>(&packed), std::max<uint64_t>(max_groups, 1) * P.hstride * 8,
                      "group gather allocation failed"));
    TGP_CUDA(launch_gather_groups(P.htab, hcap, P.hstride, packed, max_groups, P.counters + 2, ctx->sms, ctx->stream,
                                  P.hdirect != 0));
    unsigned long long ng = 0;
    TGP_CUDA(cudaMemcpyAsync(&ng, P.counters + 2, 8, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    result->ngroups = ng;
    if (!tn && ng > group_cap) {
        dev_free(ctx, packed);
        return fail(ctx, TGP_CAPACITY, "group buffer too small");
    }
    if (nagg <= static_cast<uint32_t>(kMaxFormatAggs)) {
        // Sort by packed key (= ascending lexicographic key order, key 0 in
        // the top bits) and format on the device; copy the caller's arrays once.
        const HashFormat F = hash_format();
        // Top-N: only the first min(limit, ng) groups in the aggregate's order
        // are formatted and copied.
        const uint64_t nout = tn ? std::min<uint64_t>(tn->limit, ng) : ng;
        const size_t sbytes = format_hash_groups_scratch(ng, tn ? 64u : total_bits);
        const size_t kbytes = (keys_out ? nout * q->ngroup * 8 : 0),
                     vbytes = (vals_out ? nout * nagg * sizeof(tgp_agg_value) : 0);
        uint8_t* buf = nullptr;
        const size_t kofs = (sbytes + 255) & ~size_t{255}, vofs = kofs + ((kbytes + 255) & ~size_t{255});
        if (int st = dev_alloc(ctx, reinterpret_cast<void**>(&buf), vofs + vbytes, "group format allocation failed")) {
            dev_free(ctx, packed);
            return st;
        }
        uint64_t* dkeys = kbytes ? reinterpret_cast<uint64_t*>(buf + kofs) : nullptr;
        tgp_agg_value* dvals = vbytes ? reinterpret_cast<tgp_agg_value*>(buf + vofs) : nullptr;
        cudaError_t e;
        if (tn) {
            TopNSpec S;
            std::memset(&S, 0, sizeof(S));
            S.val = amap[tn->agg].val;
            S.kind = static_cast<uint8_t>(S.val >= 0 ? P.val[S.val].kind : VK_SUM);
            S.func = static_cast<uint8_t>(amap[tn->agg].func);
            S.desc = tn->desc ? 1 : 0;
            S.sum64 = P.sum64 ? 1 : 0;
            e = topn_hash_groups(packed, ng, F, total_bits, S, nout, buf, sbytes, dkeys, dvals, ctx->sms, ctx->stream);
            result->ngroups = nout;
        } else {
            e = format_hash_groups(packed, ng, F, total_bits, buf, sbytes, dkeys, dvals, ctx->sms, ctx->stream);
        }
        if (e == cudaSuccess && kbytes) e = cudaMemcpyAsync(keys_out, dkeys, kbytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess && vbytes) e = cudaMemcpyAsync(vals_out, dvals, vbytes, cudaMemcpyDeviceToHost, ctx->stream);
        dev_free(ctx, buf);
        dev_free(ctx, packed);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return fail(ctx, TGP_DEVICE_ERROR, std::string("group format: ") + cudaGetErrorString(e));
        return TGP_OK;
    }
    if (tn) {
        dev_free(ctx, packed);
        return fail(ctx, TGP_UNSUPPORTED, "ORDER BY with more aggregates than the device formatter takes");
    }
    std::vector<unsigned long long> slots(ng * P.hstride);
    if (ng) TGP_CUDA(cudaMemcpyAsync(slots.data(), packed, ng * P.hstride * 8, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    dev_free(ctx, packed);
    // Packed key order == ascending lexicographic key order (key 0 in the top bits).
    std::vector<uint64_t> order(ng);
    for (uint64_t i = 0; i < ng; ++i) order[i] = i;
    std::sort(order.begin(), order.end(),
              [&](uint64_t x, uint64_t y) { return slots[x * P.hstride] < slots[y * P.hstride]; });
    std::vector<unsigned long long> tmp(nv1 * 2);
    for (uint64_t i = 0; i < ng; ++i) {
        const unsigned long long* s = &slots[order[i] * P.hstride];
        if (keys_out) {
            for (uint32_t k = 0; k < q->ngroup; ++k) {
                const uint64_t mask = bits[k] >= 64 ? ~0ull : ((1ull << bits[k]) - 1);
                const uint64_t rel = (s[0] >> P.gkey[k].shift) & mask;
                keys_out[i * q->ngroup + k] = static_cast<uint64_t>(kmin[k]) + rel;
            }
        }
        if (vals_out) {
            tmp[0] = s[1];
            tmp[1] = 0;
            for (uint32_t v = 0; v < P.nval; ++v) {
                tmp[2 * (v + 1)] = s[2 + 2 * v];
                tmp[2 * (v + 1) + 1] = s[3 + 2 * v];
            }
            for (uint32_t a = 0; a < nagg; ++a) fill_value(amap[a], tmp.data(), P, &vals_out[i * nagg + a]);
        }
    }
    return TGP_OK;
}

int tgp_execute(tgp_ctx* ctx, const tgp_query* q, uint64_t* keys_out, tgp_agg_value* vals_out, uint64_t group_cap,
                tgp_query_result* result) {
    return execute_impl(ctx, q, keys_out, vals_out, group_cap, result, nullptr);
}

int tgp_execute_topn(tgp_ctx* ctx, const tgp_query* q, uint32_t order_agg, int descending, uint64_t limit,
                     uint64_t* keys_out, tgp_agg_value* vals_out, tgp_query_result* result) {
    const TopNReq tn{order_agg, descending != 0, limit};
    return execute_impl(ctx, q, keys_out, vals_out, limit, result, &tn);
}

int tgp_query_footprint(tgp_ctx* ctx, const tgp_query* q, uint64_t* device_bytes) {
    if (!ctx || !q || !device_bytes) return fail(ctx, TGP_INVALID_ARG, "null argument");
    QueryState qs;
    TGP_TRY(plan_query(ctx, q, qs, scan_kernel_static_smem(), nullptr, /*dry=*/true));
    plan_one_word_slots(qs, q, false);
    const Plan& P = qs.b->P;
    // What execute_impl carves or allocates for one run of the query.
    uint64_t bytes = qs.block_words() * 8 + 1024 + qs.pending_dev_bytes;
    if (qs.mode == MODE_GROUP_HASH) {
        const uint64_t slot_bytes = static_cast<uint64_t>(P.hstride) * 8;
        const uint64_t max_groups =
            std::min<uint64_t>(qs.hcap, static_cast<uint64_t>(std::min<unsigned __int128>(qs.D, qs.hcap)));
        bytes += qs.hcap * slot_bytes;                                    // the group table
        if (P.hdirect && q->nagg <= static_cast<uint32_t>(kMaxFormatAggs)) {
            bytes += direct_groups_scratch(qs.hcap);                      // prefix counts of occupied slots
        } else {
            bytes += max_groups * slot_bytes;                             // gathered occupied slots
            bytes += format_hash_groups_scratch(max_groups, qs.total_bits);  // device sort
        }
        bytes += max_groups * (8ull * q->ngroup + sizeof(tgp_agg_value) * q->nagg) + 512;  // formatted result
    }
    *device_bytes = bytes;
    return TGP_OK;
}

int tgp_debug_fail_next_scan(tgp_ctx* ctx, uint64_t tile, uint64_t wait_ns) {
    if (!ctx) return TGP_INVALID_ARG;
    if (wait_ns < 1000000ull || wait_ns > 1000000000ull)
        return fail(ctx, TGP_INVALID_ARG, "wait limit between 1 ms and 1 s");
    ctx->dbg_skip_tile1 = tile + 1;
    ctx->dbg_wait_ns = wait_ns;
    return TGP_OK;
}

// --------------------------------------------------------------------------
// String columns and LIKE
// --------------------------------------------------------------------------
int tgp_strings_register(tgp_ctx* ctx, const uint8_t* bytes, uint64_t nbytes, const uint64_t* offsets, uint64_t n,
                         tgp_strings_id* out) {
    if (!ctx || !out || !offsets || (nbytes && !bytes)) return fail(ctx, TGP_INVALID_ARG, "null argument");
    if (is_device_ptr(offsets) || (bytes && is_device_ptr(bytes)))
        return fail(ctx, TGP_INVALID_ARG, "string columns are registered from host memory");
    // The kernel trusts the offsets: check them here.
    if (offsets[0] != 0 || offsets[n] != nbytes) return fail(ctx, TGP_INVALID_ARG, "offsets must run from 0 to nbytes");
    for (uint64_t i = 0; i < n; ++i) {
        if (offsets[i + 1] < offsets[i]) return fail(ctx, TGP_INVALID_ARG, "offsets must not decrease");
        if (offsets[i + 1] - offsets[i] >= (1ull << 31)) return fail(ctx, TGP_UNSUPPORTED, "a string of 2 GiB or more");
    }
    StringColumn c;
    c.n = n;
    c.nbytes = nbytes;
    if (int st = dev_alloc(ctx, reinterpret_cast<void**>(&c.offs), (n + 1) * 8, "string offsets allocation failed"))
        return st;
    if (int st = dev_alloc(ctx, reinterpret_cast<void**>(&c.bytes), std::max<uint64_t>(nbytes, 16), "string bytes allocation failed")) {
        dev_free(ctx, c.offs);
        return st;
    }
    int st = upload(ctx, c.offs, offsets, (n + 1) * 8);
    if (st == TGP_OK && nbytes) st = upload(ctx, c.bytes, bytes, nbytes);
    if (st == TGP_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) st = fail(ctx, TGP_DEVICE_ERROR, "string upload");
    if (st != TGP_OK) {
        dev_free(ctx, c.offs);
        dev_free(ctx, c.bytes);
        return st;
    }
    const uint64_t id = ctx->next_id++;
    ctx->strings.emplace(id, c);
    *out = id;
    return TGP_OK;
}

int tgp_strings_drop(tgp_ctx* ctx, tgp_strings_id id) {
    if (!ctx) return TGP_INVALID_ARG;
    auto it = ctx->strings.find(id);
    if (it == ctx->strings.end()) return fail(ctx, TGP_NOT_FOUND, "unknown string column id");
    cudaStreamSynchronize(ctx->stream);
    dev_free(ctx, it->second.offs);
    dev_free(ctx, it->second.bytes);
    ctx->strings.erase(it);
    return TGP_OK;
}

int tgp_like(tgp_ctx* ctx, tgp_strings_id id, const char* pattern, uint32_t pattern_len, int negated,
             uint8_t* bitmap_out, uint64_t* count_out) {
    if (!ctx || !count_out || (pattern_len && !pattern)) return fail(ctx, TGP_INVALID_ARG, "null argument");
    if (pattern_len > kLikeMaxPattern) return fail(ctx, TGP_UNSUPPORTED, "LIKE pattern longer than 256 bytes");
    auto it = ctx->strings.find(id);
    if (it == ctx->strings.end()) return fail(ctx, TGP_NOT_FOUND, "unknown string column id");
    const StringColumn& c = it->second;
    LikePattern P;
    std::memset(&P, 0, sizeof(P));
    P.len = pattern_len;
    if (pattern_len) std::memcpy(P.b, pattern, pattern_len);
    const uint64_t nwords = (c.n + 31) / 32;
    Carve cv;
    TGP_TRY(arena_reserve(ctx, nwords * 4 + 1024, &cv));
    unsigned long long* block = cv.take<unsigned long long>(4);   // [count][error]
    uint32_t* words = cv.take<uint32_t>(std::max<uint64_t>(nwords, 1));
    TGP_CUDA(cudaMemsetAsync(block, 0, 32, ctx->stream));
    TGP_CUDA(launch_like(c.bytes, c.offs, c.n, P, negated != 0, words, block, reinterpret_cast<uint32_t*>(block + 1),
                         ctx->sms, ctx->stream));
    if (bitmap_out && c.n)
        TGP_CUDA(cudaMemcpyAsync(bitmap_out, words, (c.n + 7) / 8, cudaMemcpyDefault, ctx->stream));
    unsigned long long hb[2] = {0, 0};
    TGP_CUDA(cudaMemcpyAsync(hb, block, 16, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    if (hb[1]) return fail(ctx, TGP_DEVICE_ERROR, "LIKE matching exceeded its step bound");
    *count_out = hb[0];
    return TGP_OK;
}

// --------------------------------------------------------------------------
// Scan variants and the autotuner
// --------------------------------------------------------------------------
static Knobs knobs_from(const tgp_variant& v) {
    Knobs k;
    k.threads = v.threads == 256 ? 256 : v.threads == 512 ? 512 : 0;
    k.max_stages = v.max_stages ? std::min<int>(static_cast<int>(v.max_stages), kMaxStages) : kMaxStages;
    k.placement = v.placement <= 4 ? static_cast<int>(v.placement) : 0;
    k.presum = v.presum != 0;
    k.dense = v.dense != 0;
    k.shapes = v.shapes != 0;
    k.payload = v.payload != 0;
    k.ctas_per_sm = v.ctas_per_sm == 2 ? 2 : 1;
    k.l2_ahead = static_cast<int>(std::min<uint32_t>(v.l2_ahead, 64));
    return k;
}

static tgp_variant variant_of(const Knobs& k) {
    tgp_variant v;
    std::memset(&v, 0, sizeof(v));
    v.threads = static_cast<uint32_t>(k.threads);
    v.max_stages = static_cast<uint32_t>(k.max_stages);
    v.placement = static_cast<uint32_t>(k.placement);
    v.presum = k.presum;
    v.dense = k.dense;
    v.shapes = k.shapes;
    v.payload = k.payload;
    v.ctas_per_sm = static_cast<uint32_t>(k.ctas_per_sm);
    v.l2_ahead = static_cast<uint32_t>(k.l2_ahead);
    return v;
}

static bool same_knobs(const Knobs& a, const Knobs& b) {
    return a.threads == b.threads && a.max_stages == b.max_stages && a.placement == b.placement &&
           a.presum == b.presum && a.dense == b.dense && a.shapes == b.shapes && a.payload == b.payload &&
           a.ctas_per_sm == b.ctas_per_sm && a.l2_ahead == b.l2_ahead;
}

int tgp_set_default_variant(tgp_ctx* ctx, const tgp_variant* v) {
    if (!ctx || !v) return fail(ctx, TGP_INVALID_ARG, "null argument");
    ctx->knobs = knobs_from(*v);
    return TGP_OK;
}

int tgp_get_default_variant(tgp_ctx* ctx, tgp_variant* v) {
    if (!ctx || !v) return fail(ctx, TGP_INVALID_ARG, "null argument");
    *v = variant_of(ctx->knobs);
    return TGP_OK;
}

int tgp_batch_config(tgp_ctx* ctx, uint32_t morsel_tiles, int shared_scans, uint64_t share_extra_max) {
    if (!ctx || morsel_tiles == 0) return fail(ctx, TGP_INVALID_ARG, "morsel_tiles must be at least 1");
    ctx->morsel_tiles = static_cast<int>(std::min<uint32_t>(morsel_tiles, 1u << 20));
    ctx->shared_scans = shared_scans != 0;
    ctx->share_extra_max = static_cast<size_t>(share_extra_max);
    return TGP_OK;
}

int tgp_tune_class(tgp_ctx* ctx, const tgp_query* q, uint64_t* key) {
    if (!ctx || !q || !key) return fail(ctx, TGP_INVALID_ARG, "null argument");
    QueryState qs;
    TGP_TRY(plan_query(ctx, q, qs, scan_kernel_static_smem(), nullptr, /*dry=*/true));
    *key = qs.tune_key;
    return TGP_OK;
}

int tgp_tune_set(tgp_ctx* ctx, uint64_t key, const tgp_variant* v) {
    if (!ctx || !v) return fail(ctx, TGP_INVALID_ARG, "null argument");
    ctx->tuned[key] = knobs_from(*v);
    return TGP_OK;
}

int tgp_tune_get(tgp_ctx* ctx, uint64_t key, tgp_variant* v, int* found) {
    if (!ctx || !v || !found) return fail(ctx, TGP_INVALID_ARG, "null argument");
    auto it = ctx->tuned.find(key);
    *found = it != ctx->tuned.end();
    *v = variant_of(*found ? it->second : ctx->knobs);
    return TGP_OK;
}

int tgp_tune_count(tgp_ctx* ctx, uint32_t* n) {
    if (!ctx || !n) return fail(ctx, TGP_INVALID_ARG, "null argument");
    *n = static_cast<uint32_t>(ctx->tuned.size());
    return TGP_OK;
}

int tgp_tune_at(tgp_ctx* ctx, uint32_t i, uint64_t* key, tgp_variant* v) {
    if (!ctx || !key || !v) return fail(ctx, TGP_INVALID_ARG, "null argument");
    if (i >= ctx->tuned.size()) return fail(ctx, TGP_INVALID_ARG, "tuned entry index out of range");
    std::vector<uint64_t> keys;
    keys.reserve(ctx->tuned.size());
    for (const auto& kv : ctx->tuned) keys.push_back(kv.first);
    std::sort(keys.begin(), keys.end());
    *key = keys[i];
    *v = variant_of(ctx->tuned[keys[i]]);
    return TGP_OK;
}

int tgp_tune_clear(tgp_ctx* ctx) {
    if (!ctx) return TGP_INVALID_ARG;
    ctx->tuned.clear();
    return TGP_OK;
}

namespace {

// One run of a query into host vectors (grown to its group count).
struct HostResult {
    std::vector<uint64_t> keys;
    std::vector<tgp_agg_value> vals;
    tgp_query_result res{};
};

int run_into(tgp_ctx* ctx, const tgp_query* q, HostResult* r) {
    uint64_t cap = std::max<uint64_t>(1, r->res.ngroups);
    for (int attempt = 0; attempt < 3; ++attempt) {
        r->keys.assign(std::max<uint64_t>(1, cap * std::max<uint32_t>(1, q->ngroup)), 0);
        r->vals.assign(std::max<uint64_t>(1, cap * std::max<uint32_t>(1, q->nagg)), tgp_agg_value{});
        const int st = execute_impl(ctx, q, r->keys.data(), r->vals.data(), cap, &r->res, nullptr);
        if (st != TGP_CAPACITY) return st;
        cap = r->res.ngroups;
    }
    return fail(ctx, TGP_CAPACITY, "group count kept growing");
}

bool same_results(const tgp_query* q, const HostResult& a, const HostResult& b) {
    if (a.res.rows_scanned != b.res.rows_scanned || a.res.rows_selected != b.res.rows_selected ||
        a.res.ngroups != b.res.ngroups || a.res.flags != b.res.flags)
        return false;
    const uint64_t nk = a.res.ngroups * q->ngroup, nv = a.res.ngroups * q->nagg;
    if (nk && std::memcmp(a.keys.data(), b.keys.data(), nk * 8) != 0) return false;
    for (uint64_t i = 0; i < nv; ++i) {
        const tgp_agg_value &x = a.vals[i], &y = b.vals[i];
        if (x.lo != y.lo || x.hi != y.hi || x.count != y.count || std::memcmp(&x.as_f64, &y.as_f64, 8) != 0) return false;
    }
    return true;
}

}  // namespace

int tgp_autotune(tgp_ctx* ctx, const tgp_query* q, uint32_t reps, tgp_tune_entry* entries, uint32_t cap,
                 uint32_t* n_out, uint32_t* best_out, uint64_t* key_out) {
    if (!ctx || !q || !n_out || !best_out || !key_out || (cap && !entries))
        return fail(ctx, TGP_INVALID_ARG, "null argument");
    if (ctx->profile) return fail(ctx, TGP_INVALID_ARG, "turn launch profiling off before tuning");
    reps = std::max<uint32_t>(1, std::min<uint32_t>(reps, 64));
    QueryState base;
    TGP_TRY(plan_query(ctx, q, base, scan_kernel_static_smem(), nullptr, /*dry=*/true));
    const uint64_t key = base.tune_key;
    const bool hash = base.mode == MODE_GROUP_HASH;

    // Candidates: the planner's rules first, then threads x stage cap x
    // accumulator placement (direct groups) or pre-aggregation (hash).
    std::vector<Knobs> cands;
    cands.push_back(ctx->knobs);
    for (int nt : {512, 256})
        for (int stg : {2, 4, kMaxStages}) {
            Knobs k = ctx->knobs;
            k.threads = nt;
            k.max_stages = stg;
            if (hash) {
                for (bool ps : {true, false}) {
                    k.presum = ps;
                    cands.push_back(k);
                }
            } else {
                for (int pl : {1, 2, 3, 4}) {
                    k.placement = pl;
                    if (pl == 1) {
                        for (bool dn : {true, false}) {
                            k.dense = dn;
                            cands.push_back(k);
                        }
                        k.dense = ctx->knobs.dense;
                    } else {
                        cands.push_back(k);
                    }
                }
            }
        }

    // Reference result: the planner's rules.
    HostResult ref;
    ctx->force_knobs = &cands[0];
    int st = run_into(ctx, q, &ref);
    ctx->force_knobs = nullptr;
    TGP_TRY(st);

    uint32_t n = 0, best = 0;
    double best_ms = 0.0;
    std::vector<std::pair<Knobs, double>> measured;
    for (size_t c = 0; c < cands.size(); ++c) {
        const Knobs& k = cands[c];
        bool dup = false;
        for (size_t d = 0; d < c && !dup; ++d) dup = same_knobs(cands[d], k);
        if (dup) continue;
        tgp_tune_entry e;
        std::memset(&e, 0, sizeof(e));
        e.variant = variant_of(k);
        ctx->force_knobs = &k;
        QueryState qs;
        e.status = plan_query(ctx, q, qs, scan_kernel_static_smem(), nullptr, /*dry=*/true);
        if (e.status == TGP_OK) {
            e.threads_used = qs.mode == MODE_GROUP_PRIVATE ? qs.b->P.nthreads : 512u;
            e.mode_used = qs.mode;
            Plan P = qs.b->P;
            if (size_smem(ctx, P, qs.extra, scan_kernel_static_smem(), &qs.kn) == TGP_OK) e.stages_used = P.nstages;
            HostResult r;
            r.res.ngroups = ref.res.ngroups;
            e.status = run_into(ctx, q, &r);
            e.same_result = (e.status == TGP_OK && same_results(q, ref, r)) ? 1u : 0u;
        }
        if (e.status == TGP_OK && e.same_result) {
            // Gated timing of the scan launch of each run.
            std::vector<double> t;
            HostResult r;
            r.res.ngroups = ref.res.ngroups;
            ctx->profile = true;
            ctx->profile_gate = true;
            for (uint32_t i = 0; i < reps && e.status == TGP_OK; ++i) {
                ctx->prof_used = 0;
                e.status = run_into(ctx, q, &r);
                double ms = 0.0;
                for (size_t j = 0; j < ctx->prof_used; ++j) {
                    float f = 0.f;
                    if (cudaEventElapsedTime(&f, ctx->prof_events[j].first, ctx->prof_events[j].second) == cudaSuccess)
                        ms += f;
                }
                t.push_back(ms);
            }
            ctx->profile = false;
            ctx->profile_gate = false;
            ctx->prof_used = 0;
            std::sort(t.begin(), t.end());
            e.ms = t.empty() ? 0.0 : t[t.size() / 2];
            if (e.status == TGP_OK && (measured.empty() || e.ms < best_ms)) {
                best_ms = e.ms;
                best = n;
            }
            if (e.status == TGP_OK) measured.push_back({k, e.ms});
        }
        ctx->force_knobs = nullptr;
        cudaGetLastError();
        if (n < cap) entries[n] = e;
        ++n;
    }
    ctx->force_knobs = nullptr;
    if (measured.empty()) return fail(ctx, TGP_DEVICE_ERROR, "no candidate variant ran");
    // Install the fastest variant that returned the reference result.
    const Knobs* win = nullptr;
    double wms = 0.0;
    for (const auto& m : measured)
        if (!win || m.second < wms) {
            win = &m.first;
            wms = m.second;
        }
    ctx->tuned[key] = *win;
    *n_out = n;
    *best_out = best;
    *key_out = key;
    return TGP_OK;
}

// --------------------------------------------------------------------------
// Batches
// --------------------------------------------------------------------------
static uint8_t* pinned_acquire(tgp_ctx* ctx, size_t bytes) {
    for (auto& b : ctx->pinned_pool)
        if (!b.busy && b.cap >= bytes) {
            b.busy = true;
            return b.p;
        }
    void* p = nullptr;
    const size_t cap = std::max<size_t>(bytes, 1 << 20);
    if (cudaMallocHost(&p, cap) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    ctx->pinned_pool.push_back({static_cast<uint8_t*>(p), cap, true});
    return static_cast<uint8_t*>(p);
}

static void pinned_release(tgp_ctx* ctx, uint8_t* p) {
    for (auto& b : ctx->pinned_pool)
        if (b.p == p) b.busy = false;
}

// A class of batch queries answered by one merged scan: same table, join,
// aggregates and group keys, WHERE a conjunction whose literals differ only
// on one column C. The merged query groups additionally by the bucket of C
// (cells accepted by the same members share a bucket; a per-cell table maps
// C to its bucket) under the hull of the members' ranges on C; a member's
// groups are the exact sums (MIN / MAX: extremes) of the buckets it accepts.
struct MergeCol {
    uint32_t column = 0;
    std::vector<uint64_t> bucket_mask;   // per bucket: the members that accept its cells
    std::vector<uint8_t> hlut;           // bucket of each cell of the column's [min, max]
    size_t lut_off = 0;
};

struct MergeRec {
    std::vector<uint32_t> members;       // batch item indices (bit k of a mask = members[k])
    std::vector<MergeCol> cols;          // the columns whose literals differ, one bucket key each
    std::vector<tgp_pred_node> pred;     // common leaves AND each column in its hull
    std::vector<tgp_group_key> group;    // [bucket keys] + the members' group keys
    tgp_query q{};
    // Joins: the members' rows_selected count probe rows passing WHERE,
    // matched or not: a count query per bucket (no join) gives them.
    std::vector<tgp_group_key> cgroup;
    tgp_agg count_agg{};
    tgp_query cq{};
    bool has_count = false;
    QueryState qs, cqs;
    size_t block_off = 0, cblock_off = 0;
    uint64_t nbucket_tuples() const {
        uint64_t n = 1;
        for (const MergeCol& c : cols) n *= c.bucket_mask.size();
        return n;
    }
};

struct BatchRec {
    tgp_batch_item* items = nullptr;
    uint32_t n = 0;
    std::vector<QueryState> qs;
    std::vector<uint8_t> batched;     // item runs in the persistent launch
    std::vector<size_t> block_off;    // its result block's byte offset in the readback area
    std::vector<std::unique_ptr<MergeRec>> merges;
    std::vector<int> merged_of;       // item -> merge record, or -1
    uint8_t* dev = nullptr;
    uint8_t* host = nullptr;
    size_t readback_off = 0;          // host offset of the readback area
    size_t blocks_off = 0;            // device / host offset of the first result block
    cudaEvent_t done = nullptr;
};

void tgp_batch_free_rec(tgp_ctx* ctx, void* r) {
    BatchRec* B = static_cast<BatchRec*>(r);
    if (!B) return;
    dev_free(ctx, B->dev);
    if (B->host) pinned_release(ctx, B->host);
    if (B->done) cudaEventDestroy(B->done);
    delete B;
}

static size_t align256(size_t x) { return (x + 255) & ~size_t{255}; }

// Whether a cell passes a comparison leaf with its column's comparison type
// (Int signed, Date unsigned, = / <> bitwise: apply_comparison, expr.rs:
// 1468-1530; BETWEEN / NOT BETWEEN, expr.rs:687-760).
static bool leaf_passes(const Column& c, const tgp_pred_node& n, int64_t cell) {
    const bool sgn = c.coltype == TGP_CT_INT;
    auto lt = [&](uint64_t a, uint64_t b) {
        return sgn ? static_cast<int64_t>(a) < static_cast<int64_t>(b) : a < b;
    };
    const uint64_t x = static_cast<uint64_t>(cell);
    switch (n.cmp) {
        case TGP_CMP_EQ: return x == n.lit;
        case TGP_CMP_NE: return x != n.lit;
        case TGP_CMP_LT: return lt(x, n.lit);
        case TGP_CMP_LE: return !lt(n.lit, x);
        case TGP_CMP_GT: return lt(n.lit, x);
        case TGP_CMP_GE: return !lt(x, n.lit);
        case TGP_CMP_BETWEEN: return !lt(x, n.lit) && !lt(n.lit2, x);
        default: return lt(x, n.lit) || lt(n.lit2, x);
    }
}

// A WHERE program that is a conjunction of leaves (postfix: leaves and ANDs).
static bool pure_conjunction(const tgp_query* q) {
    uint32_t leaves = 0, ands = 0;
    int depth = 0;
    for (uint32_t i = 0; i < q->npred; ++i) {
        const tgp_pred_node& nd = q->pred[i];
        if (nd.kind == TGP_PN_LEAF) {
            ++leaves;
            ++depth;
        } else if (nd.kind == TGP_PN_AND) {
            if (depth < 2) return false;
            ++ands;
            --depth;
        } else {
            return false;
        }
    }
    return leaves >= 1 && ands + 1 == leaves && depth == 1;
}

// The merge class of a query: everything but its leaf literals.
static std::string merge_key(const tgp_query* q) {
    std::string k;
    auto put = [&](const void* p, size_t n) { k.append(static_cast<const char*>(p), n); };
    put(&q->table, 8);
    put(&q->join, 8);
    put(&q->probe_key_column, 4);
    put(&q->flags, 4);
    put(&q->ngroup, 4);
    put(&q->nagg, 4);
    if (q->ngroup) put(q->group, sizeof(tgp_group_key) * q->ngroup);
    if (q->nagg) put(q->aggs, sizeof(tgp_agg) * q->nagg);
    for (uint32_t i = 0; i < q->npred; ++i) {
        put(&q->pred[i].kind, 4);
        put(&q->pred[i].column, 4);
        put(&q->pred[i].cmp, 4);
    }
    return k;
}

constexpr uint64_t kMergeMaxCells = 1ull << 20;   // bucket table bytes (cells of a column's range)
constexpr uint32_t kMergeMaxBuckets = 255;
constexpr uint64_t kMergeMaxTuples = 1ull << 14;  // bucket combinations x groups of one merged query
constexpr size_t kMergeChunk = 64;                // members per merged query (one u64 mask)

// Builds the bucket table of one varying column for a chunk of members.
// Every member's acceptance of a cell is constant between consecutive
// breakpoints (the cells where one of its leaves on the column can change:
// a literal, or the cell after one), so it is evaluated once per segment,
// not once per cell. Returns false if the column cannot be bucketed.
static bool bucket_column(const BatchRec& B, const std::vector<uint32_t>& members, const Column& col,
                          uint32_t C, MergeCol* out, uint64_t* rmin_out, uint64_t* rmax_out) {
    const uint64_t cells = static_cast<uint64_t>(col.max - col.min) + 1;
    out->column = C;
    out->bucket_mask.assign(1, 0);
    out->hlut.assign(cells, 0);
    // Each member's leaves on C.
    std::vector<std::vector<const tgp_pred_node*>> leaves(members.size());
    std::vector<uint64_t> cuts{0, cells};
    auto add_cut = [&](uint64_t lit_bits) {
        // The cell `lit` and the one after it, as offsets into [0, cells]
        // (a literal outside the range changes nothing inside it; the
        // column's minimum is not negative, so an unsigned literal above
        // INT64_MAX reads as negative and is outside too).
        const int64_t v = static_cast<int64_t>(lit_bits);
        if (v >= col.min && v <= col.max) {
            const uint64_t o = static_cast<uint64_t>(v - col.min);
            cuts.push_back(o);
            cuts.push_back(o + 1);
        }
    };
    for (size_t k = 0; k < members.size(); ++k) {
        const tgp_query* qk = B.items[members[k]].query;
        for (uint32_t j = 0; j < qk->npred; ++j)
            if (qk->pred[j].kind == TGP_PN_LEAF && qk->pred[j].column == C) {
                leaves[k].push_back(&qk->pred[j]);
                add_cut(qk->pred[j].lit);
                if (qk->pred[j].cmp == TGP_CMP_BETWEEN || qk->pred[j].cmp == TGP_CMP_NOT_BETWEEN)
                    add_cut(qk->pred[j].lit2);
            }
    }
    std::sort(cuts.begin(), cuts.end());
    cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
    std::unordered_map<uint64_t, uint8_t> bucket_of;
    bucket_of[0] = 0;
    uint64_t rmin = cells, rmax = 0;
    for (size_t s = 0; s + 1 < cuts.size(); ++s) {
        const uint64_t r0 = cuts[s], r1 = cuts[s + 1];   // cells [r0, r1)
        const int64_t cell = col.min + static_cast<int64_t>(r0);
        uint64_t mask = 0;
        for (size_t k = 0; k < members.size(); ++k) {
            bool acc = true;
            for (const tgp_pred_node* nd : leaves[k]) acc = acc && leaf_passes(col, *nd, cell);
            if (acc) mask |= 1ull << k;
        }
        auto it = bucket_of.find(mask);
        uint8_t b;
        if (it == bucket_of.end()) {
            if (out->bucket_mask.size() > kMergeMaxBuckets) return false;
            b = static_cast<uint8_t>(out->bucket_mask.size());
            bucket_of.emplace(mask, b);
            out->bucket_mask.push_back(mask);
        } else {
            b = it->second;
        }
        std::fill(out->hlut.begin() + static_cast<std::ptrdiff_t>(r0), out->hlut.begin() + static_cast<std::ptrdiff_t>(r1), b);
        if (mask) {
            rmin = std::min(rmin, r0);
            rmax = std::max(rmax, r1 - 1);
        }
    }
    if (rmin > rmax) return false;
    *rmin_out = rmin;
    *rmax_out = rmax;
    return true;
}

// Finds the merge classes among the planned, direct-grouped items of a batch:
// queries whose literals differ on at most three columns, each with a
// bounded cell range. A member accepts a combination of buckets when every
// one of its columns' buckets accepts it.
static void find_merges(tgp_ctx* ctx, BatchRec& B) {
    std::unordered_map<std::string, std::vector<uint32_t>> classes;
    std::vector<std::string> order;
    for (uint32_t i = 0; i < B.n; ++i) {
        const tgp_query* q = B.items[i].query;
        if (!B.qs[i].b || B.qs[i].mode == MODE_GROUP_HASH || !q->npred || !pure_conjunction(q)) continue;
        std::string key = merge_key(q);
        auto it = classes.find(key);
        if (it == classes.end()) {
            order.push_back(key);
            classes.emplace(key, std::vector<uint32_t>{i});
        } else {
            it->second.push_back(i);
        }
    }
    for (const std::string& key : order) {
        const std::vector<uint32_t>& all = classes[key];
        if (all.size() < 2) continue;
        const tgp_query* q0 = B.items[all[0]].query;
        const Table* T = B.qs[all[0]].T;
        const uint64_t D = B.qs[all[0]].ngroups_direct;
        // The columns whose leaf literals differ among the members.
        std::vector<uint32_t> vary;
        for (uint32_t j = 0; j < q0->npred; ++j) {
            const tgp_pred_node& a = q0->pred[j];
            if (a.kind != TGP_PN_LEAF) continue;
            bool varies = false;
            for (uint32_t i : all) {
                const tgp_pred_node& b = B.items[i].query->pred[j];
                varies = varies || b.lit != a.lit || b.lit2 != a.lit2;
            }
            if (varies && std::find(vary.begin(), vary.end(), a.column) == vary.end()) vary.push_back(a.column);
        }
        if (vary.empty()) vary.push_back(q0->pred[0].column);   // identical queries: any leaf column
        if (vary.size() > 3 || q0->ngroup + vary.size() > static_cast<size_t>(kMaxGroupKeys)) continue;
        bool ok = true;
        for (uint32_t C : vary) {
            if (C >= T->cols.size()) { ok = false; break; }
            const Column& col = T->cols[C];
            ok = ok && col.coltype != TGP_CT_FLOAT && col.min >= 0 && col.max >= col.min &&
                 static_cast<uint64_t>(col.max - col.min) + 1 <= kMergeMaxCells;
        }
        if (!ok) continue;
        // Chunks of members, halved until the bucket combinations x groups of
        // a chunk stay small enough for shared-memory tables.
        size_t start = 0;
        size_t chunk = kMergeChunk;
        while (start + 1 < all.size()) {
            const size_t cnt = std::min(chunk, all.size() - start);
            if (cnt < 2) break;
            std::unique_ptr<MergeRec> M(new MergeRec());
            M->members.assign(all.begin() + start, all.begin() + start + cnt);
            std::vector<std::pair<uint64_t, uint64_t>> hull;
            bool fits = true;
            for (uint32_t C : vary) {
                MergeCol mc;
                uint64_t rmin = 0, rmax = 0;
                if (!bucket_column(B, M->members, T->cols[C], C, &mc, &rmin, &rmax)) {
                    fits = false;
                    break;
                }
                hull.push_back({rmin, rmax});
                M->cols.push_back(std::move(mc));
            }
            if (fits && M->nbucket_tuples() * D > kMergeMaxTuples && cnt > 2) {
                chunk = std::max<size_t>(2, cnt / 2);   // fewer members: fewer buckets
                continue;
            }
            start += cnt;
            if (!fits || M->nbucket_tuples() * D > kMergeMaxTuples) continue;
            // Merged WHERE: the common leaves AND each varying column within
            // the hull of its accepted cells.
            auto push_and = [&]() {
                if (M->pred.size() > 1) {
                    tgp_pred_node a{};
                    a.kind = TGP_PN_AND;
                    M->pred.push_back(a);
                }
            };
            for (uint32_t j = 0; j < q0->npred; ++j) {
                const tgp_pred_node& nd = q0->pred[j];
                if (nd.kind != TGP_PN_LEAF || std::find(vary.begin(), vary.end(), nd.column) != vary.end()) continue;
                M->pred.push_back(nd);
                push_and();
            }
            for (size_t c = 0; c < vary.size(); ++c) {
                const Column& col = T->cols[vary[c]];
                tgp_pred_node h{};
                h.kind = TGP_PN_LEAF;
                h.column = vary[c];
                h.cmp = TGP_CMP_BETWEEN;
                h.lit = static_cast<uint64_t>(col.min + static_cast<int64_t>(hull[c].first));
                h.lit2 = static_cast<uint64_t>(col.min + static_cast<int64_t>(hull[c].second));
                M->pred.push_back(h);
                push_and();
            }
            for (uint32_t C : vary) {
                tgp_group_key bk{};
                bk.column = C;
                bk.side = TGP_SIDE_PROBE;
                M->group.push_back(bk);
            }
            for (uint32_t k = 0; k < q0->ngroup; ++k) M->group.push_back(q0->group[k]);
            M->q = *q0;
            M->q.pred = M->pred.data();
            M->q.npred = static_cast<uint32_t>(M->pred.size());
            M->q.group = M->group.data();
            M->q.ngroup = static_cast<uint32_t>(M->group.size());
            if (q0->join) {
                M->has_count = true;
                M->cgroup.assign(M->group.begin(), M->group.begin() + vary.size());
                M->count_agg.func = TGP_AGG_COUNT_STAR;
                M->cq = M->q;
                M->cq.join = 0;
                M->cq.group = M->cgroup.data();
                M->cq.ngroup = static_cast<uint32_t>(M->cgroup.size());
                M->cq.aggs = &M->count_agg;
                M->cq.nagg = 1;
            }
            B.merges.push_back(std::move(M));
        }
    }
    (void)ctx;
}

// A member's result block [counters 4][error 2][accumulators] rebuilt from
// the merged blocks: each group's slots summed (MIN / MAX: extremes) over the
// bucket combinations the member accepts, values as full int128 limbs.
static void member_block(const MergeRec& M, size_t k, const QueryState& mqs, const unsigned long long* hb,
                         const unsigned long long* hc, const QueryState& cqs,
                         std::vector<unsigned long long>* out) {
    const Plan& MP = M.qs.b->P;
    const uint32_t nv1 = mqs.nv1;
    const uint64_t D = mqs.ngroups_direct;
    out->assign(6 + D * nv1 * 2, 0);
    unsigned long long* blk = out->data();
    blk[4] = hb[4] | (hc ? hc[4] : 0);
    // The bucket combinations this member accepts, as merged group-index
    // prefixes (the bucket keys are the most significant digits).
    std::vector<uint64_t> tuples(1, 0);
    for (const MergeCol& c : M.cols) {
        std::vector<uint64_t> next;
        for (uint64_t t : tuples)
            for (size_t b = 1; b < c.bucket_mask.size(); ++b)
                if ((c.bucket_mask[b] >> k) & 1) next.push_back(t * c.bucket_mask.size() + b);
        tuples.swap(next);
    }
    const unsigned long long* macc = hb + 6;
    auto read = [&](const unsigned long long* acc, uint64_t slot, bool sum64) -> __int128 {
        const uint64_t lo = acc[2 * slot];
        const int64_t hi = sum64 ? (static_cast<int64_t>(lo) >> 63) : static_cast<int64_t>(acc[2 * slot + 1]);
        return static_cast<__int128>((static_cast<unsigned __int128>(static_cast<uint64_t>(hi)) << 64) | lo);
    };
    __int128 selected = 0;
    for (uint64_t g = 0; g < D; ++g)
        for (uint32_t v = 0; v < nv1; ++v) {
            const uint8_t kind = v == 0 ? VK_SUM : MP.val[v - 1].kind;
            const bool ext = kind == VK_MIN || kind == VK_MAX;
            __int128 acc = ext ? (kind == VK_MIN ? static_cast<__int128>(0x7fffffffffffffffll)
                                                 : static_cast<__int128>(static_cast<int64_t>(0x8000000000000000ull)))
                               : 0;
            for (uint64_t t : tuples) {
                const uint64_t slot = (t * D + g) * nv1 + v;
                if (ext) {
                    const int64_t x = static_cast<int64_t>(macc[2 * slot]);
                    acc = kind == VK_MIN ? std::min<__int128>(acc, x) : std::max<__int128>(acc, x);
                } else {
                    acc += read(macc, slot, MP.sum64 != 0);
                }
            }
            if (v == 0 && !M.has_count) selected += acc;
            const uint64_t o = 6 + (g * nv1 + v) * 2;
            blk[o] = static_cast<uint64_t>(acc);
            blk[o + 1] = ext ? 0 : static_cast<uint64_t>(acc >> 64);
        }
    if (M.has_count) {
        const Plan& CP = cqs.b->P;
        for (uint64_t t : tuples) selected += read(hc + 6, t * cqs.nv1, CP.sum64 != 0);
    }
    blk[0] = static_cast<uint64_t>(selected);
}

int tgp_batch_submit(tgp_ctx* ctx, tgp_batch_item* items, uint32_t n, tgp_batch_id* out) {
    if (!ctx || !out || (n && !items)) return fail(ctx, TGP_INVALID_ARG, "null argument");
    std::unique_ptr<BatchRec> B(new BatchRec());
    B->items = items;
    B->n = n;
    B->qs.resize(n);
    B->batched.assign(n, 0);
    B->block_off.assign(n, 0);
    const size_t bstatic = batch_kernel_static_smem();
    const size_t budget = ctx->max_dyn_smem - bstatic;
    // 1. Plan each query as tgp_execute would. Hash grouping runs now, alone
    // (its result size is only known after the scan). A direct-indexed query
    // goes to the persistent kernel when it is small (a launch of its own
    // would leave most SMs idle) or shares its table with other light
    // queries (a shared scan); every other one gets a launch of its own in
    // this batch's stream, with no synchronization between queries.
    std::vector<uint32_t> take, solo;
    const uint64_t small_tiles = static_cast<uint64_t>(ctx->sms) * 4;
    std::unordered_map<uint64_t, uint32_t> light_per_table;
    for (uint32_t i = 0; i < n; ++i) {
        tgp_batch_item& it = items[i];
        std::memset(&it.result, 0, sizeof(it.result));
        it.status = TGP_OK;
        QueryState& qs = B->qs[i];
        int st = plan_query(ctx, it.query, qs, scan_kernel_static_smem());
        if (st == TGP_OK && qs.mode != MODE_GROUP_HASH) {
            if (qs.mode == MODE_GROUP_PRIVATE && ((qs.extra + 127) & ~size_t{127}) <= ctx->share_extra_max)
                ++light_per_table[it.query->table];
            continue;
        }
        if (st == TGP_OK) st = tgp_execute(ctx, it.query, it.keys_out, it.vals_out, it.group_cap, &it.result);
        it.status = st;
        B->qs[i].b.reset();
    }
    // Merged scans: each class of same-shape queries becomes one grouped scan
    // (plus a per-bucket count scan for joins), planned as a query of its own.
    B->merged_of.assign(n, -1);
    if (ctx->shared_scans) {
        find_merges(ctx, *B);
        std::vector<std::unique_ptr<MergeRec>> kept;
        for (auto& M : B->merges) {
            // The bucket table's device address is set once the batch region
            // exists; the plan only needs a non-null placeholder now.
            BucketSpec bs{};
            bs.nkeys = static_cast<uint32_t>(M->cols.size());
            for (size_t c = 0; c < M->cols.size(); ++c) {
                bs.lut[c] = reinterpret_cast<const uint8_t*>(M.get());
                bs.nbuckets[c] = static_cast<uint32_t>(M->cols[c].bucket_mask.size());
            }
            int st = plan_query(ctx, &M->q, M->qs, scan_kernel_static_smem(), nullptr, false, &bs);
            if (st == TGP_OK) st = size_smem(ctx, M->qs.b->P, M->qs.extra, scan_kernel_static_smem(), &M->qs.kn);
            if (st == TGP_OK && M->has_count) {
                st = plan_query(ctx, &M->cq, M->cqs, scan_kernel_static_smem(), nullptr, false, &bs);
                if (st == TGP_OK) st = size_smem(ctx, M->cqs.b->P, M->cqs.extra, scan_kernel_static_smem(), &M->cqs.kn);
                if (st == TGP_OK && M->cqs.mode == MODE_GROUP_HASH) st = TGP_UNSUPPORTED;
            }
            if (st != TGP_OK || M->qs.mode == MODE_GROUP_HASH) {
                ctx->err.clear();
                continue;   // its members run unmerged
            }
            bound_presum(ctx, M->qs);
            if (M->has_count) bound_presum(ctx, M->cqs);
            for (uint32_t i : M->members) B->merged_of[i] = static_cast<int>(kept.size());
            kept.push_back(std::move(M));
        }
        B->merges = std::move(kept);
    }
    for (uint32_t i = 0; i < n; ++i) {
        QueryState& qs = B->qs[i];
        if (!qs.b || B->merged_of[i] >= 0) continue;
        const uint64_t T = (qs.b->P.nrows + kTileRows - 1) / kTileRows;
        const bool light = qs.mode == MODE_GROUP_PRIVATE && ((qs.extra + 127) & ~size_t{127}) <= ctx->share_extra_max;
        const bool shared = ctx->shared_scans && light && light_per_table[items[i].query->table] > 1;
        if (qs.mode == MODE_GROUP_PRIVATE && (T < small_tiles || shared)) {
            QueryState re;
            if (plan_query(ctx, items[i].query, re, bstatic) == TGP_OK && re.mode == MODE_GROUP_PRIVATE) {
                qs = std::move(re);
                take.push_back(i);
                continue;
            }
        }
        const int sst = size_smem(ctx, qs.b->P, qs.extra, scan_kernel_static_smem(), &qs.kn);
        if (sst == TGP_OK) bound_presum(ctx, qs);
        if (sst != TGP_OK) {
            items[i].status = tgp_execute(ctx, items[i].query, items[i].keys_out, items[i].vals_out, items[i].group_cap,
                                          &items[i].result);
            qs.b.reset();
            continue;
        }
        solo.push_back(i);
    }
    // 2. Shared scans: queries over one table are re-planned over the union of
    // their columns (when it fits the stage's slots) and packed into groups
    // whose accumulator regions fit beside two stages.
    struct Group {
        bool acc128;
        uint32_t nt;
        std::vector<uint32_t> q;
        size_t extra = 0;
        bool light = true;
        bool fast = false;   // every plan: scalar register fast path over the first plan's leaf columns / values
    };
    // Scalar plans whose register images differ only in their leaf bounds
    // and negations (the same statement with other literals) run a shared
    // tile with the leaf cells loaded once (fast_group_tile).
    auto fast_plan = [](const QueryState& qs) {
        const Plan& P = qs.b->P;
        return !qs.acc128 && P.ngroups == 1 && P.count_by_tile && P.rb.vals_on && P.rb.leaf_n > 0;
    };
    auto fast_compatible = [](const Plan& a, const Plan& b) {
        const RegBlock &x = a.rb, &y = b.rb;
        if (x.leaf_n != y.leaf_n || x.vals_nv != y.vals_nv || a.flush_limit != b.flush_limit) return false;
        for (uint32_t i = 0; i < x.leaf_n; ++i)
            if (x.leaf_soff[i] != y.leaf_soff[i]) return false;
        for (int v = 0; v < 2; ++v) {
            if (x.vals_nf[v] != y.vals_nf[v]) return false;
            for (int f = 0; f < 2; ++f)
                if (x.vals_soff[v][f] != y.vals_soff[v][f] || x.vals_dt[v][f] != y.vals_dt[v][f] ||
                    x.vals_mul[v][f] != y.vals_mul[v][f] || x.vals_add[v][f] != y.vals_add[v][f])
                    return false;
        }
        return true;
    };
    std::vector<Group> groups;
    std::unordered_map<uint64_t, std::vector<uint32_t>> by_table;
    std::vector<uint64_t> table_order;
    for (uint32_t i : take) {
        const uint64_t tid = items[i].query->table;
        if (!by_table.count(tid)) table_order.push_back(tid);
        by_table[tid].push_back(i);
    }
    for (uint64_t tid : table_order) {
        std::vector<uint32_t>& qi = by_table[tid];
        std::vector<uint32_t> cols;
        for (uint32_t i : qi) {
            const std::vector<int>& c2s = B->qs[i].b->col2slot;
            for (uint32_t c = 0; c < c2s.size(); ++c)
                if (c2s[c] >= 0 && std::find(cols.begin(), cols.end(), c) == cols.end()) cols.push_back(c);
        }
        const bool share = ctx->shared_scans && qi.size() > 1 && cols.size() <= static_cast<size_t>(kMaxSlots);
        for (uint32_t i : qi) {
            QueryState& qs = B->qs[i];
            if (share && ((qs.extra + 127) & ~size_t{127}) <= ctx->share_extra_max) {
                QueryState re;
                if (plan_query(ctx, items[i].query, re, bstatic, &cols) == TGP_OK && re.mode == MODE_GROUP_PRIVATE)
                    qs = std::move(re);
            }
            Plan& P = qs.b->P;
            // The int64 batch kernels carry the fixed-shape dense path.
            P.shape = (!qs.acc128 && !qs.J && P.dense_vec && qs.kn.shapes && dense_shape_of(P) == 1) ? 1u : 0u;
            fill_reg_block(P);
            const bool fast = fast_plan(qs);
            const size_t extra = (qs.extra + 127) & ~size_t{127};
            Group* g = nullptr;
            // Plans with a large accumulator table (dense grouping, joins) are
            // compute-bound: they run in their own group, whose layout keeps
            // the most stages and threads; light plans share scans.
            const bool light = extra <= ctx->share_extra_max;
            if (share && light)
                for (auto& k : groups)
                    if (k.light && k.acc128 == qs.acc128 && k.nt == P.nthreads && k.q.size() < static_cast<size_t>(kMaxShare) &&
                        items[k.q[0]].query->table == tid &&
                        B->qs[k.q[0]].b->P.stage_bytes == P.stage_bytes &&
                        k.fast == fast && (!fast || fast_compatible(B->qs[k.q[0]].b->P, P)) &&
                        k.extra + extra + (k.q.size() + 1) * sizeof(Plan) + 2ull * P.stage_bytes + kBarrierBytes + 256 <=
                            budget)
                        g = &k;
            if (!g) {
                groups.push_back(Group{qs.acc128, P.nthreads, {}, 0, light, fast});
                g = &groups.back();
            }
            g->q.push_back(i);
            g->extra += extra;
        }
    }
    // 3. Shared-memory layout per group: the barriers, the group's plans, the
    // stages, then each plan's accumulator region.
    for (const Group& g : groups)
        for (uint32_t i : g.q) B->qs[i].b->P.group_fast = (g.fast && g.q.size() > 1) ? 1u : 0u;
    for (const Group& g : groups) {
        const Plan& P0 = B->qs[g.q[0]].b->P;
        const size_t stage = P0.stage_bytes;
        const size_t stage_off = (kBarrierBytes + g.q.size() * sizeof(Plan) + 127) & ~size_t{127};
        const size_t fixed = stage_off + 128 + g.extra;
        const size_t avail = budget > fixed ? budget - fixed : 0;
        const uint32_t S = stage ? static_cast<uint32_t>(std::min<size_t>(avail / stage, static_cast<size_t>(ctx->knobs.max_stages))) : 1u;
        if (S == 0) return fail(ctx, TGP_UNSUPPORTED, "batched query does not fit in shared memory");
        size_t off = (stage_off + static_cast<size_t>(S) * stage + 127) & ~size_t{127};
        for (uint32_t i : g.q) {
            Plan& P = B->qs[i].b->P;
            P.nstages = S;
            P.l2_ahead = 0;
            P.stage_off = static_cast<uint32_t>(stage_off);
            P.extra_off = static_cast<uint32_t>(off);
            off += (B->qs[i].extra + 127) & ~size_t{127};
        }
        for (uint32_t i : g.q) B->qs[i].b->P.smem_bytes = static_cast<uint32_t>(off);
    }
    uint32_t nplans = 0;
    std::vector<uint32_t> plan_index(n, 0);
    std::vector<uint8_t> in_group(n, 0);
    for (const Group& g : groups)
        for (uint32_t i : g.q) {
            B->batched[i] = 1;
            in_group[i] = 1;
            plan_index[i] = nplans++;
        }
    for (uint32_t i : solo) B->batched[i] = 1;
    if (nplans == 0 && solo.empty() && B->merges.empty()) {
        const uint64_t id = ctx->next_id++;
        ctx->batches.emplace(id, B.release());
        *out = id;
        return TGP_OK;
    }
    // 4. Launch classes (acc128, NT) and morsels: a group over T tiles becomes
    // min(grid, ceil(T / morsel_tiles)) ranges, handed out largest first.
    struct Class {
        bool acc128;
        uint32_t nt;
        size_t smem = 0;
        int grid = 0;
        std::vector<Morsel> morsels;
    };
    std::vector<Class> classes;
    std::vector<size_t> group_class(groups.size());
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const Group& g = groups[gi];
        size_t k = 0;
        while (k < classes.size() && !(classes[k].acc128 == g.acc128 && classes[k].nt == g.nt)) ++k;
        if (k == classes.size()) classes.push_back(Class{g.acc128, g.nt});
        classes[k].smem = std::max<size_t>(classes[k].smem, B->qs[g.q[0]].b->P.smem_bytes);
        group_class[gi] = k;
    }
    for (auto& c : classes) {
        const int occ = batch_occupancy(c.acc128, static_cast<int>(c.nt), c.smem);
        if (occ <= 0) return fail(ctx, TGP_DEVICE_ERROR, "batch kernel cannot be resident with this shared memory");
        c.grid = ctx->sms * occ;
    }
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const Group& g = groups[gi];
        Class& c = classes[group_class[gi]];
        const uint64_t T = (B->qs[g.q[0]].b->P.nrows + kTileRows - 1) / kTileRows;
        if (T == 0) continue;
        const uint64_t per = static_cast<uint64_t>(ctx->morsel_tiles);
        const uint64_t nm = std::max<uint64_t>(1, std::min<uint64_t>(static_cast<uint64_t>(c.grid), (T + per - 1) / per));
        const uint64_t size = (T + nm - 1) / nm;
        for (uint64_t b0 = 0; b0 < T; b0 += size)
            c.morsels.push_back(Morsel{plan_index[g.q[0]], static_cast<uint32_t>(g.q.size()), b0, std::min(T, b0 + size)});
    }
    for (auto& c : classes)
        std::stable_sort(c.morsels.begin(), c.morsels.end(), [](const Morsel& a, const Morsel& b) {
            return (a.tile_end - a.tile_begin) * a.count > (b.tile_end - b.tile_begin) * b.count;
        });
    // 5. One device region: [plans][morsels per class][counters][result blocks].
    size_t off = align256(static_cast<size_t>(nplans) * sizeof(Plan));
    std::vector<size_t> morsel_off(classes.size());
    for (size_t k = 0; k < classes.size(); ++k) {
        morsel_off[k] = off;
        off = align256(off + classes[k].morsels.size() * sizeof(Morsel));
    }
    const size_t counter_off = off;
    off = align256(off + classes.size() * 4);
    for (auto& M : B->merges) {
        for (MergeCol& c : M->cols) {
            c.lut_off = off;
            off = align256(off + c.hlut.size());
        }
    }
    const size_t blocks_off = off;
    B->blocks_off = blocks_off;
    for (uint32_t i = 0; i < n; ++i) {
        if (!B->batched[i]) continue;
        B->block_off[i] = off - blocks_off;
        off = align256(off + B->qs[i].block_words() * 8);
    }
    for (auto& M : B->merges) {
        M->block_off = off - blocks_off;
        off = align256(off + M->qs.block_words() * 8);
        if (M->has_count) {
            M->cblock_off = off - blocks_off;
            off = align256(off + M->cqs.block_words() * 8);
        }
    }
    const size_t total = off, blocks_bytes = total - blocks_off;
    TGP_TRY(dev_alloc(ctx, reinterpret_cast<void**>(&B->dev), total, "batch allocation failed"));
    B->readback_off = align256(total);
    B->host = pinned_acquire(ctx, B->readback_off + blocks_bytes);
    if (!B->host) {
        dev_free(ctx, B->dev);
        B->dev = nullptr;
        return fail(ctx, TGP_OOM, "pinned batch staging allocation failed");
    }
    uint8_t* h = B->host;
    std::memset(h, 0, total);
    Plan* hplans = reinterpret_cast<Plan*>(h);
    for (uint32_t i = 0; i < n; ++i) {
        if (!B->batched[i]) continue;
        Plan& P = B->qs[i].b->P;
        unsigned long long* blk = reinterpret_cast<unsigned long long*>(B->dev + blocks_off + B->block_off[i]);
        P.counters = blk;
        P.err = reinterpret_cast<uint32_t*>(blk + 4);
        P.acc = blk + 6;
        if (B->qs[i].has_minmax()) {
            std::vector<unsigned long long> img;
            init_acc_image(P, B->qs[i].ngroups_direct, &img);
            std::memcpy(h + blocks_off + B->block_off[i] + 48, img.data(), img.size() * 8);
        }
        if (in_group[i]) {
            fill_reg_block(P);
            hplans[plan_index[i]] = P;
        }
    }
    for (size_t k = 0; k < classes.size(); ++k)
        if (!classes[k].morsels.empty())
            std::memcpy(h + morsel_off[k], classes[k].morsels.data(), classes[k].morsels.size() * sizeof(Morsel));
    // Merged scans: bucket tables, result pointers (the blocks are zero:
    // merged queries hold no MIN / MAX identities beyond their own images).
    for (auto& M : B->merges) {
        for (const MergeCol& c : M->cols) std::memcpy(h + c.lut_off, c.hlut.data(), c.hlut.size());
        auto place = [&](QueryState& qs, size_t boff) {
            Plan& P = qs.b->P;
            unsigned long long* blk = reinterpret_cast<unsigned long long*>(B->dev + blocks_off + boff);
            P.counters = blk;
            P.err = reinterpret_cast<uint32_t*>(blk + 4);
            P.acc = blk + 6;
            for (size_t c = 0; c < M->cols.size(); ++c) P.gkey[c].lut = B->dev + M->cols[c].lut_off;
            if (qs.has_minmax()) {
                std::vector<unsigned long long> img;
                init_acc_image(P, qs.ngroups_direct, &img);
                std::memcpy(h + blocks_off + boff + 48, img.data(), img.size() * 8);
            }
        };
        place(M->qs, M->block_off);
        if (M->has_count) place(M->cqs, M->cblock_off);
    }
    // 6. One upload, the queries with launches of their own, the persistent
    // launches, one readback.
    TGP_CUDA(cudaMemcpyAsync(B->dev, h, total, cudaMemcpyHostToDevice, ctx->stream));
    for (uint32_t i : solo) {
        const QueryState& qs = B->qs[i];
        bool done = false;
        TGP_TRY(try_launch_q1(ctx, qs.b->P, qs.mode, qs.acc128, qs.ngroups_direct, qs.b->max_abs_val, &done));
        if (!done) TGP_TRY(launch(ctx, qs.b->P, qs.mode, qs.acc128));
    }
    for (auto& M : B->merges) {
        TGP_TRY(launch(ctx, M->qs.b->P, M->qs.mode, M->qs.acc128));
        if (M->has_count) TGP_TRY(launch(ctx, M->cqs.b->P, M->cqs.mode, M->cqs.acc128));
    }
    for (size_t k = 0; k < classes.size(); ++k) {
        const Class& c = classes[k];
        if (c.morsels.empty()) continue;
        BatchDesc D;
        std::memset(&D, 0, sizeof(D));
        D.plans = reinterpret_cast<const Plan*>(B->dev);
        D.morsels = reinterpret_cast<const Morsel*>(B->dev + morsel_off[k]);
        D.nmorsels = static_cast<uint32_t>(c.morsels.size());
        D.next = reinterpret_cast<unsigned int*>(B->dev + counter_off) + k;
        const int grid = static_cast<int>(std::min<size_t>(static_cast<size_t>(c.grid), c.morsels.size()));
        std::pair<cudaEvent_t, cudaEvent_t>* ev = nullptr;
        if (ctx->profile) {
            if (ctx->prof_used == ctx->prof_events.size()) {
                std::pair<cudaEvent_t, cudaEvent_t> pe;
                TGP_CUDA(cudaEventCreate(&pe.first));
                TGP_CUDA(cudaEventCreate(&pe.second));
                ctx->prof_events.push_back(pe);
            }
            ev = &ctx->prof_events[ctx->prof_used++];
            TGP_CUDA(cudaEventRecord(ev->first, ctx->stream));
        }
        const cudaError_t e = launch_batch(D, c.acc128, static_cast<int>(c.nt), grid, c.smem, ctx->stream);
        if (e != cudaSuccess) return fail(ctx, TGP_DEVICE_ERROR, std::string("batch launch: ") + cudaGetErrorString(e));
        if (ev) TGP_CUDA(cudaEventRecord(ev->second, ctx->stream));
    }
    // The readback: the SMs store the result blocks into the page-locked
    // staging buffer (mapped into the device's address space), so it uses no
    // copy engine.
    TGP_CUDA(launch_copy_to_host(h + B->readback_off, B->dev + blocks_off, blocks_bytes, ctx->stream));
    TGP_CUDA(cudaEventCreateWithFlags(&B->done, cudaEventDisableTiming));
    TGP_CUDA(cudaEventRecord(B->done, ctx->stream));
    const uint64_t id = ctx->next_id++;
    ctx->batches.emplace(id, B.release());
    *out = id;
    return TGP_OK;
}

int tgp_batch_poll(tgp_ctx* ctx, tgp_batch_id id, int wait) {
    if (!ctx) return TGP_INVALID_ARG;
    auto it = ctx->batches.find(id);
    if (it == ctx->batches.end()) return fail(ctx, TGP_NOT_FOUND, "unknown batch id");
    BatchRec* B = static_cast<BatchRec*>(it->second);
    if (B->done) {
        if (!wait) {
            const cudaError_t q = cudaEventQuery(B->done);
            if (q == cudaErrorNotReady) return TGP_PENDING;
            if (q != cudaSuccess) return fail(ctx, TGP_DEVICE_ERROR, std::string("batch: ") + cudaGetErrorString(q));
        } else if (cudaEventSynchronize(B->done) != cudaSuccess) {
            return fail(ctx, TGP_DEVICE_ERROR, "batch synchronization failed");
        }
    }
    for (uint32_t i = 0; i < B->n; ++i) {
        if (!B->batched[i]) continue;
        tgp_batch_item& itm = B->items[i];
        const unsigned long long* hb =
            reinterpret_cast<const unsigned long long*>(B->host + B->readback_off + B->block_off[i]);
        itm.status = decode_direct(ctx, B->qs[i], hb, itm.keys_out, itm.vals_out, itm.group_cap, &itm.result);
    }
    std::vector<unsigned long long> blk;
    for (auto& M : B->merges) {
        const unsigned long long* hb =
            reinterpret_cast<const unsigned long long*>(B->host + B->readback_off + M->block_off);
        const unsigned long long* hc =
            M->has_count ? reinterpret_cast<const unsigned long long*>(B->host + B->readback_off + M->cblock_off)
                         : nullptr;
        for (size_t k = 0; k < M->members.size(); ++k) {
            const uint32_t i = M->members[k];
            tgp_batch_item& itm = B->items[i];
            member_block(*M, k, B->qs[i], hb, hc, M->cqs, &blk);
            itm.status = decode_direct(ctx, B->qs[i], blk.data(), itm.keys_out, itm.vals_out, itm.group_cap,
                                       &itm.result);
        }
    }
    tgp_batch_free_rec(ctx, B);
    ctx->batches.erase(it);
    return TGP_OK;
}

// --------------------------------------------------------------------------
// Captured queries
// --------------------------------------------------------------------------
namespace {

// One captured query: its plan, the graph (clear, scan, readback) and the
// buffers the graph reads and writes, plus what it was captured against.
struct GraphRec {
    QueryState qs;
    tgp_query q{};                          // counts only (pointers cleared)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long* block = nullptr;   // device result block
    unsigned long long* image = nullptr;   // MIN/MAX identity image of the accumulators
    unsigned long long* host = nullptr;    // pinned readback of the block
    uint64_t block_words = 0;
    tgp_table_id table = 0;
    const Table* T = nullptr;
    std::vector<const uint8_t*> cols;      // device column pointers at capture
    std::vector<std::pair<int64_t, int64_t>> stats;  // column min / max at capture
    tgp_join_id join = 0;
    const JoinTable* J = nullptr;
    const unsigned long long* jtab = nullptr;
    const uint32_t* jpay = nullptr;
    std::vector<uint64_t> jsig;            // layout of the payload array the plan reads
};

void graph_release(GraphRec* g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->block) cudaFree(g->block);
    if (g->image) cudaFree(g->image);
    if (g->host) cudaFreeHost(g->host);
    delete g;
}

// The table / join the graph reads must be the ones it was captured against,
// with the statistics its plan's bounds were proven from.
int graph_check(tgp_ctx* ctx, const GraphRec& g) {
    auto it = ctx->tables.find(g.table);
    if (it == ctx->tables.end() || &it->second != g.T || it->second.rows != g.qs.T->rows ||
        it->second.cols.size() != g.cols.size())
        return fail(ctx, TGP_NOT_FOUND, "captured query: table dropped or replaced; capture again");
    for (size_t c = 0; c < g.cols.size(); ++c) {
        const Column& col = it->second.cols[c];
        if (col.dptr != g.cols[c] || col.min != g.stats[c].first || col.max != g.stats[c].second)
            return fail(ctx, TGP_NOT_FOUND, "captured query: column moved or its min / max changed; capture again");
    }
    if (g.join) {
        auto jt = ctx->joins.find(g.join);
        if (jt == ctx->joins.end() || &jt->second != g.J || jt->second.tab != g.jtab ||
            (g.jpay && (jt->second.pays.count(g.jsig) == 0 || jt->second.pays.at(g.jsig).ptr != g.jpay)))
            return fail(ctx, TGP_NOT_FOUND, "captured query: join dropped or rebuilt; capture again");
    }
    return TGP_OK;
}

}  // namespace

void tgp_graph_free_rec(void* r) { graph_release(static_cast<GraphRec*>(r)); }

int tgp_graph_capture(tgp_ctx* ctx, const tgp_query* q, tgp_graph_id* out) {
    if (!ctx || !q || !out) return fail(ctx, TGP_INVALID_ARG, "null argument");
    *out = 0;
    std::unique_ptr<GraphRec, void (*)(GraphRec*)> rec(new GraphRec(), graph_release);
    GraphRec& g = *rec;
    QueryState& qs = g.qs;
    TGP_TRY(plan_query(ctx, q, qs, scan_kernel_static_smem()));
    if (qs.mode == MODE_GROUP_HASH)
        return fail(ctx, TGP_UNSUPPORTED, "hash-grouped queries size their result from the data and are not captured");
    Plan& P = qs.b->P;
    g.q = *q;
    g.q.pred = nullptr;
    g.q.group = nullptr;
    g.q.aggs = nullptr;
    qs.q = &g.q;
    g.table = q->table;
    g.T = qs.T;
    for (const Column& c : qs.T->cols) {
        g.cols.push_back(c.dptr);
        g.stats.emplace_back(c.min, c.max);
    }
    if (qs.J) {
        g.join = q->join;
        g.J = qs.J;
        g.jtab = qs.J->tab;
        g.jpay = P.jpay;
        if (g.jpay) g.jsig = qs.pay_sig;
    }

    g.block_words = qs.block_words();
    const uint64_t acc_words = qs.acc_words();
    TGP_CUDA(cudaMalloc(reinterpret_cast<void**>(&g.block), g.block_words * 8));
    TGP_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&g.host), g.block_words * 8, cudaHostAllocDefault));
    P.counters = g.block;
    P.err = reinterpret_cast<uint32_t*>(g.block + 4);
    P.acc = g.block + 6;
    const bool minmax = qs.has_minmax();
    if (minmax) {
        std::vector<unsigned long long> img;
        init_acc_image(P, qs.ngroups_direct, &img);
        TGP_CUDA(cudaMalloc(reinterpret_cast<void**>(&g.image), acc_words * 8));
        TGP_TRY(upload(ctx, g.image, img.data(), img.size() * 8));
    }
    TGP_TRY(size_smem(ctx, P, qs.extra, scan_kernel_static_smem(), &qs.kn));
    // Kernel attributes and occupancy are settled before the capture.
    if (scan_occupancy(qs.mode, qs.acc128, static_cast<int>(P.nthreads), P.smem_bytes, P.shape, P.two_ctas != 0) <= 0)
        return fail(ctx, TGP_DEVICE_ERROR, "scan kernel cannot be resident with this shared memory");

    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    const bool prof = ctx->profile;
    ctx->profile = false;
    int st = TGP_OK;
    std::string what;
    cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(g.block, 0, minmax ? 48 : g.block_words * 8, ctx->stream);
        if (e == cudaSuccess && minmax)
            e = cudaMemcpyAsync(g.block + 6, g.image, acc_words * 8, cudaMemcpyDeviceToDevice, ctx->stream);
        if (e == cudaSuccess) st = launch(ctx, P, qs.mode, qs.acc128);
        if (e == cudaSuccess && st == TGP_OK)
            e = cudaMemcpyAsync(g.host, g.block, g.block_words * 8, cudaMemcpyDeviceToHost, ctx->stream);
        const cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &g.graph);
        if (e == cudaSuccess) e = e2;
    }
    ctx->profile = prof;
    if (st != TGP_OK) return st;
    if (e != cudaSuccess) return fail(ctx, TGP_DEVICE_ERROR, std::string("graph capture: ") + cudaGetErrorString(e));
    TGP_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
    const uint64_t id = ctx->next_id++;
    ctx->graphs[id] = rec.release();
    *out = id;
    return TGP_OK;
}

int tgp_graph_launch(tgp_ctx* ctx, tgp_graph_id id, uint64_t* keys_out, tgp_agg_value* vals_out, uint64_t group_cap,
                     tgp_query_result* result) {
    if (!ctx || !result) return fail(ctx, TGP_INVALID_ARG, "null argument");
    std::memset(result, 0, sizeof(*result));
    auto it = ctx->graphs.find(id);
    if (it == ctx->graphs.end()) return fail(ctx, TGP_NOT_FOUND, "unknown graph id");
    GraphRec& g = *static_cast<GraphRec*>(it->second);
    TGP_TRY(graph_check(ctx, g));
    // Profiling counts the graph (one scan kernel between its clear and its
    // readback) as one timed launch.
    std::pair<cudaEvent_t, cudaEvent_t>* ev = nullptr;
    TGP_TRY(profile_begin(ctx, &ev));
    TGP_CUDA(cudaGraphLaunch(g.exec, ctx->stream));
    if (ev) TGP_CUDA(cudaEventRecord(ev->second, ctx->stream));
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    return decode_direct(ctx, g.qs, g.host, keys_out, vals_out, group_cap, result);
}

int tgp_graph_drop(tgp_ctx* ctx, tgp_graph_id id) {
    if (!ctx) return TGP_INVALID_ARG;
    auto it = ctx->graphs.find(id);
    if (it == ctx->graphs.end()) return fail(ctx, TGP_NOT_FOUND, "unknown graph id");
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    graph_release(static_cast<GraphRec*>(it->second));
    ctx->graphs.erase(it);
    return TGP_OK;
}

// --------------------------------------------------------------------------
// Joins
// --------------------------------------------------------------------------
static int build_join(tgp_ctx* ctx, const Table* T, tgp_table_id table_id, uint32_t key_col,
                      const tgp_pred_node* pred, uint32_t npred, JoinTable* out) {
    if (key_col >= T->cols.size()) return fail(ctx, TGP_INVALID_ARG, "key column out of range");
    const Column& kc = T->cols[key_col];
    if (kc.coltype == TGP_CT_FLOAT) return fail(ctx, TGP_UNSUPPORTED, "FLOAT join keys");
    Builder b(ctx, T);
    TGP_TRY(b.add_pred(pred, npred));
    int ks;
    TGP_TRY(b.slot_of(key_col, &ks));
    JoinTable J;
    J.build_table = table_id;
    J.key_col = key_col;
    J.kmin = kc.min;
    J.krange = static_cast<uint64_t>(kc.max) - static_cast<uint64_t>(kc.min);
    J.empty_range = T->rows == 0;
    J.wide = J.krange >= 0xffffffffull;
    // Directory of next_pow2(2 n) slots, as JoinHashTable::new does (join_hash_table.rs:76-86).
    J.cap = next_pow2(std::max<uint64_t>(16, 2 * T->rows));
    J.log2 = log2u(J.cap);
    const uint64_t words = J.cap * (J.wide ? 2 : 1);
    TGP_TRY(dev_alloc(ctx, reinterpret_cast<void**>(&J.tab), words * 8, "join table allocation failed"));
    if (J.wide) TGP_CUDA(cudaMemsetAsync(J.tab, 0, words * 8, ctx->stream));
    else TGP_CUDA(cudaMemsetAsync(J.tab, 0xff, words * 8, ctx->stream));
    Plan& P = b.P;
    Carve cv;
    TGP_TRY(arena_reserve(ctx, 256, &cv));
    P.counters = cv.take<unsigned long long>(4);
    P.err = cv.take<uint32_t>(4);
    P.acc = cv.take<unsigned long long>(2);
    TGP_CUDA(cudaMemsetAsync(P.counters, 0, 32, ctx->stream));
    TGP_CUDA(cudaMemsetAsync(P.err, 0, 16, ctx->stream));
    P.jtab = J.tab;
    P.jmask = J.cap - 1;
    P.jlog2 = J.log2;
    P.jwide = J.wide;
    P.jslot = ks;
    P.jkmin = J.kmin;
    P.jkrange = J.krange;
    int st = size_smem(ctx, P, 0);
    if (st == TGP_OK) st = launch(ctx, P, MODE_JOIN_BUILD, false);
    unsigned long long cnt[4] = {0, 0, 0, 0};
    uint32_t err = 0;
    if (st == TGP_OK) {
        cudaMemcpyAsync(cnt, P.counters, 32, cudaMemcpyDeviceToHost, ctx->stream);
        cudaMemcpyAsync(&err, P.err, 4, cudaMemcpyDeviceToHost, ctx->stream);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) st = fail(ctx, TGP_DEVICE_ERROR, "join build failed");
        else st = check_kernel_err(ctx, err);
    }
    if (st != TGP_OK) {
        free_join(ctx, J);
        return st;
    }
    J.entries = cnt[0];
    J.unique = !J.wide && cnt[3] == 0;
    *out = J;
    return TGP_OK;
}

int tgp_join_build(tgp_ctx* ctx, tgp_table_id build_table, uint32_t key_column, const tgp_pred_node* pred,
                   uint32_t npred, tgp_join_id* out) {
    if (!ctx || !out) return fail(ctx, TGP_INVALID_ARG, "null argument");
    const Table* T;
    TGP_TRY(get_table(ctx, build_table, &T));
    JoinTable J;
    TGP_TRY(build_join(ctx, T, build_table, key_column, pred, npred, &J));
    const uint64_t id = ctx->next_id++;
    ctx->joins.emplace(id, J);
    *out = id;
    return TGP_OK;
}

int tgp_join_build_smaller(tgp_ctx* ctx, tgp_table_id table_a, uint32_t key_a, const tgp_pred_node* pred_a,
                           uint32_t npred_a, tgp_table_id table_b, uint32_t key_b, const tgp_pred_node* pred_b,
                           uint32_t npred_b, tgp_join_id* out, uint32_t* build_is_a, uint64_t* rows_a,
                           uint64_t* rows_b) {
    if (!ctx || !out || !build_is_a || !rows_a || !rows_b) return fail(ctx, TGP_INVALID_ARG, "null argument");
    const Table *A, *B;
    TGP_TRY(get_table(ctx, table_a, &A));
    TGP_TRY(get_table(ctx, table_b, &B));
    if (key_a >= A->cols.size() || key_b >= B->cols.size()) return fail(ctx, TGP_INVALID_ARG, "key column out of range");
    // Each side's row count after its own filter (the reference joins the
    // single-table-filtered tables, join.rs:79-100), counted on the device.
    uint64_t na = 0, nb = 0;
    TGP_TRY(filter_impl(ctx, A, pred_a, npred_a, nullptr, nullptr, 0, &na, 0));
    TGP_TRY(filter_impl(ctx, B, pred_b, npred_b, nullptr, nullptr, 0, &nb, 0));
    // hash_join_with_keys (join.rs:557-575): an inner join builds on the left
    // side when it has fewer rows, else on the right.
    const bool on_a = na < nb;
    JoinTable J;
    if (on_a) TGP_TRY(build_join(ctx, A, table_a, key_a, pred_a, npred_a, &J));
    else TGP_TRY(build_join(ctx, B, table_b, key_b, pred_b, npred_b, &J));
    const uint64_t id = ctx->next_id++;
    ctx->joins.emplace(id, J);
    *out = id;
    *build_is_a = on_a ? 1u : 0u;
    *rows_a = na;
    *rows_b = nb;
    return TGP_OK;
}

int tgp_join_drop(tgp_ctx* ctx, tgp_join_id id) {
    if (!ctx) return TGP_INVALID_ARG;
    auto it = ctx->joins.find(id);
    if (it == ctx->joins.end()) return fail(ctx, TGP_NOT_FOUND, "unknown join id");
    free_join(ctx, it->second);
    ctx->joins.erase(it);
    return TGP_OK;
}

int tgp_join_probe_pairs(tgp_ctx* ctx, tgp_join_id join, tgp_table_id probe_table, uint32_t probe_key_column,
                         const tgp_pred_node* pred, uint32_t npred, uint32_t* probe_rows, uint32_t* build_rows,
                         uint64_t cap, uint64_t* npairs) {
    if (!ctx || !npairs) return fail(ctx, TGP_INVALID_ARG, "null argument");
    JoinTable* J;
    TGP_TRY(join_lookup(ctx, join, &J));
    const Table* T;
    TGP_TRY(get_table(ctx, probe_table, &T));
    if (probe_key_column >= T->cols.size()) return fail(ctx, TGP_INVALID_ARG, "probe key column out of range");
    Builder b(ctx, T);
    TGP_TRY(b.add_pred(pred, npred));
    int ks;
    TGP_TRY(b.slot_of(probe_key_column, &ks));
    Plan& P = b.P;
    attach_join(P, *J, ks);
    // Pass 1 counts pairs (out_cap 0), pass 2 writes them.
    Carve cv;
    TGP_TRY(arena_reserve(ctx, 256, &cv));
    P.counters = cv.take<unsigned long long>(4);
    P.err = cv.take<uint32_t>(4);
    P.acc = cv.take<unsigned long long>(2);
    TGP_CUDA(cudaMemsetAsync(P.counters, 0, 32, ctx->stream));
    TGP_CUDA(cudaMemsetAsync(P.err, 0, 16, ctx->stream));
    P.out_pairs = nullptr;
    P.out_cap = 0;
    TGP_TRY(size_smem(ctx, P, 0));
    TGP_TRY(launch(ctx, P, MODE_JOIN_PAIRS, false));
    unsigned long long counters[4];
    uint32_t err = 0;
    TGP_CUDA(cudaMemcpyAsync(counters, P.counters, 32, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaMemcpyAsync(&err, P.err, 4, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    TGP_TRY(check_kernel_err(ctx, err));
    const uint64_t n = counters[1];
    *npairs = n;
    if (n > cap) return fail(ctx, TGP_CAPACITY, "pair buffers too small");
    if (n == 0) return TGP_OK;
    if (!probe_rows || !build_rows) return fail(ctx, TGP_INVALID_ARG, "null pair buffers");
    size_t sort_bytes = 0;
    sort_pairs(nullptr, nullptr, n, nullptr, &sort_bytes, ctx->stream);
    const bool dev_out = is_device_ptr(probe_rows) && is_device_ptr(build_rows);
    TGP_TRY(arena_reserve(ctx, n * 16 + sort_bytes + (dev_out ? 0 : n * 8) + 1024, &cv));
    unsigned long long* pa = cv.take<unsigned long long>(n);
    unsigned long long* pb = cv.take<unsigned long long>(n);
    void* stmp = cv.take<uint8_t>(sort_bytes + 16);
    P.counters = cv.take<unsigned long long>(4);
    P.err = cv.take<uint32_t>(4);
    P.acc = cv.take<unsigned long long>(2);
    TGP_CUDA(cudaMemsetAsync(P.counters, 0, 32, ctx->stream));
    TGP_CUDA(cudaMemsetAsync(P.err, 0, 16, ctx->stream));
    P.out_pairs = pa;
    P.out_cap = n;
    TGP_TRY(launch(ctx, P, MODE_JOIN_PAIRS, false));
    TGP_CUDA(sort_pairs(pa, pb, n, stmp, &sort_bytes, ctx->stream));
    if (dev_out) {
        TGP_CUDA(launch_split_pairs(pb, n, probe_rows, build_rows, ctx->sms, ctx->stream));
    } else {
        uint32_t* sp = cv.take<uint32_t>(n);
        uint32_t* sb = cv.take<uint32_t>(n);
        TGP_CUDA(launch_split_pairs(pb, n, sp, sb, ctx->sms, ctx->stream));
        TGP_TRY(copy_out(ctx, probe_rows, sp, n * 4));
        TGP_TRY(copy_out(ctx, build_rows, sb, n * 4));
    }
    TGP_CUDA(cudaMemcpyAsync(&err, P.err, 4, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    return check_kernel_err(ctx, err);
}


// --------------------------------------------------------------------------
// Kernel-table boundary (src/kernel/mod.rs)
// --------------------------------------------------------------------------
static const tgp_kernel_info kGpuKernels[] = {
    {TGP_OP_SCAN_EQ_U64, TGP_CPU_GPU_SM100A, TGP_TIER_HBM, 0, "scan_eq_u64_sm100a_hbm"},
    {TGP_OP_SCAN_RANGE_U64, TGP_CPU_GPU_SM100A, TGP_TIER_HBM, 0, "scan_range_u64_sm100a_hbm"},
    {TGP_OP_SCAN_MULTI_PREDICATE, TGP_CPU_GPU_SM100A, TGP_TIER_HBM, 0, "scan_multi_predicate_sm100a_hbm"},
    {TGP_OP_HASH_BUILD, TGP_CPU_GPU_SM100A, TGP_TIER_HBM, 0, "hash_build_sm100a_hbm"},
    {TGP_OP_HASH_PROBE, TGP_CPU_GPU_SM100A, TGP_TIER_HBM, 0, "hash_probe_sm100a_hbm"},
    {TGP_OP_AGGREGATE_SUM_F64, TGP_CPU_GPU_SM100A, TGP_TIER_HBM, 0, "sum_f64_sm100a_hbm"},
    {TGP_OP_AGGREGATE_COUNT_DISTINCT, TGP_CPU_GPU_SM100A, TGP_TIER_HBM, 0, "count_distinct_sm100a_hbm"},
};

uint32_t tgp_kernel_count(void) { return sizeof(kGpuKernels) / sizeof(kGpuKernels[0]); }

int tgp_kernel_info_at(uint32_t i, tgp_kernel_info* out) {
    if (!out || i >= tgp_kernel_count()) return TGP_INVALID_ARG;
    *out = kGpuKernels[i];
    return TGP_OK;
}

// Places `bytes` of kernel input (host or device memory) in 16-byte-aligned
// device memory. Aligned device input is used in place.
static int stage_input(tgp_ctx* ctx, const void* input, size_t bytes, const uint8_t** dev) {
    if (bytes == 0) {
        *dev = nullptr;
        return TGP_OK;
    }
    if (is_device_ptr(input) && reinterpret_cast<uintptr_t>(input) % 16 == 0) {
        *dev = static_cast<const uint8_t*>(input);
        return TGP_OK;
    }
    const size_t need = ((bytes + 255) / 256) * 256;
    if (need > ctx->kin_cap) {
        TGP_CUDA(cudaStreamSynchronize(ctx->stream));
        if (ctx->kin) cudaFree(ctx->kin);
        ctx->kin = nullptr;
        ctx->kin_cap = 0;
        if (cudaMalloc(&ctx->kin, need) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, TGP_OOM, "kernel input staging allocation failed");
        }
        ctx->kin_cap = need;
    }
    TGP_CUDA(cudaMemcpyAsync(ctx->kin, input, bytes, cudaMemcpyDefault, ctx->stream));
    *dev = ctx->kin;
    return TGP_OK;
}

// A one-column table of u64 cells over staged device memory.
static Table cell_table(const uint8_t* dev, uint64_t n) {
    Table t;
    t.rows = n;
    Column c;
    c.dtype = DT_U64;
    c.coltype = TGP_CT_DATE;  // raw cells compare unsigned (src/kernel/scan.rs:99-115)
    c.width = 8;
    c.dptr = const_cast<uint8_t*>(dev);
    t.cols.push_back(c);
    return t;
}

static tgp_pred_node leaf_node(uint32_t cmp, uint64_t lit, uint64_t lit2 = 0) {
    tgp_pred_node n;
    std::memset(&n, 0, sizeof(n));
    n.kind = TGP_PN_LEAF;
    n.column = 0;
    n.cmp = cmp;
    n.lit = lit;
    n.lit2 = lit2;
    return n;
}

// Number of (probe, build) key matches of n staged probe cells.
static int count_matches(tgp_ctx* ctx, const Table& probe, const JoinTable& J, uint64_t* out) {
    Builder b(ctx, &probe);
    int ks;
    TGP_TRY(b.slot_of(0, &ks));
    attach_join(b.P, J, ks);
    Plan& P = b.P;
    Carve cv;
    TGP_TRY(arena_reserve(ctx, 256, &cv));
    P.acc = cv.take<unsigned long long>(2);
    P.counters = cv.take<unsigned long long>(4);
    P.err = cv.take<uint32_t>(4);
    TGP_CUDA(cudaMemsetAsync(P.acc, 0, 16, ctx->stream));
    TGP_CUDA(cudaMemsetAsync(P.counters, 0, 32, ctx->stream));
    TGP_CUDA(cudaMemsetAsync(P.err, 0, 16, ctx->stream));
    P.ngroups = 1;
    P.nthreads = 512;
    TGP_TRY(size_smem(ctx, P, 512 * 8));  // one private count slot per thread
    TGP_TRY(launch(ctx, P, MODE_GROUP_PRIVATE, false));
    unsigned long long acc[2];
    uint32_t err = 0;
    TGP_CUDA(cudaMemcpyAsync(acc, P.acc, 16, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaMemcpyAsync(&err, P.err, 4, cudaMemcpyDeviceToHost, ctx->stream));
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    TGP_TRY(check_kernel_err(ctx, err));
    *out = acc[0];
    return TGP_OK;
}

int tgp_kernel_execute(tgp_ctx* ctx, uint32_t op, const void* input, void* output, const tgp_kernel_params* p,
                       tgp_kernel_result* r) {
    if (!ctx || !p || !r) return fail(ctx, TGP_INVALID_ARG, "null argument");
    std::memset(r, 0, sizeof(*r));
    const uint64_t n = p->cell_count;
    if (n >= (1ull << 32)) return fail(ctx, TGP_UNSUPPORTED, "cell_count must be below 2^32");
    if (n && !input) return fail(ctx, TGP_INVALID_ARG, "null input");
    TGP_CUDA(cudaSetDevice(ctx->device));
    switch (op) {
        case TGP_OP_SCAN_EQ_U64:
        case TGP_OP_SCAN_RANGE_U64:
        case TGP_OP_SCAN_MULTI_PREDICATE: {
            const uint8_t* dev;
            TGP_TRY(stage_input(ctx, input, n * 8, &dev));
            Table t = cell_table(dev, n);
            tgp_pred_node prog[5];
            uint32_t np = 0;
            if (op == TGP_OP_SCAN_EQ_U64) {
                prog[np++] = leaf_node(TGP_CMP_EQ, p->target_u64);
            } else if (op == TGP_OP_SCAN_RANGE_U64) {
                prog[np++] = leaf_node(TGP_CMP_BETWEEN, p->low_u64, p->high_u64);
            } else {
                // ScanMultiPredicateScalar (src/kernel/scan.rs:124-160): AND of the
                // first min(predicate_count, 3) predicates; none = every cell.
                const uint32_t k = std::min<uint32_t>(p->predicate_count, 3);
                const uint8_t ops[3] = {p->pred1_op, p->pred2_op, p->pred3_op};
                const uint64_t tg[3] = {p->target_u64, p->target2_u64, p->target3_u64};
                for (uint32_t i = 0; i < k; ++i) {
                    const uint32_t cmp = ops[i] == TGP_PRED_GT ? TGP_CMP_GT : ops[i] == TGP_PRED_LT ? TGP_CMP_LT : TGP_CMP_EQ;
                    if (ops[i] > TGP_PRED_LT) return fail(ctx, TGP_INVALID_ARG, "bad predicate op");
                    prog[np++] = leaf_node(cmp, tg[i]);
                    if (i > 0) {
                        std::memset(&prog[np], 0, sizeof(tgp_pred_node));
                        prog[np++].kind = TGP_PN_AND;
                    }
                }
            }
            uint32_t words[2] = {0, 0};
            uint64_t cnt = 0;
            const bool want_mask = op == TGP_OP_SCAN_EQ_U64 && n > 0;
            TGP_TRY(filter_impl(ctx, &t, prog, np, want_mask ? reinterpret_cast<uint8_t*>(words) : nullptr, nullptr,
                                0, &cnt, want_mask ? 2u : 0u));
            r->count = cnt;
            if (want_mask) {
                uint64_t m = static_cast<uint64_t>(words[0]) | (static_cast<uint64_t>(words[1]) << 32);
                if (n < 64) m &= (1ull << n) - 1;
                r->mask = m;
            }
            return TGP_OK;
        }
        case TGP_OP_AGGREGATE_SUM_F64: {
            r->count = n;
            if (n == 0) return TGP_OK;
            const uint8_t* dev;
            TGP_TRY(stage_input(ctx, input, n * 8, &dev));
            const int blocks = static_cast<int>(std::min<uint64_t>((n + 255) / 256, static_cast<uint64_t>(ctx->sms) * 4));
            Carve cv;
            TGP_TRY(arena_reserve(ctx, blocks * 16 + 256, &cv));
            double* part = cv.take<double>(2 * blocks);
            TGP_CUDA(launch_sum_f64(reinterpret_cast<const double*>(dev), n, part, blocks, ctx->stream));
            std::vector<double> h(2 * blocks);
            TGP_CUDA(cudaMemcpyAsync(h.data(), part, h.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
            TGP_CUDA(cudaStreamSynchronize(ctx->stream));
            // Double-double accumulation of the per-block pairs.
            double hi = 0.0, lo = 0.0;
            for (int i = 0; i < blocks; ++i) {
                const double bh = h[2 * i], bl = h[2 * i + 1];
                const double s = hi + bh;
                const double bb = s - hi;
                double e = (hi - (s - bb)) + (bh - bb);
                e += lo + bl;
                hi = s + e;
                lo = e - (hi - s);
            }
            r->sum = hi;
            return TGP_OK;
        }
        case TGP_OP_AGGREGATE_COUNT_DISTINCT: {
            if (n == 0) return TGP_OK;
            const uint8_t* dev;
            TGP_TRY(stage_input(ctx, input, n * 8, &dev));
            const uint64_t cap = next_pow2(std::max<uint64_t>(16, 2 * n));
            Carve cv;
            TGP_TRY(arena_reserve(ctx, cap * 8 + 256, &cv));
            unsigned long long* set = cv.take<unsigned long long>(cap);
            unsigned long long* counters = cv.take<unsigned long long>(2);
            uint32_t* err = cv.take<uint32_t>(4);
            TGP_CUDA(cudaMemsetAsync(set, 0xff, cap * 8, ctx->stream));
            TGP_CUDA(cudaMemsetAsync(counters, 0, 16, ctx->stream));
            TGP_CUDA(cudaMemsetAsync(err, 0, 16, ctx->stream));
            const int blocks = static_cast<int>(std::min<uint64_t>((n + 255) / 256, static_cast<uint64_t>(ctx->sms) * 8));
            TGP_CUDA(launch_count_distinct(reinterpret_cast<const unsigned long long*>(dev), n, set, cap - 1, log2u(cap),
                                           counters, err, blocks, ctx->stream));
            unsigned long long hc[2];
            uint32_t herr = 0;
            TGP_CUDA(cudaMemcpyAsync(hc, counters, 16, cudaMemcpyDeviceToHost, ctx->stream));
            TGP_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, ctx->stream));
            TGP_CUDA(cudaStreamSynchronize(ctx->stream));
            TGP_TRY(check_kernel_err(ctx, herr));
            r->count = hc[0] + (hc[1] ? 1 : 0);
            return TGP_OK;
        }
        case TGP_OP_HASH_BUILD: {
            if (!output) return fail(ctx, TGP_INVALID_ARG, "HashBuild needs an output slot for the table handle");
            const uint8_t* dev;
            TGP_TRY(stage_input(ctx, input, n * 8, &dev));
            Table t = cell_table(dev, n);
            t.cols[0].coltype = TGP_CT_INT;
            TGP_TRY(compute_stats(ctx, t));
            JoinTable* J = new (std::nothrow) JoinTable();
            if (!J) return fail(ctx, TGP_OOM, "host allocation failed");
            int st = build_join(ctx, &t, 0, 0, nullptr, 0, J);
            if (st != TGP_OK) {
                delete J;
                return st;
            }
            ctx->hash_handles.insert(J);
            void* handle = J;
            if (is_device_ptr(output)) {
                TGP_CUDA(cudaMemcpy(output, &handle, 8, cudaMemcpyHostToDevice));
            } else {
                std::memcpy(output, &handle, 8);
            }
            r->count = n;
            return TGP_OK;
        }
        case TGP_OP_HASH_PROBE: {
            // input = [handle: 8 bytes][cell_count u64 keys] (src/kernel/hash.rs:171-178).
            void* handle = nullptr;
            if (is_device_ptr(input)) TGP_CUDA(cudaMemcpy(&handle, input, 8, cudaMemcpyDeviceToHost));
            else std::memcpy(&handle, input, 8);
            if (!ctx->hash_handles.count(handle)) return fail(ctx, TGP_INVALID_ARG, "unknown hash table handle");
            if (n == 0) return TGP_OK;
            const uint8_t* dev;
            TGP_TRY(stage_input(ctx, static_cast<const uint8_t*>(input) + 8, n * 8, &dev));
            Table t = cell_table(dev, n);
            uint64_t matches = 0;
            TGP_TRY(count_matches(ctx, t, *static_cast<JoinTable*>(handle), &matches));
            r->count = matches;
            return TGP_OK;
        }
        default:
            return fail(ctx, TGP_UNSUPPORTED, "operator has no GPU kernel");
    }
}

int tgp_hash_table_free(tgp_ctx* ctx, void* handle) {
    if (!ctx) return TGP_INVALID_ARG;
    auto it = ctx->hash_handles.find(handle);
    if (it == ctx->hash_handles.end()) return fail(ctx, TGP_INVALID_ARG, "unknown hash table handle");
    TGP_CUDA(cudaStreamSynchronize(ctx->stream));
    JoinTable* J = static_cast<JoinTable*>(handle);
    free_join(ctx, *J);
    delete J;
    ctx->hash_handles.erase(it);
    return TGP_OK;
}

}  // extern "C"
