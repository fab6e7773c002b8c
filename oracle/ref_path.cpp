// ref_path.cpp — TEST / BASELINE INFRASTRUCTURE ONLY. A C++ restatement of the
// reference's CPU execution of the benchmark queries, used as the timed CPU
// baseline (bench.py) and checked against the exact oracle in tests. The
// product never links or calls it.
//
// It follows the reference's algorithm step by step on its storage layout
// (one u64 cell per value, src/datasource/table.rs:25-30):
//   1. build_mask (src/engine/query_interpreter/expr.rs:633-760): start from an
//      all-ones Bitmap; every leaf allocates a fresh Bitmap from a full-column
//      AVX-512 filter (4 independent 8-lane compares per iteration,
//      src/exec/bitmap.rs:642-700), then mask.and_inplace(bm) (AVX-512BW, 64
//      bytes per iteration, bitmap.rs:506-531). BETWEEN = ge.and(le) into a new
//      bitmap first (expr.rs:687-705). Int compares signed, Date unsigned.
//   2. execute_grouped → scalar: indices = mask.iter_set_bits().collect()
//      (byte-skipping tzcnt iterator, bitmap.rs:278-316), then
//      SUM(Col * Col) for Int columns: sum += ca[i] as f64 * cb[i] as f64
//      (aggregate.rs:1589-1601), COUNT(*) = indices.len() (aggregate.rs:1298).
// Both steps run on one thread, as in the reference (no rayon on this path).
#include <immintrin.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

enum Cmp { EQ = 0, NE = 1, LT = 2, LE = 3, GT = 4, GE = 5 };

struct Bitmap {
    std::vector<uint8_t> bits;
    size_t len = 0;
    explicit Bitmap(size_t n) : bits((n + 7) / 8, 0), len(n) {}
    static Bitmap all_ones(size_t n) {
        Bitmap b(n);
        std::memset(b.bits.data(), 0xFF, b.bits.size());
        const unsigned unused = (8 - (n & 7)) & 7;
        if (unused && !b.bits.empty()) b.bits.back() >>= unused;
        return b;
    }
};

__attribute__((target("avx512f"))) inline __mmask8 cmp8(__m512i v, __m512i t, int op, bool sgn) {
    if (sgn) {
        switch (op) {
            case EQ: return _mm512_cmpeq_epi64_mask(v, t);
            case NE: return static_cast<__mmask8>(~_mm512_cmpeq_epi64_mask(v, t));
            case LT: return _mm512_cmplt_epi64_mask(v, t);
            case LE: return _mm512_cmple_epi64_mask(v, t);
            case GT: return _mm512_cmpgt_epi64_mask(v, t);
            default: return _mm512_cmpge_epi64_mask(v, t);
        }
    }
    switch (op) {
        case EQ: return _mm512_cmpeq_epu64_mask(v, t);
        case NE: return static_cast<__mmask8>(~_mm512_cmpeq_epu64_mask(v, t));
        case LT: return _mm512_cmplt_epu64_mask(v, t);
        case LE: return _mm512_cmple_epu64_mask(v, t);
        case GT: return _mm512_cmpgt_epu64_mask(v, t);
        default: return _mm512_cmpge_epu64_mask(v, t);
    }
}

inline bool cmp1(uint64_t c, uint64_t t, int op, bool sgn) {
    if (sgn) {
        const int64_t a = static_cast<int64_t>(c), b = static_cast<int64_t>(t);
        switch (op) {
            case EQ: return a == b;
            case NE: return a != b;
            case LT: return a < b;
            case LE: return a <= b;
            case GT: return a > b;
            default: return a >= b;
        }
    }
    switch (op) {
        case EQ: return c == t;
        case NE: return c != t;
        case LT: return c < t;
        case LE: return c <= t;
        case GT: return c > t;
        default: return c >= t;
    }
}

// filter_u64_avx512_inner: 4 vectors (32 rows) per iteration, 1-vector tail,
// scalar tail.
template <int OP, bool SGN>
__attribute__((target("avx512f"))) Bitmap filter_avx512(const uint64_t* col, size_t n, uint64_t val) {
    Bitmap bm(n);
    uint8_t* out = bm.bits.data();
    const __m512i t = _mm512_set1_epi64(static_cast<long long>(val));
    size_t i = 0;
    for (; i + 32 <= n; i += 32) {
        const __m512i v0 = _mm512_loadu_si512(col + i);
        const __m512i v1 = _mm512_loadu_si512(col + i + 8);
        const __m512i v2 = _mm512_loadu_si512(col + i + 16);
        const __m512i v3 = _mm512_loadu_si512(col + i + 24);
        out[(i >> 3) + 0] = cmp8(v0, t, OP, SGN);
        out[(i >> 3) + 1] = cmp8(v1, t, OP, SGN);
        out[(i >> 3) + 2] = cmp8(v2, t, OP, SGN);
        out[(i >> 3) + 3] = cmp8(v3, t, OP, SGN);
    }
    for (; i + 8 <= n; i += 8) out[i >> 3] = cmp8(_mm512_loadu_si512(col + i), t, OP, SGN);
    for (; i < n; ++i)
        if (cmp1(col[i], val, OP, SGN)) out[i >> 3] |= static_cast<uint8_t>(1u << (i & 7));
    return bm;
}

Bitmap filter(const uint64_t* col, size_t n, uint64_t val, int op, bool sgn) {
#define F(O)                                                                          \
    case O: return sgn ? filter_avx512<O, true>(col, n, val) : filter_avx512<O, false>(col, n, val);
    switch (op) {
        F(EQ) F(NE) F(LT) F(LE) F(GT) default: return sgn ? filter_avx512<GE, true>(col, n, val)
                                                         : filter_avx512<GE, false>(col, n, val);
    }
#undef F
}

__attribute__((target("avx512f,avx512bw"))) void and_inplace(Bitmap& dst, const Bitmap& src) {
    const size_t n = std::min(dst.bits.size(), src.bits.size());
    uint8_t* d = dst.bits.data();
    const uint8_t* s = src.bits.data();
    size_t i = 0;
    for (; i + 64 <= n; i += 64) {
        const __m512i a = _mm512_loadu_si512(d + i), b = _mm512_loadu_si512(s + i);
        _mm512_storeu_si512(d + i, _mm512_and_si512(a, b));
    }
    for (; i < n; ++i) d[i] &= s[i];
}

Bitmap and_new(const Bitmap& a, const Bitmap& b) {  // Bitmap::and (bitmap.rs:93-102)
    Bitmap out(std::min(a.len, b.len));
    const size_t n = std::min(a.bits.size(), b.bits.size());
    for (size_t i = 0; i < n; ++i) out.bits[i] = a.bits[i] & b.bits[i];
    return out;
}

// SetBitIter::next, byte at a time with tzcnt (bitmap.rs:278-316).
std::vector<size_t> iter_set_bits(const Bitmap& bm) {
    std::vector<size_t> out;
    size_t pos = 0;
    const size_t len = bm.len;
    const uint8_t* bits = bm.bits.data();
    while (pos < len) {
        const size_t byte_idx = pos >> 3, bit_idx = pos & 7;
        const uint8_t byte = bits[byte_idx];
        if (byte == 0) {
            pos = (byte_idx + 1) << 3;
            continue;
        }
        const uint8_t shifted = static_cast<uint8_t>(byte >> bit_idx);
        if (shifted == 0) {
            pos = (byte_idx + 1) << 3;
            continue;
        }
        const size_t r = pos + static_cast<size_t>(__builtin_ctz(shifted));
        if (r >= len) break;
        out.push_back(r);
        pos = r + 1;
    }
    return out;
}

}  // namespace

extern "C" {

// One leaf of a conjunction: column index, comparison, literal, signedness
// (1 = Int ColType, 0 = Date), and for BETWEEN (op = 6) the upper literal.
struct ref_leaf {
    uint32_t col;
    uint32_t op;   // 0..5 as Cmp, 6 = BETWEEN
    uint32_t sgn;
    uint32_t _pad;
    uint64_t lit;
    uint64_t lit2;
};

// WHERE <conjunction of leaves> → SUM(cells[a] * cells[b]) (f64), COUNT(*).
// cols: ncols pointers to n u64 cells. Returns wall seconds of the query.
double ref_scan_sum_mul(const uint64_t* const* cols, uint64_t n, const ref_leaf* leaves, uint32_t nleaves,
                        uint32_t a, uint32_t b, double* sum_out, uint64_t* count_out) {
    const auto t0 = std::chrono::steady_clock::now();
    Bitmap mask = Bitmap::all_ones(n);
    for (uint32_t i = 0; i < nleaves; ++i) {
        const ref_leaf& L = leaves[i];
        if (L.op == 6) {
            Bitmap ge = filter(cols[L.col], n, L.lit, GE, L.sgn != 0);
            Bitmap le = filter(cols[L.col], n, L.lit2, LE, L.sgn != 0);
            Bitmap bm = and_new(ge, le);
            and_inplace(mask, bm);
        } else {
            Bitmap bm = filter(cols[L.col], n, L.lit, static_cast<int>(L.op), L.sgn != 0);
            and_inplace(mask, bm);
        }
    }
    const std::vector<size_t> idx = iter_set_bits(mask);
    const uint64_t* ca = cols[a];
    const uint64_t* cb = cols[b];
    double sum = 0.0;
    for (size_t i : idx) sum += static_cast<double>(ca[i]) * static_cast<double>(cb[i]);
    const auto t1 = std::chrono::steady_clock::now();
    *sum_out = sum;
    *count_out = idx.size();
    return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
