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
// ref_grouped_q1 and ref_highcard restate the grouped paths (execute_grouped
// and try_accumulator_grouped), whose chunked grouping the reference runs on
// rayon's thread pool and this file on OpenMP threads.
#include <immintrin.h>

#include <omp.h>

#include <algorithm>
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

// A u64-keyed open-addressing map with values stored in place, standing in
// for the reference's FxHashMap (hashbrown: one allocation for the table, FxHash
// of the key = the key times 0x517cc1b727220a95, grown at 7/8 load). Linear
// probing on the high bits of the hash.
template <class V>
class FlatMap {
public:
    FlatMap() { reset(16); }
    // The value of key k, default-constructed when k is new.
    V& operator[](uint64_t k) {
        if ((n_ + 1) * 8 > cap_ * 7) grow();
        const size_t i = probe(k);
        if (!used_[i]) {
            used_[i] = 1;
            keys_[i] = k;
            ++n_;
        }
        return vals_[i];
    }
    V* find(uint64_t k) {
        const size_t i = probe(k);
        return used_[i] ? &vals_[i] : nullptr;
    }
    template <class F>
    void for_each(F&& f) {
        for (size_t i = 0; i < cap_; ++i)
            if (used_[i]) f(keys_[i], vals_[i]);
    }

private:
    size_t probe(uint64_t k) const {
        size_t i = static_cast<size_t>((k * 0x517cc1b727220a95ull) >> shift_);
        while (used_[i] && keys_[i] != k) i = (i + 1) & (cap_ - 1);
        return i;
    }
    void reset(size_t cap) {
        cap_ = cap;
        shift_ = 64 - __builtin_ctzll(cap);
        keys_.assign(cap, 0);
        vals_.clear();
        vals_.resize(cap);
        used_.assign(cap, 0);
        n_ = 0;
    }
    void grow() {
        std::vector<uint64_t> k = std::move(keys_);
        std::vector<V> v = std::move(vals_);
        std::vector<uint8_t> u = std::move(used_);
        reset(cap_ * 2);
        for (size_t i = 0; i < u.size(); ++i)
            if (u[i]) {
                const size_t j = probe(k[i]);
                used_[j] = 1;
                keys_[j] = k[i];
                vals_[j] = std::move(v[i]);
                ++n_;
            }
    }
    std::vector<uint64_t> keys_;
    std::vector<V> vals_;
    std::vector<uint8_t> used_;
    size_t cap_ = 0, n_ = 0;
    int shift_ = 0;
};

// Merges per-chunk hash → row-list maps in chunk order into group row lists
// (the order the reference's execute_grouped merge appends rows in).
std::vector<std::vector<size_t>> merge_groups(std::vector<FlatMap<std::vector<size_t>>>& local) {
    FlatMap<size_t> gid;
    std::vector<std::vector<size_t>> groups;
    groups.reserve(1024);
    for (auto& m : local)
        m.for_each([&](uint64_t h, std::vector<size_t>& rows) {
            size_t* g = gid.find(h);
            size_t id;
            if (!g) {
                id = groups.size();
                gid[h] = id;
                groups.emplace_back();
            } else {
                id = *g;
            }
            groups[id].insert(groups[id].end(), rows.begin(), rows.end());
        });
    return groups;
}

constexpr size_t kGroupChunk = 65536;  // GROUP_CHUNK_SIZE (aggregate.rs:582, accum_grouped.rs:197)

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

}  // extern "C"

namespace {

// build_mask over a conjunction of leaves (every leaf a fresh bitmap ANDed in).
Bitmap mask_of(const uint64_t* const* cols, uint64_t n, const ref_leaf* leaves, uint32_t nleaves) {
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
    return mask;
}

}  // namespace

extern "C" {

// WHERE <conjunction of leaves> → SUM(cells[a] * cells[b]) (f64), COUNT(*).
// cols: ncols pointers to n u64 cells. Returns wall seconds of the query.
double ref_scan_sum_mul(const uint64_t* const* cols, uint64_t n, const ref_leaf* leaves, uint32_t nleaves,
                        uint32_t a, uint32_t b, double* sum_out, uint64_t* count_out) {
    const auto t0 = std::chrono::steady_clock::now();
    Bitmap mask = mask_of(cols, n, leaves, nleaves);
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

// The grouped aggregate of the TPC-H Q1 shape the reference's way
// (execute_grouped, aggregate.rs:507-697): WHERE mask → indices; chunks of
// 65,536 indices grouped in parallel (rayon there, OpenMP here) into
// hash → row-list maps, the group key hash h = h * 0x517cc1b727220a95 + cell
// over the GROUP BY cells (aggregate.rs:594-603); the chunk maps merged in
// chunk order; then, group by group, each aggregate over the group's rows
// (eval_agg_expr / sum_vec, aggregate.rs:1291-1792):
//   COUNT(*) = rows; SUM(q), SUM(p) = wrapping i64 sums of the cells;
//   SUM(p * (100 - d)) = f64 sum of p as f64 * (100 - d) as f64;
//   SUM(p * (100 - d) * (100 + t)) = f64 sum of the exact i64 product;
//   AVG(q) = f64(SUM(q)) / rows.
// Per group out: keys[2], count, sum_q, sum_p (i64), disc_price, charge,
// avg_q (f64). Returns wall seconds; *ngroups = groups (at most cap written).
double ref_grouped_q1(const uint64_t* const* cols, uint64_t n, const ref_leaf* leaves, uint32_t nleaves,
                      uint32_t ka, uint32_t kb, uint32_t cq, uint32_t cp, uint32_t cd, uint32_t ct, int threads,
                      uint64_t cap, int64_t* keys, int64_t* ints, double* flts, uint64_t* ngroups) {
    const auto t0 = std::chrono::steady_clock::now();
    Bitmap mask = mask_of(cols, n, leaves, nleaves);
    const std::vector<size_t> idx = iter_set_bits(mask);
    const size_t nchunks = (idx.size() + kGroupChunk - 1) / kGroupChunk;
    std::vector<FlatMap<std::vector<size_t>>> local(nchunks);
    const uint64_t* gk[2] = {cols[ka], cols[kb]};
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (size_t c = 0; c < nchunks; ++c) {
        const size_t lo = c * kGroupChunk, hi = std::min(idx.size(), lo + kGroupChunk);
        auto& m = local[c];
        for (size_t i = lo; i < hi; ++i) {
            const size_t r = idx[i];
            uint64_t h = 0;
            for (int k = 0; k < 2; ++k) h = h * 0x517cc1b727220a95ull + gk[k][r];
            m[h].push_back(r);
        }
    }
    std::vector<std::vector<size_t>> groups = merge_groups(local);
    const uint64_t *q = cols[cq], *p = cols[cp], *d = cols[cd], *t = cols[ct];
    for (size_t g = 0; g < groups.size(); ++g) {
        const std::vector<size_t>& rows = groups[g];
        uint64_t sq = 0, sp = 0;
        double dp = 0.0, ch = 0.0;
        for (size_t r : rows) sq += q[r];
        for (size_t r : rows) sp += p[r];
        for (size_t r : rows)
            dp += static_cast<double>(p[r]) * static_cast<double>(100 - static_cast<int64_t>(d[r]));
        for (size_t r : rows) {
            const int64_t v = static_cast<int64_t>(static_cast<uint64_t>(static_cast<int64_t>(p[r])) *
                                                   static_cast<uint64_t>(100 - static_cast<int64_t>(d[r])) *
                                                   static_cast<uint64_t>(100 + static_cast<int64_t>(t[r])));
            ch += static_cast<double>(v);
        }
        if (g < cap) {
            keys[2 * g] = static_cast<int64_t>(gk[0][rows[0]]);
            keys[2 * g + 1] = static_cast<int64_t>(gk[1][rows[0]]);
            ints[3 * g] = static_cast<int64_t>(rows.size());
            ints[3 * g + 1] = static_cast<int64_t>(sq);
            ints[3 * g + 2] = static_cast<int64_t>(sp);
            flts[3 * g] = dp;
            flts[3 * g + 1] = ch;
            flts[3 * g + 2] = static_cast<double>(static_cast<int64_t>(sq)) / static_cast<double>(rows.size());
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    *ngroups = groups.size();
    return std::chrono::duration<double>(t1 - t0).count();
}

// GROUP BY key, COUNT(*), SUM(value) the reference's way
// (try_accumulator_grouped, accum_grouped.rs:55-300): all rows selected (no
// WHERE: an all-ones mask → indices); chunks of 65,536 indices accumulated in
// parallel into hash → slot-vector maps ([key cell, count, wrapping sum], a
// vector allocated per new group), the key hash being the key cell itself
// (h = 0 * K + cell); the chunk maps merged one by one into a global map.
// Per group out: key, count, sum (wrapping i64). Returns wall seconds.
double ref_highcard(const uint64_t* key, const uint64_t* val, uint64_t n, int threads, uint64_t cap,
                    int64_t* keys, int64_t* counts, int64_t* sums, uint64_t* ngroups) {
    const auto t0 = std::chrono::steady_clock::now();
    Bitmap mask = Bitmap::all_ones(n);
    const std::vector<size_t> idx = iter_set_bits(mask);
    const size_t nchunks = (idx.size() + kGroupChunk - 1) / kGroupChunk;
    std::vector<FlatMap<std::vector<uint64_t>>> local(nchunks);
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (size_t c = 0; c < nchunks; ++c) {
        const size_t lo = c * kGroupChunk, hi = std::min(idx.size(), lo + kGroupChunk);
        auto& m = local[c];
        for (size_t i = lo; i < hi; ++i) {
            const size_t r = idx[i];
            std::vector<uint64_t>& acc = m[key[r]];
            if (acc.empty()) acc = {key[r], 0, 0};  // slots allocated per new group
            acc[1] += 1;
            acc[2] += val[r];
        }
    }
    FlatMap<std::vector<uint64_t>> global;
    for (auto& m : local)
        m.for_each([&](uint64_t k, std::vector<uint64_t>& acc) {
            std::vector<uint64_t>* e = global.find(k);
            if (!e) {
                global[k] = std::move(acc);
            } else {
                (*e)[1] += acc[1];
                (*e)[2] += acc[2];
            }
        });
    const auto t1 = std::chrono::steady_clock::now();
    uint64_t g = 0;
    global.for_each([&](uint64_t, std::vector<uint64_t>& acc) {
        if (g < cap) {
            keys[g] = static_cast<int64_t>(acc[0]);
            counts[g] = static_cast<int64_t>(acc[1]);
            sums[g] = static_cast<int64_t>(acc[2]);
        }
        ++g;
    });
    *ngroups = g;
    return std::chrono::duration<double>(t1 - t0).count();
}

// The join + grouped aggregate the reference's way (hash_join_with_keys,
// join.rs:544-939, then execute_grouped): the build side is the dimension
// filtered on order_day < day_lt and materialised (filter_table); a chained
// hash table (directory of next_pow2(2n) heads carrying an OR of 16-bit tags,
// CRC32 hash times 0x8648DBDB00000001, join_hash_table.rs:76-200) and a bloom
// filter (10 bits per key, 3 probes by double hashing of two CRC32 passes,
// bloom_filter.rs:81-270) over its keys; the fact side probed in parallel
// chunks of 65,536 rows (bloom test, then the chain), each chunk emitting
// (probe row, build row) pairs; the joined table materialised column by
// column; then GROUP BY segment over all its rows: chunked parallel grouping
// and per group COUNT(*) and the f64 sum of price as f64 * (100 - disc) as f64.
// Per group out: segment, count, sum. Returns wall seconds.
double ref_join_group(const uint64_t* fk, const uint64_t* price, const uint64_t* disc, uint64_t nprobe,
                      const uint64_t* dkey, const uint64_t* dday, const uint64_t* dseg, uint64_t nbuild,
                      uint64_t day_lt, int threads, uint64_t cap, int64_t* keys, int64_t* counts, double* sums,
                      uint64_t* ngroups) {
    const auto t0 = std::chrono::steady_clock::now();
    // Build side: filter, then gather its columns.
    Bitmap bm = filter(dday, nbuild, day_lt, LT, false);
    const std::vector<size_t> bsel = iter_set_bits(bm);
    const size_t nb = bsel.size();
    std::vector<uint64_t> bkey(nb), bday(nb), bseg(nb);
    for (size_t i = 0; i < nb; ++i) {
        bkey[i] = dkey[bsel[i]];
        bday[i] = dday[bsel[i]];
        bseg[i] = dseg[bsel[i]];
    }
    // Chained table with tagged heads.
    size_t dir_size = 16;
    while (dir_size < 2 * nb) dir_size <<= 1;
    const int shift = 64 - __builtin_ctzll(dir_size);
    std::vector<uint64_t> dir(dir_size, 0);
    struct Entry {
        uint64_t key;
        uint32_t row, next;
    };
    std::vector<Entry> ent(nb + 1, Entry{0, 0, 0});
    auto jhash = [](uint64_t k) { return static_cast<uint64_t>(_mm_crc32_u64(0, k)) * 0x8648DBDB00000001ull; };
    auto tag_of = [](uint64_t h) { return static_cast<uint16_t>((h >> 16) | 1); };
    // Bloom filter.
    size_t nwords = 1;
    while (nwords < (nb * 10 + 63) / 64) nwords <<= 1;
    std::vector<uint64_t> bloom(nwords, 0);
    auto mix = [](uint64_t z) {
        z += 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    auto pair = [&](uint64_t k, uint64_t& h1, uint64_t& h2) {
        h1 = mix(_mm_crc32_u64(0, k));
        h2 = mix(_mm_crc32_u64(~0ull, k)) | 1;
    };
    for (size_t r = 0; r < nb; ++r) {
        const uint64_t h = jhash(bkey[r]);
        const size_t slot = h >> shift;
        const uint32_t e = static_cast<uint32_t>(r + 1);
        ent[e] = Entry{bkey[r], static_cast<uint32_t>(r), static_cast<uint32_t>(dir[slot] & 0xFFFFFFFFull)};
        const uint16_t t = static_cast<uint16_t>(dir[slot] >> 48) | tag_of(h);
        dir[slot] = (static_cast<uint64_t>(t) << 48) | e;
        uint64_t h1, h2;
        pair(bkey[r], h1, h2);
        for (int i = 0; i < 3; ++i, h1 += h2) bloom[(h1 >> 6) & (nwords - 1)] |= 1ull << (h1 & 63);
    }
    // Probe in parallel chunks.
    const size_t nchunks = (nprobe + kGroupChunk - 1) / kGroupChunk;
    std::vector<std::vector<uint32_t>> lsrc(nchunks), rsrc(nchunks);
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (size_t c = 0; c < nchunks; ++c) {
        const size_t lo = c * kGroupChunk, hi = std::min<size_t>(nprobe, lo + kGroupChunk);
        auto& L = lsrc[c];
        auto& R = rsrc[c];
        for (size_t p = lo; p < hi; ++p) {
            const uint64_t k = fk[p];
            uint64_t h1, h2;
            pair(k, h1, h2);
            bool maybe = true;
            for (int i = 0; i < 3 && maybe; ++i, h1 += h2) maybe = (bloom[(h1 >> 6) & (nwords - 1)] >> (h1 & 63)) & 1;
            if (!maybe) continue;
            const uint64_t h = jhash(k);
            const uint64_t head = dir[h >> shift];
            const uint16_t t = static_cast<uint16_t>(head >> 48), want = tag_of(h);
            if (t == 0 || (t & want) != want) continue;
            for (uint32_t e = static_cast<uint32_t>(head & 0xFFFFFFFFull); e; e = ent[e].next)
                if (ent[e].key == k) {
                    L.push_back(static_cast<uint32_t>(p));
                    R.push_back(ent[e].row);
                }
        }
    }
    // Materialise the joined table (every column of both sides).
    std::vector<size_t> off(nchunks + 1, 0);
    for (size_t c = 0; c < nchunks; ++c) off[c + 1] = off[c] + lsrc[c].size();
    const size_t nj = off[nchunks];
    std::vector<uint64_t> jfk(nj), jprice(nj), jdisc(nj), jkey(nj), jday(nj), jseg(nj);
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (size_t c = 0; c < nchunks; ++c)
        for (size_t i = 0; i < lsrc[c].size(); ++i) {
            const size_t o = off[c] + i, p = lsrc[c][i], b = rsrc[c][i];
            jfk[o] = fk[p];
            jprice[o] = price[p];
            jdisc[o] = disc[p];
            jkey[o] = bkey[b];
            jday[o] = bday[b];
            jseg[o] = bseg[b];
        }
    // GROUP BY segment over all joined rows.
    const std::vector<size_t> idx = iter_set_bits(Bitmap::all_ones(nj));
    const size_t gch = (idx.size() + kGroupChunk - 1) / kGroupChunk;
    std::vector<FlatMap<std::vector<size_t>>> local(gch);
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (size_t c = 0; c < gch; ++c) {
        const size_t lo = c * kGroupChunk, hi = std::min(idx.size(), lo + kGroupChunk);
        for (size_t i = lo; i < hi; ++i) local[c][jseg[idx[i]]].push_back(idx[i]);
    }
    std::vector<std::vector<size_t>> groups = merge_groups(local);
    for (size_t g = 0; g < groups.size(); ++g) {
        double sum = 0.0;
        for (size_t r : groups[g])
            sum += static_cast<double>(jprice[r]) * static_cast<double>(100 - static_cast<int64_t>(jdisc[r]));
        if (g < cap) {
            keys[g] = static_cast<int64_t>(jseg[groups[g][0]]);
            counts[g] = static_cast<int64_t>(groups[g].size());
            sums[g] = sum;
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    *ngroups = groups.size();
    return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
