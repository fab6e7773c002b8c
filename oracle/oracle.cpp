// oracle.cpp — TEST INFRASTRUCTURE ONLY. CPU restatement of turboGP's hot-path
// semantics, used by tests/ and bench.py's CPU-baseline leg as the parity
// checker. Nothing in the product (turbogp_b200/) links, loads or calls it.
//
// It evaluates row at a time, straight from the reference's definitions, and
// shares nothing with the CUDA path except the POD types of the C ABI header:
//   * cell of a narrow column: sign-extended (I32, I64) or zero-extended (U8),
//     i.e. the reference's u64 cell (src/datasource/table.rs:27-30);
//   * comparisons per ColType (src/engine/query_interpreter/expr.rs:1468-1530):
//     Int: EQ/NE bitwise on the cell, LT/LE/GT/GE signed i64
//     (src/exec/bitmap.rs:410-480); Date: unsigned u64 (bitmap.rs:350-409);
//     Float: ordered f64, EQ with tolerance 1e-6*max(|v|,1) (bitmap.rs:505-515),
//     NE = NOT EQ (bitmap.rs:498-500);
//   * BETWEEN = GE AND LE, NOT BETWEEN = LT OR GT (expr.rs:687-760);
//   * AND / OR / NOT over per-row booleans (expr.rs:633-679);
//   * per-row argument = wrapping i64 product of (mul * cell + add) factors,
//     the reference's Int x Int binop (expr.rs:2063-2076);
//   * SUM exact in int128 (the reference accumulates f64, aggregate.rs:1605-1622;
//     equal to it whenever every partial sum stays below 2^53);
//     COUNT(*) = rows; COUNT(col) counts cells != 0 (aggregate.rs:1364-1367);
//     AVG = f64(sum) / f64(count) (aggregate.rs:1416-1424); MIN/MAX signed
//     (aggregate.rs:1822-1836);
//   * GROUP BY on exact key tuples, groups ascending by signed key tuple;
//   * inner equi-join on exact key equality over the build rows passing the
//     build filter (join.rs:79-100, 544-794); pairs sorted (probe, build);
//   * kernel-table scalar kernels: ScanEqScalar (src/kernel/scan.rs:26-64),
//     ScanRangeScalar (scan.rs:67-101, unsigned), ScanMultiPredicateScalar
//     (scan.rs:103-160), SumF64Scalar (src/kernel/aggregate.rs:19-43, summed here
//     in binary128 as the FP64 reference value), CountDistinctScalar
//     (aggregate.rs:160-185), HashBuild/HashProbe match counts (src/kernel/hash.rs:84-200).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../include/turbogp_gpu.h"

namespace {

struct Cols {
    const tgp_column_desc* c;
    uint32_t n;
    uint64_t rows;
};

uint64_t cell(const tgp_column_desc& c, uint64_t r) {
    switch (c.dtype) {
        case TGP_DT_U8: return static_cast<const uint8_t*>(c.data)[r];
        case TGP_DT_I32: return static_cast<uint64_t>(static_cast<int64_t>(static_cast<const int32_t*>(c.data)[r]));
        default: return static_cast<const uint64_t*>(c.data)[r];
    }
}

bool leaf(const tgp_column_desc& c, const tgp_pred_node& n, uint64_t r) {
    const uint64_t x = cell(c, r);
    if (c.coltype == TGP_CT_FLOAT) {
        double v, a, b;
        std::memcpy(&v, &x, 8);
        std::memcpy(&a, &n.lit, 8);
        std::memcpy(&b, &n.lit2, 8);
        const double tol = 1e-6 * std::max(std::fabs(a), 1.0);
        switch (n.cmp) {
            case TGP_CMP_EQ: return std::fabs(v - a) <= tol;
            case TGP_CMP_NE: return !(std::fabs(v - a) <= tol);
            case TGP_CMP_LT: return v < a;
            case TGP_CMP_LE: return v <= a;
            case TGP_CMP_GT: return v > a;
            case TGP_CMP_GE: return v >= a;
            case TGP_CMP_BETWEEN: return v >= a && v <= b;
            default: return v < a || v > b;
        }
    }
    if (c.coltype == TGP_CT_INT) {
        const int64_t v = static_cast<int64_t>(x), a = static_cast<int64_t>(n.lit), b = static_cast<int64_t>(n.lit2);
        switch (n.cmp) {
            case TGP_CMP_EQ: return x == n.lit;
            case TGP_CMP_NE: return x != n.lit;
            case TGP_CMP_LT: return v < a;
            case TGP_CMP_LE: return v <= a;
            case TGP_CMP_GT: return v > a;
            case TGP_CMP_GE: return v >= a;
            case TGP_CMP_BETWEEN: return v >= a && v <= b;
            default: return v < a || v > b;
        }
    }
    const uint64_t a = n.lit, b = n.lit2;
    switch (n.cmp) {
        case TGP_CMP_EQ: return x == a;
        case TGP_CMP_NE: return x != a;
        case TGP_CMP_LT: return x < a;
        case TGP_CMP_LE: return x <= a;
        case TGP_CMP_GT: return x > a;
        case TGP_CMP_GE: return x >= a;
        case TGP_CMP_BETWEEN: return x >= a && x <= b;
        default: return x < a || x > b;
    }
}

// Returns -1 on a malformed program.
int eval_pred(const Cols& t, const tgp_pred_node* p, uint32_t np, uint64_t r) {
    if (np == 0) return 1;
    bool st[64];
    int sp = 0;
    for (uint32_t i = 0; i < np; ++i) {
        const tgp_pred_node& n = p[i];
        if (n.kind == TGP_PN_LEAF) {
            if (n.column >= t.n || sp >= 64) return -1;
            st[sp++] = leaf(t.c[n.column], n, r);
        } else if (n.kind == TGP_PN_NOT) {
            if (sp < 1) return -1;
            st[sp - 1] = !st[sp - 1];
        } else {
            if (sp < 2) return -1;
            const bool b = st[--sp];
            const bool a = st[sp - 1];
            st[sp - 1] = n.kind == TGP_PN_AND ? (a && b) : (a || b);
        }
    }
    return sp == 1 ? (st[0] ? 1 : 0) : -1;
}

struct Acc {
    uint64_t rows = 0;
    std::vector<__int128> sum;
    std::vector<int64_t> mn, mx;
    std::vector<uint64_t> nz;
};

int64_t row_arg(const tgp_agg& a, const Cols& probe, uint64_t pr, const Cols* build, uint64_t br, bool* ovf) {
    uint64_t acc = 1;
    __int128 exact = 1;
    for (uint32_t f = 0; f < a.nfactors; ++f) {
        const tgp_factor& F = a.f[f];
        uint64_t x = 0;
        if (F.column >= 0) x = F.side == TGP_SIDE_BUILD ? cell(build->c[F.column], br) : cell(probe.c[F.column], pr);
        const uint64_t t = static_cast<uint64_t>(F.mul) * x + static_cast<uint64_t>(F.add);
        const __int128 te = static_cast<__int128>(F.mul) * static_cast<int64_t>(x) + F.add;
        if (te != static_cast<__int128>(static_cast<int64_t>(t))) *ovf = true;
        if (f == 0) {
            acc = t;
            exact = static_cast<int64_t>(t);
        } else {
            const __int128 pe = static_cast<__int128>(static_cast<int64_t>(acc)) * static_cast<int64_t>(t);
            acc = acc * t;
            if (pe != static_cast<__int128>(static_cast<int64_t>(acc))) *ovf = true;
            exact = pe;
        }
    }
    (void)exact;
    return static_cast<int64_t>(acc);
}

void update(Acc& A, const tgp_query* q, const Cols& probe, uint64_t pr, const Cols* build, uint64_t br, bool* ovf) {
    A.rows += 1;
    for (uint32_t i = 0; i < q->nagg; ++i) {
        const tgp_agg& a = q->aggs[i];
        if (a.func == TGP_AGG_COUNT_STAR) continue;
        const int64_t v = row_arg(a, probe, pr, build, br, ovf);
        switch (a.func) {
            case TGP_AGG_COUNT_NONZERO: A.nz[i] += v != 0; break;
            case TGP_AGG_SUM:
            case TGP_AGG_AVG: A.sum[i] += v; break;
            case TGP_AGG_MIN: A.mn[i] = std::min(A.mn[i], v); break;
            case TGP_AGG_MAX: A.mx[i] = std::max(A.mx[i], v); break;
        }
    }
}

Acc new_acc(uint32_t nagg) {
    Acc a;
    a.sum.assign(nagg, 0);
    a.mn.assign(nagg, INT64_MAX);
    a.mx.assign(nagg, INT64_MIN);
    a.nz.assign(nagg, 0);
    return a;
}

void emit(const Acc& A, const tgp_query* q, tgp_agg_value* out) {
    for (uint32_t i = 0; i < q->nagg; ++i) {
        tgp_agg_value& v = out[i];
        v.count = A.rows;
        __int128 x = 0;
        double f = 0;
        switch (q->aggs[i].func) {
            case TGP_AGG_COUNT_STAR: x = A.rows; f = static_cast<double>(A.rows); break;
            case TGP_AGG_COUNT_NONZERO: x = A.nz[i]; f = static_cast<double>(A.nz[i]); break;
            case TGP_AGG_SUM: x = A.sum[i]; f = static_cast<double>(x); break;
            case TGP_AGG_AVG:
                x = A.sum[i];
                f = A.rows ? static_cast<double>(x) / static_cast<double>(A.rows) : 0.0;
                break;
            case TGP_AGG_MIN: x = A.mn[i]; f = static_cast<double>(A.mn[i]); break;
            case TGP_AGG_MAX: x = A.mx[i]; f = static_cast<double>(A.mx[i]); break;
        }
        v.lo = static_cast<uint64_t>(x);
        v.hi = static_cast<int64_t>(x >> 64);
        v.as_f64 = f;
    }
}

}  // namespace

extern "C" {

// Filter: LSB-first bitmap ((rows + 7) / 8 bytes, may be NULL), ascending row
// ids (may be NULL, capacity `rows`), count. Returns 0, or -1 on a bad program.
int orc_filter(const tgp_column_desc* cols, uint32_t ncols, uint64_t rows, const tgp_pred_node* pred, uint32_t npred,
               uint8_t* bitmap, uint32_t* rowids, uint64_t* count) {
    Cols t{cols, ncols, rows};
    if (bitmap) std::memset(bitmap, 0, (rows + 7) / 8);
    uint64_t c = 0;
    for (uint64_t r = 0; r < rows; ++r) {
        const int v = eval_pred(t, pred, npred, r);
        if (v < 0) return -1;
        if (v) {
            if (bitmap) bitmap[r >> 3] |= static_cast<uint8_t>(1u << (r & 7));
            if (rowids) rowids[c] = static_cast<uint32_t>(r);
            ++c;
        }
    }
    *count = c;
    return 0;
}

// Aggregation query over (probe) columns, optionally inner-joined with build
// columns on probe column q->probe_key_column = build column bkey, build rows
// filtered by bpred. Returns 0, 7 (capacity, res->ngroups set) or -1.
int orc_execute(const tgp_column_desc* cols, uint32_t ncols, uint64_t rows, const tgp_query* q,
                const tgp_column_desc* bcols, uint32_t nbcols, uint64_t brows, uint32_t bkey,
                const tgp_pred_node* bpred, uint32_t nbpred, uint64_t* keys_out, tgp_agg_value* vals_out, uint64_t cap,
                tgp_query_result* res) {
    Cols t{cols, ncols, rows};
    Cols b{bcols, nbcols, brows};
    const bool join = q->join != 0;
    std::unordered_multimap<uint64_t, uint64_t> ht;
    if (join) {
        for (uint64_t r = 0; r < brows; ++r) {
            const int v = eval_pred(b, bpred, nbpred, r);
            if (v < 0) return -1;
            if (v) ht.emplace(cell(bcols[bkey], r), r);
        }
    }
    std::map<std::vector<int64_t>, Acc> groups;
    bool ovf = false;
    uint64_t selected = 0;
    std::vector<int64_t> key(q->ngroup);
    auto key_of = [&](uint64_t pr, uint64_t br) {
        for (uint32_t k = 0; k < q->ngroup; ++k) {
            const tgp_group_key& g = q->group[k];
            key[k] = static_cast<int64_t>(g.side == TGP_SIDE_BUILD ? cell(bcols[g.column], br) : cell(cols[g.column], pr));
        }
    };
    if (q->ngroup == 0) groups.emplace(std::vector<int64_t>(), new_acc(q->nagg));
    for (uint64_t r = 0; r < rows; ++r) {
        const int v = eval_pred(t, q->pred, q->npred, r);
        if (v < 0) return -1;
        if (!v) continue;
        ++selected;
        if (!join) {
            key_of(r, 0);
            auto it = groups.find(key);
            if (it == groups.end()) it = groups.emplace(key, new_acc(q->nagg)).first;
            update(it->second, q, t, r, nullptr, 0, &ovf);
        } else {
            auto range = ht.equal_range(cell(cols[q->probe_key_column], r));
            for (auto e = range.first; e != range.second; ++e) {
                key_of(r, e->second);
                auto it = groups.find(key);
                if (it == groups.end()) it = groups.emplace(key, new_acc(q->nagg)).first;
                update(it->second, q, t, r, &b, e->second, &ovf);
            }
        }
    }
    res->rows_scanned = rows;
    res->rows_selected = selected;
    res->ngroups = groups.size();
    res->flags = ovf ? TGP_RESULT_ROW_OVERFLOW : 0;
    if (groups.size() > cap) return TGP_CAPACITY;
    uint64_t g = 0;
    for (auto& kv : groups) {
        for (uint32_t k = 0; k < q->ngroup; ++k) keys_out[g * q->ngroup + k] = static_cast<uint64_t>(kv.first[k]);
        emit(kv.second, q, vals_out + g * q->nagg);
        ++g;
    }
    return 0;
}

// Join pairs sorted by (probe_row, build_row). Returns 0, 7 (capacity) or -1.
int orc_join_pairs(const tgp_column_desc* pcols, uint32_t npcols, uint64_t prows, uint32_t pkey,
                   const tgp_pred_node* ppred, uint32_t nppred, const tgp_column_desc* bcols, uint32_t nbcols,
                   uint64_t brows, uint32_t bkey, const tgp_pred_node* bpred, uint32_t nbpred, uint32_t* probe_out,
                   uint32_t* build_out, uint64_t cap, uint64_t* npairs) {
    Cols t{pcols, npcols, prows};
    Cols b{bcols, nbcols, brows};
    std::unordered_map<uint64_t, std::vector<uint32_t>> ht;
    for (uint64_t r = 0; r < brows; ++r) {
        const int v = eval_pred(b, bpred, nbpred, r);
        if (v < 0) return -1;
        if (v) ht[cell(bcols[bkey], r)].push_back(static_cast<uint32_t>(r));
    }
    uint64_t n = 0;
    for (uint64_t r = 0; r < prows; ++r) {
        const int v = eval_pred(t, ppred, nppred, r);
        if (v < 0) return -1;
        if (!v) continue;
        auto it = ht.find(cell(pcols[pkey], r));
        if (it == ht.end()) continue;
        for (uint32_t br : it->second) {  // build rows ascending
            if (n < cap) {
                probe_out[n] = static_cast<uint32_t>(r);
                build_out[n] = br;
            }
            ++n;
        }
    }
    *npairs = n;
    return n > cap ? TGP_CAPACITY : 0;
}

// Scalar kernel-table semantics. HASH_BUILD/HASH_PROBE are folded into one
// call: `input` = build keys (cell_count), `input2` = probe keys (n2);
// result.count = matching pairs.
int orc_kernel_execute(uint32_t op, const uint64_t* input, const uint64_t* input2, uint64_t n2,
                       const tgp_kernel_params* p, tgp_kernel_result* r) {
    std::memset(r, 0, sizeof(*r));
    const uint64_t n = p->cell_count;
    switch (op) {
        case TGP_OP_SCAN_EQ_U64:
            for (uint64_t i = 0; i < n; ++i) {
                const uint64_t hit = input[i] == p->target_u64;
                r->count += hit;
                if (i < 64) r->mask |= hit << i;
            }
            return 0;
        case TGP_OP_SCAN_RANGE_U64:
            for (uint64_t i = 0; i < n; ++i) r->count += (input[i] >= p->low_u64) & (input[i] <= p->high_u64);
            return 0;
        case TGP_OP_SCAN_MULTI_PREDICATE: {
            const uint32_t k = std::min<uint32_t>(p->predicate_count, 3);
            const uint8_t ops[3] = {p->pred1_op, p->pred2_op, p->pred3_op};
            const uint64_t tg[3] = {p->target_u64, p->target2_u64, p->target3_u64};
            for (uint64_t i = 0; i < n; ++i) {
                bool all = true;
                for (uint32_t j = 0; j < k; ++j) {
                    const uint64_t c = input[i];
                    const bool h = ops[j] == TGP_PRED_EQ ? c == tg[j] : ops[j] == TGP_PRED_GT ? c > tg[j] : c < tg[j];
                    all = all && h;
                }
                r->count += all;
            }
            return 0;
        }
        case TGP_OP_AGGREGATE_SUM_F64: {
            __float128 s = 0;
            for (uint64_t i = 0; i < n; ++i) {
                double d;
                std::memcpy(&d, &input[i], 8);
                s += d;
            }
            r->sum = static_cast<double>(s);
            r->count = n;
            return 0;
        }
        case TGP_OP_AGGREGATE_COUNT_DISTINCT: {
            std::unordered_set<uint64_t> s(input, input + n);
            r->count = s.size();
            return 0;
        }
        case TGP_OP_HASH_PROBE: {
            std::unordered_map<uint64_t, uint64_t> mult;
            for (uint64_t i = 0; i < n; ++i) mult[input[i]]++;
            for (uint64_t i = 0; i < n2; ++i) {
                auto it = mult.find(input2[i]);
                if (it != mult.end()) r->count += it->second;
            }
            return 0;
        }
        default:
            return -1;
    }
}

// XXH3-64 (xxhash-rust 0.8, `xxh3_64`) of the 8 little-endian bytes of a
// cell, seed 0, default secret: the published algorithm's 4-to-8-byte case,
// restated from the xxHash specification. Only the secret's bytes 8..24 enter
// this case (as one xor constant).
static uint64_t xxh3_8bytes(uint64_t v) {
    const uint64_t lo = v & 0xffffffffull, hi = v >> 32;
    const uint64_t secret8 = 0x1cad21f72c81017cull, secret16 = 0xdb979083e96dd4deull;
    uint64_t x = (hi + (lo << 32)) ^ (secret8 ^ secret16);
    auto rotl = [](uint64_t a, int r) { return (a << r) | (a >> (64 - r)); };
    x ^= rotl(x, 49) ^ rotl(x, 24);
    x *= 0x9fb21c651e98df25ull;
    x ^= (x >> 35) + 8;
    x *= 0x9fb21c651e98df25ull;
    return x ^ (x >> 28);
}

uint64_t orc_xxh3_u64(uint64_t v) { return xxh3_8bytes(v); }

// The reference's HyperLogLog (exec/hll.rs): 2^14 u8 registers, register
// h >> 50 keeps the max of leading_zeros(h << 14) + 1, estimate with its
// small-range linear counting, truncated to u64.
uint64_t orc_hll_estimate(const uint64_t* cells, uint64_t n, const uint8_t* sel) {
    std::vector<uint8_t> reg(1u << 14, 0);
    for (uint64_t i = 0; i < n; ++i) {
        if (sel && !((sel[i >> 3] >> (i & 7)) & 1)) continue;
        const uint64_t h = xxh3_8bytes(cells[i]);
        const uint64_t w = h << 14;
        const uint8_t lz = static_cast<uint8_t>((w ? __builtin_clzll(w) : 64) + 1);
        uint8_t& r = reg[h >> 50];
        if (lz > r) r = lz;
    }
    const double m = 16384.0, alpha = 0.7213 / (1.0 + 1.079 / m);
    double sum = 0.0;
    uint64_t zeros = 0;
    for (uint8_t r : reg) {
        double p = 1.0;  // 2^-r by repeated halving (exact)
        for (int k = 0; k < r; ++k) p *= 0.5;
        sum += p;
        if (r == 0) ++zeros;
    }
    const double raw = alpha * m * m / sum;
    const double est = (raw <= 2.5 * m && zeros > 0) ? m * std::log(m / static_cast<double>(zeros)) : raw;
    return static_cast<uint64_t>(est);
}

// The estimate alone, from 2^14 registers (pins the library's host estimator).
uint64_t orc_hll_estimate_regs(const uint32_t* regs) {
    const double m = 16384.0, alpha = 0.7213 / (1.0 + 1.079 / m);
    double sum = 0.0;
    uint64_t zeros = 0;
    for (int i = 0; i < 16384; ++i) {
        double p = 1.0;
        for (uint32_t k = 0; k < regs[i]; ++k) p *= 0.5;
        sum += p;
        if (regs[i] == 0) ++zeros;
    }
    const double raw = alpha * m * m / sum;
    const double est = (raw <= 2.5 * m && zeros > 0) ? m * std::log(m / static_cast<double>(zeros)) : raw;
    return static_cast<uint64_t>(est);
}

// COUNT(DISTINCT col) as the reference evaluates it (aggregate.rs:1301-1325):
// exact below 100,000 selected rows (method 0), else the HyperLogLog
// estimate (method 1). `sel` is an LSB-first bitmap or NULL (all rows).
void orc_count_distinct(const uint64_t* cells, uint64_t n, const uint8_t* sel, uint64_t* count, uint32_t* method) {
    uint64_t nsel = 0;
    for (uint64_t i = 0; i < n; ++i) nsel += !sel || ((sel[i >> 3] >> (i & 7)) & 1);
    if (nsel < 100000) {
        std::unordered_set<uint64_t> seen;
        for (uint64_t i = 0; i < n; ++i)
            if (!sel || ((sel[i >> 3] >> (i & 7)) & 1)) seen.insert(cells[i]);
        *count = seen.size();
        *method = 0;
        return;
    }
    *count = orc_hll_estimate(cells, n, sel);
    *method = 1;
}

// Sequential f64 accumulation in row order, one running sum per group:
// out[group[i]] += terms[i] for i = 0..n-1. This is the order of the
// reference's per-group sums: each group's row index list is ascending
// (chunks of 65,536 rows merged in chunk order, aggregate.rs:580-623) and
// sum_vec adds one term per index in list order (aggregate.rs:1485-1792).
void orc_seq_sum_f64(const double* terms, const uint32_t* group, uint64_t n, uint32_t ngroups, double* out) {
    for (uint32_t g = 0; g < ngroups; ++g) out[g] = 0.0;
    for (uint64_t i = 0; i < n; ++i) out[group[i]] += terms[i];
}

// LIKE: the reference's like() (src/engine/query_interpreter/expr.rs:
// 2144-2171), one string at a time — byte-wise; a pattern byte equal to the
// string byte or '_' consumes one byte (tested in that order), '%' any run,
// with the last '%' as the only backtracking point; then trailing '%'s.
static bool like_bytes(const uint8_t* s, uint64_t n, const uint8_t* p, uint64_t m) {
    uint64_t si = 0, pi = 0, star_p = UINT64_MAX, star_s = 0;
    while (si < n) {
        if (pi < m && (p[pi] == '_' || p[pi] == s[si])) {
            ++si;
            ++pi;
        } else if (pi < m && p[pi] == '%') {
            star_p = pi;
            star_s = si;
            ++pi;
        } else if (star_p != UINT64_MAX) {
            pi = star_p + 1;
            ++star_s;
            si = star_s;
        } else {
            return false;
        }
    }
    while (pi < m && p[pi] == '%') ++pi;
    return pi == m;
}

// `col [NOT] LIKE pattern` over a flat string column (bytes + n + 1
// offsets): LSB-first bitmap of (n + 7) / 8 bytes; returns the count.
uint64_t orc_like(const uint8_t* bytes, const uint64_t* offs, uint64_t n, const uint8_t* pattern, uint64_t m,
                  int negated, uint8_t* bitmap) {
    uint64_t cnt = 0;
    for (uint64_t i = 0; i < (n + 7) / 8; ++i) bitmap[i] = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const bool hit = like_bytes(bytes + offs[i], offs[i + 1] - offs[i], pattern, m) != (negated != 0);
        if (hit) {
            bitmap[i >> 3] |= static_cast<uint8_t>(1u << (i & 7));
            ++cnt;
        }
    }
    return cnt;
}

}  // extern "C"
