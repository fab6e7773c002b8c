// noalloc.cu — tgp_aggregate_noalloc: the scalar / low-cardinality grouped
// aggregate of the scan kernel for callers that cannot allocate GPU memory.
//
// Who needs it: an embedding engine whose own allocator reserved the whole
// device at start-up (a cudaMalloc would fail or take memory that allocator
// promised elsewhere), a latency-bound serving thread that may not take the
// device-wide synchronisation cudaMalloc / cudaFree can cause, or a host whose
// policy forbids allocations after start-up. Such callers pass their own
// device columns and a host output buffer; this entry point allocates nothing.
//
// Its scratch (accumulators, row counters, error word, key min/max and the
// finished per-group values) lives in one file-scope `static __device__`
// array of TGP_NOALLOC_SCRATCH_BYTES (1 MiB). Every GPU that loads the library
// keeps that array until the process exits. All calls share it and it keeps
// the last call's contents, so each call re-initialises what it uses; calls
// whose work overlaps on the GPU (two streams, or two host threads) race on it
// and must be serialised by the caller.
//
// The host-side address of the array is only a stand-in; the device address is
// obtained once per device with cudaGetSymbolAddress while that device is
// current, and kept for the life of the process (a cudaDeviceReset of that
// device is not supported afterwards). The first call on a device performs
// that set-up, so it should be made before any stream capture begins.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "device_common.cuh"
#include "runtime.hpp"

namespace tgp {

static_assert(TGP_NOALLOC_SCRATCH_BYTES % 256 == 0, "scratch size is a multiple of 256");
static __device__ __align__(256) unsigned char g_noalloc_scratch[TGP_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
constexpr uint32_t kMaxNoAllocCols = 16;
std::mutex g_setup_mu;
void* g_scratch[kMaxDevices] = {};

int report(char* msg, size_t cap, int status, const char* text) {
    if (msg && cap) std::snprintf(msg, cap, "%s", text);
    return status;
}

#define NA_CUDA(call)                                                                                        \
    do {                                                                                                     \
        cudaError_t e_ = (call);                                                                             \
        if (e_ != cudaSuccess) {                                                                             \
            if (err_msg && err_cap) std::snprintf(err_msg, err_cap, "%s: %s", #call, cudaGetErrorString(e_)); \
            return TGP_DEVICE_ERROR;                                                                         \
        }                                                                                                    \
    } while (0)

// Device address of the scratch array on `device` (current), looked up once.
int scratch_on(int device, void** out, char* err_msg, size_t err_cap) {
    if (device < 0 || device >= kMaxDevices) return report(err_msg, err_cap, TGP_INVALID_ARG, "bad device index");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch[device]) {
        void* p = nullptr;
        NA_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch[device] = p;
    }
    *out = g_scratch[device];
    return TGP_OK;
}

struct SlotKinds {
    uint8_t kind[kMaxVals + 1];  // per value slot (slot 0 = row count)
};

__global__ void noalloc_init_kernel(unsigned long long* acc, uint64_t nslots, uint32_t nv1, SlotKinds k,
                                    long long* minmax, uint32_t nkeys, unsigned long long* counters) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i < nslots) {
        const uint8_t kind = k.kind[i % nv1];
        acc[2 * i] = kind == VK_MIN ? 0x7fffffffffffffffull : kind == VK_MAX ? 0x8000000000000000ull : 0ull;
        acc[2 * i + 1] = 0;
    }
    if (i < 2ull * nkeys) minmax[i] = (i & 1) ? static_cast<long long>(0x8000000000000000ull) : 0x7fffffffffffffffll;
    if (i < 6) counters[i] = 0;  // 4 counters + the 16-byte error word
}

struct OutMap {
    uint32_t nagg;
    int32_t val[kMaxVals];   // value index per aggregate, -1 = COUNT(*)
    uint8_t kind[kMaxVals];  // kind of that value
};

// Exact per-group results in tgp_agg_value layout (as_f64 is filled on the host).
__global__ void noalloc_finalize_kernel(const unsigned long long* acc, uint64_t ngroups, uint32_t nv1, OutMap m,
                                        tgp_agg_value* out) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= ngroups * m.nagg) return;
    const uint64_t g = i / m.nagg;
    const uint32_t a = static_cast<uint32_t>(i % m.nagg);
    const unsigned long long* slot = acc + g * nv1 * 2;
    tgp_agg_value v;
    v.count = slot[0];
    v.as_f64 = 0.0;
    if (m.val[a] < 0) {
        v.lo = slot[0];
        v.hi = 0;
    } else {
        const unsigned long long* s = slot + 2 * (m.val[a] + 1);
        if (m.kind[a] == VK_MIN || m.kind[a] == VK_MAX) {
            v.lo = s[0];
            v.hi = static_cast<long long>(s[0]) < 0 ? -1 : 0;
        } else {
            v.lo = s[0];
            v.hi = static_cast<int64_t>(s[1]);
        }
    }
    out[i] = v;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace tgp

using namespace tgp;

static int aggregate_noalloc_on(int device, void* stream, const tgp_column_desc* cols, uint32_t ncols,
                                uint64_t rows, const tgp_pred_node* pred, uint32_t npred,
                                const tgp_key_domain* keys, uint32_t nkeys, const tgp_agg* aggs, uint32_t nagg,
                                tgp_agg_value* vals_out, uint64_t vals_cap, tgp_query_result* result,
                                char* err_msg, size_t err_cap);

// Runs the aggregate with `device` current and gives the caller back the
// device that was current before the call, whatever the outcome.
extern "C" int tgp_aggregate_noalloc(int device, void* stream, const tgp_column_desc* cols, uint32_t ncols,
                                     uint64_t rows, const tgp_pred_node* pred, uint32_t npred,
                                     const tgp_key_domain* keys, uint32_t nkeys, const tgp_agg* aggs, uint32_t nagg,
                                     tgp_agg_value* vals_out, uint64_t vals_cap, tgp_query_result* result,
                                     char* err_msg, size_t err_cap) {
    if (err_msg && err_cap) err_msg[0] = '\0';
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) {
        cudaGetLastError();
        prev = -1;
    }
    const int st = aggregate_noalloc_on(device, stream, cols, ncols, rows, pred, npred, keys, nkeys, aggs, nagg,
                                        vals_out, vals_cap, result, err_msg, err_cap);
    if (prev >= 0 && prev != device && cudaSetDevice(prev) != cudaSuccess) {
        cudaGetLastError();
        if (st == TGP_OK) return report(err_msg, err_cap, TGP_DEVICE_ERROR, "could not restore the caller's device");
    }
    return st;
}

static int aggregate_noalloc_on(int device, void* stream, const tgp_column_desc* cols, uint32_t ncols,
                                uint64_t rows, const tgp_pred_node* pred, uint32_t npred,
                                const tgp_key_domain* keys, uint32_t nkeys, const tgp_agg* aggs, uint32_t nagg,
                                tgp_agg_value* vals_out, uint64_t vals_cap, tgp_query_result* result,
                                char* err_msg, size_t err_cap) {
    if (!cols || !result || !vals_out || (nagg && !aggs) || (nkeys && !keys) || (npred && !pred))
        return report(err_msg, err_cap, TGP_INVALID_ARG, "null argument");
    if (ncols == 0 || ncols > kMaxNoAllocCols) return report(err_msg, err_cap, TGP_INVALID_ARG, "1 to 16 columns");
    if (nagg == 0 || nagg > static_cast<uint32_t>(kMaxVals))
        return report(err_msg, err_cap, TGP_INVALID_ARG, "1 to 8 aggregates");
    if (nkeys > static_cast<uint32_t>(kMaxGroupKeys)) return report(err_msg, err_cap, TGP_UNSUPPORTED, "more than 4 group keys");
    if (npred > static_cast<uint32_t>(kMaxPredOps)) return report(err_msg, err_cap, TGP_UNSUPPORTED, "predicate program too long");
    if (rows >= (1ull << 32)) return report(err_msg, err_cap, TGP_UNSUPPORTED, "fewer than 2^32 rows");
    std::memset(result, 0, sizeof(*result));
    const cudaStream_t st = static_cast<cudaStream_t>(stream);

    NA_CUDA(cudaSetDevice(device));
    void* scratch = nullptr;
    if (int s = scratch_on(device, &scratch, err_msg, err_cap)) return s;
    int sms = 0, optin = 0;
    NA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    NA_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));

    // Columns: caller-owned device memory, 16-byte aligned (bulk copies).
    Column cc[kMaxNoAllocCols];
    for (uint32_t i = 0; i < ncols; ++i) {
        cc[i].dtype = cols[i].dtype;
        cc[i].coltype = cols[i].coltype;
        cc[i].width = cols[i].dtype == DT_U8 ? 1 : cols[i].dtype == DT_I32 ? 4
                      : (cols[i].dtype == DT_I64 || cols[i].dtype == DT_U64 || cols[i].dtype == DT_F64) ? 8 : 0;
        if (cc[i].width == 0 || cc[i].coltype > TGP_CT_FLOAT)
            return report(err_msg, err_cap, TGP_INVALID_ARG, "bad column dtype or coltype");
        cc[i].dptr = static_cast<uint8_t*>(const_cast<void*>(cols[i].data));
        if (rows) {
            cudaPointerAttributes pa;
            if (cudaPointerGetAttributes(&pa, cols[i].data) != cudaSuccess ||
                (pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged)) {
                cudaGetLastError();
                return report(err_msg, err_cap, TGP_INVALID_ARG, "columns must be device memory");
            }
            // Another GPU's column would be read through a peer mapping (or
            // fault without one): refuse it on the host, before any launch.
            if (pa.type == cudaMemoryTypeDevice && pa.device != device)
                return report(err_msg, err_cap, TGP_INVALID_ARG, "a column lives on another device");
            if (reinterpret_cast<uintptr_t>(cols[i].data) % 16 != 0)
                return report(err_msg, err_cap, TGP_INVALID_ARG, "device columns must be 16-byte aligned");
        }
    }

    Plan P;
    std::memset(&P, 0, sizeof(P));
    P.nrows = rows;
    P.jslot = -1;
    P.flush_limit = ~0ull;
    P.check_ovf = 1;  // no column statistics here: detect per-row wrapping instead of proving it away
    int col2slot[kMaxNoAllocCols];
    for (int& c : col2slot) c = -1;
    auto slot_of = [&](uint32_t col) -> int {
        if (col >= ncols) return -2;
        if (col2slot[col] < 0) {
            if (P.nslots >= static_cast<uint32_t>(kMaxSlots)) return -3;
            SlotDesc& s = P.slot[P.nslots];
            s.ptr = cc[col].dptr;
            s.width = cc[col].width;
            s.dtype = cc[col].dtype;
            s.smem_off = P.stage_bytes;
            P.stage_bytes += kTileRows * cc[col].width;
            col2slot[col] = static_cast<int>(P.nslots++);
        }
        return col2slot[col];
    };

    // WHERE program (postfix, as tgp_filter / tgp_execute take it).
    int depth = 0;
    uint32_t nand = 0;
    bool only_and = true;
    for (uint32_t i = 0; i < npred; ++i) {
        const tgp_pred_node& n = pred[i];
        if (n.kind == TGP_PN_LEAF) {
            if (P.nleaf >= static_cast<uint32_t>(kMaxLeaves))
                return report(err_msg, err_cap, TGP_UNSUPPORTED, "more than 16 predicate leaves");
            const int s = slot_of(n.column);
            if (s < 0) return report(err_msg, err_cap, s == -2 ? TGP_INVALID_ARG : TGP_UNSUPPORTED, "bad predicate column");
            if (lower_leaf(nullptr, cc[n.column], n, static_cast<uint8_t>(s), P.leaf[P.nleaf]) != TGP_OK)
                return report(err_msg, err_cap, TGP_INVALID_ARG, "bad predicate leaf");
            P.ops[i] = static_cast<uint8_t>(P.nleaf++);
            if (++depth > 8) return report(err_msg, err_cap, TGP_UNSUPPORTED, "predicate program deeper than 8");
        } else if (n.kind == TGP_PN_AND || n.kind == TGP_PN_OR) {
            if (depth < 2) return report(err_msg, err_cap, TGP_INVALID_ARG, "AND/OR needs two operands");
            --depth;
            P.ops[i] = n.kind == TGP_PN_AND ? OP_AND : OP_OR;
            if (n.kind == TGP_PN_AND) ++nand; else only_and = false;
        } else if (n.kind == TGP_PN_NOT) {
            if (depth < 1) return report(err_msg, err_cap, TGP_INVALID_ARG, "NOT needs one operand");
            P.ops[i] = OP_NOT;
            only_and = false;
        } else {
            return report(err_msg, err_cap, TGP_INVALID_ARG, "bad predicate node kind");
        }
    }
    if (npred && depth != 1) return report(err_msg, err_cap, TGP_INVALID_ARG, "predicate program must leave one value");
    P.nops = npred;
    P.all_and = (only_and && nand + 1 == P.nleaf) ? 1u : 0u;
    for (uint32_t i = 0; i < P.nleaf; ++i) {  // the kernel tests (x - lo) <= span on the stored word
        Leaf& L = P.leaf[i];
        if (L.kind == LK_64) L.lo64 -= L.xor64;
        else if (L.kind == LK_U8 || L.kind == LK_I32) L.lo32 -= L.xor32;
    }

    // Aggregates: one value slot per non-COUNT(*) aggregate.
    OutMap om;
    std::memset(&om, 0, sizeof(om));
    om.nagg = nagg;
    for (uint32_t a = 0; a < nagg; ++a) {
        const tgp_agg& g = aggs[a];
        om.val[a] = -1;
        if (g.func == TGP_AGG_COUNT_STAR) continue;
        if (g.func > TGP_AGG_MAX) return report(err_msg, err_cap, TGP_INVALID_ARG, "bad aggregate function");
        if (g.nfactors > static_cast<uint32_t>(kMaxFactors)) return report(err_msg, err_cap, TGP_UNSUPPORTED, "more than 4 factors");
        ValDesc& V = P.val[P.nval];
        V.kind = g.func == TGP_AGG_COUNT_NONZERO ? VK_COUNT_NZ : g.func == TGP_AGG_MIN ? VK_MIN
                 : g.func == TGP_AGG_MAX ? VK_MAX : VK_SUM;
        V.nf = static_cast<uint8_t>(g.nfactors);
        for (uint32_t f = 0; f < g.nfactors; ++f) {
            const tgp_factor& F = g.f[f];
            Factor& D = V.f[f];
            D.mul = F.mul;
            D.add = F.add;
            D.slot = -1;
            if (F.column < 0) continue;
            if (F.side != TGP_SIDE_PROBE) return report(err_msg, err_cap, TGP_UNSUPPORTED, "no join here");
            const int s = slot_of(static_cast<uint32_t>(F.column));
            if (s < 0) return report(err_msg, err_cap, s == -2 ? TGP_INVALID_ARG : TGP_UNSUPPORTED, "bad factor column");
            if (cc[F.column].coltype == TGP_CT_FLOAT)
                return report(err_msg, err_cap, TGP_UNSUPPORTED, "aggregate arguments over FLOAT columns");
            D.slot = static_cast<int8_t>(s);
            D.dtype = static_cast<uint8_t>(cc[F.column].dtype);
            D.soff = P.slot[s].smem_off;
        }
        om.val[a] = static_cast<int32_t>(P.nval);
        om.kind[a] = V.kind;
        ++P.nval;
    }
    const uint32_t nv1 = P.nval + 1;

    // Group keys over caller-declared domains [min, min + count).
    uint64_t ngroups = 1;
    for (uint32_t k = 0; k < nkeys; ++k) {
        if (keys[k].count == 0) return report(err_msg, err_cap, TGP_INVALID_ARG, "empty key domain");
        if (keys[k].column >= ncols || cc[keys[k].column].coltype == TGP_CT_FLOAT)
            return report(err_msg, err_cap, TGP_INVALID_ARG, "bad group key column");
        if (keys[k].count > (1ull << 32) || ngroups * keys[k].count > (1ull << 32))
            return report(err_msg, err_cap, TGP_CAPACITY, "too many groups for the fixed scratch");
        ngroups *= keys[k].count;
    }
    uint64_t stride = 1;
    for (int k = static_cast<int>(nkeys) - 1; k >= 0; --k) {
        const int s = slot_of(keys[k].column);
        if (s < 0) return report(err_msg, err_cap, TGP_UNSUPPORTED, "query references more than 8 columns");
        GKey& K = P.gkey[k];
        K.slot = static_cast<int8_t>(s);
        K.dtype = static_cast<uint8_t>(cc[keys[k].column].dtype);
        K.soff = P.slot[s].smem_off;
        K.min = keys[k].min;
        K.stride = stride;
        stride *= keys[k].count;
    }
    P.ngkey = nkeys;
    P.ngroups = static_cast<uint32_t>(ngroups);

    // Scratch layout inside the static array.
    const size_t off_minmax = 0;
    const size_t off_counters = align256(off_minmax + 16ull * nkeys);
    const size_t off_acc = align256(off_counters + 48);
    const size_t off_out = align256(off_acc + 16ull * ngroups * nv1);
    const size_t need = align256(off_out + sizeof(tgp_agg_value) * ngroups * nagg);
    if (need > TGP_NOALLOC_SCRATCH_BYTES) {
        if (err_msg && err_cap)
            std::snprintf(err_msg, err_cap, "query needs %zu bytes of scratch; the fixed maximum is %u bytes", need,
                          static_cast<unsigned>(TGP_NOALLOC_SCRATCH_BYTES));
        return TGP_CAPACITY;
    }
    if (vals_cap < ngroups * nagg) {
        result->ngroups = ngroups;
        return report(err_msg, err_cap, TGP_CAPACITY, "vals_out holds fewer than ngroups * nagg values");
    }
    unsigned char* base = static_cast<unsigned char*>(scratch);
    long long* minmax = reinterpret_cast<long long*>(base + off_minmax);
    unsigned long long* counters = reinterpret_cast<unsigned long long*>(base + off_counters);
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(base + off_acc);
    tgp_agg_value* outv = reinterpret_cast<tgp_agg_value*>(base + off_out);
    P.acc = acc;
    P.counters = counters;
    P.err = reinterpret_cast<uint32_t*>(counters + 4);

    SlotKinds sk;
    std::memset(&sk, 0, sizeof(sk));
    for (uint32_t v = 0; v < P.nval; ++v) sk.kind[v + 1] = P.val[v].kind;
    const uint64_t init_n = std::max<uint64_t>(ngroups * nv1, std::max<uint64_t>(2ull * nkeys, 6));
    noalloc_init_kernel<<<static_cast<unsigned>((init_n + 255) / 256), 256, 0, st>>>(acc, ngroups * nv1, nv1, sk, minmax,
                                                                                      nkeys, counters);
    NA_CUDA(cudaGetLastError());

    // Every key cell must lie in its declared domain (else the accumulator
    // index would leave the scratch): check with the column min/max kernel.
    if (nkeys && rows) {
        for (uint32_t k = 0; k < nkeys; ++k)
            NA_CUDA(launch_column_minmax(cc[keys[k].column].dptr, cc[keys[k].column].dtype, rows, minmax + 2 * k, sms, st));
        long long mm[2 * kMaxGroupKeys];
        NA_CUDA(cudaMemcpyAsync(mm, minmax, 16ull * nkeys, cudaMemcpyDeviceToHost, st));
        NA_CUDA(cudaStreamSynchronize(st));
        for (uint32_t k = 0; k < nkeys; ++k) {
            const uint64_t lo = static_cast<uint64_t>(mm[2 * k]) - static_cast<uint64_t>(keys[k].min);
            const uint64_t hi = static_cast<uint64_t>(mm[2 * k + 1]) - static_cast<uint64_t>(keys[k].min);
            if (mm[2 * k] < keys[k].min || lo >= keys[k].count || hi >= keys[k].count)
                return report(err_msg, err_cap, TGP_INVALID_ARG, "a group key column holds values outside its declared domain");
        }
    }

    // Accumulator placement and shared-memory stages, as tgp_execute chooses them.
    const size_t budget = static_cast<size_t>(optin) - scan_kernel_static_smem() - kBarrierBytes;
    const size_t per_thread = 16ull * ngroups * nv1;  // int128 partials
    uint32_t mode = MODE_GROUP_GLOBAL;
    bool acc128 = false;
    size_t extra = 0;
    P.nthreads = 512;
    for (uint32_t nt : {512u, 256u}) {
        if (per_thread * nt + 2ull * P.stage_bytes <= budget) {
            mode = MODE_GROUP_PRIVATE;
            acc128 = true;
            P.nthreads = nt;
            extra = per_thread * nt;
            break;
        }
    }
    if (mode != MODE_GROUP_PRIVATE && 16ull * ngroups * nv1 + 2ull * P.stage_bytes <= budget) {
        mode = MODE_GROUP_SHARED;
        extra = 16ull * ngroups * nv1;
    }
    P.count_by_tile = (mode == MODE_GROUP_PRIVATE && nkeys == 0) ? 1u : 0u;
    const size_t avail = budget > extra ? budget - extra : 0;
    uint32_t S = P.stage_bytes ? static_cast<uint32_t>(std::min<size_t>(avail / P.stage_bytes, kMaxStages)) : 1u;
    if (S == 0) return report(err_msg, err_cap, TGP_UNSUPPORTED, "query does not fit in shared memory");
    P.nstages = S;
    P.extra_off = (static_cast<uint32_t>(kBarrierBytes + static_cast<size_t>(S) * P.stage_bytes) + 127u) & ~127u;
    P.smem_bytes = static_cast<uint32_t>(P.extra_off + extra);

    const uint64_t ntiles = (rows + kTileRows - 1) / kTileRows;
    if (ntiles) {
        const int occ = scan_occupancy(mode, acc128, static_cast<int>(P.nthreads), P.smem_bytes, P.shape);
        if (occ <= 0) return report(err_msg, err_cap, TGP_DEVICE_ERROR, "scan kernel cannot be resident");
        const uint64_t grid = std::min<uint64_t>(ntiles, static_cast<uint64_t>(sms) * occ);
        NA_CUDA(launch_scan(P, mode, acc128, static_cast<int>(grid), st));
    }
    const uint64_t nout = ngroups * nagg;
    noalloc_finalize_kernel<<<static_cast<unsigned>((nout + 255) / 256), 256, 0, st>>>(acc, ngroups, nv1, om, outv);
    NA_CUDA(cudaGetLastError());
    unsigned long long cnt[6];
    NA_CUDA(cudaMemcpyAsync(vals_out, outv, sizeof(tgp_agg_value) * nout, cudaMemcpyDefault, st));
    NA_CUDA(cudaMemcpyAsync(cnt, counters, sizeof(cnt), cudaMemcpyDeviceToHost, st));
    NA_CUDA(cudaStreamSynchronize(st));
    const uint32_t err = static_cast<uint32_t>(cnt[4] & 0xffffffffull);
    if (err & kErrWaitTimeout) return report(err_msg, err_cap, TGP_TIMEOUT, "a bounded device wait gave up");

    // f64 views on the host, as tgp_execute computes them.
    for (uint64_t i = 0; i < nout; ++i) {
        tgp_agg_value& v = vals_out[i];
        const uint32_t a = static_cast<uint32_t>(i % nagg);
        const double f = static_cast<double>((static_cast<__int128>(v.hi) << 64) | static_cast<__int128>(v.lo));
        v.as_f64 = aggs[a].func == TGP_AGG_AVG ? (v.count ? f / static_cast<double>(v.count) : 0.0) : f;
    }
    result->rows_scanned = rows;
    result->rows_selected = cnt[0];
    result->ngroups = ngroups;
    result->flags = (err & kErrRowOverflow) ? TGP_RESULT_ROW_OVERFLOW : 0u;
    return TGP_OK;
}
