// groupby_direct.cu — streaming GROUP BY kernels, rows read straight from
// HBM without the scan engine's stage ring: (1) an unfiltered GROUP BY of one
// key over a moderate range (the reference's try_accumulator_grouped,
// aggregate.rs / accum_grouped.rs, on its high-cardinality inputs) into
// one-word direct slots; (2) the TPC-H Q1 shape (further below).
//
// A slot per key value (key - min < 2^27) holds (row count << shift) + the
// sum of (value - bias) over its rows; the host proved that neither field can
// reach the other. Rows stream straight from HBM with coalesced vector loads
// (evict-first, so the slot table stays in L2), hot keys add into a per-CTA
// shared table with native 32-bit atomics (two probes, claimed first come),
// and every other row is one non-returning 64-bit add to its key's slot.
// There is no stage ring: with no predicate and one key the rows need no
// staging, and the loads of a thread's next rows are in flight while it
// updates the current ones.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "device_common.cuh"
#include "plan.hpp"
#include "runtime.hpp"

namespace tgp {

namespace {

constexpr int kDgThreads = 512;
// Two CTAs per SM (64 registers, no spills) with two warp chunks' loads in
// flight measured faster on B200 (20M rows, 10M key range, Zipf(1.1)) than
// three CTAs with one or two chunks (40 registers) and two CTAs with three.
constexpr int kDgMinBlocks = 2;   // CTAs per SM the register budget is set for
constexpr int kDgUnroll = 2;      // warp chunks whose loads are in flight at once
constexpr uint32_t kDgEmpty = 0xffffffffu;
constexpr uint32_t kDgProbes = 2;
constexpr int kDgRows = 128;   // rows per warp chunk: lane l holds rows 2l, 2l + 1, 64 + 2l, 65 + 2l

// Two consecutive cells of a column at row `r` (even), sign- or zero-extended
// as the column type says (to T: a key's low word, or a value in its own
// width); streaming loads (evict first in L1 and L2).
template <uint32_t DT, typename T>
__device__ __forceinline__ void load_pair(const uint8_t* base, uint64_t r, T& a, T& b) {
    if constexpr (DT == DT_I64 || DT == DT_U64) {
        const longlong2 v = __ldcs(reinterpret_cast<const longlong2*>(base) + r / 2);
        a = static_cast<T>(v.x);
        b = static_cast<T>(v.y);
    } else if constexpr (DT == DT_I32) {
        const int2 v = __ldcs(reinterpret_cast<const int2*>(base) + r / 2);
        a = static_cast<T>(v.x);
        b = static_cast<T>(v.y);
    } else {  // DT_U8
        const uint16_t v = __ldcs(reinterpret_cast<const unsigned short*>(base) + r / 2);
        a = static_cast<T>(v & 0xffu);
        b = static_cast<T>(v >> 8);
    }
}

template <uint32_t DT>
__device__ __forceinline__ int64_t load_one(const uint8_t* base, uint64_t r) {
    if constexpr (DT == DT_I64 || DT == DT_U64) return reinterpret_cast<const long long*>(base)[r];
    else if constexpr (DT == DT_I32) return reinterpret_cast<const int32_t*>(base)[r];
    else return base[r];
}

struct DgTable {
    uint32_t* keys;
    uint32_t* cnt;
    int32_t* sums;
};

// Adds one row (slot `key`, value argument `x`) to its claimed shared slot
// `h` (shared-table hit).
template <bool HASV>
__device__ __forceinline__ void dg_hit(const DgTable& T, uint32_t h, int64_t x) {
    atomicAdd(&T.cnt[h], 1u);
    if constexpr (HASV) atomicAdd(&T.sums[h], static_cast<int32_t>(x));
}

// Adds one row to the key's global slot.
__device__ __forceinline__ void dg_global(const DirectGroupArgs& A, uint32_t key, int64_t x) {
    if (key > A.last) {
        atomicOr(A.err, kErrHashFull);
        return;
    }
    atomicAdd(A.slots + key, A.one + static_cast<unsigned long long>(x));
}

// Adds the N rows (keys, value arguments) of a thread. Shared table: the
// first-probe slot loads of all N rows are issued together, then each row
// adds to its slot (the common case once the hot keys hold slots) or claims
// an empty one; the rows left take their second probes the same way; the
// rest go to their global slots. A stale slot read is harmless: a claimed
// slot never changes key, and an empty one is claimed by compare-and-swap.
template <int N, bool HASV>
__device__ __forceinline__ void dg_rows(const DirectGroupArgs& A, const DgTable& T, const uint32_t (&key)[N],
                                        const int64_t (&x)[N]) {
    uint32_t glob = (1u << N) - 1u;
    if (A.hs) {
        uint32_t h[N], k[N];
#pragma unroll
        for (int r = 0; r < N; ++r) {
            h[r] = (key[r] * 0x9E3779B1u) >> A.hs_shift;
            k[r] = *reinterpret_cast<volatile uint32_t*>(&T.keys[h[r]]);
        }
#pragma unroll
        for (uint32_t n = 0; n < kDgProbes; ++n) {
            if (n) {
#pragma unroll
                for (int r = 0; r < N; ++r) {
                    if (!((glob >> r) & 1u)) continue;
                    h[r] = (h[r] + 1) & (A.hs - 1);
                    k[r] = *reinterpret_cast<volatile uint32_t*>(&T.keys[h[r]]);
                }
            }
#pragma unroll
            for (int r = 0; r < N; ++r) {
                if (!((glob >> r) & 1u)) continue;
                uint32_t kk = k[r];
                if (kk == kDgEmpty) kk = atomicCAS(&T.keys[h[r]], kDgEmpty, key[r]);
                if (kk == kDgEmpty || kk == key[r]) {
                    dg_hit<HASV>(T, h[r], x[r]);
                    glob &= ~(1u << r);
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < N; ++r)
        if ((glob >> r) & 1u) dg_global(A, key[r], x[r]);
}

template <uint32_t KDT, uint32_t VDT>
__global__ void __launch_bounds__(kDgThreads, kDgMinBlocks) direct_group_kernel(const DirectGroupArgs A) {
    constexpr bool HASV = VDT != 0;
    using VT = std::conditional_t<VDT == DT_I64 || VDT == DT_U64, int64_t, int32_t>;
    extern __shared__ __align__(16) uint8_t dg_smem[];
    DgTable T;
    T.keys = reinterpret_cast<uint32_t*>(dg_smem);
    T.cnt = T.keys + A.hs;
    T.sums = reinterpret_cast<int32_t*>(T.cnt + A.hs);
    for (uint32_t i = threadIdx.x; i < A.hs; i += kDgThreads) {
        T.keys[i] = kDgEmpty;
        T.cnt[i] = 0;
        if (HASV) T.sums[i] = 0;
    }
    __syncthreads();

    const uint32_t kmin = static_cast<uint32_t>(A.kmin);
    auto value_of = [&](int64_t v) -> int64_t {
        const int64_t a = A.ident ? v : static_cast<int64_t>(static_cast<uint64_t>(A.mul) * static_cast<uint64_t>(v) +
                                                              static_cast<uint64_t>(A.add));
        return A.nz ? (a != 0 ? 1 : 0) : a;
    };

    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * kDgThreads + threadIdx.x) >> 5;
    const uint64_t nwarps = static_cast<uint64_t>(gridDim.x) * (kDgThreads / 32);
    const uint64_t nfull = A.nrows / kDgRows;
    // Full chunks, kDgUnroll per step: the loads of all of them are issued
    // before the first chunk's rows are added.
    uint64_t c = warp;
    for (; c + (kDgUnroll - 1) * nwarps < nfull; c += kDgUnroll * nwarps) {
        uint32_t k[kDgUnroll][4];
        VT v[kDgUnroll][4];
#pragma unroll
        for (int u = 0; u < kDgUnroll; ++u) {
            const uint64_t b = (c + u * nwarps) * kDgRows + 2 * lane;
            load_pair<KDT>(A.key, b, k[u][0], k[u][1]);
            load_pair<KDT>(A.key, b + 64, k[u][2], k[u][3]);
            if constexpr (HASV) {
                load_pair<VDT>(A.val, b, v[u][0], v[u][1]);
                load_pair<VDT>(A.val, b + 64, v[u][2], v[u][3]);
            }
        }
#pragma unroll
        for (int u = 0; u < kDgUnroll; ++u) {
            uint32_t key[4];
            int64_t x[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                key[r] = k[u][r] - kmin;
                x[r] = HASV ? value_of(v[u][r]) : 0;
            }
            dg_rows<4, HASV>(A, T, key, x);
        }
    }
    for (; c < nfull; c += nwarps) {
        const uint64_t b = c * kDgRows + 2 * lane;
        uint32_t k[4];
        VT v[4];
        load_pair<KDT>(A.key, b, k[0], k[1]);
        load_pair<KDT>(A.key, b + 64, k[2], k[3]);
        if constexpr (HASV) {
            load_pair<VDT>(A.val, b, v[0], v[1]);
            load_pair<VDT>(A.val, b + 64, v[2], v[3]);
        }
        uint32_t key[4];
        int64_t x[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            key[r] = k[r] - kmin;
            x[r] = HASV ? value_of(v[r]) : 0;
        }
        dg_rows<4, HASV>(A, T, key, x);
    }
    // The partial last chunk: the warp next in turn takes it, one row per
    // lane (no warp-wide step inside, lanes may leave the loop early).
    if (warp == nfull % nwarps) {
        for (uint64_t r = nfull * kDgRows + lane; r < A.nrows; r += 32) {
            const int64_t x[1] = {HASV ? value_of(load_one<VDT>(A.val, r)) : 0};
            const uint32_t key[1] = {static_cast<uint32_t>(load_one<KDT>(A.key, r)) - kmin};
            dg_rows<1, HASV>(A, T, key, x);
        }
    }
    __syncthreads();
    // Merge the shared table: one add per occupied slot.
    for (uint32_t i = threadIdx.x; i < A.hs; i += kDgThreads) {
        const uint32_t key = T.keys[i];
        if (key == kDgEmpty) continue;
        if (key > A.last) {
            atomicOr(A.err, kErrHashFull);
            continue;
        }
        const uint64_t n = T.cnt[i];
        const int64_t s = HASV ? static_cast<int64_t>(T.sums[i]) : 0;
        atomicAdd(A.slots + key, (n << A.shift) + (static_cast<unsigned long long>(s) - n * static_cast<uint64_t>(A.bias)));
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(A.counters, static_cast<unsigned long long>(A.nrows));
}

template <uint32_t KDT, uint32_t VDT>
const void* dg_ptr() {
    return reinterpret_cast<const void*>(&direct_group_kernel<KDT, VDT>);
}

const void* dg_kernel(uint32_t kdt, uint32_t vdt) {
    const bool k64 = kdt == DT_I64 || kdt == DT_U64;
    if (!k64 && kdt != DT_I32) return nullptr;
    switch (vdt) {
        case 0: return k64 ? dg_ptr<DT_I64, 0>() : dg_ptr<DT_I32, 0>();
        case DT_U8: return k64 ? dg_ptr<DT_I64, DT_U8>() : dg_ptr<DT_I32, DT_U8>();
        case DT_I32: return k64 ? dg_ptr<DT_I64, DT_I32>() : dg_ptr<DT_I32, DT_I32>();
        case DT_I64:
        case DT_U64: return k64 ? dg_ptr<DT_I64, DT_I64>() : dg_ptr<DT_I32, DT_I64>();
        default: return nullptr;
    }
}

// ---------------------------------------------------------------------------
// The TPC-H Q1 shape (execute_grouped, aggregate.rs:45-505, on a predicate of
// at most four int32 leaves): GROUP BY two u8 keys, COUNT(*), sum(i32),
// sum(i64), sum(i64 * (k - i32)), sum(i64 * (k - i32) * (k + i32)), every
// sum proven to fit int64. Rows stream from HBM with coalesced loads (four
// consecutive rows per lane); each thread keeps private partials (u32 row
// counts, int64 sums) in shared memory, updated by plain read-modify-writes,
// with no stage ring, so two CTAs of 512 threads fit an SM; at the end each
// (group, value) is summed over the CTA's threads by one warp and added to
// the query's accumulator with one 64-bit atomic.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 ldcs4(const uint8_t* base, uint64_t byte_off) {
    return __ldcs(reinterpret_cast<const uint4*>(base + byte_off));
}

__global__ void __launch_bounds__(kDgThreads, 2) q1_group_kernel(const Q1Args A) {
    extern __shared__ __align__(16) uint8_t q1_smem[];
    constexpr uint32_t NT = kDgThreads;
    const uint32_t t = threadIdx.x, lane = t & 31u;
    uint32_t* cnt = reinterpret_cast<uint32_t*>(q1_smem);                         // [g][t]
    long long* val = reinterpret_cast<long long*>(q1_smem + A.ngroups * NT * 4);  // [g][v][t]
    for (uint32_t g = 0; g < A.ngroups; ++g) cnt[g * NT + t] = 0;
    for (uint32_t i = 0; i < A.ngroups * 4; ++i) val[i * NT + t] = 0;

    // One row: its selection mask (all ones or 0), group and column cells.
    auto add_row = [&](uint32_t sel, uint32_t g, uint32_t qty, int64_t price, uint32_t disc, uint32_t tax) {
        const uint64_t sm = static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(sel)));
        const uint64_t v1 = static_cast<uint64_t>(A.mul[0] * qty + A.add[0]) & sm;
        const uint64_t v2 = static_cast<uint64_t>(price) & sm;
        const uint64_t v3 = v2 * static_cast<uint64_t>(A.mul[1] * disc + A.add[1]);
        const uint64_t v4 = v3 * static_cast<uint64_t>(A.mul[2] * tax + A.add[2]);
        cnt[g * NT + t] += sel & 1u;
        long long* w = val + static_cast<size_t>(g) * 4 * NT + t;
        w[0] += static_cast<long long>(v1);
        w[NT] += static_cast<long long>(v2);
        w[2 * NT] += static_cast<long long>(v3);
        w[3 * NT] += static_cast<long long>(v4);
    };
    auto leaf = [&](uint32_t x, uint32_t i) { return ((x - A.leaf_lo[i]) <= A.leaf_sp[i] ? 1u : 0u) ^ ((A.leaf_neg >> i) & 1u); };

    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * NT + t) >> 5;
    const uint64_t nwarps = static_cast<uint64_t>(gridDim.x) * (NT / 32);
    const uint64_t nfull = A.nrows / kDgRows;
    for (uint64_t c = warp; c < nfull; c += nwarps) {
        const uint64_t r = c * kDgRows + 4 * lane;  // this lane's four rows
        const uint4 q = ldcs4(A.col[0], r * 4);
        const uint4 p0 = ldcs4(A.col[1], r * 8), p1 = ldcs4(A.col[1], r * 8 + 16);
        const uint4 d = ldcs4(A.col[2], r * 4);
        const uint4 x = ldcs4(A.col[3], r * 4);
        const uint32_t k0 = __ldcs(reinterpret_cast<const unsigned int*>(A.key0 + r));
        const uint32_t k1 = __ldcs(reinterpret_cast<const unsigned int*>(A.key1 + r));
        uint4 lv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (static_cast<uint32_t>(i) < A.nleaf) lv[i] = ldcs4(A.leaf_col[i], r * 4);
        const uint32_t qa[4] = {q.x, q.y, q.z, q.w}, da[4] = {d.x, d.y, d.z, d.w}, xa[4] = {x.x, x.y, x.z, x.w};
        const int64_t pa[4] = {static_cast<int64_t>((static_cast<uint64_t>(p0.y) << 32) | p0.x),
                               static_cast<int64_t>((static_cast<uint64_t>(p0.w) << 32) | p0.z),
                               static_cast<int64_t>((static_cast<uint64_t>(p1.y) << 32) | p1.x),
                               static_cast<int64_t>((static_cast<uint64_t>(p1.w) << 32) | p1.z)};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            uint32_t m = 1u;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (static_cast<uint32_t>(i) >= A.nleaf) break;
                const uint32_t cell = e == 0 ? lv[i].x : e == 1 ? lv[i].y : e == 2 ? lv[i].z : lv[i].w;
                m &= leaf(cell, static_cast<uint32_t>(i));
            }
            const uint32_t g = (((k0 >> (8 * e)) & 0xffu) - A.kmin0) * A.kstride0 +
                               (((k1 >> (8 * e)) & 0xffu) - A.kmin1) * A.kstride1;
            add_row(0u - m, g, qa[e], pa[e], da[e], xa[e]);
        }
    }
    // The partial last chunk, one row per lane of one warp.
    if (warp == nfull % nwarps) {
        for (uint64_t r = nfull * kDgRows + lane; r < A.nrows; r += 32) {
            uint32_t m = 1u;
            for (uint32_t i = 0; i < A.nleaf; ++i) m &= leaf(reinterpret_cast<const uint32_t*>(A.leaf_col[i])[r], i);
            const uint32_t g = (static_cast<uint32_t>(A.key0[r]) - A.kmin0) * A.kstride0 +
                               (static_cast<uint32_t>(A.key1[r]) - A.kmin1) * A.kstride1;
            add_row(0u - m, g, reinterpret_cast<const uint32_t*>(A.col[0])[r],
                    reinterpret_cast<const long long*>(A.col[1])[r], reinterpret_cast<const uint32_t*>(A.col[2])[r],
                    reinterpret_cast<const uint32_t*>(A.col[3])[r]);
        }
    }
    __syncthreads();
    // Merge: warp w sums (group, slot) pairs w, w + 16, ... over the CTA's
    // threads; slot 0 is the row count, slots 1-4 the sums.
    const uint32_t wib = t >> 5;
    for (uint32_t i = wib; i < A.ngroups * 5; i += NT / 32) {
        const uint32_t g = i / 5, v = i % 5;
        unsigned long long sum = 0;
        for (uint32_t k = lane; k < NT; k += 32)
            sum += v == 0 ? static_cast<unsigned long long>(cnt[g * NT + k])
                          : static_cast<unsigned long long>(val[(static_cast<size_t>(g) * 4 + v - 1) * NT + k]);
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, d);
        if (lane == 0 && sum) {
            atomicAdd(A.acc + 2ull * (g * 5 + v), sum);
            if (v == 0) atomicAdd(A.counters, sum);  // selected rows
        }
    }
}

}  // namespace

bool direct_group_supported(uint32_t kdt, uint32_t vdt) { return dg_kernel(kdt, vdt) != nullptr; }

int direct_group_ctas_per_sm(uint32_t hs, bool hasv) {
    const void* f = dg_kernel(DT_I64, hasv ? DT_I32 : 0);
    int occ = 0;
    const size_t smem = static_cast<size_t>(hs) * (hasv ? 12 : 8);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, kDgThreads, smem) != cudaSuccess) return 0;
    return occ;
}

size_t q1_group_smem(uint32_t ngroups) { return static_cast<size_t>(ngroups) * kDgThreads * (4 + 4 * 8); }

int q1_group_ctas_per_sm(uint32_t ngroups) {
    const void* f = reinterpret_cast<const void*>(&q1_group_kernel);
    const size_t smem = q1_group_smem(ngroups);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess)
        return 0;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, kDgThreads, smem) != cudaSuccess) return 0;
    return occ;
}

cudaError_t launch_q1_group(const Q1Args& A, int grid, cudaStream_t st) {
    const void* f = reinterpret_cast<const void*>(&q1_group_kernel);
    const size_t smem = q1_group_smem(A.ngroups);
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    Q1Args a = A;
    void* args[] = {&a};
    return cudaLaunchKernel(f, dim3(static_cast<unsigned>(grid)), dim3(kDgThreads), args, smem, st);
}

cudaError_t launch_direct_group(const DirectGroupArgs& A, uint32_t kdt, uint32_t vdt, int grid, cudaStream_t st) {
    const void* f = dg_kernel(kdt, vdt);
    if (!f) return cudaErrorInvalidValue;
    const size_t smem = static_cast<size_t>(A.hs) * (vdt ? 12 : 8);
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    DirectGroupArgs a = A;
    void* args[] = {&a};
    return cudaLaunchKernel(f, dim3(static_cast<unsigned>(grid)), dim3(kDgThreads), args, smem, st);
}

}  // namespace tgp
