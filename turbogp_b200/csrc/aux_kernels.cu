// aux_kernels.cu — the smaller kernels around the scan engine:
//   * column statistics (signed min / max of cells) computed at registration,
//   * bitmap → ascending row-id compaction (Bitmap::iter_set_bits,
//     src/exec/bitmap.rs:224-316),
//   * the AggregateSumF64 kernel-table operator (src/kernel/aggregate.rs:19-148)
//     with double-double compensated summation,
//   * the AggregateCountDistinct operator (src/kernel/aggregate.rs:160-185),
//     an exact hash set instead of the reference's HashSet,
//   * sorting of packed join pairs and their split into two u32 arrays.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cub/cub.cuh>

#include "device_common.cuh"
#include "plan.hpp"
#include "turbogp_gpu.h"

namespace tgp {

constexpr int kAuxThreads = 256;

// ---------------------------------------------------------------------------
// Column statistics
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kAuxThreads) column_minmax_kernel(const uint8_t* col, uint32_t dtype,
                                                                   uint64_t n, long long* out /* [min, max] */) {
    long long lo = 0x7fffffffffffffffll, hi = static_cast<long long>(0x8000000000000000ull);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        long long v;
        if (dtype == DT_U8) v = col[i];
        else if (dtype == DT_I32) v = reinterpret_cast<const int32_t*>(col)[i];
        else v = reinterpret_cast<const long long*>(col)[i];
        lo = min(lo, v);
        hi = max(hi, v);
    }
    for (int d = 16; d > 0; d >>= 1) {
        lo = min(lo, __shfl_down_sync(0xffffffffu, lo, d));
        hi = max(hi, __shfl_down_sync(0xffffffffu, hi, d));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(out, lo);
        atomicMax(out + 1, hi);
    }
}

cudaError_t launch_column_minmax(const uint8_t* col, uint32_t dtype, uint64_t n, long long* out,
                                 int sms, cudaStream_t st) {
    uint64_t blocks = (n + kAuxThreads - 1) / kAuxThreads;
    const uint64_t cap = static_cast<uint64_t>(sms) * 8;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) return cudaSuccess;
    column_minmax_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(col, dtype, n, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Narrowing of u64 cells whose values the host proved to fit the target
// width: U8 (0..255) or I32 (the i32 range). Four values per thread.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kAuxThreads) narrow_cells_kernel(const long long* __restrict__ src, uint64_t n,
                                                                  uint8_t* __restrict__ dst, uint32_t dtype) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t q = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; 4 * q < n; q += stride) {
        const uint64_t i = 4 * q;
        if (i + 4 <= n) {
            const longlong2 a = reinterpret_cast<const longlong2*>(src)[2 * q];
            const longlong2 b = reinterpret_cast<const longlong2*>(src)[2 * q + 1];
            if (dtype == DT_U8) {
                const uint32_t w = (static_cast<uint32_t>(a.x) & 0xffu) | ((static_cast<uint32_t>(a.y) & 0xffu) << 8) |
                                   ((static_cast<uint32_t>(b.x) & 0xffu) << 16) |
                                   ((static_cast<uint32_t>(b.y) & 0xffu) << 24);
                reinterpret_cast<uint32_t*>(dst)[q] = w;
            } else {
                reinterpret_cast<int4*>(dst)[q] = make_int4(static_cast<int>(a.x), static_cast<int>(a.y),
                                                            static_cast<int>(b.x), static_cast<int>(b.y));
            }
        } else {
            for (uint64_t j = i; j < n; ++j) {
                if (dtype == DT_U8) dst[j] = static_cast<uint8_t>(src[j]);
                else reinterpret_cast<int32_t*>(dst)[j] = static_cast<int32_t>(src[j]);
            }
        }
    }
}

cudaError_t launch_narrow_cells(const long long* src, uint64_t n, uint8_t* dst, uint32_t dtype, int sms,
                                cudaStream_t st) {
    uint64_t blocks = (n + 4ull * kAuxThreads - 1) / (4ull * kAuxThreads);
    const uint64_t cap = static_cast<uint64_t>(sms) * 8;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) return cudaSuccess;
    narrow_cells_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(src, n, dst, dtype);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Bitmap compaction: one CTA per scan tile (kTileRows bits = 64 words).
// tile_base[t] = exclusive prefix of selected rows before tile t.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(64) compact_rowids_kernel(const uint32_t* bitmap, uint64_t nwords,
                                                           const unsigned long long* tile_base,
                                                           uint32_t* rowids, uint64_t cap) {
    constexpr int kWordsPerTile = kTileRows / 32;
    __shared__ uint32_t scan[kWordsPerTile];
    const uint64_t t = blockIdx.x;
    const uint64_t w = t * kWordsPerTile + threadIdx.x;
    const uint32_t word = w < nwords ? bitmap[w] : 0u;
    const uint32_t c = __popc(word);
    // Block exclusive scan of 64 counts (two warps).
    uint32_t incl = c;
    const uint32_t lane = threadIdx.x & 31;
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= static_cast<uint32_t>(d)) incl += y;
    }
    scan[threadIdx.x] = incl;
    __syncthreads();
    uint32_t excl = incl - c;
    if (threadIdx.x >= 32) excl += scan[31];
    unsigned long long o = tile_base[t] + excl;
    uint32_t bits = word;
    while (bits) {
        const int b = __ffs(bits) - 1;
        bits &= bits - 1;
        if (o < cap) rowids[o] = static_cast<uint32_t>(w * 32 + b);
        ++o;
    }
}

// Exclusive prefix sum of per-tile counts (u32 → u64) with CUB.
cudaError_t tile_prefix(const uint32_t* counts, unsigned long long* out, uint64_t n, void* tmp,
                        size_t* tmp_bytes, cudaStream_t st) {
    return cub::DeviceScan::ExclusiveSum(tmp, *tmp_bytes, counts, out, static_cast<int>(n), st);
}

cudaError_t launch_compact(const uint32_t* bitmap, uint64_t nwords, uint64_t ntiles,
                           const unsigned long long* tile_base, uint32_t* rowids, uint64_t cap,
                           cudaStream_t st) {
    if (ntiles == 0) return cudaSuccess;
    compact_rowids_kernel<<<static_cast<unsigned>(ntiles), kTileRows / 32, 0, st>>>(bitmap, nwords, tile_base,
                                                                                   rowids, cap);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// AggregateSumF64: Σ f64 cells with double-double (TwoSum) accumulation, so the
// result is within a few ulps of the exactly rounded sum for inputs without
// catastrophic cancellation. Each block writes one (hi, lo) pair; the host
// adds the pairs in double-double.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    const double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

__device__ __forceinline__ void dd_add(double& hi, double& lo, double bh, double bl) {
    double s, e;
    two_sum(hi, bh, s, e);
    e += lo + bl;
    hi = s + e;
    lo = e - (hi - s);
}

__global__ void __launch_bounds__(kAuxThreads) sum_f64_kernel(const double* x, uint64_t n, double* out) {
    double hi = 0.0, lo = 0.0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        dd_add(hi, lo, x[i], 0.0);
    }
    for (int d = 16; d > 0; d >>= 1) {
        const double oh = __shfl_down_sync(0xffffffffu, hi, d);
        const double ol = __shfl_down_sync(0xffffffffu, lo, d);
        dd_add(hi, lo, oh, ol);
    }
    __shared__ double sh[kAuxThreads / 32][2];
    if ((threadIdx.x & 31) == 0) {
        sh[threadIdx.x >> 5][0] = hi;
        sh[threadIdx.x >> 5][1] = lo;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double h = sh[0][0], l = sh[0][1];
        for (int w = 1; w < kAuxThreads / 32; ++w) dd_add(h, l, sh[w][0], sh[w][1]);
        out[2 * blockIdx.x] = h;
        out[2 * blockIdx.x + 1] = l;
    }
}

cudaError_t launch_sum_f64(const double* x, uint64_t n, double* out, int blocks, cudaStream_t st) {
    sum_f64_kernel<<<blocks, kAuxThreads, 0, st>>>(x, n, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// AggregateCountDistinct: exact distinct count of u64 cells through an
// open-addressing set (EMPTY = ~0; the value ~0 itself is tracked by a flag).
// counters[0] += newly inserted keys; counters[1] |= saw ~0.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kAuxThreads) count_distinct_kernel(const unsigned long long* x, uint64_t n,
                                                                    unsigned long long* set, uint64_t mask,
                                                                    uint32_t log2cap,
                                                                    unsigned long long* counters,
                                                                    uint32_t* err) {
    unsigned long long local = 0;
    bool saw_empty = false;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const unsigned long long k = x[i];
        if (k == ~0ull) {
            saw_empty = true;
            continue;
        }
        uint64_t h = hash_slot(k, log2cap);
        bool placed = false;
        for (uint64_t p = 0; p <= mask; ++p) {
            unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(set + h);
            if (cur == k) {
                placed = true;
                break;
            }
            if (cur == ~0ull) {
                cur = atomicCAS(set + h, ~0ull, k);
                if (cur == ~0ull) {
                    ++local;
                    placed = true;
                    break;
                }
                if (cur == k) {
                    placed = true;
                    break;
                }
            }
            h = (h + 1) & mask;
        }
        if (!placed) atomicOr(err, kErrHashFull);
    }
    for (int d = 16; d > 0; d >>= 1) local += __shfl_down_sync(0xffffffffu, local, d);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(counters, local);
    if (saw_empty) atomicOr(counters + 1, 1ull);
}

cudaError_t launch_count_distinct(const unsigned long long* x, uint64_t n, unsigned long long* set,
                                  uint64_t mask, uint32_t log2cap, unsigned long long* counters,
                                  uint32_t* err, int blocks, cudaStream_t st) {
    count_distinct_kernel<<<blocks, kAuxThreads, 0, st>>>(x, n, set, mask, log2cap, counters, err);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// COUNT(DISTINCT col): the u64 cell of row i of a resident column (narrow
// values widen as the reference's cells hold them), rows filtered by an
// optional selection bitmap (LSB-first u32 words).
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long cell_at(const uint8_t* col, uint32_t dtype, uint64_t i) {
    if (dtype == DT_U8) return col[i];
    if (dtype == DT_I32)
        return static_cast<unsigned long long>(static_cast<long long>(reinterpret_cast<const int32_t*>(col)[i]));
    return reinterpret_cast<const unsigned long long*>(col)[i];
}

__device__ __forceinline__ bool row_selected(const uint32_t* bitmap, uint64_t i) {
    return !bitmap || ((bitmap[i >> 5] >> (i & 31)) & 1u);
}

// XXH3-64 of the 8 little-endian bytes of v with seed 0 and the default
// secret: the specification's 4-to-8-byte path (input = low word << 32 | high
// word, xored with secret[8..16) ^ secret[16..24), then the rrmxmx finaliser
// with length 8). This is the hash the reference's HyperLogLog applies to
// each cell (xxh3_64 of value.to_le_bytes(), exec/hll.rs:34-37).
__device__ __forceinline__ unsigned long long xxh3_u64(unsigned long long v) {
    constexpr unsigned long long kBitflip = 0x1cad21f72c81017cull ^ 0xdb979083e96dd4deull;
    constexpr unsigned long long kMul = 0x9fb21c651e98df25ull;
    unsigned long long h = ((v << 32) | (v >> 32)) ^ kBitflip;
    h ^= ((h << 49) | (h >> 15)) ^ ((h << 24) | (h >> 40));
    h *= kMul;
    h ^= (h >> 35) + 8ull;
    h *= kMul;
    return h ^ (h >> 28);
}

// Exact distinct count of the selected cells (as count_distinct_kernel).
__global__ void __launch_bounds__(kAuxThreads) distinct_cells_kernel(const uint8_t* col, uint32_t dtype, uint64_t n,
                                                                    const uint32_t* bitmap, unsigned long long* set,
                                                                    uint64_t mask, uint32_t log2cap,
                                                                    unsigned long long* counters, uint32_t* err) {
    unsigned long long local = 0;
    bool saw_empty = false;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (!row_selected(bitmap, i)) continue;
        const unsigned long long k = cell_at(col, dtype, i);
        if (k == ~0ull) {
            saw_empty = true;
            continue;
        }
        uint64_t h = hash_slot(k, log2cap);
        bool placed = false;
        for (uint64_t p = 0; p <= mask; ++p) {
            unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(set + h);
            if (cur == k) {
                placed = true;
                break;
            }
            if (cur == ~0ull) {
                cur = atomicCAS(set + h, ~0ull, k);
                if (cur == ~0ull) {
                    ++local;
                    placed = true;
                    break;
                }
                if (cur == k) {
                    placed = true;
                    break;
                }
            }
            h = (h + 1) & mask;
        }
        if (!placed) atomicOr(err, kErrHashFull);
    }
    for (int d = 16; d > 0; d >>= 1) local += __shfl_down_sync(0xffffffffu, local, d);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(counters, local);
    if (saw_empty) atomicOr(counters + 1, 1ull);
}

cudaError_t launch_distinct_cells(const uint8_t* col, uint32_t dtype, uint64_t n, const uint32_t* bitmap,
                                  unsigned long long* set, uint64_t mask, uint32_t log2cap,
                                  unsigned long long* counters, uint32_t* err, int sms, cudaStream_t st) {
    uint64_t blocks = (n + kAuxThreads - 1) / kAuxThreads;
    if (blocks > static_cast<uint64_t>(sms) * 8) blocks = static_cast<uint64_t>(sms) * 8;
    if (blocks == 0) return cudaSuccess;
    distinct_cells_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(col, dtype, n, bitmap, set, mask,
                                                                                log2cap, counters, err);
    return cudaGetLastError();
}

// HyperLogLog registers (2^14, exec/hll.rs:11-51): for each selected cell,
// h = xxh3(cell), register h >> 50 takes the max of
// leading_zeros(h << 14) + 1. Each CTA keeps its registers in shared memory
// (a shared atomic max only when the value could raise the register) and
// writes them, one byte each, to its row of `partial`; a second kernel takes
// the max over the CTAs' rows (no global atomics on 16K hot addresses).
constexpr int kHllRegs = 1 << 14;
constexpr int kHllThreads = 512;

__global__ void __launch_bounds__(kHllThreads) hll_kernel(const uint8_t* col, uint32_t dtype, uint64_t n,
                                                         const uint32_t* bitmap, uint8_t* partial) {
    extern __shared__ uint32_t sreg[];
    for (int r = threadIdx.x; r < kHllRegs; r += blockDim.x) sreg[r] = 0;
    __syncthreads();
    // Four rows per thread and pass, their loads issued before any hashing
    // (rows i, i + T, i + 2T, i + 3T for T threads: coalesced per row).
    const uint64_t T = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n; i += 4 * T) {
        unsigned long long c[4];
        bool on[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint64_t j = i + u * T;
            on[u] = j < n && row_selected(bitmap, j);
            c[u] = on[u] ? cell_at(col, dtype, j) : 0ull;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (!on[u]) continue;
            const unsigned long long h = xxh3_u64(c[u]);
            const uint32_t idx = static_cast<uint32_t>(h >> 50);
            const unsigned long long w = h << 14;
            const uint32_t lz = (w ? static_cast<uint32_t>(__clzll(static_cast<long long>(w))) : 64u) + 1u;
            if (lz > *reinterpret_cast<volatile uint32_t*>(sreg + idx)) atomicMax(sreg + idx, lz);
        }
    }
    __syncthreads();
    uint8_t* row = partial + static_cast<uint64_t>(blockIdx.x) * kHllRegs;
    for (int r = 4 * threadIdx.x; r < kHllRegs; r += 4 * blockDim.x)
        reinterpret_cast<uint32_t*>(row)[r / 4] = sreg[r] | (sreg[r + 1] << 8) | (sreg[r + 2] << 16) | (sreg[r + 3] << 24);
}

// regs[r] = max over the CTAs' rows of partial[b][r] (four registers a thread).
__global__ void __launch_bounds__(256) hll_merge_kernel(const uint8_t* partial, uint32_t rows, uint32_t* regs) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kHllRegs / 4) return;
    uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
    for (uint32_t b = 0; b < rows; ++b) {
        const uint32_t w = reinterpret_cast<const uint32_t*>(partial + static_cast<uint64_t>(b) * kHllRegs)[q];
        m0 = max(m0, w & 0xffu);
        m1 = max(m1, (w >> 8) & 0xffu);
        m2 = max(m2, (w >> 16) & 0xffu);
        m3 = max(m3, w >> 24);
    }
    regs[4 * q] = m0;
    regs[4 * q + 1] = m1;
    regs[4 * q + 2] = m2;
    regs[4 * q + 3] = m3;
}

int hll_blocks(uint64_t n, int sms) {
    uint64_t blocks = (n + kHllThreads - 1) / kHllThreads;
    if (blocks > static_cast<uint64_t>(sms) * 2) blocks = static_cast<uint64_t>(sms) * 2;
    return static_cast<int>(blocks);
}

cudaError_t launch_hll(const uint8_t* col, uint32_t dtype, uint64_t n, const uint32_t* bitmap, uint8_t* partial,
                       uint32_t* regs, int sms, cudaStream_t st) {
    const size_t smem = kHllRegs * sizeof(uint32_t);
    const cudaError_t e = cudaFuncSetAttribute(hll_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const int blocks = hll_blocks(n, sms);
    if (blocks == 0) return cudaMemsetAsync(regs, 0, kHllRegs * sizeof(uint32_t), st);
    hll_kernel<<<static_cast<unsigned>(blocks), kHllThreads, smem, st>>>(col, dtype, n, bitmap, partial);
    hll_merge_kernel<<<(kHllRegs / 4 + 255) / 256, 256, 0, st>>>(partial, static_cast<uint32_t>(blocks), regs);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Join pairs: sort packed (probe << 32 | build) pairs, then split.
// ---------------------------------------------------------------------------
cudaError_t sort_pairs(const unsigned long long* in, unsigned long long* out, uint64_t n, void* tmp,
                       size_t* tmp_bytes, cudaStream_t st) {
    return cub::DeviceRadixSort::SortKeys(tmp, *tmp_bytes, in, out, static_cast<int>(n), 0, 64, st);
}

__global__ void split_pairs_kernel(const unsigned long long* pairs, uint64_t n, uint32_t* probe,
                                   uint32_t* build) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const unsigned long long p = pairs[i];
        probe[i] = static_cast<uint32_t>(p >> 32);
        build[i] = static_cast<uint32_t>(p & 0xffffffffull);
    }
}

cudaError_t launch_split_pairs(const unsigned long long* pairs, uint64_t n, uint32_t* probe,
                               uint32_t* build, int sms, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    uint64_t blocks = (n + kAuxThreads - 1) / kAuxThreads;
    if (blocks > static_cast<uint64_t>(sms) * 8) blocks = static_cast<uint64_t>(sms) * 8;
    split_pairs_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(pairs, n, probe, build);
    return cudaGetLastError();
}

// Fill a u64 buffer with a value (hash-table EMPTY markers).
__global__ void fill_u64_kernel(unsigned long long* p, uint64_t n, unsigned long long v) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        p[i] = v;
}

// Writes the slot image `init` (stride words) into every slot of a table: one
// pass, slot i's words w at p[i * stride + w] (adjacent threads, adjacent words).
// (Slots are an even number of words, 16-byte aligned: written as pairs.)
__global__ void fill_slots_kernel(unsigned long long* p, uint64_t nslots, const SlotImage img) {
    const uint32_t pairs = img.stride / 2;
    ulonglong2* q = reinterpret_cast<ulonglong2*>(p);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < nslots;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        for (uint32_t w = 0; w < pairs; ++w) q[i * pairs + w] = make_ulonglong2(img.w[2 * w], img.w[2 * w + 1]);
}

cudaError_t launch_fill_slots(unsigned long long* p, uint64_t nslots, const SlotImage& img, int sms, cudaStream_t st) {
    if (nslots == 0) return cudaSuccess;
    if ((img.stride & 1u) || (reinterpret_cast<uintptr_t>(p) & 15u)) return cudaErrorInvalidValue;
    const uint64_t n = nslots;
    uint64_t blocks = (n + kAuxThreads - 1) / kAuxThreads;
    if (blocks > static_cast<uint64_t>(sms) * 16) blocks = static_cast<uint64_t>(sms) * 16;
    fill_slots_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(p, nslots, img);
    return cudaGetLastError();
}

cudaError_t launch_fill_u64(unsigned long long* p, uint64_t n, unsigned long long v, int sms,
                            cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    uint64_t blocks = (n + kAuxThreads - 1) / kAuxThreads;
    if (blocks > static_cast<uint64_t>(sms) * 8) blocks = static_cast<uint64_t>(sms) * 8;
    fill_u64_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(p, n, v);
    return cudaGetLastError();
}

// Scatter the occupied slots of a group hash table into a compact array
// (keys + slot words) for the host to sort; counters[0] = occupied slots.
__global__ void gather_groups_kernel(const unsigned long long* htab, uint64_t nslots, uint32_t stride,
                                     unsigned long long* out, uint64_t cap,
                                     unsigned long long* counter, bool direct) {
    // Whole warps walk the table (the loop bound is rounded up to a warp) so
    // one atomic per warp reserves the output rows of its occupied slots.
    const uint64_t step = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t end = (nslots + 31) & ~31ull;
    const uint32_t lane = threadIdx.x & 31u;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < end; i += step) {
        const unsigned long long* s = htab + i * stride;
        // A directly indexed table (slot = key) marks a slot by its count.
        const bool occ = i < nslots && (direct ? s[1] != 0ull : s[0] != ~0ull);
        const unsigned mask = __ballot_sync(0xffffffffu, occ);
        if (mask == 0) continue;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(counter, static_cast<unsigned long long>(__popc(mask)));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (!occ) continue;
        const unsigned long long o = base + __popc(mask & ((1u << lane) - 1u));
        if (o < cap) {
            for (uint32_t w = 0; w < stride; ++w) out[o * stride + w] = s[w];
            if (direct) out[o * stride] = i;
        }
    }
}

cudaError_t launch_gather_groups(const unsigned long long* htab, uint64_t nslots, uint32_t stride,
                                 unsigned long long* out, uint64_t cap, unsigned long long* counter,
                                 int sms, cudaStream_t st, bool direct) {
    if (nslots == 0) return cudaSuccess;
    uint64_t blocks = (nslots + kAuxThreads - 1) / kAuxThreads;
    if (blocks > static_cast<uint64_t>(sms) * 8) blocks = static_cast<uint64_t>(sms) * 8;
    gather_groups_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(htab, nslots, stride, out,
                                                                               cap, counter, direct);
    return cudaGetLastError();
}

// Join payload: for every entry (key_rel, row) of a packed join table with
// unique keys, pay[key_rel] = sum over build-side group keys of
// (cell[row] - min) * stride. Unset entries keep 0xffffffff (no match).
__device__ __forceinline__ int64_t pay_cell(const uint8_t* base, uint32_t dtype, uint32_t row) {
    if (dtype == DT_U8) return static_cast<int64_t>(__ldg(base + row));
    if (dtype == DT_I32) return static_cast<int64_t>(__ldg(reinterpret_cast<const int32_t*>(base) + row));
    return static_cast<int64_t>(__ldg(reinterpret_cast<const long long*>(base) + row));
}

__global__ void join_pay_kernel(const unsigned long long* tab, uint64_t cap, const PayKeys K, uint32_t* pay,
                                uint32_t width) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < cap;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const unsigned long long e = tab[i];
        if (e == ~0ull) continue;
        const uint32_t row = static_cast<uint32_t>(e & 0xffffffffull);
        uint64_t g = 0;
        for (uint32_t k = 0; k < K.n; ++k)
            g += (static_cast<uint64_t>(pay_cell(K.ptr[k], K.dtype[k], row)) - static_cast<uint64_t>(K.min[k])) *
                 K.stride[k];
        const uint64_t at = e >> 32;
        if (width == 1) reinterpret_cast<uint8_t*>(pay)[at] = static_cast<uint8_t>(g);
        else if (width == 2) reinterpret_cast<uint16_t*>(pay)[at] = static_cast<uint16_t>(g);
        else pay[at] = static_cast<uint32_t>(g);
    }
}

cudaError_t launch_join_pay(const unsigned long long* tab, uint64_t cap, const PayKeys& K, uint32_t* pay,
                            uint32_t width, uint64_t pay_entries, int sms, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(pay, 0xff, pay_entries * width, st);
    if (e != cudaSuccess) return e;
    uint64_t blocks = (cap + kAuxThreads - 1) / kAuxThreads;
    if (blocks > static_cast<uint64_t>(sms) * 8) blocks = static_cast<uint64_t>(sms) * 8;
    join_pay_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(tab, cap, K, pay, width);
    return cudaGetLastError();
}

// Hash-grouped results on the device: sort the gathered slots by packed key
// and write the caller's layout (keys per group, tgp_agg_value per aggregate).
__global__ void extract_keys_kernel(const unsigned long long* packed, uint64_t n, uint32_t stride,
                                    unsigned long long* keys, uint32_t* idx) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        keys[i] = packed[i * stride];
        idx[i] = static_cast<uint32_t>(i);
    }
}

// Output group i from its slot s ([key][count][value limbs...]).
// (key: the slot's packed key word.)
__device__ __forceinline__ void write_group(const unsigned long long* s, unsigned long long key, uint64_t i,
                                            const HashFormat& F, uint64_t* keys_out, tgp_agg_value* vals_out) {
    if (keys_out)
        for (uint32_t k = 0; k < F.nkey; ++k)
            keys_out[i * F.nkey + k] = static_cast<uint64_t>(F.key_min[k]) + ((key >> F.key_shift[k]) & F.key_mask[k]);
    if (!vals_out) return;
    // One-word slots (F.hpack): the count above `hpack_shift`, below it the
    // sum of (value - bias) over the slot's rows.
    const uint64_t cnt = F.hpack ? (F.hpack_shift < 64 ? s[0] >> F.hpack_shift : 0ull) : s[1];
    for (uint32_t a = 0; a < F.nagg; ++a) {
        tgp_agg_value o;
        o.count = cnt;
        if (F.hpack && F.val[a] >= 0) {
            const uint64_t low = F.hpack_shift ? (s[0] & ((1ull << F.hpack_shift) - 1ull)) : 0ull;
            const __int128 sum = static_cast<__int128>(low) + static_cast<__int128>(cnt) * F.hpack_bias;
            o.lo = static_cast<uint64_t>(sum);
            o.hi = static_cast<int64_t>(sum >> 64);
            const double f = i128_to_f64_rn(o.lo, o.hi);
            o.as_f64 = F.func[a] == TGP_AGG_AVG ? (cnt ? f / static_cast<double>(cnt) : 0.0) : f;
        } else if (F.val[a] < 0) {
            o.lo = cnt;
            o.hi = 0;
            o.as_f64 = static_cast<double>(cnt);
        } else {
            const unsigned long long* v = s + 2 + 2 * F.val[a];
            if (F.kind[a] == VK_MIN || F.kind[a] == VK_MAX) {
                const int64_t x = static_cast<int64_t>(v[0]);
                o.lo = static_cast<uint64_t>(x);
                o.hi = x < 0 ? -1 : 0;
                o.as_f64 = static_cast<double>(x);
            } else {
                o.lo = v[0];
                o.hi = F.sum64 ? (static_cast<int64_t>(v[0]) >> 63) : static_cast<int64_t>(v[1]);
                const double f = i128_to_f64_rn(o.lo, o.hi);
                o.as_f64 = F.func[a] == TGP_AGG_AVG ? (cnt ? f / static_cast<double>(cnt) : 0.0) : f;
            }
        }
        vals_out[i * F.nagg + a] = o;
    }
}

__global__ void format_hash_groups_kernel(const unsigned long long* packed, const uint32_t* order, uint64_t n,
                                          const HashFormat F, uint64_t* keys_out, tgp_agg_value* vals_out) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const unsigned long long* g = packed + static_cast<uint64_t>(order[i]) * F.hstride;
        write_group(g, g[0], i, F, keys_out, vals_out);
    }
}

// Directly indexed group tables (slot = key; a slot is occupied when its
// count is not zero, its key word is never written): the occupied slots, in
// slot order, are the groups in ascending key order, so the result is written
// straight from the table at positions from a prefix count of occupied
// slots, with no gather and no sort. Block b covers slots
// [b * kDirChunk, (b + 1) * kDirChunk); pass 1 counts each block's occupied
// slots, a device scan makes them offsets, pass 2 writes each block's groups
// in order (slot base + j * kAuxThreads + thread, j ascending, so a warp's
// ballot and the block's warp totals give each slot's rank).
constexpr int kDirPerThread = 16;
constexpr uint64_t kDirChunk = static_cast<uint64_t>(kAuxThreads) * kDirPerThread;

__global__ void __launch_bounds__(kAuxThreads) count_direct_kernel(const unsigned long long* htab, uint64_t nslots,
                                                                   uint32_t stride, unsigned long long* counts) {
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kDirChunk;
    // The count word: [key][count][...] slots, or the whole one-word slot.
    const uint32_t occ = stride > 1 ? 1u : 0u;
    uint32_t c = 0;
#pragma unroll 4
    for (int j = 0; j < kDirPerThread; ++j) {
        const uint64_t i = base + static_cast<uint64_t>(j) * kAuxThreads + threadIdx.x;
        c += (i < nslots && htab[i * stride + occ] != 0ull) ? 1u : 0u;
    }
    for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
    __shared__ uint32_t wsum[kAuxThreads / 32];
    if ((threadIdx.x & 31u) == 0) wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kAuxThreads / 32; ++w) t += wsum[w];
        counts[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kAuxThreads) format_direct_kernel(const unsigned long long* htab, uint64_t nslots,
                                                                    const unsigned long long* offsets, uint64_t cap,
                                                                    const HashFormat F, uint64_t* keys_out,
                                                                    tgp_agg_value* vals_out) {
    __shared__ uint32_t wsum[kAuxThreads / 32];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kDirChunk;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    unsigned long long run = offsets[blockIdx.x];
    for (int j = 0; j < kDirPerThread; ++j) {
        const uint64_t i = base + static_cast<uint64_t>(j) * kAuxThreads + threadIdx.x;
        const unsigned long long* s = htab + i * F.hstride;
        const bool occ = i < nslots && s[F.hstride > 1 ? 1 : 0] != 0ull;
        const uint32_t mask = __ballot_sync(0xffffffffu, occ);
        if (lane == 0) wsum[warp] = __popc(mask);
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t w = 0; w < kAuxThreads / 32; ++w) {
            before += w < warp ? wsum[w] : 0u;
            total += wsum[w];
        }
        const unsigned long long pos = run + before + __popc(mask & ((1u << lane) - 1u));
        if (occ && pos < cap) write_group(s, i, pos, F, keys_out, vals_out);
        run += total;
        __syncthreads();
    }
}

cudaError_t format_hash_groups(const unsigned long long* packed, uint64_t n, const HashFormat& F, uint32_t key_bits,
                               void* scratch, size_t scratch_bytes, uint64_t* keys_out, tgp_agg_value* vals_out,
                               int sms, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    // scratch: keys[2n] u64, idx[2n] u32, then CUB temporary storage.
    unsigned long long* k0 = static_cast<unsigned long long*>(scratch);
    unsigned long long* k1 = k0 + n;
    uint32_t* i0 = reinterpret_cast<uint32_t*>(k1 + n);
    uint32_t* i1 = i0 + n;
    uint8_t* tmp = reinterpret_cast<uint8_t*>(i1 + n);
    const size_t head = n * 16 + n * 8;
    size_t tmp_bytes = scratch_bytes > head ? scratch_bytes - head : 0;
    uint64_t blocks = (n + kAuxThreads - 1) / kAuxThreads;
    if (blocks > static_cast<uint64_t>(sms) * 8) blocks = static_cast<uint64_t>(sms) * 8;
    extract_keys_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(packed, n, F.hstride, k0, i0);
    cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k0, k1, i0, i1, static_cast<int>(n), 0,
                                                    static_cast<int>(key_bits ? key_bits : 1), st);
    if (e != cudaSuccess) return e;
    format_hash_groups_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(packed, i1, n, F, keys_out,
                                                                                     vals_out);
    return cudaGetLastError();
}

uint64_t direct_groups_blocks(uint64_t nslots) { return (nslots + kDirChunk - 1) / kDirChunk; }

// Scratch: counts[nb + 1], offsets[nb + 1] (u64), then CUB's scan storage.
size_t direct_groups_scratch(uint64_t nslots) {
    const uint64_t nb = direct_groups_blocks(nslots);
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, static_cast<unsigned long long*>(nullptr),
                                  static_cast<unsigned long long*>(nullptr), static_cast<int>(nb + 1));
    return (nb + 1) * 16 + tmp + 256;
}

cudaError_t count_direct_groups(const unsigned long long* htab, uint64_t nslots, uint32_t stride, void* scratch,
                                size_t scratch_bytes, unsigned long long* total, cudaStream_t st) {
    const uint64_t nb = direct_groups_blocks(nslots);
    unsigned long long* counts = static_cast<unsigned long long*>(scratch);
    unsigned long long* offsets = counts + nb + 1;
    uint8_t* tmp = reinterpret_cast<uint8_t*>(offsets + nb + 1);
    size_t tmp_bytes = scratch_bytes - (nb + 1) * 16;
    // counts[nb] = 0, so offsets[nb] is the number of occupied slots.
    cudaError_t e = cudaMemsetAsync(counts + nb, 0, 8, st);
    if (e != cudaSuccess) return e;
    if (nb) count_direct_kernel<<<static_cast<unsigned>(nb), kAuxThreads, 0, st>>>(htab, nslots, stride, counts);
    e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, counts, offsets, static_cast<int>(nb + 1), st);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(total, offsets + nb, 8, cudaMemcpyDeviceToDevice, st);
}

cudaError_t format_direct_groups(const unsigned long long* htab, uint64_t nslots, const void* scratch, uint64_t cap,
                                 const HashFormat& F, uint64_t* keys_out, tgp_agg_value* vals_out, cudaStream_t st) {
    const uint64_t nb = direct_groups_blocks(nslots);
    if (nb == 0 || cap == 0) return cudaSuccess;
    const unsigned long long* offsets = static_cast<const unsigned long long*>(scratch) + nb + 1;
    format_direct_kernel<<<static_cast<unsigned>(nb), kAuxThreads, 0, st>>>(htab, nslots, offsets, cap, F, keys_out,
                                                                            vals_out);
    return cudaGetLastError();
}

size_t format_hash_groups_scratch(uint64_t n, uint32_t key_bits) {
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, static_cast<unsigned long long*>(nullptr),
                                    static_cast<unsigned long long*>(nullptr), static_cast<uint32_t*>(nullptr),
                                    static_cast<uint32_t*>(nullptr), static_cast<int>(n), 0,
                                    static_cast<int>(key_bits ? key_bits : 1));
    return n * 24 + tmp + 256;
}

// Radix keys of one LSD pass of the top-N order: an unsigned image of the
// ordering value whose ascending order is the wanted order (complemented for
// descending). int128 sums take two passes: low limb (pass 0), then the
// signed high limb (pass 1). idx[i] carries the slot index along.
__global__ void order_keys_kernel(const unsigned long long* packed, const uint32_t* perm, uint64_t n, uint32_t hstride,
                                  const TopNSpec S, int pass, unsigned long long* keys, uint32_t* idx) {
    constexpr unsigned long long kSign = 0x8000000000000000ull;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t p = perm[i];
        const unsigned long long* s = packed + static_cast<uint64_t>(p) * hstride;
        unsigned long long k;
        if (S.val < 0) {
            k = s[1];  // row count (unsigned)
        } else {
            const unsigned long long* v = s + 2 + 2 * S.val;
            if (S.kind == VK_MIN || S.kind == VK_MAX) {
                k = v[0] ^ kSign;
            } else if (S.func == TGP_AGG_AVG) {
                const unsigned long long cnt = s[1];
                const uint64_t lo = v[0];
                const int64_t hi = S.sum64 ? (static_cast<int64_t>(v[0]) >> 63) : static_cast<int64_t>(v[1]);
                const double f = cnt ? i128_to_f64_rn(lo, hi) / static_cast<double>(cnt) : 0.0;
                const unsigned long long u = static_cast<unsigned long long>(__double_as_longlong(f));
                k = (u & kSign) ? ~u : (u | kSign);
            } else if (S.sum64) {
                k = v[0] ^ kSign;
            } else {
                k = pass == 0 ? v[0] : (v[1] ^ kSign);
            }
        }
        keys[i] = S.desc ? ~k : k;
        idx[i] = p;
    }
}

cudaError_t topn_hash_groups(const unsigned long long* packed, uint64_t n, const HashFormat& F, uint32_t key_bits,
                             const TopNSpec& S, uint64_t limit, void* scratch, size_t scratch_bytes,
                             uint64_t* keys_out, tgp_agg_value* vals_out, int sms, cudaStream_t st) {
    if (n == 0 || limit == 0) return cudaSuccess;
    unsigned long long* k0 = static_cast<unsigned long long*>(scratch);
    unsigned long long* k1 = k0 + n;
    uint32_t* i0 = reinterpret_cast<uint32_t*>(k1 + n);
    uint32_t* i1 = i0 + n;
    uint8_t* tmp = reinterpret_cast<uint8_t*>(i1 + n);
    const size_t head = n * 16 + n * 8;
    size_t tmp_bytes = scratch_bytes > head ? scratch_bytes - head : 0;
    uint64_t blocks = (n + kAuxThreads - 1) / kAuxThreads;
    if (blocks > static_cast<uint64_t>(sms) * 8) blocks = static_cast<uint64_t>(sms) * 8;
    // Key order first, so the stable value passes leave ties in key order.
    extract_keys_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(packed, n, F.hstride, k0, i0);
    cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k0, k1, i0, i1, static_cast<int>(n), 0,
                                                    static_cast<int>(key_bits ? key_bits : 1), st);
    if (e != cudaSuccess) return e;
    const bool wide = S.val >= 0 && S.kind != VK_MIN && S.kind != VK_MAX && S.func != TGP_AGG_AVG && !S.sum64;
    for (int pass = 0; pass < (wide ? 2 : 1); ++pass) {
        order_keys_kernel<<<static_cast<unsigned>(blocks), kAuxThreads, 0, st>>>(packed, i1, n, F.hstride, S, pass,
                                                                                 k0, i0);
        e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k0, k1, i0, i1, static_cast<int>(n), 0, 64, st);
        if (e != cudaSuccess) return e;
    }
    const uint64_t m = limit < n ? limit : n;
    uint64_t fb = (m + kAuxThreads - 1) / kAuxThreads;
    if (fb > static_cast<uint64_t>(sms) * 8) fb = static_cast<uint64_t>(sms) * 8;
    format_hash_groups_kernel<<<static_cast<unsigned>(fb), kAuxThreads, 0, st>>>(packed, i1, m, F, keys_out, vals_out);
    return cudaGetLastError();
}

// A bounded busy wait of one thread (profiling: keeps the GPU busy while the
// host submits the launch that follows).
__global__ void delay_kernel(uint64_t ns) {
    const uint64_t t0 = global_ns();
    while (global_ns() - t0 < ns) {
    }
}

cudaError_t launch_delay(uint64_t ns, cudaStream_t st) {
    delay_kernel<<<1, 1, 0, st>>>(ns < 1000000ull ? ns : 1000000ull);
    return cudaGetLastError();
}

// Copies 16-byte words from device memory into page-locked host memory with
// the SMs' own stores over the link: a batch's result readback then takes no
// copy engine, so it does not queue behind another stream's large
// device-to-host copy (a high-cardinality result) on the same engine.
__global__ void __launch_bounds__(256) copy_to_host_kernel(uint4* __restrict__ dst, const uint4* __restrict__ src,
                                                           uint64_t nwords) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nwords;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        dst[i] = src[i];
}

cudaError_t launch_copy_to_host(void* host_dst, const void* dev_src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return cudaSuccess;
    if ((bytes & 15u) || (reinterpret_cast<uintptr_t>(host_dst) & 15u) || (reinterpret_cast<uintptr_t>(dev_src) & 15u))
        return cudaErrorInvalidValue;
    const uint64_t nwords = bytes / 16;
    // A grid-stride copy: a few hundred blocks cover any readback size.
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((nwords + 255) / 256, 256));
    copy_to_host_kernel<<<grid, 256, 0, st>>>(static_cast<uint4*>(host_dst), static_cast<const uint4*>(dev_src),
                                              nwords);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// LIKE over a string column (flat bytes + u64 offsets, the reference's
// StringSearchColumn flat buffer, src/exec/fm_index.rs:273-277, 388-440).
// Matching is the reference's like() (src/engine/query_interpreter/expr.rs:
// 2144-2171): byte-wise, a pattern byte equal to the string byte (tested
// first, so a '%' or '_' also matches itself) or '_' consumes one byte, '%'
// any run, with one backtracking point (the last '%').
// Each warp takes 32 consecutive strings; when their bytes fit its staging
// buffer they are copied into shared memory with coalesced loads first, and
// every lane matches its own string from there.
// ---------------------------------------------------------------------------
constexpr int kLikeWarps = 8;
constexpr int kLikeStageBytes = 4096;

// Steps of one match are bounded by (n + 1) * (m + 1) + n + m + 2; a match
// that would exceed that raises kErrOutputFull on `err` and reports no match
// (it cannot happen for the algorithm above; the bound keeps the loop finite
// by construction).
__device__ __forceinline__ bool like_match(const uint8_t* s, uint32_t n, const uint8_t* p, uint32_t m, uint32_t* err) {
    uint32_t si = 0, pi = 0, star_p = 0xffffffffu, star_s = 0;
    const uint64_t limit = static_cast<uint64_t>(n + 1) * (m + 1) + n + m + 2;
    uint64_t steps = 0;
    while (si < n) {
        if (++steps > limit) {
            atomicOr(err, kErrOutputFull);
            return false;
        }
        const uint8_t c = s[si];
        if (pi < m && (p[pi] == '_' || p[pi] == c)) {
            ++si;
            ++pi;
        } else if (pi < m && p[pi] == '%') {
            star_p = pi;
            star_s = si;
            ++pi;
        } else if (star_p != 0xffffffffu) {
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

__global__ void __launch_bounds__(kLikeWarps * 32) like_kernel(const uint8_t* bytes, const unsigned long long* offs,
                                                                uint64_t n, const __grid_constant__ LikePattern P,
                                                                uint32_t negated, uint32_t* bitmap,
                                                                unsigned long long* count, uint32_t* err) {
    __shared__ uint8_t stage[kLikeWarps][kLikeStageBytes];
    __shared__ uint8_t pat[kLikeMaxPattern];
    for (uint32_t k = threadIdx.x; k < P.len; k += blockDim.x) pat[k] = P.b[k];
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint64_t nwords = (n + 31) / 32;
    unsigned long long cnt = 0;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * kLikeWarps + w; g < nwords;
         g += static_cast<uint64_t>(gridDim.x) * kLikeWarps) {
        const uint64_t row = g * 32 + lane;
        const bool valid = row < n;
        const uint64_t end_row = (g * 32 + 32 < n) ? g * 32 + 32 : n;
        const uint64_t first = offs[g * 32], last = offs[end_row];
        const uint64_t so = valid ? offs[row] : first;
        const uint32_t sl = valid ? static_cast<uint32_t>(offs[row + 1] - so) : 0u;
        bool m = false;
        if (last - first <= static_cast<uint64_t>(kLikeStageBytes)) {
            const uint32_t span = static_cast<uint32_t>(last - first);
            for (uint32_t k = lane; k < span; k += 32) stage[w][k] = bytes[first + k];
            __syncwarp();
            if (valid) m = like_match(&stage[w][so - first], sl, pat, P.len, err);
            __syncwarp();
        } else if (valid) {
            m = like_match(bytes + so, sl, pat, P.len, err);
        }
        const bool sel = valid && (m != (negated != 0));
        const uint32_t bits = __ballot_sync(0xffffffffu, sel);
        if (lane == 0) {
            bitmap[g] = bits;
            cnt += __popc(bits);
        }
    }
    if (lane == 0 && cnt) atomicAdd(count, cnt);
}

cudaError_t launch_like(const uint8_t* bytes, const unsigned long long* offs, uint64_t n, const LikePattern& P,
                        bool negated, uint32_t* bitmap, unsigned long long* count, uint32_t* err, int sms,
                        cudaStream_t st) {
    const uint64_t nwords = (n + 31) / 32;
    if (nwords == 0) return cudaSuccess;
    uint64_t blocks = (nwords + kLikeWarps - 1) / kLikeWarps;
    if (blocks > static_cast<uint64_t>(sms) * 8) blocks = static_cast<uint64_t>(sms) * 8;
    like_kernel<<<static_cast<unsigned>(blocks), kLikeWarps * 32, 0, st>>>(bytes, offs, n, P, negated ? 1u : 0u,
                                                                          bitmap, count, err);
    return cudaGetLastError();
}

}  // namespace tgp
