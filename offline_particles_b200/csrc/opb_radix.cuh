// Stable LSD radix sort of (key, index) pairs with 8-bit digits: the sort
// behind the spatial orders of opb_sort.cu.
//
// A pass over one digit runs three kernels in stream order (no CTA waits on
// another CTA):
//   k_radix_counts   per tile of keys, how many keys hold each digit value;
//   k_radix_scan     per digit value, the exclusive scan of its tile counts and
//                    the digit's total;
//   k_radix_scatter  per tile, every key's rank among the tile's keys of its
//                    digit, in index order (a warp match over the digit and
//                    per-warp counters); the tile is staged in shared memory
//                    in digit order and written out one digit run at a time,
//                    so consecutive threads store to consecutive addresses.
// The first pass makes the values itself (key i carries i), so no index array
// is read.  Every pass is stable, hence the whole sort is: its permutation is
// the one that orders the keys and keeps equal keys in index order, the same
// as that of any other stable sort of the same keys.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace opb_radix {

constexpr int kThreads = 256;  // one thread per digit value in the per-digit steps
constexpr int kWarps = kThreads / 32;
constexpr int kDigits = 256;
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;

// keys per thread of a tile (build knobs): by default 8 for 32-bit and 64-bit keys (tiles of 2048); the staged
// tile (keys and values) then takes 16 or 24 KB of shared memory.  Measured on 4,194,304 32-bit keys: 8 keys
// per thread 0.294 ms per sort with the keys, 12 keys 0.295 ms, 16 keys 0.310 ms.
#ifndef OPB_RADIX_ITEMS32
#define OPB_RADIX_ITEMS32 8
#endif
#ifndef OPB_RADIX_ITEMS64
#define OPB_RADIX_ITEMS64 8
#endif
template <class K>
__host__ __device__ constexpr int items_per_thread() {
    return sizeof(K) == 4 ? OPB_RADIX_ITEMS32 : OPB_RADIX_ITEMS64;
}

template <class K>
__host__ __device__ constexpr int tile_keys() {
    return kThreads * items_per_thread<K>();
}

template <class K>
__device__ __forceinline__ uint32_t digit_of(K key, int shift) {
    return (uint32_t)(key >> shift) & 0xFFu;
}

// exclusive prefix sum of v over the CTA's kThreads threads (thread order); ws: kWarps words of shared memory
__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t v, uint32_t *ws) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    uint32_t before = 0;
    for (int j = 0; j < w; ++j) before += ws[j];
    __syncthreads();  // ws may be written again by the next call
    return before + x - v;
}

// counts[d * ntiles + t] = number of keys of tile t whose digit at `shift` is d
template <class K>
__global__ void __launch_bounds__(kThreads) k_radix_counts(const K *__restrict__ keys, long long n, int shift,
                                                           uint32_t *__restrict__ counts, int ntiles) {
    constexpr int kItems = items_per_thread<K>();
    constexpr int kTile = tile_keys<K>();
    __shared__ uint32_t h[kWarps][kDigits];
    for (int i = threadIdx.x; i < kWarps * kDigits; i += kThreads) (&h[0][0])[i] = 0;
    const long long base = (long long)blockIdx.x * kTile;
    const int m = (int)(n - base < kTile ? n - base : kTile);
    K k[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int i = j * kThreads + (int)threadIdx.x;
        if (i < m) k[j] = keys[base + i];
    }
    __syncthreads();
    uint32_t *hw = h[threadIdx.x >> 5];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int i = j * kThreads + (int)threadIdx.x;
        if (i < m) atomicAdd(&hw[digit_of(k[j], shift)], 1u);
    }
    __syncthreads();
    const int d = threadIdx.x;  // kThreads == kDigits
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s += h[w][d];
    counts[(size_t)d * ntiles + blockIdx.x] = s;
}

// per digit d (one CTA each): counts[d * ntiles + t] <- the sum over tiles t' < t; totals[d] <- the sum over
// all tiles
__global__ void __launch_bounds__(kScanThreads) k_radix_scan(uint32_t *__restrict__ counts, int ntiles,
                                                             uint32_t *__restrict__ totals) {
    constexpr int kChunk = kScanThreads * kScanItems;
    __shared__ uint32_t ws[kScanThreads / 32];
    uint32_t *row = counts + (size_t)blockIdx.x * ntiles;
    uint32_t carry = 0;  // the same value in every thread
    for (long long start = 0; start < ntiles; start += kChunk) {
        const long long i0 = start + (long long)threadIdx.x * kScanItems;
        uint32_t v[kScanItems], sum = 0;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            v[j] = i0 + j < ntiles ? row[i0 + j] : 0u;
            sum += v[j];
        }
        uint32_t run = carry + block_exclusive_sum(sum, ws);
        const uint32_t end = run + sum;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            if (i0 + j < ntiles) row[i0 + j] = run;
            run += v[j];
        }
        if (threadIdx.x == kScanThreads - 1) ws[0] = end;  // the last thread holds the running total
        __syncthreads();
        carry = ws[0];
        __syncthreads();
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// One pass: the keys of tile blockIdx.x (and their values; with FIRST the values are the key indices) go to
// their stable position by the digit at `shift`.  counts/totals: as k_radix_scan leaves them.
template <class K, bool FIRST>
__global__ void __launch_bounds__(kThreads) k_radix_scatter(const K *__restrict__ kin, const int32_t *__restrict__ vin,
                                                            K *__restrict__ kout, int32_t *__restrict__ vout,
                                                            long long n, int shift, const uint32_t *__restrict__ counts,
                                                            const uint32_t *__restrict__ totals, int ntiles) {
    constexpr int kItems = items_per_thread<K>();
    constexpr int kTile = tile_keys<K>();
    constexpr int kWarpSpan = 32 * kItems;  // warp w ranks tile entries [w * kWarpSpan, (w + 1) * kWarpSpan)
    __shared__ uint32_t hw[kWarps][kDigits];  // per-warp digit counters, then their exclusive scan over warps
    __shared__ uint32_t run_in_tile[kDigits];  // where digit d's run starts in the staged tile
    __shared__ long long run_out[kDigits];  // the run's start in the output, minus run_in_tile
    __shared__ uint32_t ws[2][kWarps];
    __shared__ K sk[kTile];
    __shared__ int32_t sv[kTile];

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int i = tid; i < kWarps * kDigits; i += kThreads) (&hw[0][0])[i] = 0;
    const long long base = (long long)blockIdx.x * kTile;
    const int m = (int)(n - base < kTile ? n - base : kTile);
    K key[kItems];
    int32_t val[kItems];
    uint32_t rank[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int li = w * kWarpSpan + j * 32 + lane;
        if (li < m) {
            key[j] = kin[base + li];
            val[j] = FIRST ? (int32_t)(base + li) : vin[base + li];
        }
    }
    __syncthreads();  // counters cleared
    const uint32_t lower = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const bool valid = w * kWarpSpan + j * 32 + lane < m;
        const uint32_t d = valid ? digit_of(key[j], shift) : (uint32_t)kDigits;  // kDigits: no key
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = valid ? hw[w][d] : 0u;
        __syncwarp();
        if (valid && (peers & lower) == 0) hw[w][d] = before + (uint32_t)__popc(peers);  // lowest lane of the group
        __syncwarp();
        rank[j] = before + (uint32_t)__popc(peers & lower);
    }
    __syncthreads();
    {
        const int d = tid;  // kThreads == kDigits
        uint32_t in_tile = 0;
#pragma unroll
        for (int v = 0; v < kWarps; ++v) {
            const uint32_t c = hw[v][d];
            hw[v][d] = in_tile;
            in_tile += c;
        }
        const uint32_t start = block_exclusive_sum(in_tile, ws[0]);
        const uint32_t below = block_exclusive_sum(totals[d], ws[1]);  // keys of every tile with a smaller digit
        run_in_tile[d] = start;
        run_out[d] = (long long)below + counts[(size_t)d * ntiles + blockIdx.x] - start;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        if (w * kWarpSpan + j * 32 + lane < m) {
            const uint32_t d = digit_of(key[j], shift);
            const uint32_t at = run_in_tile[d] + hw[w][d] + rank[j];
            if (at < (uint32_t)kTile) {
                sk[at] = key[j];
                sv[at] = val[j];
            }
        }
    }
    __syncthreads();
    for (int i = tid; i < m; i += kThreads) {
        const K k = sk[i];
        const long long pos = run_out[digit_of(k, shift)] + i;
        if (pos >= 0 && pos < n) {
            kout[pos] = k;
            vout[pos] = sv[i];
        }
    }
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

template <class K>
inline long long tiles_for(long long n) {
    return (n + tile_keys<K>() - 1) / tile_keys<K>();
}

// device scratch of radix_sort_index for n keys: the tile counts and the digit totals
template <class K>
inline size_t temp_bytes(long long n) {
    return align256((size_t)kDigits * (size_t)tiles_for<K>(n) * 4) + align256((size_t)kDigits * 4);
}

// Sorts the n keys in `keys` by their bits [0, end_bit) stably and writes to `perm` the permutation: perm[j]
// is the index of the key at sorted position j.  keys_alt and ids_alt (n entries each) and temp
// (temp_bytes<K>(n)) are scratch; `keys` is overwritten.  *sorted (if not NULL) receives the buffer that
// holds the sorted keys (`keys` or `keys_alt`).
template <class K>
cudaError_t radix_sort_index(K *keys, K *keys_alt, int32_t *perm, int32_t *ids_alt, long long n, int end_bit,
                             void *temp, cudaStream_t st, K **sorted) {
    if (sorted) *sorted = keys;
    if (n <= 0) return cudaSuccess;
    const int passes = end_bit <= 8 ? 1 : (end_bit + 7) / 8;
    const long long ntiles = tiles_for<K>(n);
    uint32_t *counts = (uint32_t *)temp;
    uint32_t *totals = (uint32_t *)((char *)temp + align256((size_t)kDigits * (size_t)ntiles * 4));
    const K *kin = keys;
    const int32_t *vin = nullptr;
    for (int p = 0; p < passes; ++p) {
        K *kout = (kin == keys) ? keys_alt : keys;
        // the last pass writes perm, the one before it ids_alt, and so on back to the first
        int32_t *vout = ((passes - 1 - p) & 1) == 0 ? perm : ids_alt;
        const int shift = 8 * p;
        k_radix_counts<K><<<(unsigned)ntiles, kThreads, 0, st>>>(kin, n, shift, counts, (int)ntiles);
        k_radix_scan<<<kDigits, kScanThreads, 0, st>>>(counts, (int)ntiles, totals);
        if (p == 0)
            k_radix_scatter<K, true><<<(unsigned)ntiles, kThreads, 0, st>>>(kin, nullptr, kout, vout, n, shift, counts,
                                                                             totals, (int)ntiles);
        else
            k_radix_scatter<K, false><<<(unsigned)ntiles, kThreads, 0, st>>>(kin, vin, kout, vout, n, shift, counts,
                                                                              totals, (int)ntiles);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        kin = kout;
        vin = vout;
    }
    if (sorted) *sorted = const_cast<K *>(kin);
    return cudaSuccess;
}

}  // namespace opb_radix
