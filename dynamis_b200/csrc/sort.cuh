// sort.cuh - onesweep LSD radix sort and single-pass exclusive scan for sm_100a.
//
// Replaces the dynamis-sort operator (crates/dynamis-sort/src/radix.rs:321-476 with
// sort_histogram/prefix/scatter/copy.wgsl). Semantics kept: a stable LSD sort with 8-bit digits,
// the minor word's digits first and then the major word's (radix.rs:312-317), a u32 payload
// carried along. Design is new:
//   * one up-front histogram kernel counts every digit pass in a single read of the keys;
//   * each digit pass is ONE kernel: a tile of 256 threads x 8 keys ranks its keys with
//     warp __match_any_sync (stable: rounds in index order, lanes in order), publishes its digit
//     counts, and resolves its global digit prefix by decoupled look-back over earlier tiles;
//   * keys are staged in shared memory in digit order so the global scatter is coalesced runs.
// Tiles are claimed from an atomic counter, so a tile only waits on tiles already running.
// Every look-back wait is bounded (spin_limit polls per thread, kLookbackSpinLimit unless a caller
// lowers it); a wait that runs out sets DYN_STATUS_LOOKBACK_TIMEOUT in the status word it is given
// and the pass finishes without trapping.
#pragma once

#include <cstdint>

#include "dynamis_cuda.h"

namespace dyn {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys
constexpr uint32_t kLookbackSpinLimit = 1u << 22;
constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1u;

// DYN_STATUS_* bits: dynamis_cuda.h

__device__ __forceinline__ uint32_t load_relaxed(const uint32_t* p) {
    return *reinterpret_cast<const volatile uint32_t*>(p);
}
__device__ __forceinline__ void store_relaxed(uint32_t* p, uint32_t v) {
    *reinterpret_cast<volatile uint32_t*>(p) = v;
}

// Counts digit occurrences for every pass of the sort in one read. hist: passes x 256 words.
// Digit pass p reads word (p < minor_digits ? minor : major), byte (p or p - minor_digits).
static __global__ void k_sort_histogram(const uint32_t* __restrict__ major, const uint32_t* __restrict__ minor,
                                 const uint32_t* __restrict__ count_ptr, uint32_t n_fixed, uint32_t cap,
                                 int major_digits, int minor_digits, uint32_t* __restrict__ hist) {
    __shared__ uint32_t local[8][256];
    int passes = major_digits + minor_digits;
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&local[0][0])[i] = 0;
    __syncthreads();
    uint32_t n = count_ptr ? min(*count_ptr, cap) : n_fixed;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t mn = minor ? minor[i] : 0u;
        uint32_t mj = major[i];
        for (int p = 0; p < passes; ++p) {
            uint32_t word = p < minor_digits ? mn : mj;
            int byte = p < minor_digits ? p : p - minor_digits;
            atomicAdd(&local[p][(word >> (8 * byte)) & 255u], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
        uint32_t v = (&local[0][0])[i];
        if (v) atomicAdd(&hist[i], v);
    }
}

// Exclusive scan of each pass's 256 digit counts, in place (one block of 256 threads).
static __global__ void k_sort_offsets(uint32_t* hist, int passes) {
    __shared__ uint32_t buf[256];
    for (int p = 0; p < passes; ++p) {
        uint32_t v = hist[p * 256 + threadIdx.x];
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < 256; off <<= 1) {
            uint32_t t = threadIdx.x >= off ? buf[threadIdx.x - off] : 0u;
            __syncthreads();
            buf[threadIdx.x] += t;
            __syncthreads();
        }
        hist[p * 256 + threadIdx.x] = buf[threadIdx.x] - v;
        __syncthreads();
    }
}

// One digit pass. The sorted word is `key` (major or minor per pass); `other` rides along.
template <bool kTwoWords, bool kPayload>
static __global__ void __launch_bounds__(kSortThreads)
    k_onesweep(const uint32_t* __restrict__ key_in, const uint32_t* __restrict__ other_in,
               const uint32_t* __restrict__ val_in, uint32_t* __restrict__ key_out, uint32_t* __restrict__ other_out,
               uint32_t* __restrict__ val_out, const uint32_t* __restrict__ count_ptr, uint32_t n_fixed, uint32_t cap,
               int shift, const uint32_t* __restrict__ digit_base, uint32_t* __restrict__ lookback,
               uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ status, uint32_t spin_limit) {
    constexpr int kWarps = kSortThreads / 32;
    __shared__ uint32_t warp_hist[kWarps][256];
    __shared__ uint32_t tile_start[256];
    __shared__ uint32_t global_start[256];
    __shared__ uint32_t stage_key[kSortTile];
    __shared__ uint32_t stage_other[kTwoWords ? kSortTile : 1];
    __shared__ uint32_t stage_val[kPayload ? kSortTile : 1];
    __shared__ uint32_t tile_id;
    __shared__ uint32_t scan_buf[256];

    uint32_t n = count_ptr ? min(*count_ptr, cap) : n_fixed;
    if (threadIdx.x == 0) tile_id = atomicAdd(tile_counter, 1u);
    for (int i = threadIdx.x; i < kWarps * 256; i += kSortThreads) (&warp_hist[0][0])[i] = 0u;
    __syncthreads();
    const uint32_t tile = tile_id;
    const uint32_t tile_base = tile * kSortTile;
    if (tile_base >= n) return;
    const uint32_t tile_n = min((uint32_t)kSortTile, n - tile_base);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t lane_lt = (1u << lane) - 1u;

    uint32_t keys[kSortItems];
    uint32_t others[kSortItems];
    uint32_t vals[kSortItems];
    uint32_t ranks[kSortItems];
    // warp w owns items [w*256, (w+1)*256); round r, lane l -> item w*256 + r*32 + l
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        uint32_t item = warp * (32 * kSortItems) + r * 32 + lane;
        bool valid = item < tile_n;
        uint32_t g = tile_base + item;
        keys[r] = valid ? key_in[g] : 0u;
        if (kTwoWords) others[r] = valid ? other_in[g] : 0u;
        if (kPayload) vals[r] = valid ? val_in[g] : 0u;
        uint32_t digit = valid ? ((keys[r] >> shift) & 255u) : 256u;
        uint32_t peers = __match_any_sync(0xFFFFFFFFu, digit);
        uint32_t before = 0;
        if (valid) before = warp_hist[warp][digit];
        __syncwarp();
        if (valid && (peers & lane_lt) == 0u) warp_hist[warp][digit] = before + __popc(peers);
        __syncwarp();
        ranks[r] = before + __popc(peers & lane_lt);
    }
    __syncthreads();
    // thread d owns digit d: prefix over warps, tile count
    const uint32_t d = threadIdx.x;
    uint32_t count = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        uint32_t c = warp_hist[w][d];
        warp_hist[w][d] = count;
        count += c;
    }
    // decoupled look-back for this digit
    uint32_t* lb = lookback + (size_t)tile * 256u;
    uint32_t exclusive = 0;
    if (tile == 0) {
        store_relaxed(&lb[d], kFlagPrefix | count);
    } else {
        store_relaxed(&lb[d], kFlagAggregate | count);
        int32_t t = (int32_t)tile - 1;
        uint32_t spins = 0;
        while (t >= 0) {
            uint32_t word = load_relaxed(lookback + (size_t)t * 256u + d);
            uint32_t flag = word & ~kValueMask;
            if (flag == 0u) {
                if (++spins > spin_limit) {
                    atomicOr(status, DYN_STATUS_LOOKBACK_TIMEOUT);
                    break;
                }
                continue;
            }
            exclusive += word & kValueMask;
            if (flag == kFlagPrefix) break;
            --t;
        }
        __threadfence();
        store_relaxed(&lb[d], kFlagPrefix | (exclusive + count));
    }
    global_start[d] = digit_base[d] + exclusive;
    // exclusive scan over digits for the staging layout
    scan_buf[d] = count;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
        uint32_t t = d >= (uint32_t)off ? scan_buf[d - off] : 0u;
        __syncthreads();
        scan_buf[d] += t;
        __syncthreads();
    }
    tile_start[d] = scan_buf[d] - count;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        uint32_t item = warp * (32 * kSortItems) + r * 32 + lane;
        if (item < tile_n) {
            uint32_t digit = (keys[r] >> shift) & 255u;
            uint32_t pos = tile_start[digit] + warp_hist[warp][digit] + ranks[r];
            stage_key[pos] = keys[r];
            if (kTwoWords) stage_other[pos] = others[r];
            if (kPayload) stage_val[pos] = vals[r];
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < tile_n; i += kSortThreads) {
        uint32_t k = stage_key[i];
        uint32_t digit = (k >> shift) & 255u;
        uint32_t dst = global_start[digit] + (i - tile_start[digit]);
        key_out[dst] = k;
        if (kTwoWords) other_out[dst] = stage_other[i];
        if (kPayload) val_out[dst] = stage_val[i];
    }
}

// Single-pass exclusive scan of u32 values (decoupled look-back over 2048-value tiles).
// Writes out[i] = sum(in[0..i)) and, from the last tile, *total = sum(in[0..n)).
static __global__ void __launch_bounds__(kSortThreads)
    k_scan_exclusive(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, const uint32_t* __restrict__ count_ptr,
                     uint32_t n_fixed, uint32_t cap, uint32_t* __restrict__ total, uint32_t* __restrict__ lookback,
                     uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ status, uint32_t spin_limit) {
    __shared__ uint32_t tile_id;
    __shared__ uint32_t warp_sums[kSortThreads / 32];
    __shared__ uint32_t tile_exclusive;
    uint32_t n = count_ptr ? min(*count_ptr, cap) : n_fixed;
    if (threadIdx.x == 0) tile_id = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = tile_id;
    const uint32_t base = tile * kSortTile + threadIdx.x * kSortItems;
    if (tile * kSortTile >= n) {
        if (tile == 0 && threadIdx.x == 0 && total) *total = 0u;
        return;
    }
    uint32_t v[kSortItems];
    uint32_t sum = 0;
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        uint32_t i = base + r;
        v[r] = i < n ? in[i] : 0u;
        sum += v[r];
    }
    // block scan of per-thread sums
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, off);
        if (lane >= off) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t ws = lane < kSortThreads / 32 ? warp_sums[lane] : 0u;
        uint32_t wi = ws;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, wi, off);
            if (lane >= off) wi += t;
        }
        if (lane < kSortThreads / 32) warp_sums[lane] = wi - ws;
        if (lane == kSortThreads / 32 - 1) {
            uint32_t aggregate = wi;
            uint32_t exclusive = 0;
            if (tile == 0) {
                store_relaxed(&lookback[0], kFlagPrefix | aggregate);
            } else {
                store_relaxed(&lookback[tile], kFlagAggregate | aggregate);
                int32_t t = (int32_t)tile - 1;
                uint32_t spins = 0;
                while (t >= 0) {
                    uint32_t word = load_relaxed(&lookback[t]);
                    uint32_t flag = word & ~kValueMask;
                    if (flag == 0u) {
                        if (++spins > spin_limit) {
                            atomicOr(status, DYN_STATUS_LOOKBACK_TIMEOUT);
                            break;
                        }
                        continue;
                    }
                    exclusive += word & kValueMask;
                    if (flag == kFlagPrefix) break;
                    --t;
                }
                __threadfence();
                store_relaxed(&lookback[tile], kFlagPrefix | (exclusive + aggregate));
            }
            tile_exclusive = exclusive;
            if (total && (tile + 1) * kSortTile >= n) *total = exclusive + aggregate;
        }
    }
    __syncthreads();
    uint32_t run = tile_exclusive + warp_sums[warp] + (incl - sum);
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        uint32_t i = base + r;
        if (i < n) out[i] = run;
        run += v[r];
    }
}

}  // namespace dyn
