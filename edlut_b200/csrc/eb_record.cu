// Device sort of the spike recording buffer (eb_get_spikes).
//
// The update kernels append (step << 32 | neuron) records with one atomic per
// warp, so a drained buffer is in no fixed order; the API returns it sorted by
// (step, neuron), the order of the reference's output spike files
// (the output drivers see spikes as the event queue processes them: by time,
// and within one model's update step by neuron index,
// src/spike/TimeDrivenInternalSpike.cpp:182-232).  Sorting on the host took
// 13-20 ms for the ~310k records of 1,000 cerebellar-layer steps, longer than
// simulating them; this is a stable LSD radix sort on the device over only the
// key bits that vary:
//
//   rel = (step - s_lo) << cell_bits | neuron      (s_lo < every recorded step)
//
// 8-bit digits, one pass per digit, three launches per pass: per-tile digit
// histograms, one exclusive scan over them (digit-major, so each tile learns
// where its run of each digit starts), and a stable scatter.  Tiles are 4,096
// keys (256 threads x 16), striped so loads are coalesced; the scatter ranks a
// key among the tile's earlier keys of the same digit with __match_any_sync per
// warp and a per-digit running count across warps.  Every key of a drain is
// distinct (a neuron records at most one spike per step), so the result is the
// same whatever order the records were appended in.
#include <cuda_runtime.h>
#include <cstdint>

#include "eb_record.h"

namespace eb {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kNoDigit = 0xffffffffu;

__device__ __forceinline__ uint32_t digit_of(unsigned long long key, unsigned long long s_lo, int cell_bits,
                                             int shift) {
    const unsigned long long rel = (((key >> 32) - s_lo) << cell_bits) | (key & 0xffffffffull);
    return (uint32_t)(rel >> shift) & 255u;
}

__global__ void __launch_bounds__(kThreads) k_rec_hist(const unsigned long long *__restrict__ keys, int64_t n,
                                                       unsigned long long s_lo, int cell_bits, int shift,
                                                       uint32_t *__restrict__ hist, int ntiles) {
    __shared__ uint32_t h[256];
    const int t = threadIdx.x;
    h[t] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kTile;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int64_t i = base + (int64_t)j * kThreads + t;
        if (i < n) atomicAdd(&h[digit_of(keys[i], s_lo, cell_bits, shift)], 1u);
    }
    __syncthreads();
    hist[(int64_t)t * ntiles + blockIdx.x] = h[t];
}

// Exclusive scan of `total` counts in place, one block of 1024 threads: each
// thread sums a contiguous chunk, the block scans the chunk sums, each thread
// rewrites its chunk.
__global__ void __launch_bounds__(1024) k_rec_scan(uint32_t *__restrict__ hist, int64_t total) {
    __shared__ uint32_t wsum[32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int64_t chunk = (total + 1023) / 1024;
    const int64_t lo = (int64_t)t * chunk;
    const int64_t hi = lo + chunk < total ? lo + chunk : total;
    uint32_t s = 0;
    for (int64_t i = lo; i < hi; ++i) s += hist[i];
    // inclusive warp scan, then the warps' totals
    uint32_t x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t v = wsum[lane], z = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += y;
        }
        wsum[lane] = z - v;  // exclusive prefix of the warps
    }
    __syncthreads();
    uint32_t run = wsum[w] + x - s;
    for (int64_t i = lo; i < hi; ++i) {
        const uint32_t v = hist[i];
        hist[i] = run;
        run += v;
    }
}

__global__ void __launch_bounds__(kThreads) k_rec_scatter(const unsigned long long *__restrict__ keys,
                                                          unsigned long long *__restrict__ out, int64_t n,
                                                          unsigned long long s_lo, int cell_bits, int shift,
                                                          const uint32_t *__restrict__ hist, int ntiles) {
    __shared__ uint32_t off[256];
    __shared__ uint32_t run[256];
    __shared__ uint32_t wc[kWarps][256];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const unsigned lt = (1u << lane) - 1u;
    off[t] = hist[(int64_t)t * ntiles + blockIdx.x];
    run[t] = 0;
    const int64_t base = (int64_t)blockIdx.x * kTile;
    unsigned long long k[kItems];
    uint32_t pos[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int64_t i = base + (int64_t)j * kThreads + t;
        k[j] = i < n ? keys[i] : 0ull;
    }
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const bool valid = base + (int64_t)j * kThreads + t < n;
        const uint32_t d = valid ? digit_of(k[j], s_lo, cell_bits, shift) : kNoDigit;
#pragma unroll
        for (int q = 0; q < kWarps; ++q) wc[q][t] = 0;
        __syncthreads();
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const uint32_t r = (uint32_t)__popc(peers & lt);
        if (valid && r == 0) wc[w][d] = (uint32_t)__popc(peers);
        __syncthreads();
        {   // thread t: digit t's running count through the warps of this slot
            uint32_t c = run[t];
#pragma unroll
            for (int q = 0; q < kWarps; ++q) {
                const uint32_t v = wc[q][t];
                wc[q][t] = c;
                c += v;
            }
            run[t] = c;
        }
        __syncthreads();
        pos[j] = valid ? off[d] + wc[w][d] + r : 0u;
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < kItems; ++j)
        if (base + (int64_t)j * kThreads + t < n) out[pos[j]] = k[j];
}

int bit_width(unsigned long long x) { return x ? 64 - __builtin_clzll(x) : 0; }

}  // namespace

size_t record_sort_hist_words(int64_t n) { return (size_t)256 * (size_t)((n + kTile - 1) / kTile); }

cudaError_t sort_record(unsigned long long *keys, unsigned long long *tmp, uint32_t *hist, int64_t n,
                        int64_t s_lo, int64_t s_hi, int64_t n_cells, cudaStream_t st,
                        unsigned long long **sorted) {
    *sorted = keys;
    if (n <= 1) return cudaSuccess;
    const int cell_bits = bit_width((unsigned long long)(n_cells > 1 ? n_cells - 1 : 1));
    const int step_bits = bit_width((unsigned long long)(s_hi > s_lo ? s_hi - s_lo : 1));
    const int passes = (cell_bits + step_bits + 7) / 8;
    const int ntiles = (int)((n + kTile - 1) / kTile);
    const int64_t total = (int64_t)256 * ntiles;
    unsigned long long *src = keys, *dst = tmp;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        k_rec_hist<<<ntiles, kThreads, 0, st>>>(src, n, (unsigned long long)s_lo, cell_bits, shift, hist, ntiles);
        k_rec_scan<<<1, 1024, 0, st>>>(hist, total);
        k_rec_scatter<<<ntiles, kThreads, 0, st>>>(src, dst, n, (unsigned long long)s_lo, cell_bits, shift, hist,
                                                   ntiles);
        unsigned long long *x = src;
        src = dst;
        dst = x;
    }
    *sorted = src;
    return cudaGetLastError();
}

int record_sort_launches(int64_t n, int64_t s_lo, int64_t s_hi, int64_t n_cells) {
    if (n <= 1) return 0;
    const int cell_bits = bit_width((unsigned long long)(n_cells > 1 ? n_cells - 1 : 1));
    const int step_bits = bit_width((unsigned long long)(s_hi > s_lo ? s_hi - s_lo : 1));
    return 3 * ((cell_bits + step_bits + 7) / 8);
}

}  // namespace eb
