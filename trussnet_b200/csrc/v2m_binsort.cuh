// v2m_binsort.cuh -- ascending node ids within each bin of the hash's counting
// sort, after a scatter (one atomic cursor per bin) that placed them in any order.
//
// The CPU's counting sort is stable (src/v2m_particles.cpp:791-795 of
// fangq/trussnet): within a bin the ids ascend. Ids are distinct, so sorting a
// bin's segment ascending restores exactly that order. Work stays linear in the
// bin's size whatever the input:
//   - a bin of at most kSmallBin ids: one thread, insertion sort (at most
//     kSmallBin (kSmallBin - 1) / 2 moves; the common case, bins hold a few ids);
//   - a larger bin: the whole thread block, an LSD radix sort of the segment on
//     4-bit digits of (id - min id), as many passes as the id range needs (at
//     most 8), ping-ponging with a scratch segment of the same size at the same
//     offsets (bins never overlap, so every bin owns its scratch range).
// Crowded bins (coincident or clustered nodes, a caller's skewed keys) therefore
// cost O(c) block work per pass instead of O(c^2) on one thread.
#pragma once

#include <cstdint>

namespace v2m {

constexpr int kSmallBin = 64;          // one-thread bins
constexpr int kBinSortThreads = 256;   // the block of every kernel that calls block_bin_sort
constexpr int kBinSortBuckets = 16;    // 4-bit digits

// a[0, c) ascending, one thread
static __device__ __forceinline__ void small_bin_sort(int* __restrict__ a, int c) {
    for (int x = 1; x < c; ++x) {
        const int v = a[x];
        int y = x - 1;
        while (y >= 0 && a[y] > v) {
            a[y + 1] = a[y];
            --y;
        }
        a[y + 1] = v;
    }
}

// Shared memory of block_bin_sort (one per block).
struct BinSortSmem {
    int cnt[kBinSortBuckets * kBinSortThreads];   // [digit][thread], then the scatter offsets
    int part[kBinSortThreads];                    // per-thread sums of the offset scan
    int vmin[kBinSortThreads / 32], vmax[kBinSortThreads / 32];
    int lo, passes;
};

// a[0, c) (distinct values >= 0) ascending, by the whole block of
// kBinSortThreads threads; tmp[0, c) is scratch. Every thread of the block must
// call it with the same arguments. Each thread owns one contiguous chunk of the
// segment and walks it in order, so each pass is a stable counting sort on one
// digit: the column-major scan of the (digit, thread) counts gives every thread
// its own run of positions per digit.
static __device__ __noinline__ void block_bin_sort(int* __restrict__ a, int* __restrict__ tmp, int c, BinSortSmem& sm) {
    const int t = threadIdx.x;
    const int lane = t & 31, w = t >> 5;
    // the id range: its bit length fixes the number of 4-bit passes
    int lo = 0x7fffffff, hi = 0;
    for (int x = t; x < c; x += kBinSortThreads) {
        const int v = a[x];
        lo = min(lo, v);
        hi = max(hi, v);
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if (lane == 0) {
        sm.vmin[w] = lo;
        sm.vmax[w] = hi;
    }
    __syncthreads();
    if (t == 0) {
        int l = sm.vmin[0], h = sm.vmax[0];
        for (int q = 1; q < kBinSortThreads / 32; ++q) {
            l = min(l, sm.vmin[q]);
            h = max(h, sm.vmax[q]);
        }
        const unsigned range = (unsigned)(h - l);
        const int bits = range ? 32 - __clz((int)range) : 0;
        sm.lo = l;
        sm.passes = (bits + 3) / 4;
    }
    __syncthreads();
    lo = sm.lo;
    const int passes = sm.passes;
    const int chunk = (c + kBinSortThreads - 1) / kBinSortThreads;
    const int x0 = min(c, t * chunk), x1 = min(c, x0 + chunk);
    int* src = a;
    int* dst = tmp;
    for (int p = 0; p < passes; ++p) {
        const int sh = 4 * p;
        int h[kBinSortBuckets];
#pragma unroll
        for (int d = 0; d < kBinSortBuckets; ++d) {
            h[d] = 0;
        }
        for (int x = x0; x < x1; ++x) {
            const int d = ((src[x] - lo) >> sh) & (kBinSortBuckets - 1);
#pragma unroll
            for (int q = 0; q < kBinSortBuckets; ++q) {
                h[q] += q == d;
            }
        }
#pragma unroll
        for (int d = 0; d < kBinSortBuckets; ++d) {
            sm.cnt[d * kBinSortThreads + t] = h[d];
        }
        __syncthreads();
        // exclusive scan of cnt in index order (digit major, thread minor):
        // thread t takes entries [16 t, 16 t + 16)
        int s = 0;
#pragma unroll
        for (int q = 0; q < kBinSortBuckets; ++q) {
            s += sm.cnt[t * kBinSortBuckets + q];
        }
        int incl = s;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) {
                incl += y;
            }
        }
        if (lane == 31) {
            sm.part[w] = incl;
        }
        __syncthreads();
        int before = 0;
        for (int q = 0; q < w; ++q) {
            before += sm.part[q];
        }
        int run = before + incl - s;
        __syncthreads();   // (every thread has read part[] and its cnt entries)
#pragma unroll
        for (int q = 0; q < kBinSortBuckets; ++q) {
            const int e = t * kBinSortBuckets + q;
            const int v = sm.cnt[e];
            sm.cnt[e] = run;
            run += v;
        }
        __syncthreads();
#pragma unroll
        for (int d = 0; d < kBinSortBuckets; ++d) {
            h[d] = sm.cnt[d * kBinSortThreads + t];
        }
        for (int x = x0; x < x1; ++x) {
            const int v = src[x];
            const int d = ((v - lo) >> sh) & (kBinSortBuckets - 1);
            int pos = 0;
#pragma unroll
            for (int q = 0; q < kBinSortBuckets; ++q) {
                if (q == d) {
                    pos = h[q]++;
                }
            }
            dst[pos] = v;
        }
        __syncthreads();
        int* z = src;
        src = dst;
        dst = z;
    }
    if (src != a) {
        for (int x = t; x < c; x += kBinSortThreads) {
            a[x] = src[x];
        }
        __syncthreads();
    }
}

}  // namespace v2m
