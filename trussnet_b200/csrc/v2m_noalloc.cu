// v2m_noalloc.cu -- the hash's counting sort (bin counts, exclusive scan, stable
// scatter) as one entry point that allocates no device memory.
//
// Who needs it: a caller whose process owns the GPU's memory through its own
// pool -- a framework's caching allocator, or a host application (a MATLAB MEX
// host, a plugin host) that has reserved most of the device for itself. There a
// cudaMalloc from the library can fail for want of free memory, or fragment the
// pool, and cudaFree synchronizes the whole device, stalling the caller's other
// streams. Such a caller hands in its own input and output buffers; the only
// other memory this entry point touches is the scratch below.
//
// Scratch: a file-scope __device__ array holding kBins + 1 bin counters (and as
// many scatter cursors), the scan's tile sums and an id segment of kMaxKeys
// entries (the in-bin sort of crowded bins): at most V2M_NOALLOC_MAX_BINS = 2^20
// bins and V2M_NOALLOC_MAX_KEYS = 2^22 keys, about 24 MB, held by every GPU that
// loads the library until the process exits. Host code must not use the array's
// name as a device address (on the host it is only a stand-in): the address
// comes from cudaGetSymbolAddress, taken once per device, with that device
// current, on the first call made on it. A cudaDeviceReset of a device discards
// its copy of the array, and the address cached for it is then stale: do not
// call this entry point on that device again in the same process. Every call
// shares the array and leaves its contents behind; the counters and the error
// flag are cleared at the start of each call. Calls that overlap on the GPU (two
// streams, or two host threads on one device) race on the array and give wrong
// results: serialize them.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/v2m_cuda.h"
#include "v2m_binsort.cuh"

namespace v2m_na {

using v2m::kBinSortThreads;
using v2m::kSmallBin;

constexpr int kBins = V2M_NOALLOC_MAX_BINS;
constexpr int kMaxKeys = V2M_NOALLOC_MAX_KEYS;
constexpr int kTile = 1024;
constexpr int kTiles = (kBins + 1 + kTile - 1) / kTile;
constexpr int kThreads = 256;

// the scratch (see the file comment)
struct Scratch {
    int count[kBins + 1];
    int cursor[kBins + 1];
    int tile[kTiles];
    int tile_ofs[kTiles];
    int err;
    int ids[kMaxKeys];   // scratch of the in-bin sort of bins above kSmallBin ids (same offsets as sorted)
};

static __device__ __align__(256) Scratch g_scratch;

__global__ void k_clear(Scratch* sc, int nbins) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= nbins) {
        sc->count[i] = 0;
    }
    if (i == 0) {
        sc->err = 0;
    }
}

__global__ void k_count(Scratch* sc, const int* __restrict__ key, int n, int nbins) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int k = key[i];
        if (k < 0 || k >= nbins) {
            atomicCAS(&sc->err, 0, 1);
            return;
        }
        atomicAdd(&sc->count[k], 1);
    }
}

__global__ void k_tile_sums(Scratch* sc, int nbins) {
    const int t = blockIdx.x;
    int s = 0;
    for (int q = threadIdx.x; q < kTile; q += blockDim.x) {
        const int e = t * kTile + q;
        if (e <= nbins) {
            s += sc->count[e];
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
    }
    __shared__ int red[kThreads / 32];
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < kThreads / 32; ++w) {
            tot += red[w];
        }
        sc->tile[t] = tot;
    }
}

// one thread walks the (at most kTiles) tile sums in order
__global__ void k_tile_scan(Scratch* sc, int ntiles) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int run = 0;
        for (int t = 0; t < ntiles; ++t) {
            sc->tile_ofs[t] = run;
            run += sc->tile[t];
        }
    }
}

// per tile: bin starts = the tile's offset + the exclusive scan of its counts
__global__ void k_apply(Scratch* sc, int nbins, int* __restrict__ cstart) {
    constexpr int PER = kTile / kThreads;
    const int t = blockIdx.x;
    int x[PER], s = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int e = t * kTile + threadIdx.x * PER + q;
        x[q] = e <= nbins ? sc->count[e] : 0;
        s += x[q];
    }
    int incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if ((threadIdx.x & 31) >= o) {
            incl += y;
        }
    }
    __shared__ int wsum[kThreads / 32];
    if ((threadIdx.x & 31) == 31) {
        wsum[threadIdx.x >> 5] = incl;
    }
    __syncthreads();
    int before = 0;
    for (int w = 0; w < (int)(threadIdx.x >> 5); ++w) {
        before += wsum[w];
    }
    int run = sc->tile_ofs[t] + before + incl - s;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int e = t * kTile + threadIdx.x * PER + q;
        if (e <= nbins) {
            cstart[e] = run;
            sc->cursor[e] = run;
        }
        run += x[q];
    }
}

__global__ void k_scatter(Scratch* sc, const int* __restrict__ key, int n, int nbins, int* __restrict__ sorted) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int k = key[i];
        if (k < 0 || k >= nbins) {
            return;   // (flagged by k_count)
        }
        const int pos = atomicAdd(&sc->cursor[k], 1);
        if (pos >= 0 && pos < n) {
            sorted[pos] = i;
        } else {
            atomicCAS(&sc->err, 0, 2);
        }
    }
}

// Ascending ids within each bin (the stable order): a bin of at most kSmallBin
// ids on one thread, larger bins by the whole block over the scratch's id
// segment at the same offsets -- linear in the bin's size, so a caller's keys
// that crowd into one bin cannot stall a thread.
__global__ void __launch_bounds__(kBinSortThreads) k_bin_order(Scratch* sc, const int* __restrict__ cstart, int nbins,
                                                               int* __restrict__ sorted) {
    __shared__ v2m::BinSortSmem sm;
    __shared__ int big[kBinSortThreads];
    __shared__ int nbig;
    for (int base = blockIdx.x * kBinSortThreads; base < nbins; base += gridDim.x * kBinSortThreads) {
        if (threadIdx.x == 0) {
            nbig = 0;
        }
        __syncthreads();
        const int e = base + threadIdx.x;
        if (e < nbins) {
            const int s0 = cstart[e], c = cstart[e + 1] - s0;
            if (c <= kSmallBin) {
                v2m::small_bin_sort(sorted + s0, c);
            } else {
                big[atomicAdd(&nbig, 1)] = e;
            }
        }
        __syncthreads();
        const int nb = nbig;
        for (int q = 0; q < nb; ++q) {
            const int s0 = cstart[big[q]], s1 = cstart[big[q] + 1];
            v2m::block_bin_sort(sorted + s0, sc->ids + s0, s1 - s0, sm);
        }
        __syncthreads();
    }
}

thread_local std::string g_err;
std::mutex g_mu;
Scratch* g_addr[64] = {};   // per device: the scratch's device address

// once per device, with that device current
Scratch* scratch_for(int dev) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev < 0 || dev >= 64) {
        return nullptr;
    }
    if (!g_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        g_addr[dev] = static_cast<Scratch*>(p);
    }
    return g_addr[dev];
}

}  // namespace v2m_na

using namespace v2m_na;

extern "C" {

int v2m_bin_sort_noalloc(const int32_t* key, int64_t n, int64_t nbins, int32_t* sorted, int32_t* cstart,
                         void* stream) {
    if (n < 0 || nbins < 1) {
        g_err = "v2m_bin_sort_noalloc: n must be >= 0 and nbins >= 1";
        return V2M_ERR_ARG;
    }
    if (n > V2M_NOALLOC_MAX_KEYS) {
        g_err = "v2m_bin_sort_noalloc: " + std::to_string(n) + " keys exceed the fixed scratch of " +
                std::to_string(V2M_NOALLOC_MAX_KEYS) + " keys";
        return V2M_ERR_ARG;
    }
    if (nbins > V2M_NOALLOC_MAX_BINS) {
        g_err = "v2m_bin_sort_noalloc: " + std::to_string(nbins) + " bins exceed the fixed scratch of " +
                std::to_string(V2M_NOALLOC_MAX_BINS) + " bins";
        return V2M_ERR_ARG;
    }
    if ((n > 0 && (!key || !sorted)) || !cstart) {
        g_err = "v2m_bin_sort_noalloc: null buffer";
        return V2M_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        g_err = "v2m_bin_sort_noalloc: no CUDA device";
        return V2M_ERR_CUDA;
    }
    Scratch* sc = scratch_for(dev);
    if (!sc) {
        g_err = "v2m_bin_sort_noalloc: cudaGetSymbolAddress failed for the scratch array";
        return V2M_ERR_CUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nb = (int)nbins, nn = (int)n;
    const int ntiles = (nb + 1 + kTile - 1) / kTile;
    k_clear<<<(nb + 1 + kThreads - 1) / kThreads, kThreads, 0, s>>>(sc, nb);
    if (nn > 0) {
        k_count<<<(nn + kThreads - 1) / kThreads, kThreads, 0, s>>>(sc, key, nn, nb);
    }
    k_tile_sums<<<ntiles, kThreads, 0, s>>>(sc, nb);
    k_tile_scan<<<1, 32, 0, s>>>(sc, ntiles);
    k_apply<<<ntiles, kThreads, 0, s>>>(sc, nb, cstart);
    if (nn > 0) {
        k_scatter<<<(nn + kThreads - 1) / kThreads, kThreads, 0, s>>>(sc, key, nn, nb, sorted);
        k_bin_order<<<(nb + kBinSortThreads - 1) / kBinSortThreads, kBinSortThreads, 0, s>>>(sc, cstart, nb, sorted);
    }
    int err = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(&err, &sc->err, sizeof(int), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(s);
    }
    if (e != cudaSuccess) {
        g_err = std::string("v2m_bin_sort_noalloc: ") + cudaGetErrorString(e);
        return V2M_ERR_CUDA;
    }
    if (err) {
        g_err = "v2m_bin_sort_noalloc: a key is outside [0, nbins)";
        return V2M_ERR_ARG;
    }
    g_err.clear();
    return V2M_OK;
}

const char* v2m_bin_sort_noalloc_error(void) {
    return g_err.c_str();
}

}  // extern "C"
