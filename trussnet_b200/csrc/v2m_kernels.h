// v2m_kernels.h -- device buffers of a session and the kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "v2m_types.cuh"

namespace v2m {

constexpr int kScanTile = 1024;     // bin entries per scan tile (volume bin ranges are aligned to it)
constexpr int kScanThreads = 256;
constexpr int kNbrMaxThreads = 256; // k_neighbors: up to 8 warps per block, one node each
constexpr int kMoveThreads = 256;   // k_move_pre's block; volume node ranges are aligned to it
constexpr int kMainThreads = 128;   // the block of k_move_int and k_move_main
constexpr int kCtlThreads = 256;
constexpr int kNodeAlign = kMoveThreads;

// The library's stream-ordered memory pool on `device` (created on first use;
// v2m_host.cu). Freed blocks stay reserved for the next session, up to
// V2M_CUDA_POOL_KEEP_MB (default 16384; 0: returned at once), so repeated calls
// do not map fresh device memory each time. The pool is the library's own: the
// device's default pool is left as the process has it.
cudaMemPool_t library_pool(int device);

// cudaMallocFromPoolAsync from the library's pool of the current device.
inline cudaError_t pool_malloc(void** p, size_t bytes, cudaStream_t s) {
    int dev = 0;
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        return e;
    }
    cudaMemPool_t pool = library_pool(dev);
    return pool ? cudaMallocFromPoolAsync(p, bytes, pool, s) : cudaErrorMemoryAllocation;
}

// Copies between device memory and pageable host memory through two pinned
// staging buffers of the library (allocated once per process, double-buffered:
// the DMA of one chunk overlaps the host copy of the previous one).
// staged_map runs fn(chunk, bytes, offset) on the host over each chunk of
// src (device) in pinned memory and copies the chunk back to dst (device).
cudaError_t staged_d2h(void* dst, const void* src, size_t bytes, cudaStream_t s);
cudaError_t staged_map(void* dst, const void* src, size_t bytes, cudaStream_t s,
                       const std::function<void(void*, size_t, size_t)>& fn);

// Every device array of a session (flat over its volumes).
struct Dev {
    int nvol = 0;
    int sms = 148;       // multiprocessors: the grid of the grid-stride kernels
    int shape_any = 0;   // some volume has analytic shape fields (gm < 0)
    int64_t N = 0;       // nodes incl. per-volume padding
    int64_t KT = 0;      // bin-start entries incl. padding
    int ntile_key = 0;
    DVol* vols = nullptr;
    VolCtl* ctl = nullptr;
    Global* G = nullptr;
    uint16_t* nodevol = nullptr;   // volume of each node, 0xFFFF = padding
    int16_t* tilevol = nullptr;    // volume of each scan tile, -1 = none
    float4* Pq = nullptr;          // x, y, z, +-h (sign: non-interior)
    float4* F = nullptr;           // force + active bars
    float4* Vel = nullptr;         // FIRE velocity
    float4* P0 = nullptr;          // positions at the last list build
    float4* Ps = nullptr;          // bin-order positions + h at the last build
    int2* Js = nullptr;            // bin-order node id and label test (snap_info) at the last build
    uint8_t* typ = nullptr;
    uint16_t* lab = nullptr;
    uint32_t* part = nullptr;      // two uint16 partner labels
    float* mv = nullptr;
    float* pw = nullptr;
    int* key = nullptr;
    int* sorted = nullptr;
    int* sort_tmp = nullptr;       // scratch of the large bins' in-block sort (same offsets as sorted)
    int* nbr = nullptr;            // slot-major: nbr[k*N + i]
    uint8_t* nnb = nullptr;
    int* rlist = nullptr;
    float4* S = nullptr;           // queued nodes' capped step and h
    int* queue = nullptr;          // move queue: trapped from the front, interior from the back
    int* cnt = nullptr;
    int* cstart = nullptr;
    int* cursor = nullptr;
    int* tilesum = nullptr;
    int* tileofs = nullptr;
    double2* psum = nullptr;       // FIRE power and its sum of magnitudes per move block
    double* pser = nullptr;        // serial FIRE power per volume
};

void launch_keys(cudaStream_t s, const Dev& d);
void launch_scan(cudaStream_t s, const Dev& d);
void launch_scatter(cudaStream_t s, const Dev& d);
void launch_neighbors(cudaStream_t s, const Dev& d, int threads);
void launch_force(cudaStream_t s, const Dev& d, int threads);
void launch_move(cudaStream_t s, const Dev& d);
void launch_control(cudaStream_t s, const Dev& d, int serial);
void launch_xcount(cudaStream_t s, const DGrid& g, uint4* xbrick, int* xn, int nb);
void launch_xfill(cudaStream_t s, const DGrid& g, const int2* tabs, float* xphi, int ntab);
void launch_refresh(cudaStream_t s, const Dev& d, int blocks);
void launch_set_rebuild(cudaStream_t s, const Dev& d, int val);
void launch_lists_init(cudaStream_t s, const Dev& d);
void launch_lists_rowmajor(cudaStream_t s, const Dev& d, int64_t nofs, int n, int* out, int* nout);
void launch_constraint_dirs(cudaStream_t s, const Dev& d, int v, int n, bool shape, float* out);
void launch_lists_from_rowmajor(cudaStream_t s, const Dev& d, int64_t nofs, int n, const int* in, const int* nin);
void launch_pack_nodes(cudaStream_t s, const Dev& d, int v, int n, const float* P, const uint8_t* typ_all);
void launch_unpack_P(cudaStream_t s, const Dev& d, int64_t nofs, int n, float* P);
void launch_hn(cudaStream_t s, const Dev& d, int64_t nofs, int n, float* out);
void launch_set_hn(cudaStream_t s, const Dev& d, int64_t nofs, int n, const float* in);
void launch_resign(cudaStream_t s, const Dev& d, int64_t nofs, int n);
void launch_float4_to3(cudaStream_t s, const float4* a, int64_t nofs, int n, float* out);
void launch_float3_to4(cudaStream_t s, const float* in, int64_t nofs, int n, float4* a);
void launch_local_ids(cudaStream_t s, const int* a, int64_t nofs, int n, int* out);
void launch_local_cstart(cudaStream_t s, const int* a, int64_t kofs, int cnt, int64_t nofs, int* out);

// Seeding on the device (v2m_seed.cu): one grid, its size grades and the
// seed-level spacings (computed on the host with the reference's float pow).
struct SeedArgs {
    DGrid g;
    const uint8_t* grade = nullptr;
    const float* spacing = nullptr;   // per seed level
    int nseed = 1;
    int voxmode = 0;
    float jseed = 0.0f;
    int corners = 1;
    float hmax = 0.0f;
    const float* feat = nullptr;      // shape input's sharp features (host memory, tn::Grid::feat), or none
    int64_t nfeat = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
};

// The seeds (device arrays in `tmp`, freed by the caller): n nodes, P xyz, lab,
// typ, part pairs and part3 in tn::Nodes' layout.
struct SeedBuffers {
    std::vector<void*> tmp;
    float* P = nullptr;
    uint16_t* lab = nullptr;
    uint8_t* typ = nullptr;
    uint16_t* part = nullptr;
    uint16_t* part3 = nullptr;
    int n = 0;
};

cudaError_t seed_run(const SeedArgs& A, SeedBuffers& B, std::string& err);

}  // namespace v2m
