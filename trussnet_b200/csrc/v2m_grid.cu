// v2m_grid.cu -- the relaxation's fields built on the device from a label
// volume: tn::build_grid_cpu (src/v2m_grid.cpp:47-722 of fangq/trussnet) for
// label input, stage by stage and bit for bit.
//
//   k_maxlabel      highest label (the label count of the sizing)
//   k_brick_labels  labels within R of each 8^3 brick, one warp per brick    [v2m_brick_labels, src/opencl/v2m_grid_body.cl:28-69]
//   (scan)          one slot per (mixed brick, label), in brick order        [src/v2m_grid.cpp:123-144]
//   k_smooth        separable Gaussian of a slot's indicator, one block per  [smooth_all, src/v2m_grid.cpp:168-228]
//                   slot, the (8+2R)^3 tile in shared memory, the reference's
//                   pass order and summation order
//   k_size          per-voxel size: own label, strongest competitor,         [v2m_size_voxel / v2m_kappa_max, src/opencl/v2m_grid_body.cl:321-475]
//                   curvature bound 1/(K |kappa|)
//   k_thick_peak_bricks  per voxel, the largest own-label phi within +-2    [v2m_thick_voxel, src/opencl/v2m_grid_body.cl:241-276]
//                   voxels; one block per brick, the halo's labels and phi
//                   in shared memory
//   k_thick_pick    the voxels whose thickness needs erfinv, listed; the
//                   host maps their peaks (erfinv needs the host's logf) and
//   k_thick_put     scatters the thicknesses back
//   k_axis_min /    the thin-layer blend weight: min filter, smoothstep,     [src/v2m_grid.cpp:465-527]
//   k_smoothstep /  Gaussian blur, separable passes on the dense grid
//   k_axis_blur
//   k_blend         phi = w phi(sigma) + (1 - w) phi(sigma_thin)
//   k_preserve      own label on top at voxel centres (preserve > 0)         [v2m_preserve_voxel, src/opencl/v2m_grid_body.cl:282-314]
//   k_limit         one Jacobi sweep of the gradient limit |grad h| <= g     [v2m_limit_voxel, src/opencl/v2m_grid_body.cl:477-495]
//   k_grade         the 256 log-spaced size grades, from thresholds the host  [v2m_grade, src/opencl/v2m_grid_body.cl:498-506]
//                   finds with its own logf
//
// Where the reference calls logf (the thickness's erfinv, the grades), the host
// evaluates it: the host C library's logf is not correctly rounded, so the
// device cannot reproduce it with its own log. Everything else is device work.
// The Gaussian weights are computed on the host with the reference's
// expression (host expf), as the reference does.
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/v2m_cuda.h"
#include "v2m_field.cuh"
#include "v2m_grid.h"
#include "v2m_kernels.h"

namespace v2m {
namespace {

constexpr int kMaxR = 6;
constexpr int kSmoothThreads = 256;

struct Dims {
    int nx, ny, nz, nbx, nby, nbz;
    float vx, vy, vz;
};

__device__ __forceinline__ int lab_at(const uint16_t* __restrict__ L, const Dims& d, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= d.nx || j >= d.ny || k >= d.nz) {
        return 0;
    }
    return L[i + (size_t)d.nx * (j + (size_t)d.ny * k)];
}

__global__ void k_maxlabel(const uint16_t* __restrict__ L, int64_t nv, int* out) {
    int m = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        m = max(m, (int)L[v]);
    }
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, m);
    }
}

// One warp per brick: the labels of the brick's box dilated by R voxels (the
// outside of the grid is label 0), scanned in the reference's order (z, y, x):
// the first V2M_BL distinct labels met are kept, ascending; more than V2M_BL:
// count V2M_BL + 1. A batch of 32 voxels at a time; the labels not yet listed
// are taken in lane order (the scan order) by their first lane.
__global__ void k_brick_labels(const uint16_t* __restrict__ L, Dims d, int R, int* __restrict__ bl_cnt,
                               uint16_t* __restrict__ bl_lab, int nb) {
    __shared__ int s_lab[8][V2M_BL];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int b = blockIdx.x * (blockDim.x >> 5) + w;
    if (b >= nb) {
        return;
    }
    const int bx = b % d.nbx, by = (b / d.nbx) % d.nby, bz = b / (d.nbx * d.nby);
    const int W = V2M_BS + 2 * R + 1;   // (x0 .. x1 inclusive)
    const int x0 = bx * V2M_BS - R, y0 = by * V2M_BS - R, z0 = bz * V2M_BS - R;
    const int total = W * W * W;
    int n = 0, ovf = 0;
    for (int base = 0; base < total; base += 32) {
        const int e = base + lane;
        int l = -1;
        if (e < total) {
            const int x = e % W, y = (e / W) % W, z = e / (W * W);
            l = lab_at(L, d, x0 + x, y0 + y, z0 + z);
        }
        bool seen = l < 0;
        for (int q = 0; q < n && !seen; ++q) {
            seen = s_lab[w][q] == l;
        }
        const bool fresh = !seen;
        const unsigned peers = __match_any_sync(0xffffffffu, fresh ? l : -2 - lane);
        unsigned firsts = __ballot_sync(0xffffffffu, fresh && (__ffs(peers) - 1) == lane);
        while (firsts) {
            const int src = __ffs(firsts) - 1;
            firsts &= firsts - 1;
            const int nl = __shfl_sync(0xffffffffu, l, src);
            if (n >= V2M_BL) {
                ovf = 1;
                continue;
            }
            if (lane == 0) {   // insertion keeps the list ascending
                int k = n;
                while (k > 0 && s_lab[w][k - 1] > nl) {
                    s_lab[w][k] = s_lab[w][k - 1];
                    --k;
                }
                s_lab[w][k] = nl;
            }
            ++n;
            __syncwarp();
        }
    }
    if (lane == 0) {
        bl_cnt[b] = ovf ? V2M_BL + 1 : n;
    }
    if (lane < V2M_BL) {
        bl_lab[(size_t)b * V2M_BL + lane] = lane < n ? (uint16_t)s_lab[w][lane] : (uint16_t)0xFFFF;
    }
}

// slots per brick: min(count, V2M_BL) when more than one, else none
__global__ void k_slot_count(const int* __restrict__ bl_cnt, int* __restrict__ c, int nb) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb) {
        const int n = min(bl_cnt[b], V2M_BL);
        c[b] = n <= 1 ? 0 : n;
    }
}

__global__ void k_slot_fill(const int* __restrict__ c, const int* __restrict__ ofs, const uint16_t* __restrict__ bl_lab,
                            int* __restrict__ bl_slot, int* __restrict__ slot_brick, uint16_t* __restrict__ slot_label,
                            int nb) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) {
        return;
    }
    const int n = c[b];
    bl_slot[b] = n ? ofs[b] : -1;
    for (int q = 0; q < n; ++q) {
        slot_brick[ofs[b] + q] = b;
        slot_label[ofs[b] + q] = bl_lab[(size_t)b * V2M_BL + q];
    }
}

struct GaussW {
    float w[2 * kMaxR + 1];
};

// One block per slot: the label's indicator on the brick's (8+2R)^3 tile, then
// x (centre columns), y (centre rows), z (the 512 centre voxels), each a sum
// over dd = -R..R in that order, from 0 -- the reference's loops.
__global__ void __launch_bounds__(kSmoothThreads) k_smooth(const uint16_t* __restrict__ L, Dims d,
                                                          const int* __restrict__ slot_brick,
                                                          const uint16_t* __restrict__ slot_label, GaussW gw, int R,
                                                          float* __restrict__ phi) {
    extern __shared__ float sm[];
    const int T = V2M_BS + 2 * R;
    float* A = sm;
    float* B = sm + T * T * T;
    const int s = blockIdx.x;
    const int b = slot_brick[s];
    const int l = slot_label[s];
    const int x0 = (b % d.nbx) * V2M_BS - R, y0 = ((b / d.nbx) % d.nby) * V2M_BS - R,
              z0 = (b / (d.nbx * d.nby)) * V2M_BS - R;
    for (int e = threadIdx.x; e < T * T * T; e += kSmoothThreads) {
        const int x = e % T, y = (e / T) % T, z = e / (T * T);
        A[e] = lab_at(L, d, x0 + x, y0 + y, z0 + z) == l ? 1.0f : 0.0f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < T * T * V2M_BS; e += kSmoothThreads) {   // x
        const int x = R + e % V2M_BS, y = (e / V2M_BS) % T, z = e / (V2M_BS * T);
        float v = 0.0f;
        for (int dd = -R; dd <= R; ++dd) {
            v += gw.w[dd + R] * A[x + dd + T * (y + T * z)];
        }
        B[x + T * (y + T * z)] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < T * V2M_BS * V2M_BS; e += kSmoothThreads) {   // y
        const int x = R + e % V2M_BS, y = R + (e / V2M_BS) % V2M_BS, z = e / (V2M_BS * V2M_BS);
        float v = 0.0f;
        for (int dd = -R; dd <= R; ++dd) {
            v += gw.w[dd + R] * B[x + T * (y + dd + T * z)];
        }
        A[x + T * (y + T * z)] = v;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < V2M_SLOT; t += kSmoothThreads) {   // z
        const int x = t % V2M_BS + R, y = (t / V2M_BS) % V2M_BS + R, z = t / (V2M_BS * V2M_BS) + R;
        float v = 0.0f;
        for (int dd = -R; dd <= R; ++dd) {
            v += gw.w[dd + R] * A[x + T * (y + T * (z + dd))];
        }
        phi[(size_t)s * V2M_SLOT + t] = v;
    }
}

// Largest principal curvature of the level set of psi_ab through voxel
// (i,j,k), central differences with stride st (v2m_kappa_max,
// src/opencl/v2m_grid_body.cl:321-392), the reference's expressions.
__device__ __noinline__ float kappa_max(const DGrid& g, int a, int b, int i, int j, int k, int st) {
    float f[27];
    for (int n = 0; n < 27; ++n) {
        const int dx = (n % 3 - 1) * st, dy = ((n / 3) % 3 - 1) * st, dz = (n / 9 - 1) * st;
        f[n] = phi_voxel(g, a, i + dx, j + dy, k + dz) - phi_voxel(g, b, i + dx, j + dy, k + dz);
    }
#define F3(dx, dy, dz) f[((dx) + 1) + 3 * ((dy) + 1) + 9 * ((dz) + 1)]
    const float hx = g.vx * st, hy = g.vy * st, hz = g.vz * st;
    float gr[3], H[9];
    gr[0] = (F3(1, 0, 0) - F3(-1, 0, 0)) / (2 * hx);
    gr[1] = (F3(0, 1, 0) - F3(0, -1, 0)) / (2 * hy);
    gr[2] = (F3(0, 0, 1) - F3(0, 0, -1)) / (2 * hz);
    H[0] = (F3(1, 0, 0) - 2 * F3(0, 0, 0) + F3(-1, 0, 0)) / (hx * hx);
    H[4] = (F3(0, 1, 0) - 2 * F3(0, 0, 0) + F3(0, -1, 0)) / (hy * hy);
    H[8] = (F3(0, 0, 1) - 2 * F3(0, 0, 0) + F3(0, 0, -1)) / (hz * hz);
    H[1] = H[3] = (F3(1, 1, 0) - F3(1, -1, 0) - F3(-1, 1, 0) + F3(-1, -1, 0)) / (4 * hx * hy);
    H[2] = H[6] = (F3(1, 0, 1) - F3(1, 0, -1) - F3(-1, 0, 1) + F3(-1, 0, -1)) / (4 * hx * hz);
    H[5] = H[7] = (F3(0, 1, 1) - F3(0, 1, -1) - F3(0, -1, 1) + F3(0, -1, -1)) / (4 * hy * hz);
#undef F3
    const float gn = sqrtf(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
    if (gn < 1e-6f) {
        return 0.0f;
    }
    float n[3], Pm[9], HP[9];
    n[0] = gr[0] / gn;
    n[1] = gr[1] / gn;
    n[2] = gr[2] / gn;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            Pm[3 * r + c] = (r == c ? 1.0f : 0.0f) - n[r] * n[c];
        }
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            HP[3 * r + c] = H[3 * r] * Pm[c] + H[3 * r + 1] * Pm[3 + c] + H[3 * r + 2] * Pm[6 + c];
        }
    }
    float T = 0.0f, F = 0.0f, PHP[9];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            PHP[3 * r + c] = Pm[3 * r] * HP[c] + Pm[3 * r + 1] * HP[3 + c] + Pm[3 * r + 2] * HP[6 + c];
            F += PHP[3 * r + c] * PHP[3 * r + c];
        }
    }
    T = (PHP[0] + PHP[4] + PHP[8]) / gn;
    F /= gn * gn;
    const float disc = 2.0f * F - T * T;
    return 0.5f * (fabsf(T) + sqrtf(disc > 0.0f ? disc : 0.0f));
}

struct SizeArgs {
    const float* hlab;
    int nlab;
    float hbase, hmin, hmax, K, hcurv;
};

// Initial size at each voxel (v2m_size_voxel, src/opencl/v2m_grid_body.cl:413-475;
// no interface sizes, no analytic curvature: label input).
__global__ void k_size(DGrid g, SizeArgs A, float* __restrict__ h) {
    const int64_t nv = (int64_t)g.nx * g.ny * g.nz;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(v % g.nx), j = (int)((v / g.nx) % g.ny), k = (int)(v / ((int64_t)g.nx * g.ny));
        const int a = g.L[v];
        float hh = (a < A.nlab && A.hlab[a] > 0.0f) ? A.hlab[a] : A.hbase;
        if (a == 0) {
            h[v] = A.hmax;
            continue;
        }
        const int bk = brick_index(g, i, j, k);
        if (g.bl_slot[bk] >= 0) {
            const float pa = phi_voxel(g, a, i, j, k);
            int best = -1;
            float pb = -1.0f;
            const int cnt = g.bl_cnt[bk];
            for (int s = 0; s < cnt && s < V2M_BL; ++s) {
                const int l = g.bl_lab[(size_t)bk * V2M_BL + s];
                if (l == a) {
                    continue;
                }
                const float pv = phi_voxel(g, l, i, j, k);
                if (pv > pb) {
                    pb = pv;
                    best = l;
                }
            }
            if (best >= 0 && pa - pb < 0.45f) {
                if (best < A.nlab && A.hlab[best] > 0.0f) {
                    hh = fminf(hh, A.hlab[best]);
                }
                const float kap = kappa_max(g, a, best, i, j, k, 1);
                if (kap > 0.0f) {
                    hh = fminf(hh, fmaxf(1.0f / (A.K * kap), A.hcurv));
                }
            }
        }
        h[v] = hh < A.hmin ? A.hmin : (hh > A.hmax ? A.hmax : hh);
    }
}

// The voxels whose thickness needs erfinv (peak m in [0, 0.9999)) listed for the
// host, the others set to "no thickness" (1e30) here. The list's order varies
// from run to run; each entry carries its voxel, so the results do not.
__global__ void k_thick_pick(float* __restrict__ tv, int64_t nv, int* __restrict__ cnt, int* __restrict__ idx,
                             float* __restrict__ val) {
    const int lane = threadIdx.x & 31;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < nv; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = base + threadIdx.x;
        const float m = v < nv ? tv[v] : -1.0f;
        const bool need = v < nv && m >= 0.0f && m < 0.9999f;
        if (v < nv && !need) {
            tv[v] = 1e30f;
        }
        const unsigned b = __ballot_sync(0xffffffffu, need);
        int at = 0;
        if (lane == 0 && b) {
            at = atomicAdd(cnt, __popc(b));
        }
        at = __shfl_sync(0xffffffffu, at, 0);
        if (need) {
            const int k = at + __popc(b & ((1u << lane) - 1u));
            idx[k] = (int)v;
            val[k] = m;
        }
    }
}

__global__ void k_thick_put(float* __restrict__ tv, const int* __restrict__ idx, const float* __restrict__ val,
                            int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        tv[idx[k]] = val[k];
    }
}

// The thickness's device half (v2m_thick_voxel): the largest phi of the
// voxel's own label over the own-label voxels within +-2; -1 in a uniform
// brick. One block per brick, 2 voxels a thread. A mixed
// brick stages the labels of its (8+4)^3 halo (0 outside the grid, as
// label_at) and, for each listed label that some voxel of the brick owns, that
// label's phi over the halo (phi_voxel, outside the grid included); the voxels
// of that label then take the maximum over their own-label neighbours from
// shared memory. The maximum starts at +0 and takes f > m, so its value does
// not depend on the visiting order. A voxel whose label is not among the
// brick's first V2M_BL (an overflowing brick) takes the per-voxel loop.
constexpr int kPeakR = 2;
constexpr int kPeakT = V2M_BS + 2 * kPeakR;   // 12

__global__ void __launch_bounds__(256) k_thick_peak_bricks(DGrid g, float* __restrict__ out) {
    __shared__ uint16_t lt[kPeakT * kPeakT * kPeakT];
    __shared__ float pt[kPeakT * kPeakT * kPeakT];
    const int b = blockIdx.x;
    const int bx = b % g.nbx, by = (b / g.nbx) % g.nby, bz = b / (g.nbx * g.nby);
    const int i0 = bx * V2M_BS, j0 = by * V2M_BS, k0 = bz * V2M_BS;
    int vi[2], vj[2], vk[2], own[2];
    bool in[2];
    float m[2] = { 0.0f, 0.0f };
    bool done[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int t = threadIdx.x + 256 * q;
        vi[q] = i0 + (t & 7);
        vj[q] = j0 + ((t >> 3) & 7);
        vk[q] = k0 + (t >> 6);
        in[q] = vi[q] < g.nx && vj[q] < g.ny && vk[q] < g.nz;
        done[q] = !in[q];
    }
    const size_t sx = (size_t)g.nx, sxy = (size_t)g.nx * g.ny;
    if (g.bl_slot[b] < 0) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (in[q]) {
                out[vi[q] + sx * vj[q] + sxy * vk[q]] = -1.0f;
            }
        }
        return;
    }
    for (int e = threadIdx.x; e < kPeakT * kPeakT * kPeakT; e += 256) {
        const int u = i0 - kPeakR + e % kPeakT, w = j0 - kPeakR + (e / kPeakT) % kPeakT,
                  z = k0 - kPeakR + e / (kPeakT * kPeakT);
        lt[e] = (uint16_t)label_at(g, u, w, z);
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        own[q] = in[q] ? g.L[vi[q] + sx * vj[q] + sxy * vk[q]] : -1;
    }
    const int cnt = min(g.bl_cnt[b], V2M_BL);
    for (int s = 0; s < cnt; ++s) {
        const int l = g.bl_lab[(size_t)b * V2M_BL + s];
        if (!__syncthreads_or(own[0] == l || own[1] == l)) {
            continue;
        }
        for (int e = threadIdx.x; e < kPeakT * kPeakT * kPeakT; e += 256) {
            pt[e] = phi_voxel(g, l, i0 - kPeakR + e % kPeakT, j0 - kPeakR + (e / kPeakT) % kPeakT,
                              k0 - kPeakR + e / (kPeakT * kPeakT));
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (!done[q] && own[q] == l) {
                const int c = (vi[q] - i0) + kPeakT * ((vj[q] - j0) + kPeakT * (vk[q] - k0));
                float mm = 0.0f;
                for (int dz = 0; dz <= 2 * kPeakR; ++dz) {
                    for (int dy = 0; dy <= 2 * kPeakR; ++dy) {
                        for (int dx = 0; dx <= 2 * kPeakR; ++dx) {
                            const int e = c + dx + kPeakT * (dy + kPeakT * dz);
                            if (lt[e] == l) {
                                const float f = pt[e];
                                mm = f > mm ? f : mm;
                            }
                        }
                    }
                }
                m[q] = mm;
                done[q] = true;
            }
        }
        __syncthreads();   // pt is refilled for the next label
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        if (!in[q]) {
            continue;
        }
        if (!done[q]) {   // own label beyond the brick's list: the per-voxel loop
            const int a = own[q];
            float mm = 0.0f;
            for (int dz = -kPeakR; dz <= kPeakR; ++dz) {
                for (int dy = -kPeakR; dy <= kPeakR; ++dy) {
                    for (int dx = -kPeakR; dx <= kPeakR; ++dx) {
                        const int u = vi[q] + dx, w = vj[q] + dy, z = vk[q] + dz;
                        if (label_at(g, u, w, z) != a) {
                            continue;
                        }
                        const float f = phi_voxel(g, a, u, w, z);
                        mm = f > mm ? f : mm;
                    }
                }
            }
            m[q] = mm;
        }
        out[vi[q] + sx * vj[q] + sxy * vk[q]] = m[q];
    }
}

// thin-layer sizing: h <= max(floor, t vmin / thick) where t is finite
__global__ void k_thick_size(const float* __restrict__ tv, float* __restrict__ h, int64_t nv, float floor_mm, float vmin,
                             float thick) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        const float t = tv[v];
        if (t < 1e29f) {
            h[v] = fminf(h[v], fmaxf(floor_mm, t * vmin / thick));
        }
    }
}

// one separable pass along `axis`, indices clamped to the grid: min over
// radius r (mn) or the kernel-weighted sum (src/v2m_grid.cpp:470-487)
__global__ void k_axis_pass(const float* __restrict__ src, float* __restrict__ dst, Dims d, int axis, int r, int mn,
                            GaussW ker) {
    const int64_t nv = (int64_t)d.nx * d.ny * d.nz;
    const int64_t st = axis == 0 ? 1 : (axis == 1 ? d.nx : (int64_t)d.nx * d.ny);
    const int nlen = axis == 0 ? d.nx : (axis == 1 ? d.ny : d.nz);
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)((v / st) % nlen);
        float acc = mn ? 1e30f : 0.0f;
        for (int dd = -r; dd <= r; ++dd) {
            const int cc = min(nlen - 1, max(0, c + dd));
            const float x = src[v + (cc - c) * st];
            acc = mn ? (x < acc ? x : acc) : acc + ker.w[dd + r] * x;
        }
        dst[v] = acc;
    }
}

__global__ void k_smoothstep(float* __restrict__ w, int64_t nv, float lo, float den) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        float x = (w[v] - lo) / den;
        x = fminf(1.0f, fmaxf(0.0f, x));
        w[v] = x * x * (3.0f - 2.0f * x);
    }
}

// phi <- w phi_s + (1 - w) phi (the sharp field), voxels inside the grid
__global__ void k_blend(const int* __restrict__ slot_brick, const float* __restrict__ wv, const float* __restrict__ phi_s,
                        float* __restrict__ phi, Dims d, int64_t ns) {
    const int64_t tot = ns * V2M_SLOT;
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < tot; o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = o / V2M_SLOT;
        const int t = (int)(o % V2M_SLOT);
        const int b = slot_brick[s];
        const int i = (b % d.nbx) * V2M_BS + t % V2M_BS, j = ((b / d.nbx) % d.nby) * V2M_BS + (t / V2M_BS) % V2M_BS,
                  k = (b / (d.nbx * d.nby)) * V2M_BS + t / (V2M_BS * V2M_BS);
        if (i >= d.nx || j >= d.ny || k >= d.nz) {
            continue;
        }
        const float w = wv[i + (size_t)d.nx * (j + (size_t)d.ny * k)];
        phi[o] = w * phi_s[o] + (1.0f - w) * phi[o];
    }
}

// v2m_preserve_voxel: the voxel's own label at least margin m above the others
__global__ void k_preserve(DGrid g, float* __restrict__ phi, float m) {
    const int64_t nv = (int64_t)g.nx * g.ny * g.nz;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(v % g.nx), j = (int)((v / g.nx) % g.ny), k = (int)(v / ((int64_t)g.nx * g.ny));
        const int b = brick_index(g, i, j, k);
        const int slot = g.bl_slot[b];
        if (slot < 0) {
            continue;
        }
        const int a = g.L[v];
        const size_t t = (size_t)(i & 7) + V2M_BS * ((j & 7) + V2M_BS * (k & 7));
        const int n = g.bl_cnt[b] < V2M_BL ? g.bl_cnt[b] : V2M_BL;
        int sa = -1;
        float mo = 0.0f;
        for (int s = 0; s < n; ++s) {
            const float x = phi[(size_t)(slot + s) * V2M_SLOT + t];
            if (g.bl_lab[(size_t)b * V2M_BL + s] == a) {
                sa = slot + s;
            } else if (x > mo) {
                mo = x;
            }
        }
        if (sa >= 0 && phi[(size_t)sa * V2M_SLOT + t] < mo + m) {
            phi[(size_t)sa * V2M_SLOT + t] = mo + m;
        }
    }
}

struct LimitW {
    float d[27];   // g |x - x_n| for each of the 26 neighbours (n = 13: the voxel itself, unused)
};

// One Jacobi sweep (v2m_limit_voxel): hn = min(h, h_n + g |x - x_n|) over the 26
// neighbours inside the grid; *changed = 1 if some value dropped.
__global__ void k_limit(const float* __restrict__ h, float* __restrict__ hn, Dims d, LimitW lw, int* changed) {
    const int64_t nv = (int64_t)d.nx * d.ny * d.nz;
    int any = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(v % d.nx), j = (int)((v / d.nx) % d.ny), k = (int)(v / ((int64_t)d.nx * d.ny));
        const float h0 = h[v];
        float m = h0;
        for (int n = 0; n < 27; ++n) {
            const int dx = n % 3 - 1, dy = (n / 3) % 3 - 1, dz = n / 9 - 1;
            const int x = i + dx, y = j + dy, z = k + dz;
            if (n == 13 || x < 0 || y < 0 || z < 0 || x >= d.nx || y >= d.ny || z >= d.nz) {
                continue;
            }
            m = fminf(m, h[x + (size_t)d.nx * (y + (size_t)d.ny * z)] + lw.d[n]);
        }
        hn[v] = m;
        any |= m < h0;
    }
    if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0) {
        *changed = 1;
    }
}

// grade = the number of thresholds at or below h (the host found, with its own
// logf, the smallest size of each grade 1..255)
__global__ void k_grade(const float* __restrict__ h, int64_t nv, const float* __restrict__ th, uint8_t* __restrict__ grade) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        const float x = h[v];
        int lo = 0, hi = 255;   // count of th[0..255) <= x
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (th[mid] <= x) {
                lo = mid + 1;
            } else {
                hi = mid;
            }
        }
        grade[v] = (uint8_t)lo;
    }
}

// ---- host ----------------------------------------------------------------------
// The reference's float expressions for what stays on the host (compiled
// without contraction, as the reference's host build).
float gauss_weight(int dd, float sigma) {
    return std::exp(-0.5f * (float)(dd * dd) / (sigma * sigma));
}

GaussW gauss_weights(float sigma, int R) {
    GaussW g{};
    float ws = 0.0f;
    for (int dd = -R; dd <= R; ++dd) {
        g.w[dd + R] = gauss_weight(dd, sigma);
        ws += g.w[dd + R];
    }
    for (int dd = 0; dd <= 2 * R; ++dd) {
        g.w[dd] /= ws;
    }
    return g;
}

// erfinv in single precision by M. Giles' published approximation ("Approximating
// the erfinv function", GPU Computing Gems, 2010), as the reference's
// v2m_erfinv evaluates it (src/opencl/v2m_grid_body.cl:204-233).
float erfinv_giles(float x) {
    float w = -std::log((1.0f - x) * (1.0f + x)), p;
    if (w < 5.0f) {
        w -= 2.5f;
        p = 2.81022636e-08f;
        p = 3.43273939e-07f + p * w;
        p = -3.5233877e-06f + p * w;
        p = -4.39150654e-06f + p * w;
        p = 0.00021858087f + p * w;
        p = -0.00125372503f + p * w;
        p = -0.00417768164f + p * w;
        p = 0.246640727f + p * w;
        p = 1.50140941f + p * w;
    } else {
        w = std::sqrt(w) - 3.0f;
        p = -0.000200214257f;
        p = 0.000100950558f + p * w;
        p = 0.00134934322f + p * w;
        p = -0.00367342844f + p * w;
        p = 0.00573950773f + p * w;
        p = -0.0076224613f + p * w;
        p = 0.00943887047f + p * w;
        p = 1.00167406f + p * w;
        p = 2.83297682f + p * w;
    }
    return p * x;
}

// v2m_grade (src/opencl/v2m_grid_body.cl:498-506) with the host's logf
uint8_t grade_of(float h, float hmin, float hmax) {
    if (hmax <= hmin * 1.0001f) {
        return 0;
    }
    float t = std::log(h / hmin) / std::log(hmax / hmin);
    t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
    return (uint8_t)(t * 255.0f + 0.5f);
}

// th[k-1] = the smallest positive float whose grade is >= k (k = 1..255), by
// bisection over the float bit patterns (grade_of is non-decreasing in h: the
// host logf is monotone, checked over every float in [2^-30, 2^30)); +inf
// where no float reaches grade k.
std::vector<float> grade_thresholds(float hmin, float hmax) {
    std::vector<float> th(255, INFINITY);
    if (hmax <= hmin * 1.0001f) {
        return th;
    }
    auto f_of = [](uint32_t u) {
        float f;
        std::memcpy(&f, &u, 4);
        return f;
    };
    const uint32_t top = 0x7f7fffffu;   // the largest finite float
    for (int k = 1; k <= 255; ++k) {
        if (grade_of(f_of(top), hmin, hmax) < k) {
            continue;
        }
        uint32_t lo = 1, hi = top;   // grade(f(hi)) >= k
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (grade_of(f_of(mid), hmin, hmax) >= k) {
                hi = mid;
            } else {
                lo = mid + 1;
            }
        }
        th[k - 1] = f_of(lo);
    }
    return th;
}

unsigned gs_blocks(int64_t n, int sms) {
    const int64_t need = (n + 255) / 256;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * 16));
}

}  // namespace

cudaError_t grid_build(const GridBuildArgs& A, GridBuildOut& O, std::string& err) {
    cudaStream_t st = A.stream;
    const Dims d{ A.nx, A.ny, A.nz, (A.nx + 7) / 8, (A.ny + 7) / 8, (A.nz + 7) / 8, A.vs[0], A.vs[1], A.vs[2] };
    const int64_t nv = (int64_t)A.nx * A.ny * A.nz;
    const int nb = d.nbx * d.nby * d.nbz;
    const GridParamsH& p = A.prm;
    std::vector<void*>& tmp = O.tmp;
    auto lap = [&](const char* what) {
        if (A.lap) {
            A.lap(what);
        }
    };
    auto dalloc = [&](size_t bytes) -> void* {
        void* q = nullptr;
        if (pool_malloc(&q, std::max<size_t>(bytes, 16), st) != cudaSuccess) {
            return nullptr;
        }
        tmp.push_back(q);
        return q;
    };
#define V2M_TRY(x)                    \
    do {                              \
        const cudaError_t e_ = (x);   \
        if (e_ != cudaSuccess) {      \
            return e_;                \
        }                             \
    } while (0)
#define V2M_ALLOC(ptr, T, count)                                       \
    do {                                                               \
        ptr = static_cast<T*>(dalloc(sizeof(T) * (size_t)(count)));    \
        if (!ptr) {                                                    \
            return cudaErrorMemoryAllocation;                          \
        }                                                              \
    } while (0)
    // the reference's derived sizes (src/v2m_grid.cpp:58-80)
    const int Ri = std::min(6, std::max(1, (int)std::ceil(3.0f * p.sigma)));
    const int Rc = std::min(6, std::max(1, (int)std::ceil(3.0f * p.sigma_curv)));
    const int R = std::max(Ri, Rc);
    const float vmin = std::min(A.vs[0], std::min(A.vs[1], A.vs[2]));
    float hbase = p.hbase > 0 ? p.hbase : 3.0f * vmin;
    float hmin = p.hmin > 0 ? p.hmin : hbase / 3.0f;
    float hmax = p.hmax > 0 ? p.hmax : hbase;
    for (float v : p.hlab) {
        if (v > 0) {
            hmax = std::max(hmax, v);
            hmin = std::min(hmin, v);
        }
    }
    const float hcurv = hmin;
    O.R = R;
    O.hbase = hbase;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, A.device);
    // labels
    uint16_t* L;
    V2M_ALLOC(L, uint16_t, nv);
    V2M_TRY(cudaMemcpyAsync(L, A.L, 2 * (size_t)nv, cudaMemcpyHostToDevice, st));
    int* dmax;
    V2M_ALLOC(dmax, int, 1);
    V2M_TRY(cudaMemsetAsync(dmax, 0, 4, st));
    k_maxlabel<<<gs_blocks(nv, sms), 256, 0, st>>>(L, nv, dmax);
    int maxlabel = 0;
    V2M_TRY(cudaMemcpyAsync(&maxlabel, dmax, 4, cudaMemcpyDeviceToHost, st));
    // 1. labels near each brick
    int* bl_cnt;
    uint16_t* bl_lab;
    int* bl_slot;
    V2M_ALLOC(bl_cnt, int, nb);
    V2M_ALLOC(bl_lab, uint16_t, (size_t)nb * V2M_BL);
    V2M_ALLOC(bl_slot, int, nb);
    lap("upload");
    k_brick_labels<<<(nb + 7) / 8, 256, 0, st>>>(L, d, R, bl_cnt, bl_lab, nb);
    V2M_TRY(cudaGetLastError());
    lap("brick labels");
    // 2. slots, in brick order
    int *cnt, *ofs;
    V2M_ALLOC(cnt, int, nb + 1);
    V2M_ALLOC(ofs, int, nb + 1);
    k_slot_count<<<(nb + 255) / 256, 256, 0, st>>>(bl_cnt, cnt, nb);
    V2M_TRY(cudaMemsetAsync(cnt + nb, 0, 4, st));
    size_t cub_bytes = 0;
    V2M_TRY(cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, cnt, ofs, nb + 1, st));
    void* cub_tmp = dalloc(cub_bytes);
    if (!cub_tmp) {
        return cudaErrorMemoryAllocation;
    }
    V2M_TRY(cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, cnt, ofs, nb + 1, st));
    int ns = 0;
    V2M_TRY(cudaMemcpyAsync(&ns, ofs + nb, 4, cudaMemcpyDeviceToHost, st));
    V2M_TRY(cudaStreamSynchronize(st));
    O.nlab = maxlabel + 1;
    O.nslots = ns;
    int* slot_brick;
    uint16_t* slot_label;
    float *phi, *phi2;
    V2M_ALLOC(slot_brick, int, ns);
    V2M_ALLOC(slot_label, uint16_t, ns);
    V2M_ALLOC(phi, float, (size_t)ns * V2M_SLOT);
    V2M_ALLOC(phi2, float, (size_t)ns * V2M_SLOT);
    k_slot_fill<<<(nb + 255) / 256, 256, 0, st>>>(cnt, ofs, bl_lab, bl_slot, slot_brick, slot_label, nb);
    auto smooth = [&](float sigma, int Rs, float* out) -> cudaError_t {
        if (ns == 0) {
            return cudaSuccess;
        }
        const int T = V2M_BS + 2 * Rs;
        const size_t smem = 2 * sizeof(float) * (size_t)T * T * T;
        V2M_TRY(cudaFuncSetAttribute(k_smooth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_smooth<<<ns, kSmoothThreads, smem, st>>>(L, d, slot_brick, slot_label, gauss_weights(sigma, Rs), Rs, out);
        return cudaGetLastError();
    };
    // 3. the wide (curvature) smoothing, for the sizing
    lap("slots");
    V2M_TRY(smooth(p.sigma_curv, Rc, phi));
    lap("curvature smoothing");
    DGrid g;
    std::memset(&g, 0, sizeof(g));
    g.nx = A.nx;
    g.ny = A.ny;
    g.nz = A.nz;
    g.nbx = d.nbx;
    g.nby = d.nby;
    g.nbz = d.nbz;
    g.vx = A.vs[0];
    g.vy = A.vs[1];
    g.vz = A.vs[2];
    g.L = L;
    g.bl_cnt = bl_cnt;
    g.bl_lab = bl_lab;
    g.bl_slot = bl_slot;
    g.phi = phi;
    // 4. sizing
    std::vector<float> hlab(std::max(1, maxlabel + 1), 0.0f);
    for (size_t l = 0; l < p.hlab.size() && l < hlab.size(); ++l) {
        hlab[l] = p.hlab[l];
    }
    float* dhlab;
    V2M_ALLOC(dhlab, float, hlab.size());
    V2M_TRY(cudaMemcpyAsync(dhlab, hlab.data(), 4 * hlab.size(), cudaMemcpyHostToDevice, st));
    float *h, *hn;
    V2M_ALLOC(h, float, nv);
    V2M_ALLOC(hn, float, nv);
    SizeArgs sa{ dhlab, (int)hlab.size(), hbase, hmin, hmax, p.K, hcurv };
    k_size<<<gs_blocks(nv, sms), 256, 0, st>>>(g, sa, h);
    V2M_TRY(cudaGetLastError());
    lap("sizing");
    // thickness (for the thin-layer sizing and blend): the peak on the device,
    // its erfinv on the host (the host's logf, as the reference)
    float* tv = nullptr;
    if (p.thick > 0.0f || p.sigma_thin > 0.0f) {
        V2M_ALLOC(tv, float, nv);
        k_thick_peak_bricks<<<(unsigned)((int64_t)g.nbx * g.nby * g.nbz), 256, 0, st>>>(g, tv);
        lap("thickness peak");
        // only the voxels with a peak in [0, 0.9999) need erfinv: listed on the
        // device, their peaks mapped on the host through the pinned staging
        // buffers, chunk by chunk, in place, and scattered back
        int* npick;
        int* pidx;
        float* pval;
        V2M_ALLOC(npick, int, 1);
        V2M_ALLOC(pidx, int, nv);
        V2M_ALLOC(pval, float, nv);
        V2M_TRY(cudaMemsetAsync(npick, 0, 4, st));
        k_thick_pick<<<gs_blocks(nv, sms), 256, 0, st>>>(tv, (int64_t)nv, npick, pidx, pval);
        V2M_TRY(cudaGetLastError());
        int hpick = 0;
        V2M_TRY(cudaMemcpyAsync(&hpick, npick, 4, cudaMemcpyDeviceToHost, st));
        V2M_TRY(cudaStreamSynchronize(st));
        const float sg = p.sigma_curv;
        const unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        V2M_TRY(staged_map(pval, pval, 4 * (size_t)hpick, st, [&](void* buf, size_t bytes, size_t) {
            float* t = static_cast<float*>(buf);
            const int64_t cnt = (int64_t)(bytes / 4);
            const unsigned nt = (unsigned)std::max<int64_t>(1, std::min<int64_t>(nth, cnt / 65536));
            auto run = [=](unsigned q) {
                const int64_t a = cnt * q / nt, b = cnt * (q + 1) / nt;
                for (int64_t v = a; v < b; ++v) {
                    t[v] = 2.8284271f * sg * erfinv_giles(t[v]);
                }
            };
            std::vector<std::thread> pool;
            for (unsigned q = 1; q < nt; ++q) {
                pool.emplace_back(run, q);
            }
            run(0);
            for (auto& th : pool) {
                th.join();
            }
        }));
        if (hpick > 0) {
            k_thick_put<<<gs_blocks(hpick, sms), 256, 0, st>>>(tv, pidx, pval, hpick);
            V2M_TRY(cudaGetLastError());
        }
        lap(("thickness erfinv (host, " + std::to_string(hpick) + " voxels)").c_str());
    }
    if (p.thick > 0.0f) {
        const float floor_mm = p.thin_floor * vmin;
        k_thick_size<<<gs_blocks(nv, sms), 256, 0, st>>>(tv, h, nv, floor_mm, vmin, p.thick);
        hmin = std::min(hmin, floor_mm);
    }
    // 5. the interface fields: sigma, then the thin-layer blend with sigma_thin
    V2M_TRY(smooth(p.sigma, Ri, phi));
    lap("interface smoothing");
    if (p.sigma_thin > 0.0f) {
        float* w = tv;   // (the thickness, consumed into the blend weight)
        float* wt;
        V2M_ALLOC(wt, float, nv);
        GaussW none{};
        for (int a = 0; a < 3; ++a) {
            k_axis_pass<<<gs_blocks(nv, sms), 256, 0, st>>>(w, wt, d, a, 2, 1, none);
            std::swap(w, wt);
        }
        k_smoothstep<<<gs_blocks(nv, sms), 256, 0, st>>>(w, nv, p.thin_lo, std::max(1e-3f, p.thin_hi - p.thin_lo));
        GaussW ker{};
        float ks = 0.0f;
        for (int dd = -3; dd <= 3; ++dd) {
            ker.w[dd + 3] = gauss_weight(dd, 1.0f);
            ks += ker.w[dd + 3];
        }
        for (int q = 0; q < 7; ++q) {
            ker.w[q] /= ks;
        }
        for (int a = 0; a < 3; ++a) {
            k_axis_pass<<<gs_blocks(nv, sms), 256, 0, st>>>(w, wt, d, a, 3, 0, ker);
            std::swap(w, wt);
        }
        const int Rt = std::min(6, std::max(1, (int)std::ceil(3.0f * p.sigma_thin)));
        V2M_TRY(smooth(p.sigma_thin, Rt, phi2));   // the sharp field
        if (ns > 0) {
            k_blend<<<gs_blocks((int64_t)ns * V2M_SLOT, sms), 256, 0, st>>>(slot_brick, w, phi, phi2, d, ns);
        }
        std::swap(phi, phi2);   // phi: the blend
        g.phi = phi;
        lap("thin-layer blend");
    }
    if (p.preserve > 0.0f) {
        k_preserve<<<gs_blocks(nv, sms), 256, 0, st>>>(g, phi, p.preserve);
    }
    V2M_TRY(cudaGetLastError());
    // 6. gradient limiting: Jacobi sweeps until nothing changes
    LimitW lw{};
    for (int n = 0; n < 27; ++n) {
        const int dx = n % 3 - 1, dy = (n / 3) % 3 - 1, dz = n / 9 - 1;
        const float ex = dx * A.vs[0], ey = dy * A.vs[1], ez = dz * A.vs[2];
        lw.d[n] = p.g * std::sqrt(ex * ex + ey * ey + ez * ez);
    }
    int* changed;
    V2M_ALLOC(changed, int, 1);
    O.limit_sweeps = 0;
    for (;;) {
        V2M_TRY(cudaMemsetAsync(changed, 0, 4, st));
        k_limit<<<gs_blocks(nv, sms), 256, 0, st>>>(h, hn, d, lw, changed);
        std::swap(h, hn);
        int c = 0;
        V2M_TRY(cudaMemcpyAsync(&c, changed, 4, cudaMemcpyDeviceToHost, st));
        V2M_TRY(cudaStreamSynchronize(st));
        ++O.limit_sweeps;
        if (!c) {
            break;
        }
    }
    lap("gradient limit");
    // 7. grades
    const std::vector<float> th = grade_thresholds(hmin, hmax);
    float* dth;
    V2M_ALLOC(dth, float, 255);
    V2M_TRY(cudaMemcpyAsync(dth, th.data(), 4 * 255, cudaMemcpyHostToDevice, st));
    uint8_t* grade;
    V2M_ALLOC(grade, uint8_t, nv);
    k_grade<<<gs_blocks(nv, sms), 256, 0, st>>>(h, nv, dth, grade);
    V2M_TRY(cudaGetLastError());
    lap("grades");
    O.hmin = hmin;
    O.hmax = hmax;
    O.L = L;
    O.bl_cnt = bl_cnt;
    O.bl_lab = bl_lab;
    O.bl_slot = bl_slot;
    O.phi = phi;
    O.h = h;
    O.grade = grade;
    O.overflow_bricks = 0;
    (void)err;
#undef V2M_TRY
#undef V2M_ALLOC
    return cudaSuccess;
}

}  // namespace v2m
