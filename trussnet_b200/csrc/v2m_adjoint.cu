// v2m_adjoint.cu -- the differentiable relaxation unroll and its hand-written
// adjoint, for sm_100a.
//
// The unroll is the relaxation step (v2m_force + the Jacobi branch of
// v2m_move, src/opencl/v2m_particle_body.cl:161-184, 898-900 of
// fangq/trussnet) with its discrete decisions frozen:
//   h_i  = H(x_i), trilinear in the sizing grid G (m0 x m1 x m2 values at
//          x = (a cs0, b cs1, c cs2), x fastest), the point clamped to G's box;
//   the lists are fixed (one list build before the unroll);
//   the active bars of every step are recorded on a tape (24-bit mask per node
//          and step) by the forward pass and replayed by the backward pass, so
//          the stiffness c_i = popcount(mask) is frozen (its jumps would make the
//          step discontinuous);
//   x_i' = x_i + dt sum_k f_k (x_i - x_j) / max(c_i, 1), f = (l0 - l) / l,
//          l0 = a_ij (h_i + h_j), a_ij = fsurf/2 (both non-INTERIOR) or fscale/2;
//          CORNER nodes stay.
// Optional taped constraints (v2m_unroll_set_constraints) freeze the trapped
// move's geometry the way the tape freezes the active bars: node i's increment
// is projected, x_i' = x_i + P_i (s_i F_i), with P_i = I - n n^T for an
// INTERFACE node (it glides in the tangent plane of its interface, unit normal
// n) or P_i = t t^T for a JUNCTION node (it moves along the junction line, unit
// direction t); the directions are constants of the unroll, taken once from the
// field at the starting positions. P_i is symmetric, so the reverse step's
// increment adjoint is mu_i = s_i P_i lam_i.
// Loss: sum over every list entry (i, j) of (l_ij / hm_ij - 1)^2, hm = (h_i+h_j)/2.
//
// Reverse mode with checkpoints every `ckpt` steps: the backward pass recomputes
// each segment's states (and sizes) from its checkpoint, then walks it
// backwards. Each node gathers the reverse terms of its own bars and of the bars
// pointing at it (the lists' transpose, built once), in a fixed order, in
// double; the sizing grid's 8-corner contributions are added as 64-bit fixed
// point (2^-32) with integer atomics, exact and associative. The gradients are
// bit-identical run to run.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/v2m_cuda.h"

namespace v2m_adj {

// an NVTX range over a call of the unroll's C ABI (header-only NVTX: a branch
// when no profiler is attached)
struct Trace {
    explicit Trace(const char* name) {
        nvtxRangePushA(name);
    }
    ~Trace() {
        nvtxRangePop();
    }
    Trace(const Trace&) = delete;
    Trace& operator=(const Trace&) = delete;
};

constexpr double kFix = 4294967296.0;   // 2^32
constexpr int kT = 256;

struct Dims {
    int m0, m1, m2;
    float cs0, cs1, cs2;
};

__device__ __forceinline__ void fx_add(unsigned long long* a, double v) {
    const long long q = __double2ll_rn(v * kFix);
    atomicAdd(a, (unsigned long long)q);
}

__device__ __forceinline__ double fx_get(unsigned long long a) {
    return (double)(long long)a / kFix;
}

// h at p, optionally its gradient, the 8 corner ids and weights
__device__ __forceinline__ float size_at(const Dims& D, const float* __restrict__ G, float px, float py, float pz,
                                         float* grad, int* idx, float* w) {
    const float ms[3] = { (float)(D.m0 - 1), (float)(D.m1 - 1), (float)(D.m2 - 1) };
    const float cs[3] = { D.cs0, D.cs1, D.cs2 };
    const int mm[3] = { D.m0, D.m1, D.m2 };
    const float p[3] = { px, py, pz };
    float f[3];
    int i0[3], inside[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        float v = p[d] / cs[d];
        inside[d] = v > 0.0f && v < ms[d];
        v = fminf(fmaxf(v, 0.0f), ms[d]);
        int a = (int)floorf(v);
        if (a > mm[d] - 2) {
            a = mm[d] > 1 ? mm[d] - 2 : 0;
        }
        i0[d] = a;
        f[d] = v - (float)a;
    }
    float c[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        int a = min(i0[0] + (k & 1), D.m0 - 1), b = min(i0[1] + ((k >> 1) & 1), D.m1 - 1),
            cc = min(i0[2] + (k >> 2), D.m2 - 1);
        const int id = a + D.m0 * (b + D.m1 * cc);
        c[k] = __ldg(G + id);
        if (idx) {
            idx[k] = id;
        }
    }
    float h = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float wk = ((k & 1) ? f[0] : 1.0f - f[0]) * (((k >> 1) & 1) ? f[1] : 1.0f - f[1]) *
                         ((k >> 2) ? f[2] : 1.0f - f[2]);
        if (w) {
            w[k] = wk;
        }
        h += wk * c[k];
    }
    if (grad) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            float g = 0.0f;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                float prod = ((k >> d) & 1) ? 1.0f : -1.0f;
#pragma unroll
                for (int e = 0; e < 3; ++e) {
                    if (e != d) {
                        prod *= ((k >> e) & 1) ? f[e] : 1.0f - f[e];
                    }
                }
                g += prod * c[k];
            }
            grad[d] = inside[d] ? g / cs[d] : 0.0f;
        }
    }
    return h;
}

// ---- packed node records ---------------------------------------------------------
// A state is float4 xh[i] = (x_i, h_i): one 16-byte load brings a neighbour's
// position and size. List entries carry the neighbour's "not INTERIOR" flag in
// bit 31 (ids are below 2^30), so no type byte is gathered per bar.

constexpr int kIdMask = 0x7FFFFFFF;

__device__ __forceinline__ float4 with_size(const Dims& D, const float* __restrict__ G, float x, float y, float z) {
    return make_float4(x, y, z, size_at(D, G, x, y, z, nullptr, nullptr, nullptr));
}

// xh = (x, H(x)) from [n, 3] positions
__global__ void k_pack_size(Dims D, const float* __restrict__ G, const float* __restrict__ x3, float4* __restrict__ xh,
                            int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        xh[i] = with_size(D, G, x3[3 * i], x3[3 * i + 1], x3[3 * i + 2]);
    }
}

__global__ void k_pack(const float* __restrict__ x3, float4* __restrict__ x4, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        x4[i] = make_float4(x3[3 * i], x3[3 * i + 1], x3[3 * i + 2], 0.0f);
    }
}

__global__ void k_unpack(const float4* __restrict__ x4, float* __restrict__ x3, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const float4 p = x4[i];
        x3[3 * i] = p.x;
        x3[3 * i + 1] = p.y;
        x3[3 * i + 2] = p.z;
    }
}

// P_i v in place: kind (d.w) 1 removes the component along d (a plane), kind 2
// keeps only it (a line), kind 0 leaves v.
__device__ __forceinline__ void project(const float4* __restrict__ dirs, int i, float& x, float& y, float& z) {
    if (!dirs) {
        return;
    }
    const float4 d = __ldg(dirs + i);
    if (d.w == 0.0f) {
        return;
    }
    const float t = x * d.x + y * d.y + z * d.z;
    if (d.w == 1.0f) {
        x = x - t * d.x;
        y = y - t * d.y;
        z = z - t * d.z;
    } else {
        x = t * d.x;
        y = t * d.y;
        z = t * d.z;
    }
}

// one step xh -> yh (the new state's sizes included); records (replay = 0) or
// replays the active-bar masks. A replay visits only the taped bars, in the same
// ascending slot order as the recording. Ids and positions are loaded kB at a
// time (independent gathers in flight); the bars are added in slot order.
constexpr int kB = 4;

__global__ void k_step(Dims D, const float* __restrict__ G, const float4* __restrict__ xh,
                       const int* __restrict__ nbrf, const uint8_t* __restrict__ nnb, const uint8_t* __restrict__ typ,
                       float fscale, float fsurf, float dt, const float4* __restrict__ dirs,
                       uint32_t* __restrict__ mask, int replay, float4* __restrict__ yh, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const float4 p = xh[i];
    const int ti = typ[i];
    if (ti == V2M_CORNER) {
        yh[i] = p;   // y = x, so H(y) = H(x)
        if (!replay) {
            mask[i] = 0u;
        }
        return;
    }
    const bool ni = ti != V2M_INTERIOR;
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    int act = 0;
    // the slots to visit: every listed one (recording) or the taped ones (replay)
    const int c = nnb[i];
    uint32_t todo = replay ? mask[i] : (c >= 32 ? 0xFFFFFFFFu : ((1u << c) - 1u));
    uint32_t bits = 0u;
    while (todo) {
        int ks[kB], es[kB];
        float4 qs[kB];
        int m = 0;
#pragma unroll
        for (int q = 0; q < kB; ++q) {
            ks[q] = -1;
            if (todo) {
                ks[q] = __ffs(todo) - 1;
                todo &= todo - 1u;
                m = q + 1;
            }
        }
#pragma unroll
        for (int q = 0; q < kB; ++q) {
            if (q < m) {
                es[q] = __ldg(nbrf + (size_t)ks[q] * n + i);
            }
        }
#pragma unroll
        for (int q = 0; q < kB; ++q) {
            if (q < m) {
                qs[q] = __ldg(xh + (es[q] & kIdMask));
            }
        }
#pragma unroll
        for (int q = 0; q < kB; ++q) {
            if (q < m) {
                const float ex = p.x - qs[q].x, ey = p.y - qs[q].y, ez = p.z - qs[q].z;
                const float l = sqrtf(ex * ex + ey * ey + ez * ez);
                const float l0 = ((ni && es[q] < 0) ? fsurf : fscale) * 0.5f * (p.w + qs[q].w);
                if (replay || (l < l0 && l > 0.0f)) {
                    bits |= 1u << ks[q];
                    const float f = (l0 - l) / l;
                    fx += f * ex;
                    fy += f * ey;
                    fz += f * ez;
                    ++act;
                }
            }
        }
    }
    if (!replay) {
        mask[i] = bits;
    }
    const float s = dt / (float)(act > 1 ? act : 1);
    float ix = s * fx, iy = s * fy, iz = s * fz;
    project(dirs, i, ix, iy, iz);
    yh[i] = with_size(D, G, p.x + ix, p.y + iy, p.z + iz);
}

__global__ void k_loss(const float4* __restrict__ xh, const int* __restrict__ nbrf, const uint8_t* __restrict__ nnb,
                       double* __restrict__ part, int n) {
    __shared__ double red[kT / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s = 0.0;
    if (i < n) {
        const float4 p = xh[i];
        for (int k = 0; k < nnb[i]; ++k) {
            const int j = __ldg(nbrf + (size_t)k * n + i) & kIdMask;
            const float4 q = __ldg(xh + j);
            const float ex = p.x - q.x, ey = p.y - q.y, ez = p.z - q.z;
            const float l = sqrtf(ex * ex + ey * ey + ez * ez);
            const float r = l / (0.5f * (p.w + q.w)) - 1.0f;
            s += (double)r * (double)r;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kT / 32; ++w) {
            t += red[w];
        }
        part[blockIdx.x] = t;
    }
}

// ---- gather form of the reverse passes --------------------------------------------
// The lists are frozen, so their transpose (for every node j, the entries
// (i, k) with nbr[i][k] = j, by ascending i then k) is built once. Each node then
// sums, in a fixed order and in double, the terms of its own bars and of the
// bars that point at it: no atomics, and the same bits on every run. Only the
// sizing grid's 8-corner scatter stays on fixed-point atomics.
//
// The reverse of step t reads, for every node, one 32-byte record: the state
// (x_t, h_t), mu = s_t P lam_{t+1} (s_t = dt / max(c_t, 1), the node's step scale,
// P its taped projection or I)
// and the step's taped mask. A bar pointing at j then costs one load of its
// source's record.
struct __align__(32) Rec {
    float4 xh;    // x_t, h_t
    float4 mub;   // mu (3 floats), the taped mask (bits)
};

__device__ __forceinline__ Rec make_rec(const float4& xh, const float4& lam, uint32_t bits, float dt,
                                        const float4* __restrict__ dirs, int i) {
    const int act = __popc(bits);
    const float s = dt / (float)(act > 1 ? act : 1);
    float mx = s * lam.x, my = s * lam.y, mz = s * lam.z;
    project(dirs, i, mx, my, mz);
    Rec r;
    r.xh = xh;
    r.mub = make_float4(mx, my, mz, __uint_as_float(bits));
    return r;
}

__global__ void k_rec(const float4* __restrict__ xh, const float4* __restrict__ lam, const uint32_t* __restrict__ mask,
                      float dt, const float4* __restrict__ dirs, Rec* __restrict__ rec, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        rec[i] = make_rec(xh[i], lam[i], mask[i], dt, dirs, i);
    }
}

// the size term of node j, in the same thread that summed dL/dh_j: lam_j +=
// dL/dh_j dH/dx_j, and the grid's 8 corners get dL/dh_j w (fixed-point atomics)
__device__ __forceinline__ void size_tail(const Dims& D, const float* __restrict__ G, const float4& p, double gh,
                                          double* l3, unsigned long long* __restrict__ gG) {
    const float g = (float)gh;
    if (g == 0.0f) {
        return;
    }
    float gr[3], w[8];
    int idx[8];
    size_at(D, G, p.x, p.y, p.z, gr, idx, w);
    for (int d = 0; d < 3; ++d) {
        l3[d] += (double)(g * gr[d]);
    }
    for (int k = 0; k < 8; ++k) {
        fx_add(gG + idx[k], (double)g * (double)w[k]);
    }
}

// d(loss)/dx and d(loss)/dh at x (loss = sum over list entries of (l/hm - 1)^2)
__global__ void k_loss_bwd_g(Dims D, const float* __restrict__ G, const float4* __restrict__ xh,
                             const int* __restrict__ nbrf, const uint8_t* __restrict__ nnb,
                             const uint8_t* __restrict__ indeg, const int* __restrict__ tsrcf, float gscale,
                             float4* __restrict__ lam, unsigned long long* __restrict__ gG, int n) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) {
        return;
    }
    const float4 pj = xh[j];
    double l3[3] = { 0.0, 0.0, 0.0 }, g = 0.0;
    // own entries (j -> k): + dl e/l
    for (int k = 0; k < nnb[j]; ++k) {
        const float4 q = __ldg(xh + (__ldg(nbrf + (size_t)k * n + j) & kIdMask));
        const float e[3] = { pj.x - q.x, pj.y - q.y, pj.z - q.z };
        const float l = sqrtf(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        const float hm = 0.5f * (pj.w + q.w);
        const float r = l / hm - 1.0f;
        const float dl = gscale * 2.0f * r / hm, dhm = -gscale * 2.0f * r * l / (hm * hm);
        for (int d = 0; d < 3; ++d) {
            l3[d] += (double)(dl * (e[d] / l));
        }
        g += 0.5 * (double)dhm;
    }
    // entries pointing at j (i -> j): - dl e/l
    const int cin = indeg[j];
    for (int t = 0; t < cin; ++t) {
        const float4 pi = __ldg(xh + (__ldg(tsrcf + (size_t)t * n + j) & kIdMask));
        const float e[3] = { pi.x - pj.x, pi.y - pj.y, pi.z - pj.z };
        const float l = sqrtf(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        const float hm = 0.5f * (pi.w + pj.w);
        const float r = l / hm - 1.0f;
        const float dl = gscale * 2.0f * r / hm, dhm = -gscale * 2.0f * r * l / (hm * hm);
        for (int d = 0; d < 3; ++d) {
            l3[d] -= (double)(dl * (e[d] / l));
        }
        g += 0.5 * (double)dhm;
    }
    size_tail(D, G, pj, g, l3, gG);
    lam[j] = make_float4((float)l3[0], (float)l3[1], (float)l3[2], 0.0f);
}

// one bar's reverse terms: v = (d phi / d e)^T mu and s = (e . mu) / l, with
// phi = f e, f = (l0 - l) / l (the hardware reciprocal square root of l^2, a
// few ulps: the reverse pass needs the FP64 gradient to 1e-4, not bit-parity)
__device__ __forceinline__ void bar_vjp(const float* e, float l0, float a, const float* mu, float* v, float* sa) {
    const float l2 = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
    const float il = rsqrtf(l2);
    const float l = l2 * il;
    const float f = (l0 - l) * il;
    const float em = e[0] * mu[0] + e[1] * mu[1] + e[2] * mu[2];
    const float c = -l0 * il * il * il * em;   // d f / d l * (e . mu) / l
    for (int d = 0; d < 3; ++d) {
        v[d] = f * mu[d] + c * e[d];
    }
    *sa = a * em * il;
}

// reverse of step t: lam_in = dL/dx_{t+1} -> lam_out = dL/dx_t (with the size
// term). kRoles threads per node, in different warps of the block: for the
// block's kBwdNodes nodes, role 0 sums each node's own taped bars and roles
// 1 .. kRoles-1 consecutive parts of the taped bars pointing at it, each in
// its fixed order (in float: the node's result is a float) with kB gathers in
// flight (kRoles = 2: one thread for the own bars, one for the incoming ones;
// more roles only duplicate the per-node loads). The other roles hand their
// sums over through shared memory; role 0
// adds them in role order, then the size term. When step t - 1 follows in the
// same segment, it also writes node j's record for it (state x_{t-1},
// mask_{t-1}, mu from lam_out).
constexpr int kRoles = 2;
constexpr int kBwdNodes = kT / kRoles;

__global__ void __launch_bounds__(kT, 4) k_step_bwd_g(Dims D, const float* __restrict__ G, const Rec* __restrict__ rec,
                             const float4* __restrict__ lam_in, const int* __restrict__ nbrf,
                             const uint8_t* __restrict__ typ, float fscale, float fsurf, float dt,
                             const float4* __restrict__ dirs, const uint8_t* __restrict__ indeg, const int* __restrict__ tsrcf,
                             const uint8_t* __restrict__ tslot, float4* __restrict__ lam_out,
                             const float4* __restrict__ xh_prev, const uint32_t* __restrict__ mask_prev,
                             Rec* __restrict__ rec_prev, unsigned long long* __restrict__ gG, int n) {
    __shared__ float hand[kRoles - 1][4][kBwdNodes];
    const int slot = threadIdx.x % kBwdNodes;
    const int role = threadIdx.x / kBwdNodes;   // warp-uniform
    const int j = blockIdx.x * kBwdNodes + slot;
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, ag = 0.0f;
    Rec rj;
    rj.xh = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    bool nj = false;
    if (j < n) {
        rj = rec[j];
        nj = typ[j] != V2M_INTERIOR;
        const float4 pj = rj.xh;
        if (role == 0) {
            // own bars (a CORNER's mask is empty): + v
            const float mu[3] = { rj.mub.x, rj.mub.y, rj.mub.z };
            uint32_t todo = __float_as_uint(rj.mub.w);
            while (todo) {
                int es[kB];
                float4 qs[kB];
                int ks[kB], m = 0;
#pragma unroll
                for (int q = 0; q < kB; ++q) {
                    ks[q] = 0;
                    if (todo) {
                        ks[q] = __ffs(todo) - 1;
                        todo &= todo - 1u;
                        m = q + 1;
                    }
                }
#pragma unroll
                for (int q = 0; q < kB; ++q) {
                    if (q < m) {
                        es[q] = __ldg(nbrf + (size_t)ks[q] * n + j);
                    }
                }
#pragma unroll
                for (int q = 0; q < kB; ++q) {
                    if (q < m) {
                        qs[q] = __ldg(&rec[es[q] & kIdMask].xh);
                    }
                }
#pragma unroll
                for (int q = 0; q < kB; ++q) {
                    if (q < m) {
                        const float e[3] = { pj.x - qs[q].x, pj.y - qs[q].y, pj.z - qs[q].z };
                        const float a = ((nj && es[q] < 0) ? fsurf : fscale) * 0.5f;
                        const float l0 = a * (pj.w + qs[q].w);
                        float v[3], sa;
                        bar_vjp(e, l0, a, mu, v, &sa);
                        a0 += v[0];
                        a1 += v[1];
                        a2 += v[2];
                        ag += sa;
                    }
                }
            }
        } else {
            // the role's part of the bars pointing at j: - v
            const int cin = indeg[j];
            const int part = (cin + kRoles - 2) / (kRoles - 1);
            const int t0 = (role - 1) * part, t1 = min(cin, t0 + part);
            for (int t = t0; t < t1; t += kB) {
                int es[kB], ks[kB];
                float4 mb[kB];
#pragma unroll
                for (int q = 0; q < kB; ++q) {
                    if (t + q < t1) {
                        es[q] = __ldg(tsrcf + (size_t)(t + q) * n + j);
                        ks[q] = __ldg(tslot + (size_t)(t + q) * n + j);
                    }
                }
#pragma unroll
                for (int q = 0; q < kB; ++q) {
                    if (t + q < t1) {
                        mb[q] = __ldg(reinterpret_cast<const float4*>(rec + (es[q] & kIdMask)) + 1);
                    }
                }
#pragma unroll
                for (int q = 0; q < kB; ++q) {
                    if (t + q < t1 && ((__float_as_uint(mb[q].w) >> ks[q]) & 1u)) {
                        const float4 pi = __ldg(reinterpret_cast<const float4*>(rec + (es[q] & kIdMask)));
                        const float mu[3] = { mb[q].x, mb[q].y, mb[q].z };
                        const float e[3] = { pi.x - pj.x, pi.y - pj.y, pi.z - pj.z };
                        const float a = ((es[q] < 0 && nj) ? fsurf : fscale) * 0.5f;
                        const float l0 = a * (pi.w + pj.w);
                        float v[3], sa;
                        bar_vjp(e, l0, a, mu, v, &sa);
                        a0 -= v[0];
                        a1 -= v[1];
                        a2 -= v[2];
                        ag += sa;
                    }
                }
            }
        }
    }
    if (role > 0) {
        hand[role - 1][0][slot] = a0;
        hand[role - 1][1][slot] = a1;
        hand[role - 1][2][slot] = a2;
        hand[role - 1][3][slot] = ag;
    }
    __syncthreads();
    if (j >= n || role > 0) {
        return;
    }
    double s0 = a0, s1 = a1, s2 = a2, sg = ag;
#pragma unroll
    for (int r = 0; r < kRoles - 1; ++r) {
        s0 += (double)hand[r][0][slot];
        s1 += (double)hand[r][1][slot];
        s2 += (double)hand[r][2][slot];
        sg += (double)hand[r][3][slot];
    }
    const float4 lj = lam_in[j];
    double l3[3] = { (double)lj.x + s0, (double)lj.y + s1, (double)lj.z + s2 };
    size_tail(D, G, rj.xh, sg, l3, gG);
    const float4 lo = make_float4((float)l3[0], (float)l3[1], (float)l3[2], 0.0f);
    lam_out[j] = lo;
    if (rec_prev) {
        rec_prev[j] = make_rec(xh_prev[j], lo, mask_prev[j], dt, dirs, j);
    }
}

__global__ void k_add(float* __restrict__ a, const float* __restrict__ b, int m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        a[i] += b[i];
    }
}

__global__ void k_fix_to_float(unsigned long long* __restrict__ a, float* __restrict__ out, int m, int clear) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        out[i] = (float)fx_get(a[i]);
        if (clear) {
            a[i] = 0ull;
        }
    }
}

// row-major [n][K] lists -> slot-major, each entry flagged (bit 31) when its node is not INTERIOR
__global__ void k_lists(const int* __restrict__ rowmajor, const int* __restrict__ cnt, const uint8_t* __restrict__ typ,
                        int* __restrict__ slot, uint8_t* __restrict__ nnb, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * V2M_K) {
        return;
    }
    const int i = t / V2M_K, k = t % V2M_K;
    const int c = cnt[i];
    const int j = k < c ? rowmajor[t] : i;
    slot[(size_t)k * n + i] = j | (typ[j] != V2M_INTERIOR ? (int)0x80000000u : 0);
    if (k == 0) {
        nnb[i] = (uint8_t)c;
    }
}

}  // namespace v2m_adj

using namespace v2m_adj;

struct v2m_unroll {
    int device = 0, n = 0, K = 0, ckpt = 10, nck = 0;
    Dims D{};
    float fscale = 1.2f, fsurf = 1.0f, dt = 0.2f;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;  // the backward pass's segment recomputation
    std::vector<cudaEvent_t> seg_ready, seg_done;   // per segment: recomputed (stream2), walked back (stream)
    int* nbr = nullptr;              // slot-major lists, bit 31 = the neighbour is not INTERIOR
    uint8_t* nnb = nullptr;
    uint8_t* typ = nullptr;
    float4* dirs = nullptr;          // taped constraints (direction, kind), or null
    float4* dirs_buf = nullptr;      // their buffer (kept when they are cleared)
    uint32_t* tape = nullptr;        // K x n
    float4* ck = nullptr;            // nck checkpoints x n
    float4* seg = nullptr;           // (ckpt + 1) x n segment states (x, h)
    float4* seg2 = nullptr;          // a second segment buffer (the backward pass alternates)
    float4* lamf = nullptr;
    unsigned long long* gG = nullptr;
    double* part = nullptr;
    // transpose of the lists, slot-major like nbr: node j's t-th incoming entry
    // (by ascending i, then k) at [t * n + j], t < indeg[j] <= maxin
    int maxin = 0;
    uint8_t* indeg = nullptr;
    int* tsrc = nullptr;             // its source node i (bit 31: i is not INTERIOR)
    uint8_t* tslot = nullptr;        // its slot k in i's list
    float4* lamb = nullptr;          // second adjoint buffer
    Rec* rec = nullptr;              // 2 x n reverse-step records (double buffer)
    int have_tape = 0;
    float ms_fwd = 0.0f, ms_bwd = 0.0f;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<void*> allocs;
    template <typename T>
    T* alloc(size_t count) {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(count * sizeof(T), 16)) != cudaSuccess) {
            throw std::runtime_error("cudaMalloc failed");
        }
        allocs.push_back(p);
        return (T*)p;
    }
    ~v2m_unroll() {
        for (void* p : allocs) {
            cudaFree(p);
        }
        if (e0) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
        }
        for (cudaEvent_t e : seg_ready) {
            cudaEventDestroy(e);
        }
        for (cudaEvent_t e : seg_done) {
            cudaEventDestroy(e);
        }
        if (stream2) {
            cudaStreamDestroy(stream2);
        }
        if (stream) {
            cudaStreamDestroy(stream);
        }
    }
};

namespace {

thread_local std::string g_uerr;

void uck(cudaError_t e, const char* where) {
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string(where) + ": CUDA error " + std::to_string((int)e) + " (" +
                                 cudaGetErrorString(e) + ")");
    }
}

template <typename F>
int uguard(F&& f) {
    try {
        f();
        return V2M_OK;
    } catch (const std::invalid_argument& e) {
        g_uerr = e.what();
        return V2M_ERR_ARG;
    } catch (const std::exception& e) {
        g_uerr = e.what();
        return V2M_ERR_CUDA;
    }
}

unsigned blocks(int n) {
    return (unsigned)((n + kT - 1) / kT);
}

// forward over steps [t0, t1) from the state xh, writing state t + 1 to seg[t - t0 + 1]
void run_steps(v2m_unroll* u, const float* G, const float4* xh, int t0, int t1, float4* seg, int replay,
               cudaStream_t st) {
    const int n = u->n;
    const float4* cur = xh;
    for (int t = t0; t < t1; ++t) {
        float4* nxt = seg + (size_t)(t - t0 + 1) * n;
        k_step<<<blocks(n), kT, 0, st>>>(u->D, G, cur, u->nbr, u->nnb, u->typ, u->fscale, u->fsurf, u->dt, u->dirs,
                                         u->tape + (size_t)t * n, replay, nxt, n);
        cur = nxt;
    }
}

}  // namespace

extern "C" {

const char* v2m_unroll_last_error(void) {
    return g_uerr.c_str();
}

int v2m_unroll_create(int64_t n, const int32_t* nbr, const int32_t* nnb, const uint8_t* typ, const int32_t* m,
                      const float* cs, float fscale, float fsurf, float dt, int K, int ckpt, int device,
                      v2m_unroll** out) {
    v2m_adj::Trace trace("v2m_unroll_create");
    return uguard([&] {
        if (!out || n < 1 || n > (1 << 29) || !nbr || !nnb || !typ || !m || !cs || K < 1 || ckpt < 1) {
            throw std::invalid_argument("bad argument");
        }
        if (m[0] < 1 || m[1] < 1 || m[2] < 1 || !(cs[0] > 0 && cs[1] > 0 && cs[2] > 0)) {
            throw std::invalid_argument("bad sizing grid");
        }
        for (int64_t i = 0; i < n; ++i) {
            if (nnb[i] < 0 || nnb[i] > V2M_K || typ[i] > V2M_CORNER) {
                throw std::invalid_argument("list length or type out of range");
            }
            for (int k = 0; k < nnb[i]; ++k) {
                if (nbr[i * V2M_K + k] < 0 || nbr[i * V2M_K + k] >= n) {
                    throw std::invalid_argument("neighbour id out of range");
                }
            }
        }
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
            cudaGetLastError();
            throw std::runtime_error("no CUDA device available");
        }
        const int dev = device < 0 ? 0 : device;
        uck(cudaSetDevice(dev), "cudaSetDevice");
        v2m_unroll* u = new v2m_unroll();
        try {
            u->device = dev;
            u->n = (int)n;
            u->K = K;
            u->ckpt = ckpt;
            u->nck = (K + ckpt - 1) / ckpt;
            u->D = Dims{ m[0], m[1], m[2], cs[0], cs[1], cs[2] };
            u->fscale = fscale;
            u->fsurf = fsurf;
            u->dt = dt;
            uck(cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking), "stream");
            uck(cudaStreamCreateWithFlags(&u->stream2, cudaStreamNonBlocking), "stream");
            u->seg_ready.assign(u->nck, nullptr);
            u->seg_done.assign(u->nck, nullptr);
            for (int c = 0; c < u->nck; ++c) {
                uck(cudaEventCreateWithFlags(&u->seg_ready[c], cudaEventDisableTiming), "event");
                uck(cudaEventCreateWithFlags(&u->seg_done[c], cudaEventDisableTiming), "event");
            }
            uck(cudaEventCreate(&u->e0), "event");
            uck(cudaEventCreate(&u->e1), "event");
            const size_t nn = (size_t)n;
            u->nbr = u->alloc<int>(nn * V2M_K);
            u->nnb = u->alloc<uint8_t>(nn);
            u->typ = u->alloc<uint8_t>(nn);
            u->tape = u->alloc<uint32_t>(nn * K);
            u->ck = u->alloc<float4>(nn * u->nck);
            u->seg = u->alloc<float4>(nn * (ckpt + 1));
            u->seg2 = u->alloc<float4>(nn * (ckpt + 1));
            u->lamf = u->alloc<float4>(nn);
            u->gG = u->alloc<unsigned long long>((size_t)m[0] * m[1] * m[2]);
            u->part = u->alloc<double>(nn / kT + 1);
            u->lamb = u->alloc<float4>(nn);
            u->rec = u->alloc<Rec>(2 * nn);
            // the transpose of the lists: incoming entries of every node, by (i, k)
            std::vector<int> deg(nn, 0);
            for (int64_t i = 0; i < n; ++i) {
                for (int k = 0; k < nnb[i]; ++k) {
                    ++deg[nbr[i * V2M_K + k]];
                }
            }
            const int maxin = std::max(1, *std::max_element(deg.begin(), deg.end()));
            if (maxin > 255) {
                throw std::invalid_argument("a node is in more than 255 lists");
            }
            u->maxin = maxin;
            std::vector<int> tsrc(nn * maxin, 0);
            std::vector<uint8_t> tslot(nn * maxin, 0), indeg(nn, 0);
            for (int64_t i = 0; i < n; ++i) {
                for (int k = 0; k < nnb[i]; ++k) {
                    const int j = nbr[i * V2M_K + k];
                    const size_t e = (size_t)indeg[j] * nn + j;
                    tsrc[e] = (int)i | (typ[i] != V2M_INTERIOR ? (int)0x80000000u : 0);
                    tslot[e] = (uint8_t)k;
                    ++indeg[j];
                }
            }
            u->indeg = u->alloc<uint8_t>(nn);
            u->tsrc = u->alloc<int>(tsrc.size());
            u->tslot = u->alloc<uint8_t>(tslot.size());
            uck(cudaMemcpy(u->indeg, indeg.data(), nn, cudaMemcpyHostToDevice), "upload");
            uck(cudaMemcpy(u->tsrc, tsrc.data(), 4 * tsrc.size(), cudaMemcpyHostToDevice), "upload");
            uck(cudaMemcpy(u->tslot, tslot.data(), tslot.size(), cudaMemcpyHostToDevice), "upload");
            int* tmp = u->alloc<int>(nn * V2M_K + nn);
            uck(cudaMemcpyAsync(tmp, nbr, 4 * nn * V2M_K, cudaMemcpyHostToDevice, u->stream), "upload");
            uck(cudaMemcpyAsync(tmp + nn * V2M_K, nnb, 4 * nn, cudaMemcpyHostToDevice, u->stream), "upload");
            uck(cudaMemcpyAsync(u->typ, typ, nn, cudaMemcpyHostToDevice, u->stream), "upload");
            k_lists<<<(unsigned)((nn * V2M_K + kT - 1) / kT), kT, 0, u->stream>>>(tmp, tmp + nn * V2M_K, u->typ, u->nbr,
                                                                               u->nnb, (int)n);
            uck(cudaMemsetAsync(u->gG, 0, 8 * (size_t)m[0] * m[1] * m[2], u->stream), "memset");
            uck(cudaGetLastError(), "launch");
            uck(cudaStreamSynchronize(u->stream), "synchronize");
        } catch (...) {
            delete u;
            throw;
        }
        *out = u;
    });
}

int v2m_unroll_destroy(v2m_unroll* u) {
    return uguard([&] {
        if (u) {
            cudaSetDevice(u->device);
            cudaStreamSynchronize(u->stream);
            delete u;
        }
    });
}

int v2m_unroll_forward(v2m_unroll* u, const float* x0, const float* G, float* xK, int replay) {
    v2m_adj::Trace trace("v2m_unroll_forward");
    return uguard([&] {
        if (!u || !x0 || !G || !xK) {
            throw std::invalid_argument("bad argument");
        }
        if (replay && !u->have_tape) {
            throw std::invalid_argument("no tape recorded yet");
        }
        uck(cudaSetDevice(u->device), "cudaSetDevice");
        const int n = u->n;
        uck(cudaEventRecord(u->e0, u->stream), "event");
        k_pack_size<<<blocks(n), kT, 0, u->stream>>>(u->D, G, x0, u->seg, n);
        for (int c = 0; c < u->nck; ++c) {
            const int t0 = c * u->ckpt, t1 = std::min(u->K, t0 + u->ckpt);
            uck(cudaMemcpyAsync(u->ck + (size_t)c * n, u->seg, 16 * (size_t)n, cudaMemcpyDeviceToDevice, u->stream),
                "checkpoint");
            run_steps(u, G, u->ck + (size_t)c * n, t0, t1, u->seg, replay, u->stream);
            uck(cudaMemcpyAsync(u->seg, u->seg + (size_t)(t1 - t0) * n, 16 * (size_t)n, cudaMemcpyDeviceToDevice,
                                u->stream), "segment");
        }
        k_unpack<<<blocks(n), kT, 0, u->stream>>>(u->seg, xK, n);
        uck(cudaEventRecord(u->e1, u->stream), "event");
        uck(cudaGetLastError(), "launch");
        uck(cudaStreamSynchronize(u->stream), "synchronize");
        uck(cudaEventElapsedTime(&u->ms_fwd, u->e0, u->e1), "elapsed");
        u->have_tape = 1;
    });
}

int v2m_unroll_loss(v2m_unroll* u, const float* x, const float* G, double* loss) {
    return uguard([&] {
        if (!u || !x || !G || !loss) {
            throw std::invalid_argument("bad argument");
        }
        uck(cudaSetDevice(u->device), "cudaSetDevice");
        const int n = u->n;
        float4* xh = u->lamf;   // scratch
        k_pack_size<<<blocks(n), kT, 0, u->stream>>>(u->D, G, x, xh, n);
        k_loss<<<blocks(n), kT, 0, u->stream>>>(xh, u->nbr, u->nnb, u->part, n);
        std::vector<double> part(blocks(n));
        uck(cudaMemcpyAsync(part.data(), u->part, 8 * part.size(), cudaMemcpyDeviceToHost, u->stream), "read");
        uck(cudaStreamSynchronize(u->stream), "synchronize");
        double s = 0.0;
        for (double p : part) {
            s += p;
        }
        *loss = s;
    });
}

// gx = gscale * dLoss/dx at x; gG += gscale * dLoss/dG (gG overwritten when accumulate == 0)
int v2m_unroll_loss_backward(v2m_unroll* u, const float* x, const float* G, float gscale, float* gx, float* gG,
                             int accumulate) {
    v2m_adj::Trace trace("v2m_unroll_loss_backward");
    return uguard([&] {
        if (!u || !x || !G || !gx || !gG) {
            throw std::invalid_argument("bad argument");
        }
        uck(cudaSetDevice(u->device), "cudaSetDevice");
        const int n = u->n, mg = u->D.m0 * u->D.m1 * u->D.m2;
        float4* xh = u->seg;
        k_pack_size<<<blocks(n), kT, 0, u->stream>>>(u->D, G, x, xh, n);
        if (!accumulate) {
            uck(cudaMemsetAsync(u->gG, 0, 8 * (size_t)mg, u->stream), "memset");
        }
        k_loss_bwd_g<<<blocks(n), kT, 0, u->stream>>>(u->D, G, xh, u->nbr, u->nnb, u->indeg, u->tsrc, gscale,
                                                      u->lamf, u->gG, n);
        k_unpack<<<blocks(n), kT, 0, u->stream>>>(u->lamf, gx, n);
        k_fix_to_float<<<blocks(mg), kT, 0, u->stream>>>(u->gG, gG, mg, 0);
        uck(cudaGetLastError(), "launch");
        uck(cudaStreamSynchronize(u->stream), "synchronize");
    });
}

// reverse of the last forward pass: gxK = dL/dxK in, gx0 = dL/dx0 out,
// gG (overwritten) = dL/dG through the steps, plus gG_in (may be null) from other terms
int v2m_unroll_backward(v2m_unroll* u, const float* G, const float* gxK, float* gx0, float* gG, const float* gG_in) {
    v2m_adj::Trace trace("v2m_unroll_backward");
    return uguard([&] {
        if (!u || !G || !gxK || !gx0 || !gG) {
            throw std::invalid_argument("bad argument");
        }
        if (!u->have_tape) {
            throw std::invalid_argument("backward before forward");
        }
        uck(cudaSetDevice(u->device), "cudaSetDevice");
        const int n = u->n, mg = u->D.m0 * u->D.m1 * u->D.m2;
        uck(cudaEventRecord(u->e0, u->stream), "event");
        uck(cudaMemsetAsync(u->gG, 0, 8 * (size_t)mg, u->stream), "memset");
        k_pack<<<blocks(n), kT, 0, u->stream>>>(gxK, u->lamf, n);
        // Segment c's states are recomputed from its checkpoint on stream2 into
        // buffer c % 2 while stream walks segment c + 1 back from the other buffer:
        // the recomputation waits for the walk that last used its buffer, the
        // walk for its segment's recomputation.
        float4* buf[2] = { u->seg, u->seg2 };
        uck(cudaStreamWaitEvent(u->stream2, u->e0, 0), "wait");
        auto recompute = [&](int c) {
            const int t0 = c * u->ckpt, t1 = std::min(u->K, t0 + u->ckpt);
            float4* b = buf[c & 1];
            if (c + 2 < u->nck) {
                uck(cudaStreamWaitEvent(u->stream2, u->seg_done[c + 2], 0), "wait");
            }
            uck(cudaMemcpyAsync(b, u->ck + (size_t)c * n, 16 * (size_t)n, cudaMemcpyDeviceToDevice, u->stream2),
                "segment");
            run_steps(u, G, b, t0, t1 - 1, b, 1, u->stream2);
            uck(cudaEventRecord(u->seg_ready[c], u->stream2), "event");
        };
        recompute(u->nck - 1);
        for (int c = u->nck - 1; c >= 0; --c) {
            if (c > 0) {
                recompute(c - 1);
            }
            const int t0 = c * u->ckpt, t1 = std::min(u->K, t0 + u->ckpt);
            float4* b = buf[c & 1];
            uck(cudaStreamWaitEvent(u->stream, u->seg_ready[c], 0), "wait");
            Rec* rc = u->rec;
            Rec* rp = u->rec + n;
            k_rec<<<blocks(n), kT, 0, u->stream>>>(b + (size_t)(t1 - 1 - t0) * n, u->lamf,
                                                   u->tape + (size_t)(t1 - 1) * n, u->dt, u->dirs, rc, n);
            for (int t = t1 - 1; t >= t0; --t) {
                const bool more = t > t0;
                k_step_bwd_g<<<(unsigned)((n + kBwdNodes - 1) / kBwdNodes), kT, 0, u->stream>>>(
                    u->D, G, rc, u->lamf, u->nbr, u->typ, u->fscale, u->fsurf, u->dt, u->dirs, u->indeg, u->tsrc,
                    u->tslot,
                    u->lamb, more ? b + (size_t)(t - 1 - t0) * n : nullptr,
                    more ? u->tape + (size_t)(t - 1) * n : nullptr, more ? rp : nullptr, u->gG, n);
                std::swap(u->lamf, u->lamb);
                std::swap(rc, rp);
            }
            uck(cudaEventRecord(u->seg_done[c], u->stream), "event");
        }
        k_unpack<<<blocks(n), kT, 0, u->stream>>>(u->lamf, gx0, n);
        k_fix_to_float<<<blocks(mg), kT, 0, u->stream>>>(u->gG, gG, mg, 1);
        uck(cudaEventRecord(u->e1, u->stream), "event");
        uck(cudaGetLastError(), "launch");
        uck(cudaStreamSynchronize(u->stream), "synchronize");
        uck(cudaEventElapsedTime(&u->ms_bwd, u->e0, u->e1), "elapsed");
        if (gG_in) {
            k_add<<<blocks(mg), kT, 0, u->stream>>>(gG, gG_in, mg);
            uck(cudaGetLastError(), "launch");
            uck(cudaStreamSynchronize(u->stream), "synchronize");
        }
    });
}

// Taped constraints from dirs (host, float [3n]; null clears them): an INTERFACE
// node's unit interface normal, a JUNCTION node's unit junction-line direction
// (V2M_ARR_DIRS of a session gives both); entries of other types are ignored,
// and a zero direction leaves its node free. Directions are normalised here.
// Invalidates the tape: the next forward pass records a new one.
int v2m_unroll_set_constraints(v2m_unroll* u, const float* dirs) {
    return uguard([&] {
        if (!u) {
            throw std::invalid_argument("bad argument");
        }
        uck(cudaSetDevice(u->device), "cudaSetDevice");
        uck(cudaStreamSynchronize(u->stream), "synchronize");
        if (!dirs) {
            u->dirs = nullptr;
            u->have_tape = 0;
            return;
        }
        const size_t nn = (size_t)u->n;
        std::vector<uint8_t> typ(nn);
        uck(cudaMemcpy(typ.data(), u->typ, nn, cudaMemcpyDeviceToHost), "read types");
        std::vector<float4> h(nn);
        for (size_t i = 0; i < nn; ++i) {
            const float x = dirs[3 * i], y = dirs[3 * i + 1], z = dirs[3 * i + 2];
            const float kind = typ[i] == V2M_INTERFACE ? 1.0f : (typ[i] == V2M_JUNCTION ? 2.0f : 0.0f);
            const double r = std::sqrt((double)x * x + (double)y * y + (double)z * z);
            if (!std::isfinite(r)) {
                throw std::invalid_argument("constraint direction not finite");
            }
            h[i] = (kind == 0.0f || r == 0.0) ? make_float4(0.0f, 0.0f, 0.0f, 0.0f)
                                              : make_float4((float)(x / r), (float)(y / r), (float)(z / r), kind);
        }
        if (!u->dirs_buf) {
            u->dirs_buf = u->alloc<float4>(nn);
        }
        uck(cudaMemcpy(u->dirs_buf, h.data(), 16 * nn, cudaMemcpyHostToDevice), "upload");
        u->dirs = u->dirs_buf;
        u->have_tape = 0;
    });
}

int v2m_unroll_tape(v2m_unroll* u, uint32_t* host, int64_t count) {
    return uguard([&] {
        if (!u || !host || count < (int64_t)u->n * u->K) {
            throw std::invalid_argument("bad argument");
        }
        uck(cudaSetDevice(u->device), "cudaSetDevice");
        uck(cudaMemcpy(host, u->tape, 4 * (size_t)u->n * u->K, cudaMemcpyDeviceToHost), "read tape");
    });
}

// device milliseconds of the last forward (all K steps) and backward passes
int v2m_unroll_timing(v2m_unroll* u, float* ms_forward, float* ms_backward) {
    return uguard([&] {
        if (!u) {
            throw std::invalid_argument("bad argument");
        }
        if (ms_forward) {
            *ms_forward = u->ms_fwd;
        }
        if (ms_backward) {
            *ms_backward = u->ms_bwd;
        }
    });
}

}  // extern "C"
