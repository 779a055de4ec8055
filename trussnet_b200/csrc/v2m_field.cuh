// v2m_field.cuh -- device-side point queries of the relaxation and the per-node
// move, for sm_100a.
//
// These restate, for one CUDA thread per node, what the reference evaluates per
// node in src/opencl/v2m_grid_body.cl:110-200 (brick-sparse phi lookups),
// src/opencl/v2m_seed_body.cl:33-420 (labels near a point, owner label, psi and
// its gradient, bracketed projections) and src/opencl/v2m_particle_body.cl
// (crossing, glide, third label, valid branch, voxel trapping, move_step, move)
// of fangq/trussnet. Every floating-point expression keeps the reference's
// operand order; the library is compiled with --fmad=false and IEEE div/sqrt, so
// a node's result is the reference CPU's bit for bit.
//
// Register-resident label lists: a brick's 16 labels are one 32-byte load kept
// as 8 registers (LabList), so the label loops do not spill to local memory.
#pragma once

#include <climits>
#include <cstdint>

#include "v2m_sdf.cuh"
#include "v2m_types.cuh"

namespace v2m {
// (internal linkage: the header is compiled into more than one source)
namespace {

// ---- grid lookups ---------------------------------------------------------------
__device__ __forceinline__ int label_at(const DGrid& g, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= g.nx || j >= g.ny || k >= g.nz) {
        return 0;
    }
    return g.L[i + (size_t)g.nx * (j + (size_t)g.ny * k)];
}

__device__ __forceinline__ int brick_index(const DGrid& g, int i, int j, int k) {
    return (i >> 3) + g.nbx * ((j >> 3) + g.nby * (k >> 3));
}

// The 16 labels of a brick as 8 packed registers.
struct LabList {
    uint32_t w[8];
    __device__ __forceinline__ int get(int s) const {
        return (int)((w[s >> 1] >> ((s & 1) * 16)) & 0xFFFFu);
    }
};

__device__ __forceinline__ LabList load_labels(const DGrid& g, int b) {
    const uint4* p = reinterpret_cast<const uint4*>(g.bl_lab + (size_t)b * V2M_BL);
    const uint4 a = __ldg(p), c = __ldg(p + 1);
    LabList r;
    r.w[0] = a.x; r.w[1] = a.y; r.w[2] = a.z; r.w[3] = a.w;
    r.w[4] = c.x; r.w[5] = c.y; r.w[6] = c.z; r.w[7] = c.w;
    return r;
}

// Slot of label l in brick b (-1: uniform brick or l not listed); *has = listed.
// (src/opencl/v2m_grid_body.cl:122-134) The 16 labels are compared two at a
// time with 16-bit SIMD compares; the first listed match wins, as in the loop.
__device__ __forceinline__ int slot_lookup(const DGrid& g, int b, int l, int* has) {
    const int n = __ldg(g.bl_cnt + b);
    const LabList ll = load_labels(g, b);
    const unsigned pat = (unsigned)(l & 0xFFFF) * 0x00010001u;
    unsigned bits = 0u;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        const unsigned m = __vcmpeq2(ll.w[w], pat);
        bits |= ((m & 1u) | ((m >> 15) & 2u)) << (2 * w);
    }
    const int nn = n < V2M_BL ? n : V2M_BL;
    bits &= nn >= 32 ? 0xFFFFFFFFu : ((1u << nn) - 1u);
    if (!bits) {
        *has = 0;
        return -1;
    }
    *has = 1;
    const int idx = __ffs(bits) - 1;
    const int first = __ldg(g.bl_slot + b);
    if (kChecked && first >= 0 && (int64_t)first + idx >= g.nslots) {
        check_fail(g.chk, 20, b);   // a brick's slot beyond the phi array
        return -1;
    }
    return first < 0 ? -1 : first + idx;
}

// phi_l at voxel (i,j,k) (src/opencl/v2m_grid_body.cl:137-153)
__device__ __noinline__ float phi_voxel(const DGrid& g, int l, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= g.nx || j >= g.ny || k >= g.nz) {
        return l == 0 ? 1.0f : 0.0f;
    }
    int has;
    const int s = slot_lookup(g, brick_index(g, i, j, k), l, &has);
    if (s < 0) {
        return (has && g.L[i + (size_t)g.nx * (j + (size_t)g.ny * k)] == l) ? 1.0f : 0.0f;
    }
    return __ldg(g.phi + (size_t)s * V2M_SLOT + (i & 7) + V2M_BS * ((j & 7) + V2M_BS * (k & 7)));
}

// Trilinear blend of 8 corners at fractions (fx,fy,fz), the reference's order.
__device__ __forceinline__ float trilerp8(const float* c, float fx, float fy, float fz) {
    const float x00 = c[0] + fx * (c[1] - c[0]), x10 = c[2] + fx * (c[3] - c[2]);
    const float x01 = c[4] + fx * (c[5] - c[4]), x11 = c[6] + fx * (c[7] - c[6]);
    const float y0 = x00 + fy * (x10 - x00), y1 = x01 + fy * (x11 - x01);
    return y0 + fz * (y1 - y0);
}

// The trilinear cell under a point, computed once and shared by every label
// evaluated there: corner voxel, fractions and -- when the cell's base voxel
// lies inside the grid -- its brick's corner-table list (labels, count, first
// table). cell_corners reads the table, whose values are the reference's
// per-voxel phi (v2m_phi_cell, src/opencl/v2m_grid_body.cl:159-186, corner by
// corner), so the corners equal the reference's in both its one-brick case and
// its per-corner case.
struct Cell {
    int i0, j0, k0;
    float fx, fy, fz;
    int fast;
    int n, first;
    LabList ll;
};

__device__ __forceinline__ void cell_at(const DGrid& g, float px, float py, float pz, Cell& c) {
    const float u = px / g.vx, v = py / g.vy, w = pz / g.vz;
    c.i0 = (int)floorf(u);
    c.j0 = (int)floorf(v);
    c.k0 = (int)floorf(w);
    c.fx = u - c.i0;
    c.fy = v - c.j0;
    c.fz = w - c.k0;
    c.fast = 0;
    c.n = 0;
    c.first = -1;
    if (c.i0 >= 0 && c.j0 >= 0 && c.k0 >= 0 && c.i0 < g.nx && c.j0 < g.ny && c.k0 < g.nz) {
        const int b = brick_index(g, c.i0, c.j0, c.k0);
        const uint4* p = g.xbrick + (size_t)3 * b;
        const uint4 a = __ldg(p), e = __ldg(p + 1), f = __ldg(p + 2);
        const int n = (int)a.x;
        if (n >= 0) {
            c.fast = 1;
            c.n = n;
            c.first = (int)a.y;
            c.ll.w[0] = a.z; c.ll.w[1] = a.w; c.ll.w[2] = e.x; c.ll.w[3] = e.y;
            c.ll.w[4] = e.z; c.ll.w[5] = e.w; c.ll.w[6] = f.x; c.ll.w[7] = f.y;
        }
    }
}

// index of label l among the first n of a brick's labels, -1 if absent
__device__ __forceinline__ int lab_index(const LabList& ll, int n, int l) {
    const unsigned pat = (unsigned)(l & 0xFFFF) * 0x00010001u;
    unsigned bits = 0u;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        const unsigned m = __vcmpeq2(ll.w[w], pat);
        bits |= ((m & 1u) | ((m >> 15) & 2u)) << (2 * w);
    }
    const int nn = n < V2M_BL ? n : V2M_BL;
    bits &= (1u << nn) - 1u;
    return bits ? __ffs(bits) - 1 : -1;
}

// the 8 corners of phi_l in a cell whose base voxel lies inside the grid
// (c.fast): from its brick's corner table, or the uniform value
__device__ __forceinline__ void table_corners(const DGrid& g, const Cell& c, int l, float* out) {
    const int idx = lab_index(c.ll, c.n, l);
    if (kChecked && idx >= 0 && c.first >= 0 && (int64_t)c.first + idx >= g.ntab) {
        check_fail(g.chk, 21, c.first);   // a brick's corner table beyond the tables
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            out[n] = 0.0f;
        }
        return;
    }
    if (idx >= 0 && c.first >= 0) {
        const float* base = g.xphi + (size_t)(c.first + idx) * 729 + (c.i0 & 7) + 9 * ((c.j0 & 7) + 9 * (c.k0 & 7));
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            out[n] = __ldg(base + (n & 1) + 9 * ((n >> 1) & 1) + 81 * (n >> 2));
        }
    } else {
        const float f = idx >= 0 ? 1.0f : 0.0f;   // uniform table: its label everywhere; absent label: 0
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            out[n] = f;
        }
    }
}

// the 8 corners of phi_l in the cell
__device__ __forceinline__ void cell_corners(const DGrid& g, const Cell& c, int l, float* out) {
    if (c.fast) {
        table_corners(g, c, l, out);
        return;
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        out[n] = phi_voxel(g, l, c.i0 + (n & 1), c.j0 + ((n >> 1) & 1), c.k0 + ((n >> 2) & 1));
    }
}

__device__ __forceinline__ float cell_phi(const DGrid& g, const Cell& c, int l) {
    float v[8];
    cell_corners(g, c, l, v);
    return trilerp8(v, c.fx, c.fy, c.fz);
}

// phi_l at p, located in cell c: the analytic fields' own value, else the cell's
// (src/opencl/v2m_seed_body.cl:33-39)
template <bool kShape>
__device__ __forceinline__ float field_phi(const DGrid& g, const Cell& c, int l, float px, float py, float pz) {
    if constexpr (kShape) {
        return sdf_phi(g, l, px, py, pz);
    } else {
        return cell_phi(g, c, l);
    }
}

// phi_l trilinear at p (src/opencl/v2m_grid_body.cl:189-200)
template <bool kShape>
__device__ __noinline__ float phi_point(const DGrid& g, int l, float px, float py, float pz) {
    if constexpr (kShape) {
        return sdf_phi(g, l, px, py, pz);
    }
    Cell c;
    cell_at(g, px, py, pz, c);
    return cell_phi(g, c, l);
}

// The labels that may appear at p: its brick's list (src/opencl/v2m_seed_body.cl:42-59).
// Outside the grid: label 0 only.
__device__ __forceinline__ int labels_near(const DGrid& g, float px, float py, float pz, LabList& out) {
    const int i = (int)floorf(px / g.vx + 0.5f), j = (int)floorf(py / g.vy + 0.5f), k = (int)floorf(pz / g.vz + 0.5f);
    if (i < 0 || j < 0 || k < 0 || i >= g.nx || j >= g.ny || k >= g.nz) {
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            out.w[s] = 0u;
        }
        return 1;
    }
    const int b = brick_index(g, i, j, k);
    const int c = __ldg(g.bl_cnt + b);
    out = load_labels(g, b);
    return c < V2M_BL ? c : V2M_BL;
}

// ---- gray-scale fields (src/opencl/v2m_seed_body.cl:65-114) ---------------------
__device__ __forceinline__ float gray_sample(const DGrid& g, float px, float py, float pz, float* gr) {
    const float u = px / g.vx, v = py / g.vy, w = pz / g.vz;
    const int i0 = (int)floorf(u), j0 = (int)floorf(v), k0 = (int)floorf(w);
    const float fx = u - i0, fy = v - j0, fz = w - k0;
    const float outside = g.gTW[0] - g.gTW[g.gm];
    float c[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const int ii = i0 + (n & 1), jj = j0 + ((n >> 1) & 1), kk = k0 + ((n >> 2) & 1);
        c[n] = (ii < 0 || jj < 0 || kk < 0 || ii >= g.nx || jj >= g.ny || kk >= g.nz)
                   ? outside : __ldg(g.gI + ii + (size_t)g.nx * (jj + (size_t)g.ny * kk));
    }
    const float x00 = c[0] + fx * (c[1] - c[0]), x10 = c[2] + fx * (c[3] - c[2]);
    const float x01 = c[4] + fx * (c[5] - c[4]), x11 = c[6] + fx * (c[7] - c[6]);
    const float y0 = x00 + fy * (x10 - x00), y1 = x01 + fy * (x11 - x01);
    if (gr) {
        const float dx0 = (c[1] - c[0]) + fy * ((c[3] - c[2]) - (c[1] - c[0]));
        const float dx1 = (c[5] - c[4]) + fy * ((c[7] - c[6]) - (c[5] - c[4]));
        gr[0] = (dx0 + fz * (dx1 - dx0)) / g.vx;
        gr[1] = ((x10 - x00) + fz * ((x11 - x01) - (x10 - x00))) / g.vy;
        gr[2] = (y1 - y0) / g.vz;
    }
    return y0 + fz * (y1 - y0);
}

// psi_ab straight from the field's own formula: the analytic shape fields
// (gm < 0), or the intensity for adjacent gray labels; 0 if not applicable
// (then psi comes from the sampled cells)
template <bool kShape>
__device__ __forceinline__ int gray_psi(const DGrid& g, int a, int b, float px, float py, float pz, float* val, float* gr) {
    if constexpr (kShape) {
        *val = sdf_psi(g, a, b, px, py, pz, gr);
        return 1;
    }
    if (g.gm <= 0 || (a - b != 1 && b - a != 1)) {
        return 0;
    }
    const int k = a < b ? a : b;
    const float sg = (a > b ? 2.0f : -2.0f) / g.gTW[g.gm + k];
    *val = sg * (gray_sample(g, px, py, pz, gr) - g.gTW[k]);
    if (gr) {
        gr[0] *= sg;
        gr[1] *= sg;
        gr[2] *= sg;
    }
    return 1;
}

// The label owning p: argmax phi_l (smooth mode) or the voxel's label (voxel
// mode), with the runner-up and the margin (src/opencl/v2m_seed_body.cl:116-175).
template <bool kShape>
__device__ __forceinline__ int owner_label(const DGrid& g, int voxmode, float px, float py, float pz, int* second,
                                           float* margin) {
    const int i = (int)floorf(px / g.vx + 0.5f), j = (int)floorf(py / g.vy + 0.5f), k = (int)floorf(pz / g.vz + 0.5f);
    if (g.gm > 0 && !voxmode) {
        const float I = gray_sample(g, px, py, pz, nullptr);
        int l = 0;
        while (l < g.gm && I >= g.gTW[l]) {
            ++l;
        }
        const float dl = l > 0 ? (I - g.gTW[l - 1]) / g.gTW[g.gm + l - 1] : 1e30f;
        const float du = l < g.gm ? (g.gTW[l] - I) / g.gTW[g.gm + l] : 1e30f;
        *second = (dl < du) ? l - 1 : (l < g.gm ? l + 1 : V2M_NOLAB);
        *margin = 2.0f * fminf(dl, du);
        return l;
    }
    LabList ll;
    const int n = labels_near(g, px, py, pz, ll);
    int best = ll.get(0), sec = V2M_NOLAB;
    float pb = kShape ? -1e30f : -1.0f, ps = pb;
    if (n == 1) {
        *second = V2M_NOLAB;
        *margin = 1.0f;
        return best;
    }
    if constexpr (kShape) {
        // analytic fields: ranked by s itself (phi saturates beyond w / 2 of a
        // surface); the margin in phi units
#pragma unroll 1
        for (int s = 0; s < n; ++s) {
            const int l = ll.get(s);
            const float v = sdf_value(g, l, px, py, pz);
            if (v > pb) {
                ps = pb;
                sec = best;
                pb = v;
                best = l;
            } else if (v > ps) {
                ps = v;
                sec = l;
            }
        }
        const float w = sdf_at(g, 1);
        pb = fminf(1.0f, fmaxf(0.0f, 0.5f + pb / w));
        ps = sec == V2M_NOLAB ? 0.0f : fminf(1.0f, fmaxf(0.0f, 0.5f + ps / w));
        *second = sec;
        *margin = pb - ps;
        return voxmode ? label_at(g, i, j, k) : best;
    }
    Cell cl;
    cell_at(g, px, py, pz, cl);
    // two labels per turn: both labels' corner loads are in flight together;
    // the ranking still takes the labels one by one in list order
#pragma unroll 1
    for (int s = 0; s < n; s += 2) {
        const int l0 = ll.get(s);
        const bool two = s + 1 < n;
        const int l1 = two ? ll.get(s + 1) : l0;
        float c0[8], c1[8];
        cell_corners(g, cl, l0, c0);
        cell_corners(g, cl, l1, c1);
        const float v0 = trilerp8(c0, cl.fx, cl.fy, cl.fz), v1 = trilerp8(c1, cl.fx, cl.fy, cl.fz);
        if (v0 > pb) {
            ps = pb;
            sec = best;
            pb = v0;
            best = l0;
        } else if (v0 > ps) {
            ps = v0;
            sec = l0;
        }
        if (two) {
            if (v1 > pb) {
                ps = pb;
                sec = best;
                pb = v1;
                best = l1;
            } else if (v1 > ps) {
                ps = v1;
                sec = l1;
            }
        }
    }
    *second = sec;
    *margin = pb - ps;
    if (voxmode) {
        return label_at(g, i, j, k);
    }
    return best;
}

// owner_label's label-field branch (gm == 0), also handing out the cell it
// ranked the labels on (*ranked = 1; not when the brick lists one label)
__device__ __forceinline__ int owner_on_cell(const DGrid& g, float px, float py, float pz, int* second, Cell& cl,
                                             int* ranked) {
    LabList ll;
    const int n = labels_near(g, px, py, pz, ll);
    int best = ll.get(0), sec = V2M_NOLAB;
    float pb = -1.0f, ps = pb;
    *ranked = 0;
    if (n == 1) {
        *second = V2M_NOLAB;
        return best;
    }
    cell_at(g, px, py, pz, cl);
    *ranked = 1;
#pragma unroll 1
    for (int s = 0; s < n; s += 2) {
        const int l0 = ll.get(s);
        const bool two = s + 1 < n;
        const int l1 = two ? ll.get(s + 1) : l0;
        float c0[8], c1[8];
        cell_corners(g, cl, l0, c0);
        cell_corners(g, cl, l1, c1);
        const float v0 = trilerp8(c0, cl.fx, cl.fy, cl.fz), v1 = trilerp8(c1, cl.fx, cl.fy, cl.fz);
        if (v0 > pb) {
            ps = pb;
            sec = best;
            pb = v0;
            best = l0;
        } else if (v0 > ps) {
            ps = v0;
            sec = l0;
        }
        if (two) {
            if (v1 > pb) {
                ps = pb;
                sec = best;
                pb = v1;
                best = l1;
            } else if (v1 > ps) {
                ps = v1;
                sec = l1;
            }
        }
    }
    *second = sec;
    return best;
}

// psi_ab = phi_a - phi_b at p (src/opencl/v2m_seed_body.cl:179-205)
template <bool kShape>
__device__ __noinline__ float psi(const DGrid& g, int a, int b, float px, float py, float pz) {
    float gv;
    if (gray_psi<kShape>(g, a, b, px, py, pz, &gv, nullptr)) {
        return gv;
    }
    Cell cl;
    cell_at(g, px, py, pz, cl);
    float c[8], e[8];
    cell_corners(g, cl, a, c);
    cell_corners(g, cl, b, e);
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        c[n] -= e[n];
    }
    return trilerp8(c, cl.fx, cl.fy, cl.fz);
}

// psi's value and cell-analytic gradient from the corner differences
// c = phi_a - phi_b and the fractions: (gradient, value)
__device__ __forceinline__ float4 psi_grad_diff(const DGrid& g, const float* c, float fx, float fy, float fz) {
    float gr[3];
    const float x00 = c[0] + fx * (c[1] - c[0]), x10 = c[2] + fx * (c[3] - c[2]);
    const float x01 = c[4] + fx * (c[5] - c[4]), x11 = c[6] + fx * (c[7] - c[6]);
    const float y0 = x00 + fy * (x10 - x00), y1 = x01 + fy * (x11 - x01);
    const float dx0 = (c[1] - c[0]) + fy * ((c[3] - c[2]) - (c[1] - c[0]));
    const float dx1 = (c[5] - c[4]) + fy * ((c[7] - c[6]) - (c[5] - c[4]));
    gr[0] = (dx0 + fz * (dx1 - dx0)) / g.vx;
    gr[1] = ((x10 - x00) + fz * ((x11 - x01) - (x10 - x00))) / g.vy;
    gr[2] = (y1 - y0) / g.vz;
    return make_float4(gr[0], gr[1], gr[2], y0 + fz * (y1 - y0));
}

// psi_ab's value and cell-analytic gradient on a cell already located: (gradient, value)
__device__ __forceinline__ float4 psi_grad_on(const DGrid& g, const Cell& cl, int a, int b) {
    float c[8], e[8];
    cell_corners(g, cl, a, c);
    cell_corners(g, cl, b, e);
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        c[n] -= e[n];
    }
    return psi_grad_diff(g, c, cl.fx, cl.fy, cl.fz);
}

// The corner differences phi_a - phi_b of the last cell a search evaluated psi_ab
// on (label fields): the probes of a bracketed search mostly stay in one cell,
// and there psi and its gradient need no memory access. The values are the
// ones psi / psi_grad4 read (same cell, same corners), so the results are too.
struct PsiCache {
    int i0, j0, k0;   // i0 == INT_MIN: empty
    float d[8];
};

__device__ __forceinline__ PsiCache psi_cache_empty() {
    PsiCache pc;
    pc.i0 = pc.j0 = pc.k0 = INT_MIN;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        pc.d[n] = 0.0f;
    }
    return pc;
}

// p's cell into the cache (read from the tables unless it is the cached one); its fractions out
__device__ __forceinline__ void psi_cache_at(const DGrid& g, int a, int b, float px, float py, float pz, PsiCache& pc,
                                             float& fx, float& fy, float& fz) {
    const float u = px / g.vx, v = py / g.vy, w = pz / g.vz;
    const int i0 = (int)floorf(u), j0 = (int)floorf(v), k0 = (int)floorf(w);
    fx = u - i0;
    fy = v - j0;
    fz = w - k0;
    if (i0 != pc.i0 || j0 != pc.j0 || k0 != pc.k0) {
        Cell cl;
        cell_at(g, px, py, pz, cl);
        float c[8], e[8];
        cell_corners(g, cl, a, c);
        cell_corners(g, cl, b, e);
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            pc.d[n] = c[n] - e[n];
        }
        pc.i0 = i0;
        pc.j0 = j0;
        pc.k0 = k0;
    }
}

// psi_ab and its cell-analytic gradient (src/opencl/v2m_seed_body.cl:211-247)
// (one out-of-line copy returning (gradient, value); psi_grad below unpacks it)
template <bool kShape>
__device__ __noinline__ float4 psi_grad4(const DGrid& g, int a, int b, float px, float py, float pz) {
    float gv, gr[3];
    if (gray_psi<kShape>(g, a, b, px, py, pz, &gv, gr)) {
        return make_float4(gr[0], gr[1], gr[2], gv);
    }
    Cell cl;
    cell_at(g, px, py, pz, cl);
    return psi_grad_on(g, cl, a, b);
}

// psi and psi_grad4 through a PsiCache (the gray-scale branch bypasses it)
template <bool kShape>
__device__ __forceinline__ float psi_c(const DGrid& g, int a, int b, float px, float py, float pz, PsiCache& pc) {
    float gv;
    if (gray_psi<kShape>(g, a, b, px, py, pz, &gv, nullptr)) {
        return gv;
    }
    float fx, fy, fz;
    psi_cache_at(g, a, b, px, py, pz, pc, fx, fy, fz);
    return trilerp8(pc.d, fx, fy, fz);
}

template <bool kShape>
__device__ __forceinline__ float4 psi_grad4_c(const DGrid& g, int a, int b, float px, float py, float pz, PsiCache& pc) {
    float gv, gr[3];
    if (gray_psi<kShape>(g, a, b, px, py, pz, &gv, gr)) {
        return make_float4(gr[0], gr[1], gr[2], gv);
    }
    float fx, fy, fz;
    psi_cache_at(g, a, b, px, py, pz, pc, fx, fy, fz);
    return psi_grad_diff(g, pc.d, fx, fy, fz);
}

template <bool kShape>
__device__ __forceinline__ float psi_grad(const DGrid& g, int a, int b, float px, float py, float pz, float* gr) {
    const float4 r = psi_grad4<kShape>(g, a, b, px, py, pz);
    gr[0] = r.x;
    gr[1] = r.y;
    gr[2] = r.z;
    return r.w;
}

// Bracketed root of psi_ab along unit direction u from p, within rad: doubling
// probes from the Newton guess tg, then Illinois regula falsi
// (src/opencl/v2m_seed_body.cl:255-320). Returns (the moved p, 1) on success,
// (p, 0) otherwise. (The out-of-line helpers take and return points by value,
// so their callers' points stay in registers; the pointer forms below wrap them.)
template <bool kShape>
__device__ __noinline__ float4 bisect_dirv(const DGrid& g, int a, int b, float px, float py, float pz, float ux,
                                           float uy, float uz, float v0, float rad, float tg, PsiCache pc) {
    const float p[3] = { px, py, pz }, u[3] = { ux, uy, uz };
    if (v0 == 0.0f) {
        return make_float4(px, py, pz, 1.0f);
    }
    const float sg = v0 > 0.0f ? -1.0f : 1.0f;
    float t0 = 0.0f, t1 = -1.0f, f0 = v0, f1 = 0.0f;
    float t = (tg > 0.0f && tg < rad) ? tg : 0.25f * rad;
    for (int k = 0; k < 8; ++k) {
        const float v = psi_c<kShape>(g, a, b, p[0] + sg * t * u[0], p[1] + sg * t * u[1], p[2] + sg * t * u[2], pc);
        if ((v > 0.0f) != (v0 > 0.0f) || v == 0.0f) {
            t1 = t;
            f1 = v;
            break;
        }
        t0 = t;
        f0 = v;
        if (t >= rad) {
            break;
        }
        t = fminf(2.0f * t, rad);
    }
    if (t1 < 0.0f) {
        return make_float4(px, py, pz, 0.0f);
    }
    int side = 0;
    for (int it = 0; it < 8 && f1 != 0.0f && fabsf(t1 - t0) > 1e-4f * rad; ++it) {
        const float tm = (f0 != f1) ? t1 - f1 * (t1 - t0) / (f1 - f0) : 0.5f * (t0 + t1);
        const float v = psi_c<kShape>(g, a, b, p[0] + sg * tm * u[0], p[1] + sg * tm * u[1], p[2] + sg * tm * u[2], pc);
        if ((v > 0.0f) == (f1 > 0.0f)) {
            t1 = tm;
            f1 = v;
            if (side == -1) {
                f0 *= 0.5f;
            }
            side = -1;
        } else {
            t0 = t1;
            f0 = f1;
            t1 = tm;
            f1 = v;
            side = 1;
        }
    }
    return make_float4(p[0] + sg * t1 * u[0], p[1] + sg * t1 * u[1], p[2] + sg * t1 * u[2], 1.0f);
}

template <bool kShape>
__device__ __forceinline__ int bisect_dir(const DGrid& g, int a, int b, float* p, const float* u, float v0, float rad,
                                          float tg) {
    const float4 r = bisect_dirv<kShape>(g, a, b, p[0], p[1], p[2], u[0], u[1], u[2], v0, rad, tg, psi_cache_empty());
    p[0] = r.x;
    p[1] = r.y;
    p[2] = r.z;
    return r.w != 0.0f;
}

// Projection onto psi_ab = 0 along the local normal within rad (src/opencl/v2m_seed_body.cl:324-335)
// (pc: a cache of psi_ab's corners from the caller, or empty)
template <bool kShape>
__device__ __noinline__ float4 project1v(const DGrid& g, int a, int b, float px, float py, float pz, float rad,
                                         PsiCache pc) {
    const float4 r4 = psi_grad4_c<kShape>(g, a, b, px, py, pz, pc);
    const float gr[3] = { r4.x, r4.y, r4.z };
    const float v = r4.w;
    const float gn = sqrtf(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
    if (gn < 1e-9f) {
        return make_float4(px, py, pz, 0.0f);
    }
    return bisect_dirv<kShape>(g, a, b, px, py, pz, gr[0] / gn, gr[1] / gn, gr[2] / gn, v, rad, 1.5f * fabsf(v) / gn, pc);
}

template <bool kShape>
__device__ __forceinline__ int project1(const DGrid& g, int a, int b, float* p, float rad) {
    const float4 r = project1v<kShape>(g, a, b, p[0], p[1], p[2], rad, psi_cache_empty());
    p[0] = r.x;
    p[1] = r.y;
    p[2] = r.z;
    return r.w != 0.0f;
}

// Projection onto the junction curve psi_ab = psi_ac = 0 by alternating
// bracketed legs (src/opencl/v2m_seed_body.cl:342-420).
template <bool kShape>
__device__ __noinline__ float4 project2v(const DGrid& g, int a, int b, int c, float px, float py, float pz,
                                         float rad) {
    const float p[3] = { px, py, pz };
    float q[3] = { px, py, pz };
    if constexpr (kShape) {
        // analytic fields: of the three pairs' constraints, solve the two whose
        // gradients are the most independent (the largest cross product), with
        // the label they share as the pivot a (T-junctions of exact CSG have two
        // parallel constraints there)
        float gab[3], gac[3], gbc[3];
        psi_grad<kShape>(g, a, b, q[0], q[1], q[2], gab);
        psi_grad<kShape>(g, a, c, q[0], q[1], q[2], gac);
        psi_grad<kShape>(g, b, c, q[0], q[1], q[2], gbc);
        const float xa[3] = { gab[1] * gac[2] - gab[2] * gac[1], gab[2] * gac[0] - gab[0] * gac[2],
                              gab[0] * gac[1] - gab[1] * gac[0] };
        const float xb[3] = { gab[1] * gbc[2] - gab[2] * gbc[1], gab[2] * gbc[0] - gab[0] * gbc[2],
                              gab[0] * gbc[1] - gab[1] * gbc[0] };
        const float xc[3] = { gac[1] * gbc[2] - gac[2] * gbc[1], gac[2] * gbc[0] - gac[0] * gbc[2],
                              gac[0] * gbc[1] - gac[1] * gbc[0] };
        const float na = xa[0] * xa[0] + xa[1] * xa[1] + xa[2] * xa[2];
        const float nb = xb[0] * xb[0] + xb[1] * xb[1] + xb[2] * xb[2];
        const float nc = xc[0] * xc[0] + xc[1] * xc[1] + xc[2] * xc[2];
        if (nb > na && nb >= nc) {   // pivot b: psi_ba, psi_bc
            const int t = a;
            a = b;
            b = t;
        } else if (nc > na && nc > nb) {   // pivot c: psi_ca, psi_cb
            const int t = a;
            a = c;
            c = b;
            b = t;
        }
    }
    for (int it = 0; it < 3; ++it) {
        float g1[3], g2[3];
        if (!project1<kShape>(g, a, b, q, rad)) {
            return make_float4(px, py, pz, 0.0f);
        }
        psi_grad<kShape>(g, a, b, q[0], q[1], q[2], g1);
        const float v2 = psi_grad<kShape>(g, a, c, q[0], q[1], q[2], g2);
        const float a11 = g1[0] * g1[0] + g1[1] * g1[1] + g1[2] * g1[2];
        if (a11 < 1e-18f) {
            return make_float4(px, py, pz, 0.0f);
        }
        const float pr = (g1[0] * g2[0] + g1[1] * g2[1] + g1[2] * g2[2]) / a11;
        float u[3] = { g2[0] - pr * g1[0], g2[1] - pr * g1[1], g2[2] - pr * g1[2] };
        const float un = sqrtf(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        if (un < 1e-9f) {
            return make_float4(px, py, pz, 0.0f);
        }
        u[0] /= un;
        u[1] /= un;
        u[2] /= un;
        if (!bisect_dir<kShape>(g, a, c, q, u, v2, rad, 1.5f * fabsf(v2) / un)) {
            return make_float4(px, py, pz, 0.0f);
        }
    }
    if (!project1<kShape>(g, a, b, q, rad)) {
        return make_float4(px, py, pz, 0.0f);
    }
    const float m2 = (q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) + (q[2] - p[2]) * (q[2] - p[2]);
    if (m2 > rad * rad) {
        return make_float4(px, py, pz, 0.0f);
    }
    return make_float4(q[0], q[1], q[2], 1.0f);
}

template <bool kShape>
__device__ __forceinline__ int project2(const DGrid& g, int a, int b, int c, float* p, float rad) {
    const float4 r = project2v<kShape>(g, a, b, c, p[0], p[1], p[2], rad);
    p[0] = r.x;
    p[1] = r.y;
    p[2] = r.z;
    return r.w != 0.0f;
}

// Crossing of p -> q with psi_ab = 0: 6 bisections and a secant (src/opencl/v2m_particle_body.cl:188-212)
template <bool kShape>
__device__ __noinline__ float4 crossingv(const DGrid& g, int a, int b, float px, float py, float pz, float qx,
                                         float qy, float qz) {
    const float p[3] = { px, py, pz }, q[3] = { qx, qy, qz };
    PsiCache pc = psi_cache_empty();
    float t0 = 0.0f, t1 = 1.0f;
    float v0 = psi_c<kShape>(g, a, b, p[0], p[1], p[2], pc);
    float v1 = psi_c<kShape>(g, a, b, q[0], q[1], q[2], pc);
    for (int it = 0; it < 6; ++it) {
        const float tm = 0.5f * (t0 + t1);
        const float vm = psi_c<kShape>(g, a, b, p[0] + tm * (q[0] - p[0]), p[1] + tm * (q[1] - p[1]), p[2] + tm * (q[2] - p[2]), pc);
        if (vm > 0.0f) {
            t0 = tm;
            v0 = vm;
        } else {
            t1 = tm;
            v1 = vm;
        }
    }
    const float t = (v0 - v1) != 0.0f ? t0 + (t1 - t0) * v0 / (v0 - v1) : 0.5f * (t0 + t1);
    return make_float4(p[0] + t * (q[0] - p[0]), p[1] + t * (q[1] - p[1]), p[2] + t * (q[2] - p[2]), 0.0f);
}

template <bool kShape>
__device__ __forceinline__ void crossing(const DGrid& g, int a, int b, const float* p, const float* q, float* c) {
    const float4 r = crossingv<kShape>(g, a, b, p[0], p[1], p[2], q[0], q[1], q[2]);
    c[0] = r.x;
    c[1] = r.y;
    c[2] = r.z;
}

// Drop v's component along psi_ab's normal at p (src/opencl/v2m_particle_body.cl:215-229)
template <bool kShape>
__device__ __forceinline__ void tangential(const DGrid& g, int a, int b, const float* p, float* v) {
    float gr[3];
    psi_grad<kShape>(g, a, b, p[0], p[1], p[2], gr);
    const float gn2 = gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2];
    if (gn2 < 1e-12f) {
        return;
    }
    const float vn = (v[0] * gr[0] + v[1] * gr[1] + v[2] * gr[2]) / gn2;
    for (int k = 0; k < 3; ++k) {
        v[k] -= vn * gr[k];
    }
}

// A third label competing at q (phi_c > 0.5 phi_a), or NOLAB (src/opencl/v2m_particle_body.cl:232-260)
template <bool kShape>
__device__ __noinline__ int third_labelv(const DGrid& g, int a, int b, float qx, float qy, float qz) {
    const float q[3] = { qx, qy, qz };
    LabList ll;
    const int n = labels_near(g, q[0], q[1], q[2], ll);
    int other = 0;
#pragma unroll
    for (int s = 0; s < V2M_BL; ++s) {
        if (s < n) {
            const int l = ll.get(s);
            other |= l != a && l != b;
        }
    }
    if (!other) {
        return V2M_NOLAB;
    }
    Cell cl;
    cell_at(g, q[0], q[1], q[2], cl);
    const float pa = field_phi<kShape>(g, cl, a, q[0], q[1], q[2]);
    int c = V2M_NOLAB;
    float pc = 0.5f * pa;
#pragma unroll 1
    for (int s = 0; s < n; ++s) {
        const int l = ll.get(s);
        if (l != a && l != b) {
            const float w = field_phi<kShape>(g, cl, l, q[0], q[1], q[2]);
            if (w > pc) {
                pc = w;
                c = l;
            }
        }
    }
    return c;
}

template <bool kShape>
__device__ __forceinline__ int third_label(const DGrid& g, int a, int b, const float* q) {
    return third_labelv<kShape>(g, a, b, q[0], q[1], q[2]);
}

// Do the node's labels dominate at q? (src/opencl/v2m_particle_body.cl:266-291)
template <bool kShape>
__device__ __noinline__ int valid_onv(const DGrid& g, int a, int b, int c, float qx, float qy, float qz) {
    const float q[3] = { qx, qy, qz };
    LabList ll;
    const int n = labels_near(g, q[0], q[1], q[2], ll);
    int other = 0;
#pragma unroll
    for (int s = 0; s < V2M_BL; ++s) {
        if (s < n) {
            const int l = ll.get(s);
            other |= l != a && l != b && l != c;
        }
    }
    if (!other) {
        return 1;
    }
    Cell cl;
    cell_at(g, q[0], q[1], q[2], cl);
    float mine = fminf(field_phi<kShape>(g, cl, a, q[0], q[1], q[2]), field_phi<kShape>(g, cl, b, q[0], q[1], q[2]));
    if (c != V2M_NOLAB) {
        mine = fminf(mine, field_phi<kShape>(g, cl, c, q[0], q[1], q[2]));
    }
#pragma unroll 1
    for (int s = 0; s < n; ++s) {
        const int l = ll.get(s);
        if (l != a && l != b && l != c && field_phi<kShape>(g, cl, l, q[0], q[1], q[2]) > mine + 0.02f) {
            return 0;
        }
    }
    return 1;
}

template <bool kShape>
__device__ __forceinline__ int valid_on(const DGrid& g, int a, int b, int c, const float* q) {
    return valid_onv<kShape>(g, a, b, c, q[0], q[1], q[2]);
}

// third_label(a, b, q) and valid_on(a, b, NOLAB, q) together: one label list,
// one cell and one phi evaluation per label serve both (the same values as
// the two calls). Returns (third label or NOLAB, valid).
template <bool kShape>
__device__ __noinline__ int2 third_and_valid(const DGrid& g, int a, int b, float qx, float qy, float qz) {
    LabList ll;
    const int n = labels_near(g, qx, qy, qz, ll);
    int other = 0;
#pragma unroll
    for (int s = 0; s < V2M_BL; ++s) {
        if (s < n) {
            const int l = ll.get(s);
            other |= l != a && l != b;
        }
    }
    if (!other) {
        return make_int2(V2M_NOLAB, 1);
    }
    Cell cl;
    cell_at(g, qx, qy, qz, cl);
    const float pa = field_phi<kShape>(g, cl, a, qx, qy, qz);
    const float mine = fminf(pa, field_phi<kShape>(g, cl, b, qx, qy, qz));
    int c = V2M_NOLAB, valid = 1;
    float pc = 0.5f * pa;
#pragma unroll 1
    for (int s = 0; s < n; ++s) {
        const int l = ll.get(s);
        if (l != a && l != b) {
            const float w = field_phi<kShape>(g, cl, l, qx, qy, qz);
            if (w > pc) {
                pc = w;
                c = l;
            }
            if (w > mine + 0.02f) {
                valid = 0;
            }
        }
    }
    return make_int2(c, valid);
}

// ---- voxel trap mode (src/opencl/v2m_particle_body.cl:358-650) -------------------
// Walk p -> p + s through label-a voxels (one face at a time); on the first face
// into another label write the face point to x, that label to *lb and return
// the ray fraction; -1 if the step stays inside label a.
__device__ __noinline__ float dda_hit(const DGrid& g, int a, const float* p, const float* s, float* x, int* lb) {
    const float vsz[3] = { g.vx, g.vy, g.vz };
    float u[3], w[3];
    int id[3];
    for (int k = 0; k < 3; ++k) {
        u[k] = p[k] / vsz[k] + 0.5f;
        w[k] = s[k] / vsz[k];
        id[k] = (int)floorf(u[k]);
    }
    int l = label_at(g, id[0], id[1], id[2]);
    if (l != a) {
        x[0] = p[0];
        x[1] = p[1];
        x[2] = p[2];
        *lb = l;
        return 0.0f;
    }
    float t = 0.0f;
    for (int it = 0; it < 64; ++it) {
        float ht[3];
        for (int k = 0; k < 3; ++k) {
            ht[k] = w[k] != 0.0f ? fabsf(((float)id[k] + (w[k] > 0.0f ? 1.0f : 0.0f) - u[k]) / w[k]) : 1e30f;
        }
        const float dt = fminf(fminf(ht[0], ht[1]), ht[2]);
        const int ax = dt == ht[0] ? 0 : (dt == ht[1] ? 1 : 2);
        if (t + dt >= 1.0f) {
            return -1.0f;
        }
        t += dt;
        for (int k = 0; k < 3; ++k) {
            u[k] += dt * w[k];
        }
        u[ax] = (float)id[ax] + (w[ax] > 0.0f ? 1.0f : 0.0f);
        id[ax] += w[ax] > 0.0f ? 1 : -1;
        l = label_at(g, id[0], id[1], id[2]);
        if (l != a) {
            for (int k = 0; k < 3; ++k) {
                x[k] = (u[k] - 0.5f) * vsz[k];
            }
            *lb = l;
            return t;
        }
    }
    return -1.0f;
}

// Nearest point to q on the a|b voxel faces (c == NOLAB) or on the a|b|c voxel
// edges, within R voxels; squared distance or -1 (src/opencl/v2m_particle_body.cl:437-529).
__device__ __noinline__ float vox_nearest(const DGrid& g, int a, int b, int c, const float* q, int R, float* out) {
    const float vsz[3] = { g.vx, g.vy, g.vz };
    float u[3];
    int ci[3];
    for (int k = 0; k < 3; ++k) {
        u[k] = q[k] / vsz[k] + 0.5f;
        ci[k] = (int)floorf(u[k]);
    }
    float best = -1.0f;
    for (int vk = ci[2] - R; vk <= ci[2] + R; ++vk)
        for (int vj = ci[1] - R; vj <= ci[1] + R; ++vj)
            for (int vi = ci[0] - R; vi <= ci[0] + R; ++vi) {
                if (label_at(g, vi, vj, vk) != a) {
                    continue;
                }
                const int v[3] = { vi, vj, vk };
                for (int ax = 0; ax < 3; ++ax) {
                    const int o1 = (ax + 1) % 3, o2 = (ax + 2) % 3;
                    if (c == V2M_NOLAB) {
                        for (int sd = 0; sd < 2; ++sd) {
                            int nn[3] = { v[0], v[1], v[2] };
                            nn[ax] += sd ? 1 : -1;
                            if (label_at(g, nn[0], nn[1], nn[2]) != b) {
                                continue;
                            }
                            float y[3];
                            y[ax] = (float)(v[ax] + sd);
                            y[o1] = fminf(fmaxf(u[o1], (float)v[o1]), (float)(v[o1] + 1));
                            y[o2] = fminf(fmaxf(u[o2], (float)v[o2]), (float)(v[o2] + 1));
                            float d2 = 0.0f;
                            for (int k = 0; k < 3; ++k) {
                                y[k] = (y[k] - 0.5f) * vsz[k];
                                d2 += (y[k] - q[k]) * (y[k] - q[k]);
                            }
                            if (best < 0.0f || d2 < best) {
                                best = d2;
                                out[0] = y[0];
                                out[1] = y[1];
                                out[2] = y[2];
                            }
                        }
                    } else {
                        for (int e = 0; e < 4; ++e) {
                            const int e1 = e & 1, e2 = e >> 1;
                            int hb = 0, hc = 0;
                            for (int m = 0; m < 4; ++m) {
                                int nn[3] = { v[0], v[1], v[2] };
                                nn[o1] += e1 - 1 + (m & 1);
                                nn[o2] += e2 - 1 + (m >> 1);
                                const int ln = label_at(g, nn[0], nn[1], nn[2]);
                                hb |= ln == b;
                                hc |= ln == c;
                            }
                            if (!hb || !hc) {
                                continue;
                            }
                            float y[3];
                            y[ax] = fminf(fmaxf(u[ax], (float)v[ax]), (float)(v[ax] + 1));
                            y[o1] = (float)(v[o1] + e1);
                            y[o2] = (float)(v[o2] + e2);
                            float d2 = 0.0f;
                            for (int k = 0; k < 3; ++k) {
                                y[k] = (y[k] - 0.5f) * vsz[k];
                                d2 += (y[k] - q[k]) * (y[k] - q[k]);
                            }
                            if (best < 0.0f || d2 < best) {
                                best = d2;
                                out[0] = y[0];
                                out[1] = y[1];
                                out[2] = y[2];
                            }
                        }
                    }
                }
            }
    return best;
}

__device__ __forceinline__ int vox_third(const DGrid& g, int a, int b, const float* p) {
    const int i0 = (int)floorf(p[0] / g.vx), j0 = (int)floorf(p[1] / g.vy), k0 = (int)floorf(p[2] / g.vz);
    for (int m = 0; m < 8; ++m) {
        const int l = label_at(g, i0 + (m & 1), j0 + ((m >> 1) & 1), k0 + (m >> 2));
        if (l != a && l != b) {
            return l;
        }
    }
    return V2M_NOLAB;
}

// ---- the size field at a point ----------------------------------------------------
// hmode 0: the nearest voxel, clamped (src/opencl/v2m_particle_body.cl:30-36);
// hmode 1: trilinear between voxel centres, clamped to the grid (extension).
__device__ __forceinline__ float size_at(const DGrid& g, int hmode, float px, float py, float pz) {
    if (hmode == 0) {
        int i = (int)floorf(px / g.vx + 0.5f), j = (int)floorf(py / g.vy + 0.5f), k = (int)floorf(pz / g.vz + 0.5f);
        i = i < 0 ? 0 : (i >= g.nx ? g.nx - 1 : i);
        j = j < 0 ? 0 : (j >= g.ny ? g.ny - 1 : j);
        k = k < 0 ? 0 : (k >= g.nz ? g.nz - 1 : k);
        return __ldg(g.hvox + i + (size_t)g.nx * (j + (size_t)g.ny * k));
    }
    float u = px / g.vx, v = py / g.vy, w = pz / g.vz;
    u = fminf(fmaxf(u, 0.0f), (float)(g.nx - 1));
    v = fminf(fmaxf(v, 0.0f), (float)(g.ny - 1));
    w = fminf(fmaxf(w, 0.0f), (float)(g.nz - 1));
    int i0 = (int)floorf(u), j0 = (int)floorf(v), k0 = (int)floorf(w);
    i0 = i0 > g.nx - 2 ? (g.nx > 1 ? g.nx - 2 : 0) : i0;
    j0 = j0 > g.ny - 2 ? (g.ny > 1 ? g.ny - 2 : 0) : j0;
    k0 = k0 > g.nz - 2 ? (g.nz > 1 ? g.nz - 2 : 0) : k0;
    const float fx = u - i0, fy = v - j0, fz = w - k0;
    const int i1 = i0 + 1 < g.nx ? i0 + 1 : i0, j1 = j0 + 1 < g.ny ? j0 + 1 : j0, k1 = k0 + 1 < g.nz ? k0 + 1 : k0;
    float c[8];
    const int ii[2] = { i0, i1 }, jj[2] = { j0, j1 }, kk[2] = { k0, k1 };
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        c[n] = __ldg(g.hvox + ii[n & 1] + (size_t)g.nx * (jj[(n >> 1) & 1] + (size_t)g.ny * kk[n >> 2]));
    }
    return trilerp8(c, fx, fy, fz);
}

// ---- the move --------------------------------------------------------------------
// Node state a move reads and writes, held in registers.
struct NodeState {
    float p[3];   // position
    int a;        // own label
    int ty;       // type
    int pb, pc;   // partner labels (part[2i], part[2i+1])
    float hn;     // h at the node
};

// Voxel-mode move with step s (src/opencl/v2m_particle_body.cl:549-650).
__device__ __noinline__ float move_voxel(const DGrid& g, int hmode, float h, float snap, const float* s, NodeState& st) {
    const float vmin = fminf(fminf(g.vx, g.vy), g.vz);
    float p[3], q[3], x[3];
    p[0] = st.p[0];
    p[1] = st.p[1];
    p[2] = st.p[2];
    const int a = st.a;
    int ty = st.ty, b = st.pb, c = st.pc;
    const float sl = sqrtf(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    const int R = 1 + (int)ceilf(sl / vmin);
    for (int k = 0; k < 3; ++k) {
        q[k] = p[k] + s[k];
    }
    if (ty == V2M_INTERIOR) {
        int l;
        const float t = dda_hit(g, a, p, s, x, &l);
        if (t >= 0.0f) {
            b = l;
            if (vox_nearest(g, a, b, V2M_NOLAB, q, R, q) < 0.0f) {
                q[0] = x[0];
                q[1] = x[1];
                q[2] = x[2];
            }
            ty = V2M_INTERFACE;
        } else if (snap > 0.0f) {
            const int Rs = 1 + (int)ceilf(snap * h / vmin);
            float best = -1.0f, y[3];
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int l2 = label_at(g, (int)floorf(q[0] / g.vx + 0.5f) + dx * Rs,
                                                (int)floorf(q[1] / g.vy + 0.5f) + dy * Rs,
                                                (int)floorf(q[2] / g.vz + 0.5f) + dz * Rs);
                        if (l2 == a || l2 == b) {
                            continue;
                        }
                        const float d2 = vox_nearest(g, a, l2, V2M_NOLAB, q, Rs, y);
                        if (d2 >= 0.0f && d2 < snap * snap * h * h && (best < 0.0f || d2 < best)) {
                            best = d2;
                            b = l2;
                            x[0] = y[0];
                            x[1] = y[1];
                            x[2] = y[2];
                        }
                    }
            if (best >= 0.0f) {
                q[0] = x[0];
                q[1] = x[1];
                q[2] = x[2];
                ty = V2M_INTERFACE;
            }
        }
    } else if (ty == V2M_INTERFACE) {
        if (vox_nearest(g, a, b, V2M_NOLAB, q, R, q) < 0.0f) {
            return 0.0f;
        }
    } else {
        if (vox_nearest(g, a, b, c, q, R, q) < 0.0f) {
            return 0.0f;
        }
    }
    if (ty == V2M_INTERFACE) {
        const int cc = vox_third(g, a, b, q);
        if (cc != V2M_NOLAB) {
            float r[3];
            const float d2 = vox_nearest(g, a, b, cc, q, 1, r);
            if (d2 >= 0.0f && d2 < 0.0625f * h * h) {
                q[0] = r[0];
                q[1] = r[1];
                q[2] = r[2];
                ty = V2M_JUNCTION;
                c = cc;
            }
        }
    }
    const float mv = sqrtf((q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) + (q[2] - p[2]) * (q[2] - p[2]));
    st.p[0] = q[0];
    st.p[1] = q[1];
    st.p[2] = q[2];
    st.ty = ty;
    st.pb = ty == V2M_INTERIOR ? V2M_NOLAB : b;
    st.pc = ty >= V2M_JUNCTION ? c : V2M_NOLAB;
    st.hn = size_at(g, hmode, q[0], q[1], q[2]);
    return mv / h;
}

// The trapped move with the (capped) step s (src/opencl/v2m_particle_body.cl:659-833).
// ty0 is the type before the move; st is updated in place exactly where the
// reference writes the node's arrays.
template <bool kShape>
__device__ __forceinline__ float move_step(const DGrid& g, int hmode, float h, float* s, float maxstep, float snap,
                                        int voxmode, NodeState& st) {
    float p[3], q[3];
    p[0] = st.p[0];
    p[1] = st.p[1];
    p[2] = st.p[2];
    const int a = st.a;
    const int ty_in = st.ty;
    int ty = ty_in;
    if (voxmode) {
        return move_voxel(g, hmode, h, snap, s, st);
    }
    int b = st.pb;
    const int c = st.pc;
    if (ty == V2M_INTERIOR) {
        for (int k = 0; k < 3; ++k) {
            q[k] = p[k] + s[k];
        }
        int sec, ranked = 0;
        float mg;
        Cell oc;
        const int l = (kShape || g.gm > 0) ? owner_label<kShape>(g, 0, q[0], q[1], q[2], &sec, &mg)
                                           : owner_on_cell(g, q[0], q[1], q[2], &sec, oc, &ranked);
        if (l != a) {
            b = l;
            float x[3], r[3];
            crossing<kShape>(g, a, b, p, q, x);
            for (int k = 0; k < 3; ++k) {
                r[k] = q[k] - x[k];
            }
            tangential<kShape>(g, a, b, x, r);
            for (int k = 0; k < 3; ++k) {
                q[k] = x[k] + r[k];
            }
            if (!project1<kShape>(g, a, b, q, 0.5f * h)) {
                q[0] = x[0];
                q[1] = x[1];
                q[2] = x[2];
            }
            ty = V2M_INTERFACE;
            st.pb = b;
        } else if (sec != V2M_NOLAB && snap > 0.0f) {
            // psi_grad(a, sec) at q; on the cell the ranking located (the same cell psi_grad4 finds)
            const float4 r = ranked ? psi_grad_on(g, oc, a, sec) : psi_grad4<kShape>(g, a, sec, q[0], q[1], q[2]);
            const float gq[3] = { r.x, r.y, r.z };
            const float v = r.w;
            const float gn = sqrtf(gq[0] * gq[0] + gq[1] * gq[1] + gq[2] * gq[2]);
            if (gn > 1e-9f && v / gn < snap * h && project1<kShape>(g, a, sec, q, 1.2f * snap * h)) {
                ty = V2M_INTERFACE;
                b = sec;
                st.pb = sec;
            }
        }
    } else if (ty == V2M_INTERFACE) {
        // tangential(p, s), then project1(q, h / 2) through one psi cache
        PsiCache pc = psi_cache_empty();
        {
            const float4 r4 = psi_grad4_c<kShape>(g, a, b, p[0], p[1], p[2], pc);
            const float gr[3] = { r4.x, r4.y, r4.z };
            const float gn2 = gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2];
            if (!(gn2 < 1e-12f)) {
                const float vn = (s[0] * gr[0] + s[1] * gr[1] + s[2] * gr[2]) / gn2;
                for (int k = 0; k < 3; ++k) {
                    s[k] -= vn * gr[k];
                }
            }
        }
        for (int k = 0; k < 3; ++k) {
            q[k] = p[k] + s[k];
        }
        const float4 pr = project1v<kShape>(g, a, b, q[0], q[1], q[2], 0.5f * h, pc);
        if (pr.w == 0.0f) {
            return 0.0f;
        }
        q[0] = pr.x;
        q[1] = pr.y;
        q[2] = pr.z;
    } else {
        float g1[3], g2[3], td[3];
        psi_grad<kShape>(g, a, b, p[0], p[1], p[2], g1);
        psi_grad<kShape>(g, a, c, p[0], p[1], p[2], g2);
        td[0] = g1[1] * g2[2] - g1[2] * g2[1];
        td[1] = g1[2] * g2[0] - g1[0] * g2[2];
        td[2] = g1[0] * g2[1] - g1[1] * g2[0];
        const float tl2 = td[0] * td[0] + td[1] * td[1] + td[2] * td[2];
        const float stp = tl2 > 1e-20f ? (s[0] * td[0] + s[1] * td[1] + s[2] * td[2]) / tl2 : 0.0f;
        for (int k = 0; k < 3; ++k) {
            q[k] = p[k] + stp * td[k];
        }
        if (!project2<kShape>(g, a, b, c, q, 0.5f * h)) {
            return 0.0f;
        }
    }
    // an interface node meeting a third label joins the junction curve
    // (third_and_valid also gives valid_on's answer for q as an INTERFACE node)
    int valid_here = -1;
    if (ty == V2M_INTERFACE) {
        const int2 tv = third_and_valid<kShape>(g, a, b, q[0], q[1], q[2]);
        const int cc = tv.x;
        valid_here = tv.y;
        if (cc != V2M_NOLAB) {
            float r[3] = { q[0], q[1], q[2] };
            if (project2<kShape>(g, a, b, cc, r, 0.5f * h)) {
                q[0] = r[0];
                q[1] = r[1];
                q[2] = r[2];
                ty = V2M_JUNCTION;
                st.pc = cc;
            }
        }
    }
    // safety net: a displacement beyond the step cap plus the projection reach (or NaN) stays
    {
        const float lim = (maxstep + fmaxf(snap, 0.5f)) * h;
        const float m2 = (q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) + (q[2] - p[2]) * (q[2] - p[2]);
        if (!(m2 <= lim * lim)) {
            if (ty_in == V2M_INTERIOR) {
                st.pb = V2M_NOLAB;
            }
            return 0.0f;
        }
    }
    // refuse a move onto an invalid branch of the constraint
    if (ty != V2M_INTERIOR &&
        !(ty == V2M_INTERFACE && valid_here >= 0 ? valid_here
                                                  : valid_on<kShape>(g, a, st.pb, ty >= V2M_JUNCTION ? st.pc : V2M_NOLAB, q))) {
        if (ty == V2M_INTERFACE || ty_in == V2M_INTERIOR) {
            const int cc = third_label<kShape>(g, a, st.pb, q);
            float r[3] = { q[0], q[1], q[2] };
            if (cc != V2M_NOLAB && project2<kShape>(g, a, st.pb, cc, r, 0.5f * h) && valid_on<kShape>(g, a, st.pb, cc, r)) {
                q[0] = r[0];
                q[1] = r[1];
                q[2] = r[2];
                ty = V2M_JUNCTION;
                st.pc = cc;
            } else {
                // the node keeps its old type (an interior one drops its partner)
                if (ty_in == V2M_INTERIOR) {
                    st.pb = V2M_NOLAB;
                }
                return 0.0f;
            }
        } else {
            return 0.0f;
        }
    }
    const float mv = sqrtf((q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) + (q[2] - p[2]) * (q[2] - p[2]));
    st.p[0] = q[0];
    st.p[1] = q[1];
    st.p[2] = q[2];
    st.ty = ty;
    st.hn = size_at(g, hmode, q[0], q[1], q[2]);
    return mv / h;
}

}  // namespace
}  // namespace v2m
