// v2m_seed.cu -- seeding on the device: the graded HCP lattice, its
// classification onto interfaces and junction curves, the junction-line seeds and
// the corner nodes of tn::seed_cpu (src/v2m_particles.cpp:637-726, 75-244; the
// bodies src/opencl/v2m_seed_body.cl:420-596, 603-748 and
// src/opencl/v2m_particle_body.cl:302-356).
//
// Every stage is count -> scan -> fill over voxels, nodes or grid vertices, so
// the nodes come out in the reference's order; the point queries are the
// relaxation's own (v2m_field.cuh), so the positions, labels, types and partner
// labels are the reference's bit for bit. The junction seeds are deduplicated by
// a stable two-pass radix sort of their keys (the reference sorts them with
// std::sort by key, then vertex), and the lattice nodes near a kept seed are
// dropped through a sorted uniform hash of the seeds.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <string>
#include <utility>
#include <vector>

#include "v2m_field.cuh"
#include "v2m_kernels.h"

namespace v2m {

namespace {

constexpr int kSeedThreads = 256;

__device__ __forceinline__ int seed_level(int grade, int nseed) {
    return nseed <= 1 ? 0 : (int)floorf((float)grade * (float)(nseed - 1) / 255.0f + 0.5f);
}

// HCP point (i, j, k) of spacing s (src/opencl/v2m_seed_body.cl:424-429)
__device__ __forceinline__ void hcp_point(float s, int i, int j, int k, float* p) {
    const float dy = s * 0.8660254f, dz = s * 0.8164966f;
    p[0] = i * s + ((j & 1) ? 0.5f * s : 0.0f) + ((k & 1) ? 0.5f * s : 0.0f);
    p[1] = j * dy + ((k & 1) ? dy / 3.0f : 0.0f);
    p[2] = k * dz;
}

// The lattice points of voxel v's seed level inside its box whose label is not
// the exterior: counted (P == nullptr) or written from `out` on
// (src/opencl/v2m_seed_body.cl:452-500).
template <bool kShape>
__device__ int seed_voxel(const DGrid& g, const uint8_t* __restrict__ grade, const float* __restrict__ spacing,
                          int nseed, int voxmode, int i, int j, int k, float* P, uint16_t* lab, int out) {
    const size_t v = i + (size_t)g.nx * (j + (size_t)g.ny * k);
    if (__ldg(g.L + v) == 0) {
        return 0;
    }
    const float s = __ldg(spacing + seed_level(__ldg(grade + v), nseed));
    const float dy = s * 0.8660254f, dz = s * 0.8164966f;
    const float x0 = (i - 0.5f) * g.vx, x1 = (i + 0.5f) * g.vx;
    const float y0 = (j - 0.5f) * g.vy, y1 = (j + 0.5f) * g.vy;
    const float z0 = (k - 0.5f) * g.vz, z1 = (k + 0.5f) * g.vz;
    int n = 0;
    const int k0 = (int)ceilf(z0 / dz), k1 = (int)ceilf(z1 / dz);
    for (int kk = k0; kk < k1; ++kk) {
        const float oy = (kk & 1) ? dy / 3.0f : 0.0f;
        const int j0 = (int)ceilf((y0 - oy) / dy), j1 = (int)ceilf((y1 - oy) / dy);
        for (int jj = j0; jj < j1; ++jj) {
            const float ox = ((jj & 1) ? 0.5f * s : 0.0f) + ((kk & 1) ? 0.5f * s : 0.0f);
            const int i0 = (int)ceilf((x0 - ox) / s), i1 = (int)ceilf((x1 - ox) / s);
            for (int ii = i0; ii < i1; ++ii) {
                float p[3];
                hcp_point(s, ii, jj, kk, p);
                int sec;
                float mg;
                const int l = owner_label<kShape>(g, voxmode, p[0], p[1], p[2], &sec, &mg);
                if (l == 0 || l == V2M_NOLAB) {
                    continue;
                }
                if (P) {
                    P[3 * (size_t)(out + n)] = p[0];
                    P[3 * (size_t)(out + n) + 1] = p[1];
                    P[3 * (size_t)(out + n) + 2] = p[2];
                    lab[out + n] = (uint16_t)l;
                }
                ++n;
            }
        }
    }
    return n;
}

// cnt[v + 1] = the voxel's count (write == 0); the points at cnt[v] (write == 1,
// cnt scanned)
template <bool kShape>
__global__ void __launch_bounds__(kSeedThreads) k_seed_voxels(DGrid g, const uint8_t* __restrict__ grade,
                                                            const float* __restrict__ spacing, int nseed, int voxmode,
                                                            int* __restrict__ cnt, int write, float* __restrict__ P,
                                                            uint16_t* __restrict__ lab) {
    const int64_t nv = (int64_t)g.nx * g.ny * g.nz;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(v % g.nx), j = (int)((v / g.nx) % g.ny), k = (int)(v / ((int64_t)g.nx * g.ny));
        if (!write) {
            cnt[v + 1] = seed_voxel<kShape>(g, grade, spacing, nseed, voxmode, i, j, k, nullptr, nullptr, 0);
        } else if (cnt[v + 1] != cnt[v]) {
            seed_voxel<kShape>(g, grade, spacing, nseed, voxmode, i, j, k, P, lab, cnt[v]);
        }
    }
}

// Node i after seeding: projected onto its interface within half a spacing
// (INTERFACE), onto a junction curve where a third label competes (JUNCTION);
// only the lower label's nodes of an internal interface are projected
// (src/opencl/v2m_seed_body.cl:509-596).
template <bool kShape>
__global__ void __launch_bounds__(kSeedThreads) k_seed_classify(DGrid g, int n, float* __restrict__ P,
                                                              const uint16_t* __restrict__ lab, uint8_t* __restrict__ typ,
                                                              uint16_t* __restrict__ part) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float p[3] = { P[3 * (size_t)i], P[3 * (size_t)i + 1], P[3 * (size_t)i + 2] };
        typ[i] = V2M_INTERIOR;
        part[2 * (size_t)i] = part[2 * (size_t)i + 1] = V2M_NOLAB;
        const int a = lab[i];
        LabList ll;
        const int nl = labels_near(g, p[0], p[1], p[2], ll);
        if (nl < 2) {
            continue;
        }
        int b = V2M_NOLAB;
        float pb = -1.0f;
        for (int s = 0; s < nl; ++s) {
            const int l = ll.get(s);
            if (l != a) {
                const float v = phi_point<kShape>(g, l, p[0], p[1], p[2]);
                if (v > pb) {
                    pb = v;
                    b = l;
                }
            }
        }
        if (b == V2M_NOLAB || (b != 0 && b < a)) {
            continue;
        }
        int vi = (int)floorf(p[0] / g.vx + 0.5f), vj = (int)floorf(p[1] / g.vy + 0.5f), vk = (int)floorf(p[2] / g.vz + 0.5f);
        vi = vi < 0 ? 0 : (vi >= g.nx ? g.nx - 1 : vi);   // (inside for every lattice point)
        vj = vj < 0 ? 0 : (vj >= g.ny ? g.ny - 1 : vj);
        vk = vk < 0 ? 0 : (vk >= g.nz ? g.nz - 1 : vk);
        const float hs = __ldg(g.hvox + vi + (size_t)g.nx * (vj + (size_t)g.ny * vk));
        float gr[3];
        const float v = psi_grad<kShape>(g, a, b, p[0], p[1], p[2], gr);
        const float gn = sqrtf(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
        if (gn < 1e-9f || fabsf(v) / gn > 0.5f * hs) {
            continue;
        }
        float q[3] = { p[0], p[1], p[2] };
        if (!project1<kShape>(g, a, b, q, 0.6f * hs)) {
            continue;
        }
        typ[i] = V2M_INTERFACE;
        part[2 * (size_t)i] = (uint16_t)b;
        int c = V2M_NOLAB;
        float pc = -1.0f;
        const float pa = phi_point<kShape>(g, a, q[0], q[1], q[2]);
        for (int s = 0; s < nl; ++s) {
            const int l = ll.get(s);
            if (l != a && l != b) {
                const float w = phi_point<kShape>(g, l, q[0], q[1], q[2]);
                if (w > pc) {
                    pc = w;
                    c = l;
                }
            }
        }
        if (c != V2M_NOLAB && pc > 0.5f * pa) {
            float r[3] = { q[0], q[1], q[2] };
            if (project2<kShape>(g, a, b, c, r, 0.5f * hs)) {
                q[0] = r[0];
                q[1] = r[1];
                q[2] = r[2];
                typ[i] = V2M_JUNCTION;
                part[2 * (size_t)i + 1] = (uint16_t)c;
            }
        }
        P[3 * (size_t)i] = q[0];
        P[3 * (size_t)i + 1] = q[1];
        P[3 * (size_t)i + 2] = q[2];
    }
}

// The distinct labels of the 8 voxels around grid vertex (i, j, k), in first-seen
// order (src/opencl/v2m_seed_body.cl:611-629)
__device__ __forceinline__ int vertex_nlab(const DGrid& g, int i, int j, int k, int* labs) {
    int n = 0;
    for (int m = 0; m < 8; ++m) {
        const int l = label_at(g, i + (m & 1), j + ((m >> 1) & 1), k + (m >> 2));
        int seen = 0;
        for (int x = 0; x < n; ++x) {
            seen |= labs[x] == l;
        }
        if (!seen) {
            labs[n++] = l;
        }
    }
    return n;
}

__device__ __forceinline__ void vertex_ijk(const DGrid& g, int64_t v, int& i, int& j, int& k) {
    const int vx1 = g.nx + 1, vy1 = g.ny + 1;
    i = (int)(v % vx1) - 1;
    j = (int)((v / vx1) % vy1) - 1;
    k = (int)(v / ((int64_t)vx1 * vy1)) - 1;
}

__device__ __forceinline__ float det3(const float M[3][3]) {
    return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
}

// A CORNER node at a grid vertex where >= 4 labels meet, kept at the local
// minimum of a cluster of such vertices; its position the Newton solution of the
// three psi constraints when within half a voxel (src/opencl/v2m_seed_body.cl:631-748).
template <bool kShape>
__device__ int corner_vertex(const DGrid& g, int i, int j, int k, bool write, float* P, uint16_t* lab, uint8_t* typ,
                             uint16_t* part, uint16_t* part3, int out) {
    int labs[8];
    const int n = vertex_nlab(g, i, j, k, labs);
    if (n < 4) {
        return 0;
    }
    for (int dz = -1; dz <= 1; ++dz) {
        for (int dy = -1; dy <= 1; ++dy) {
            for (int dx = -1; dx <= 1; ++dx) {
                if (dz < 0 || (dz == 0 && (dy < 0 || (dy == 0 && dx < 0)))) {
                    int l2[8];
                    if (vertex_nlab(g, i + dx, j + dy, k + dz, l2) >= 4) {
                        return 0;
                    }
                }
            }
        }
    }
    if (!write) {
        return 1;
    }
    float x[3] = { (i + 0.5f) * g.vx, (j + 0.5f) * g.vy, (k + 0.5f) * g.vz };
    float ph[8];
    for (int s = 0; s < n; ++s) {
        ph[s] = phi_point<kShape>(g, labs[s], x[0], x[1], x[2]);
    }
    for (int s = 0; s < n; ++s) {   // labels by phi, descending (the reference's exchange order)
        for (int t = s + 1; t < n; ++t) {
            if (ph[t] > ph[s]) {
                const float f = ph[s];
                ph[s] = ph[t];
                ph[t] = f;
                const int l = labs[s];
                labs[s] = labs[t];
                labs[t] = l;
            }
        }
    }
    int ia = 0;
    while (ia < 4 && labs[ia] == 0) {
        ++ia;
    }
    const int a = labs[ia];
    int o[3], no = 0;
    for (int s = 0; s < 4; ++s) {
        if (s != ia) {
            o[no++] = labs[s];
        }
    }
    float q[3] = { x[0], x[1], x[2] };
    int ok = 1;
    for (int it = 0; it < 5 && ok; ++it) {
        float J[3][3], v[3];
        for (int r = 0; r < 3; ++r) {
            v[r] = psi_grad<kShape>(g, a, o[r], q[0], q[1], q[2], J[r]);
        }
        const float det = det3(J);
        if (fabsf(det) < 1e-12f) {
            ok = 0;
            break;
        }
        float dlt[3];
        for (int c = 0; c < 3; ++c) {   // Cramer: J dlt = -v
            float M[3][3];
            for (int r = 0; r < 3; ++r) {
                for (int cc = 0; cc < 3; ++cc) {
                    M[r][cc] = cc == c ? -v[r] : J[r][cc];
                }
            }
            dlt[c] = det3(M) / det;
        }
        for (int c = 0; c < 3; ++c) {
            q[c] += dlt[c];
        }
    }
    const float ex = (q[0] - x[0]) / g.vx, ey = (q[1] - x[1]) / g.vy, ez = (q[2] - x[2]) / g.vz;
    if (ok && ex * ex + ey * ey + ez * ez <= 0.25f) {
        x[0] = q[0];
        x[1] = q[1];
        x[2] = q[2];
    }
    P[3 * (size_t)out] = x[0];
    P[3 * (size_t)out + 1] = x[1];
    P[3 * (size_t)out + 2] = x[2];
    lab[out] = (uint16_t)a;
    typ[out] = V2M_CORNER;
    part[2 * (size_t)out] = (uint16_t)o[0];
    part[2 * (size_t)out + 1] = (uint16_t)o[1];
    part3[out] = (uint16_t)o[2];
    return 1;
}

template <bool kShape>
__global__ void __launch_bounds__(kSeedThreads) k_seed_corners(DGrid g, int* __restrict__ cnt, int write, int out0,
                                                             float* __restrict__ P, uint16_t* __restrict__ lab,
                                                             uint8_t* __restrict__ typ, uint16_t* __restrict__ part,
                                                             uint16_t* __restrict__ part3) {
    const int64_t nvert = (int64_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvert; v += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        vertex_ijk(g, v, i, j, k);
        if (!write) {
            cnt[v + 1] = corner_vertex<kShape>(g, i, j, k, false, nullptr, nullptr, nullptr, nullptr, nullptr, 0);
        } else if (cnt[v + 1] != cnt[v]) {
            corner_vertex<kShape>(g, i, j, k, true, P, lab, typ, part, part3, out0 + cnt[v]);
        }
    }
}

// A junction-line candidate at a grid vertex where exactly 3 labels meet,
// projected onto the a|b|c curve within a voxel and valid there; its key is its
// seed level and its cell of jseed x the level's spacing
// (src/opencl/v2m_particle_body.cl:302-356).
template <bool kShape>
__device__ int junction_vertex(const DGrid& g, const uint8_t* __restrict__ grade, const float* __restrict__ spacing,
                               int nseed, float cellfac, int i, int j, int k, float* x, int* lab3, int* key) {
    int labs[8];
    const int n = vertex_nlab(g, i, j, k, labs);
    if (n != 3) {
        return 0;
    }
    x[0] = (i + 0.5f) * g.vx;
    x[1] = (j + 0.5f) * g.vy;
    x[2] = (k + 0.5f) * g.vz;
    int a = -1;
    float pa = -1.0f;
    for (int s = 0; s < 3; ++s) {
        if (labs[s] != 0) {
            const float f = phi_point<kShape>(g, labs[s], x[0], x[1], x[2]);
            if (f > pa) {
                pa = f;
                a = labs[s];
            }
        }
    }
    int o[2], no = 0;
    for (int s = 0; s < 3; ++s) {
        if (labs[s] != a) {
            o[no++] = labs[s];
        }
    }
    const float vmin = fminf(fminf(g.vx, g.vy), g.vz);
    if (!project2<kShape>(g, a, o[0], o[1], x, vmin) || !valid_on<kShape>(g, a, o[0], o[1], x)) {
        return 0;
    }
    const int vi = (int)floorf(x[0] / g.vx + 0.5f), vj = (int)floorf(x[1] / g.vy + 0.5f), vk = (int)floorf(x[2] / g.vz + 0.5f);
    if (vi < 0 || vj < 0 || vk < 0 || vi >= g.nx || vj >= g.ny || vk >= g.nz) {
        return 0;
    }
    const int lev = seed_level(__ldg(grade + vi + (size_t)g.nx * (vj + (size_t)g.ny * vk)), nseed);
    const float c = cellfac * __ldg(spacing + lev);
    lab3[0] = a;
    lab3[1] = o[0];
    lab3[2] = o[1];
    key[0] = lev;
    key[1] = (int)floorf(x[0] / c);
    key[2] = (int)floorf(x[1] / c);
    key[3] = (int)floorf(x[2] / c);
    return 1;
}

// junction candidates: counted, then written with their two sort keys -- hi:
// level and cell (18 bits per cell coordinate, biased), lo: the sorted label
// triple -- and the positions and labels
constexpr int kCellBits = 18;
constexpr int kCellBias = 1 << (kCellBits - 1);

template <bool kShape>
__global__ void __launch_bounds__(kSeedThreads) k_seed_junctions(DGrid g, const uint8_t* __restrict__ grade,
                                                               const float* __restrict__ spacing, int nseed,
                                                               float cellfac, int* __restrict__ cnt, int write,
                                                               float* __restrict__ cx, int* __restrict__ clab,
                                                               unsigned long long* __restrict__ khi,
                                                               unsigned long long* __restrict__ klo,
                                                               int* __restrict__ err) {
    const int64_t nvert = (int64_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvert; v += (int64_t)gridDim.x * blockDim.x) {
        if (write && cnt[v + 1] == cnt[v]) {
            continue;
        }
        int i, j, k, l3[3], key[4];
        float x[3];
        vertex_ijk(g, v, i, j, k);
        const int f = junction_vertex<kShape>(g, grade, spacing, nseed, cellfac, i, j, k, x, l3, key);
        if (!write) {
            cnt[v + 1] = f;
            continue;
        }
        const int e = cnt[v];
        cx[3 * (size_t)e] = x[0];
        cx[3 * (size_t)e + 1] = x[1];
        cx[3 * (size_t)e + 2] = x[2];
        clab[3 * (size_t)e] = l3[0];
        clab[3 * (size_t)e + 1] = l3[1];
        clab[3 * (size_t)e + 2] = l3[2];
        int t0 = l3[0], t1 = l3[1], t2 = l3[2];   // the triple sorted
        if (t0 > t1) {
            const int t = t0;
            t0 = t1;
            t1 = t;
        }
        if (t1 > t2) {
            const int t = t1;
            t1 = t2;
            t2 = t;
        }
        if (t0 > t1) {
            const int t = t0;
            t0 = t1;
            t1 = t;
        }
        unsigned long long hi = (unsigned long long)key[0];
        for (int a = 1; a < 4; ++a) {
            const int b = key[a] + kCellBias;
            if (b < 0 || b >= (1 << kCellBits)) {
                atomicExch(err, 1);
            }
            hi = (hi << kCellBits) | (unsigned long long)(b & ((1 << kCellBits) - 1));
        }
        khi[e] = hi;
        klo[e] = ((unsigned long long)t0 << 32) | ((unsigned long long)t1 << 16) | (unsigned long long)t2;
    }
}

// After the stable sort (by lo, then hi): the first of each key group is kept
__global__ void k_seed_jfirst(int m, const unsigned long long* __restrict__ khi, const unsigned long long* __restrict__ klo,
                              int* __restrict__ flag) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        flag[e + 1] = e == 0 || khi[e] != khi[e - 1] || klo[e] != klo[e - 1];
    }
}

// the kept seeds in key order, and their cells of the drop hash
struct DropHash {
    float cell, vs[3];
    int hd[3];
};

__device__ __forceinline__ long long drop_key(const DropHash& H, const float* p, int* c3) {
    for (int e = 0; e < 3; ++e) {
        const int c = (int)floorf((p[e] + H.vs[e]) / H.cell);
        c3[e] = min(H.hd[e] - 1, max(0, c));
    }
    return c3[0] + H.hd[0] * (c3[1] + (long long)H.hd[1] * c3[2]);
}

__global__ void k_seed_jkeep(int m, const int* __restrict__ order, const int* __restrict__ flag,
                             const float* __restrict__ cx, const int* __restrict__ clab, DropHash H,
                             float* __restrict__ sx, int* __restrict__ slab, long long* __restrict__ bkey,
                             int* __restrict__ bidx) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        if (flag[e + 1] == flag[e]) {
            continue;
        }
        const int s = flag[e], c = order[e];
        float p[3] = { cx[3 * (size_t)c], cx[3 * (size_t)c + 1], cx[3 * (size_t)c + 2] };
        sx[3 * (size_t)s] = p[0];
        sx[3 * (size_t)s + 1] = p[1];
        sx[3 * (size_t)s + 2] = p[2];
        slab[3 * (size_t)s] = clab[3 * (size_t)c];
        slab[3 * (size_t)s + 1] = clab[3 * (size_t)c + 1];
        slab[3 * (size_t)s + 2] = clab[3 * (size_t)c + 2];
        int c3[3];
        bkey[s] = drop_key(H, p, c3);
        bidx[s] = s;
    }
}

// a lattice node within 0.4 h of a kept seed is dropped; keep[i + 1] = kept
__global__ void __launch_bounds__(kSeedThreads) k_seed_jdrop(DGrid g, int n, const float* __restrict__ P,
                                                           const uint8_t* __restrict__ typ, DropHash H, int ns,
                                                           const long long* __restrict__ bkey,
                                                           const int* __restrict__ bidx, const float* __restrict__ sx,
                                                           int* __restrict__ keep) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int drop = 0;
        if (typ[i] != V2M_CORNER) {
            const float p[3] = { P[3 * (size_t)i], P[3 * (size_t)i + 1], P[3 * (size_t)i + 2] };
            const float h = size_at(g, 0, p[0], p[1], p[2]);
            int c3[3];
            drop_key(H, p, c3);
            for (int dz = -1; dz <= 1 && !drop; ++dz) {
                for (int dy = -1; dy <= 1 && !drop; ++dy) {
                    for (int dx = -1; dx <= 1 && !drop; ++dx) {
                        const int x = c3[0] + dx, y = c3[1] + dy, z = c3[2] + dz;
                        if (x < 0 || y < 0 || z < 0 || x >= H.hd[0] || y >= H.hd[1] || z >= H.hd[2]) {
                            continue;
                        }
                        const long long kk = x + H.hd[0] * (y + (long long)H.hd[1] * z);
                        int lo = 0, hi = ns;   // first entry with key >= kk
                        while (lo < hi) {
                            const int mid = (lo + hi) >> 1;
                            if (bkey[mid] < kk) {
                                lo = mid + 1;
                            } else {
                                hi = mid;
                            }
                        }
                        for (int e = lo; e < ns && bkey[e] == kk; ++e) {
                            const int s = bidx[e];
                            const float ex = p[0] - sx[3 * (size_t)s], ey = p[1] - sx[3 * (size_t)s + 1],
                                        ez = p[2] - sx[3 * (size_t)s + 2];
                            if (ex * ex + ey * ey + ez * ez < 0.16f * h * h) {
                                drop = 1;
                                break;
                            }
                        }
                    }
                }
            }
        }
        keep[i + 1] = !drop;
    }
}

// the kept lattice nodes compacted, then the seeds appended (JUNCTION nodes)
__global__ void k_seed_jcompact(int n, const int* __restrict__ keep, const float* __restrict__ P,
                                const uint16_t* __restrict__ lab, const uint8_t* __restrict__ typ,
                                const uint16_t* __restrict__ part, int ns, const float* __restrict__ sx,
                                const int* __restrict__ slab, float* __restrict__ P2, uint16_t* __restrict__ lab2,
                                uint8_t* __restrict__ typ2, uint16_t* __restrict__ part2) {
    const int nk = keep[n];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + ns; i += gridDim.x * blockDim.x) {
        if (i < n) {
            if (keep[i + 1] == keep[i]) {
                continue;
            }
            const int o = keep[i];
            P2[3 * (size_t)o] = P[3 * (size_t)i];
            P2[3 * (size_t)o + 1] = P[3 * (size_t)i + 1];
            P2[3 * (size_t)o + 2] = P[3 * (size_t)i + 2];
            lab2[o] = lab[i];
            typ2[o] = typ[i];
            part2[2 * (size_t)o] = part[2 * (size_t)i];
            part2[2 * (size_t)o + 1] = part[2 * (size_t)i + 1];
        } else {
            const int s = i - n, o = nk + s;
            P2[3 * (size_t)o] = sx[3 * (size_t)s];
            P2[3 * (size_t)o + 1] = sx[3 * (size_t)s + 1];
            P2[3 * (size_t)o + 2] = sx[3 * (size_t)s + 2];
            lab2[o] = (uint16_t)slab[3 * (size_t)s];
            typ2[o] = V2M_JUNCTION;
            part2[2 * (size_t)o] = (uint16_t)slab[3 * (size_t)s + 1];
            part2[2 * (size_t)o + 1] = (uint16_t)slab[3 * (size_t)s + 2];
        }
    }
}

// ---- 5. shape features (tn::seed_cpu's add_feature_nodes, src/v2m_particles.cpp:298-623) ----
// The curves' geometry (sample points, bisection midpoints, arc length and the
// resampled points) is computed on the host, in the reference's float and double
// arithmetic and with the host's cos / sin for circles; every point query (the
// labels round a point, h at a point) runs here on the device, through the
// relaxation's own field code.

// the labels round each point x: x and six axis samples at 0.2 h (mask_at)
template <bool kShape>
__global__ void __launch_bounds__(kSeedThreads) k_feat_mask(DGrid g, int n, const float* __restrict__ X,
                                                           unsigned long long* __restrict__ mask) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const float x[3] = { X[3 * (size_t)t], X[3 * (size_t)t + 1], X[3 * (size_t)t + 2] };
        const float e = 0.2f * size_at(g, 0, x[0], x[1], x[2]);
        const float dir[7][3] = { { 0, 0, 0 }, { 1, 0, 0 }, { -1, 0, 0 }, { 0, 1, 0 }, { 0, -1, 0 }, { 0, 0, 1 }, { 0, 0, -1 } };
        unsigned long long m = 0ull;
#pragma unroll 1
        for (int d = 0; d < 7; ++d) {
            int sec;
            float mg;
            const int l = owner_label<kShape>(g, 0, x[0] + e * dir[d][0], x[1] + e * dir[d][1], x[2] + e * dir[d][2],
                                              &sec, &mg);
            m |= l < 64 ? 1ull << l : 0ull;
        }
        mask[t] = m;
    }
}

// h at each point (v2m_h_at: the nearest voxel's)
__global__ void k_feat_hat(DGrid g, int n, const float* __restrict__ X, float* __restrict__ out) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        out[t] = size_at(g, 0, X[3 * (size_t)t], X[3 * (size_t)t + 1], X[3 * (size_t)t + 2]);
    }
}

constexpr int kFeatWarps = 4;
constexpr int kFeatMaxDirs = 160;

// Each candidate's labels round it: the labels at 0.25 h along the ndir
// directions, counted; up to four of them in the order (tissue labels first,
// then by count, descending, then by label), with their number (0 when the
// point lies outside the grid or inside one region). One warp per candidate:
// the lanes sample the directions, lane 0 ranks the labels.
template <bool kShape>
__global__ void __launch_bounds__(32 * kFeatWarps) k_feat_classify(DGrid g, int n, const float* __restrict__ X,
                                                                  const float* __restrict__ dirs, int ndir,
                                                                  int4* __restrict__ ls, int* __restrict__ nls,
                                                                  float* __restrict__ hx) {
    __shared__ int lb[kFeatWarps][kFeatMaxDirs];
    __shared__ int dl[kFeatWarps][kFeatMaxDirs], dc[kFeatWarps][kFeatMaxDirs];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nw = gridDim.x * kFeatWarps;
    for (int c = blockIdx.x * kFeatWarps + w; c < n; c += nw) {
        const float x[3] = { X[3 * (size_t)c], X[3 * (size_t)c + 1], X[3 * (size_t)c + 2] };
        const float h = size_at(g, 0, x[0], x[1], x[2]);
        const bool out = x[0] < 0 || x[1] < 0 || x[2] < 0 || x[0] > (g.nx - 1) * g.vx || x[1] > (g.ny - 1) * g.vy ||
                         x[2] > (g.nz - 1) * g.vz;
        if (lane == 0) {
            hx[c] = h;
        }
        if (out) {
            if (lane == 0) {
                nls[c] = 0;
                ls[c] = make_int4(V2M_NOLAB, V2M_NOLAB, V2M_NOLAB, V2M_NOLAB);
            }
            continue;
        }
        const float e = 0.25f * h;
        for (int d = lane; d < ndir; d += 32) {
            int sec;
            float mg;
            lb[w][d] = owner_label<kShape>(g, 0, x[0] + e * dirs[3 * d], x[1] + e * dirs[3 * d + 1],
                                           x[2] + e * dirs[3 * d + 2], &sec, &mg);
        }
        __syncwarp();
        if (lane == 0) {
            int nd = 0;   // distinct labels and their counts
            for (int d = 0; d < ndir; ++d) {
                const int l = lb[w][d];
                int q = 0;
                while (q < nd && dl[w][q] != l) {
                    ++q;
                }
                if (q == nd) {
                    dl[w][nd] = l;
                    dc[w][nd] = 0;
                    ++nd;
                }
                ++dc[w][q];
            }
            int L[4] = { V2M_NOLAB, V2M_NOLAB, V2M_NOLAB, V2M_NOLAB };
            int m = 0;
            if (nd >= 2) {
                // the first four in (label 0 last, count descending, label ascending) order
                for (; m < 4 && m < nd; ++m) {
                    int best = -1;
                    for (int q = 0; q < nd; ++q) {
                        if (dc[w][q] < 0) {
                            continue;
                        }
                        if (best < 0) {
                            best = q;
                            continue;
                        }
                        const int lq = dl[w][q], lb_ = dl[w][best];
                        const bool zq = lq == 0, zb = lb_ == 0;
                        const bool before = zq != zb ? !zq
                                                     : (dc[w][q] != dc[w][best] ? dc[w][q] > dc[w][best] : lq < lb_);
                        if (before) {
                            best = q;
                        }
                    }
                    L[m] = dl[w][best];
                    dc[w][best] = -1;
                }
                if (m > 0 && L[0] == 0) {
                    m = 0;   // (no tissue round it)
                }
            }
            ls[c] = make_int4(L[0], L[1], L[2], L[3]);
            nls[c] = m;
        }
        __syncwarp();
    }
}

// the seeds within 0.4 h of a kept feature node are dropped, found through the
// reference's uniform cells of side `cell` (keys: the sorted packed cells of
// the feature nodes); keep[i + 1] = kept
constexpr long long kFeatCellOff = 1ll << 20;

__device__ __host__ __forceinline__ bool feat_cell_key(long long i, long long j, long long k, unsigned long long* key) {
    i += kFeatCellOff;
    j += kFeatCellOff;
    k += kFeatCellOff;
    if (i < 0 || j < 0 || k < 0 || i >= 2 * kFeatCellOff || j >= 2 * kFeatCellOff || k >= 2 * kFeatCellOff) {
        return false;
    }
    *key = ((unsigned long long)i << 42) | ((unsigned long long)j << 21) | (unsigned long long)k;
    return true;
}

__global__ void __launch_bounds__(kSeedThreads) k_feat_drop(DGrid g, int n, const float* __restrict__ P, float cell,
                                                          int nk, const unsigned long long* __restrict__ keys,
                                                          const int* __restrict__ kidx, const float* __restrict__ kp,
                                                          int* __restrict__ keep) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float x[3] = { P[3 * (size_t)i], P[3 * (size_t)i + 1], P[3 * (size_t)i + 2] };
        const float r = 0.4f * size_at(g, 0, x[0], x[1], x[2]);
        const long long ci = (long long)floorf(x[0] / cell), cj = (long long)floorf(x[1] / cell),
                        ck = (long long)floorf(x[2] / cell);
        const long long reach = (long long)ceilf(r / cell);
        int drop = 0;
        for (long long a = -reach; a <= reach && !drop; ++a) {
            for (long long b = -reach; b <= reach && !drop; ++b) {
                for (long long c = -reach; c <= reach && !drop; ++c) {
                    unsigned long long kk;
                    if (!feat_cell_key(ci + a, cj + b, ck + c, &kk)) {
                        continue;
                    }
                    int lo = 0, hi = nk;   // first entry with key >= kk
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (keys[mid] < kk) {
                            lo = mid + 1;
                        } else {
                            hi = mid;
                        }
                    }
                    for (int e = lo; e < nk && keys[e] == kk; ++e) {
                        const int k = kidx[e];
                        const float dx = kp[3 * (size_t)k] - x[0], dy = kp[3 * (size_t)k + 1] - x[1],
                                    dz = kp[3 * (size_t)k + 2] - x[2];
                        if (dx * dx + dy * dy + dz * dz < r * r) {
                            drop = 1;
                            break;
                        }
                    }
                }
            }
        }
        keep[i + 1] = !drop;
    }
}

// the kept seeds compacted in order, then the feature nodes appended (CORNER
// nodes: own label the first of their labels, partners the next three)
__global__ void k_feat_compact(int n, const int* __restrict__ keep, const float* __restrict__ P,
                               const uint16_t* __restrict__ lab, const uint8_t* __restrict__ typ,
                               const uint16_t* __restrict__ part, const uint16_t* __restrict__ part3, int nk,
                               const float* __restrict__ kp, const int4* __restrict__ kl, const int* __restrict__ kn,
                               float* __restrict__ P2, uint16_t* __restrict__ lab2, uint8_t* __restrict__ typ2,
                               uint16_t* __restrict__ part2, uint16_t* __restrict__ part32) {
    const int nkeep = keep[n];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + nk; i += gridDim.x * blockDim.x) {
        if (i < n) {
            if (keep[i + 1] == keep[i]) {
                continue;
            }
            const int o = keep[i];
            P2[3 * (size_t)o] = P[3 * (size_t)i];
            P2[3 * (size_t)o + 1] = P[3 * (size_t)i + 1];
            P2[3 * (size_t)o + 2] = P[3 * (size_t)i + 2];
            lab2[o] = lab[i];
            typ2[o] = typ[i];
            part2[2 * (size_t)o] = part[2 * (size_t)i];
            part2[2 * (size_t)o + 1] = part[2 * (size_t)i + 1];
            part32[o] = part3[i];
        } else {
            const int k = i - n, o = nkeep + k;
            const int4 L = kl[k];
            const int m = kn[k];
            P2[3 * (size_t)o] = kp[3 * (size_t)k];
            P2[3 * (size_t)o + 1] = kp[3 * (size_t)k + 1];
            P2[3 * (size_t)o + 2] = kp[3 * (size_t)k + 2];
            lab2[o] = (uint16_t)L.x;
            typ2[o] = V2M_CORNER;
            part2[2 * (size_t)o] = (uint16_t)(m > 1 ? L.y : V2M_NOLAB);
            part2[2 * (size_t)o + 1] = (uint16_t)(m > 2 ? L.z : V2M_NOLAB);
            part32[o] = (uint16_t)(m > 3 ? L.w : V2M_NOLAB);
        }
    }
}

__global__ void k_iota(int n, int* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[i] = i;
    }
}

__global__ void k_gather_u64(int n, const int* __restrict__ idx, const unsigned long long* __restrict__ in,
                             unsigned long long* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[i] = in[idx[i]];
    }
}

unsigned gs_blocks(int64_t items, int sms) {
    const int64_t need = (items + kSeedThreads - 1) / kSeedThreads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * 8));
}

// CUB scratch for one call
struct Scratch {
    cudaStream_t s;
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t need(size_t b) {
        if (b <= bytes) {
            return cudaSuccess;
        }
        if (p) {
            cudaFreeAsync(p, s);
        }
        bytes = b;
        return pool_malloc(&p, b, s);
    }
    ~Scratch() {
        if (p) {
            cudaFreeAsync(p, s);
        }
    }
};

// inclusive scan of cnt[1..n] in place (cnt[0] == 0): cnt[v] = the exclusive start
cudaError_t scan_counts(Scratch& sc, int* cnt, int64_t n) {
    size_t b = 0;
    cudaError_t e = cub::DeviceScan::InclusiveSum(nullptr, b, cnt + 1, cnt + 1, n, sc.s);
    if (e == cudaSuccess) {
        e = sc.need(b);
    }
    if (e == cudaSuccess) {
        e = cub::DeviceScan::InclusiveSum(sc.p, b, cnt + 1, cnt + 1, n, sc.s);
    }
    return e;
}

}  // namespace

// ---- 5. shape features: the host's part -------------------------------------------------
// One feature curve of tn::Grid::feat: 2 a segment (a, b), 3 a circle (centre,
// normal, radius), 4 a polyline (n, then n points). at() is the reference's
// curve point at parameter t in [0, 1] (src/v2m_particles.cpp:347-369), the
// circle's frame its orthonormal pair about the normal (:330-345): the same
// float expressions, in the same order (this file is compiled without
// contraction), with the host's cos / sin.
struct FeatCurve {
    int type = 0;
    const float* q = nullptr;
    float u[3] = { 0, 0, 0 }, w[3] = { 0, 0, 0 };

    FeatCurve(int ty, const float* qq) : type(ty), q(qq) {
        if (type == 3) {
            const float* n = q + 3;
            const float a0 = std::fabs(n[0]) < 0.9f ? 1.0f : 0.0f, a1 = a0 > 0 ? 0.0f : 1.0f;
            u[0] = n[1] * 0 - n[2] * a1;
            u[1] = n[2] * a0 - n[0] * 0;
            u[2] = n[0] * a1 - n[1] * a0;
            const float lu = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
            for (float& x : u) {
                x /= lu;
            }
            w[0] = n[1] * u[2] - n[2] * u[1];
            w[1] = n[2] * u[0] - n[0] * u[2];
            w[2] = n[0] * u[1] - n[1] * u[0];
        }
    }

    void at(float t, float* o) const {
        if (type == 4) {
            const int n = static_cast<int>(q[0]);
            const float uu = t * static_cast<float>(n - 1);
            const int i = std::min(n - 2, std::max(0, static_cast<int>(uu)));
            const float f = uu - static_cast<float>(i);
            for (int a = 0; a < 3; ++a) {
                o[a] = q[1 + 3 * i + a] + f * (q[1 + 3 * (i + 1) + a] - q[1 + 3 * i + a]);
            }
        } else if (type == 2) {
            for (int a = 0; a < 3; ++a) {
                o[a] = q[a] + t * (q[3 + a] - q[a]);
            }
        } else {
            const float th = 6.28318531f * t, c = std::cos(th), sn = std::sin(th);
            for (int a = 0; a < 3; ++a) {
                o[a] = q[a] + q[6] * (c * u[a] + sn * w[a]);
            }
        }
    }
};

// The feature pass over the seeds in B (src/v2m_particles.cpp:304-623): the
// candidates (corners; then where the labels round a curve change, bisected;
// then points spaced by h along each curve), each given the labels round it;
// one kept per 0.3 h in that order (two or more labels); the seeds within 0.4 h
// of a kept one dropped; the kept ones appended as CORNER nodes.
template <bool kShape, class Alloc>
cudaError_t feature_pass(const SeedArgs& A, SeedBuffers& B, Scratch& sc, Alloc& alloc, std::string& err) {
    const DGrid& g = A.g;
    cudaStream_t s = A.stream;
    constexpr int nsamp = 256;
    cudaError_t e;
    // the point queries: masks or sizes of host points, through device buffers
    float* dX = nullptr;
    size_t capX = 0;
    auto points = [&](const std::vector<float>& X) -> cudaError_t {
        const size_t n = X.size() / 3;
        if (n > capX) {
            capX = std::max<size_t>(n, 1024);
            dX = (float*)alloc(sizeof(float) * 3 * capX);
            if (!dX) {
                return cudaErrorMemoryAllocation;
            }
        }
        return cudaMemcpyAsync(dX, X.data(), sizeof(float) * X.size(), cudaMemcpyHostToDevice, s);
    };
    unsigned long long* dM = nullptr;
    size_t capM = 0;
    auto masks = [&](const std::vector<float>& X, std::vector<unsigned long long>& out) -> cudaError_t {
        const int n = (int)(X.size() / 3);
        out.assign((size_t)n, 0ull);
        if (n == 0) {
            return cudaSuccess;
        }
        cudaError_t r = points(X);
        if (r != cudaSuccess) {
            return r;
        }
        if ((size_t)n > capM) {
            capM = std::max<size_t>(n, 1024);
            dM = (unsigned long long*)alloc(8 * capM);
            if (!dM) {
                return cudaErrorMemoryAllocation;
            }
        }
        k_feat_mask<kShape><<<gs_blocks(n, A.sms), kSeedThreads, 0, s>>>(g, n, dX, dM);
        if ((r = cudaMemcpyAsync(out.data(), dM, 8 * (size_t)n, cudaMemcpyDeviceToHost, s)) != cudaSuccess) {
            return r;
        }
        return cudaStreamSynchronize(s);
    };
    auto sizes = [&](const std::vector<float>& X, std::vector<float>& out) -> cudaError_t {
        const int n = (int)(X.size() / 3);
        out.assign((size_t)n, 0.0f);
        if (n == 0) {
            return cudaSuccess;
        }
        cudaError_t r = points(X);
        if (r != cudaSuccess) {
            return r;
        }
        float* dH = (float*)alloc(sizeof(float) * (size_t)n);
        if (!dH) {
            return cudaErrorMemoryAllocation;
        }
        k_feat_hat<<<gs_blocks(n, A.sms), kSeedThreads, 0, s>>>(g, n, dX, dH);
        if ((r = cudaMemcpyAsync(out.data(), dH, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s)) != cudaSuccess) {
            return r;
        }
        return cudaStreamSynchronize(s);
    };
    // the features: corners, then the curves (a polyline needs two points)
    std::vector<float> fp;
    std::vector<FeatCurve> curves;
    for (int64_t k = 0; k < A.nfeat;) {
        const int type = static_cast<int>(A.feat[k]);
        const int64_t len = type == 1 ? 4 : type == 2 ? 7 : type == 3 ? 8
                          : type == 4 && k + 1 < A.nfeat ? 2 + 3 * static_cast<int64_t>(A.feat[k + 1]) : -1;
        if (len < 0 || k + len > A.nfeat || (type == 4 && A.feat[k + 1] < 0)) {
            err = "the feature list is malformed at float " + std::to_string(k);
            return cudaErrorInvalidValue;
        }
        const float* q = A.feat + k + 1;
        if (type == 1) {
            fp.insert(fp.end(), { q[0], q[1], q[2] });
        } else if (type != 4 || q[0] >= 2) {
            curves.emplace_back(type, q);
        }
        k += len;
    }
    const size_t ncv = curves.size();
    // the curves' samples and the labels round them
    std::vector<float> pts(ncv * 3 * (nsamp + 1));
    for (size_t c = 0; c < ncv; ++c) {
        for (int k = 0; k <= nsamp; ++k) {
            curves[c].at(static_cast<float>(k) / nsamp, &pts[3 * (c * (nsamp + 1) + k)]);
        }
    }
    std::vector<unsigned long long> mk;
    if ((e = masks(pts, mk)) != cudaSuccess) {
        return e;
    }
    // where the labels change: 14 bisection steps, every change at once
    struct Job {
        size_t c;
        float lo, hi;
        unsigned long long m0;
    };
    std::vector<Job> jobs;
    for (size_t c = 0; c < ncv; ++c) {
        const unsigned long long* m = &mk[c * (nsamp + 1)];
        for (int k = 1; k <= nsamp; ++k) {
            if (m[k] != m[k - 1]) {
                jobs.push_back({ c, static_cast<float>(k - 1) / nsamp, static_cast<float>(k) / nsamp, m[k - 1] });
            }
        }
    }
    if (!jobs.empty()) {
        std::vector<float> X(3 * jobs.size());
        std::vector<unsigned long long> mm;
        for (int it = 0; it < 14; ++it) {
            for (size_t j = 0; j < jobs.size(); ++j) {
                curves[jobs[j].c].at(0.5f * (jobs[j].lo + jobs[j].hi), &X[3 * j]);
            }
            if ((e = masks(X, mm)) != cudaSuccess) {
                return e;
            }
            for (size_t j = 0; j < jobs.size(); ++j) {
                const float mid = 0.5f * (jobs[j].lo + jobs[j].hi);
                if (mm[j] == jobs[j].m0) {
                    jobs[j].lo = mid;
                } else {
                    jobs[j].hi = mid;
                }
            }
        }
        for (size_t j = 0; j < jobs.size(); ++j) {
            float x[3];
            curves[jobs[j].c].at(0.5f * (jobs[j].lo + jobs[j].hi), x);
            fp.insert(fp.end(), x, x + 3);
        }
    }
    // arc length in units of h, then the regular points
    std::vector<float> mids(ncv * 3 * nsamp);
    for (size_t c = 0; c < ncv; ++c) {
        for (int k = 1; k <= nsamp; ++k) {
            const float* a = &pts[3 * (c * (nsamp + 1) + k - 1)];
            const float* b = &pts[3 * (c * (nsamp + 1) + k)];
            float* m = &mids[3 * (c * nsamp + k - 1)];
            m[0] = 0.5f * (a[0] + b[0]);
            m[1] = 0.5f * (a[1] + b[1]);
            m[2] = 0.5f * (a[2] + b[2]);
        }
    }
    std::vector<float> hm;
    if ((e = sizes(mids, hm)) != cudaSuccess) {
        return e;
    }
    for (size_t c = 0; c < ncv; ++c) {
        const int type = curves[c].type;
        const float* P = &pts[3 * c * (nsamp + 1)];
        std::vector<double> acc(nsamp + 1, 0.0);
        for (int k = 1; k <= nsamp; ++k) {
            const float* a = &P[3 * (k - 1)];
            const float* b = &P[3 * k];
            const float ds = std::sqrt((b[0] - a[0]) * (b[0] - a[0]) + (b[1] - a[1]) * (b[1] - a[1]) +
                                       (b[2] - a[2]) * (b[2] - a[2]));
            acc[k] = acc[k - 1] + ds / std::max(hm[c * nsamp + k - 1], 1e-6f);
        }
        const double per = type == 4 ? 2.0 : 1.0;
        const int ns = std::max(type == 3 ? 6 : 1, static_cast<int>(std::lround(per * acc[nsamp])));
        for (int q = type == 3 || type == 4 ? 0 : 1; q < ns; ++q) {
            const double target = acc[nsamp] * q / ns;
            int k = 1;
            while (k < nsamp && acc[k] < target) {
                ++k;
            }
            const double f = acc[k] > acc[k - 1] ? (target - acc[k - 1]) / (acc[k] - acc[k - 1]) : 0.0;
            for (int a = 0; a < 3; ++a) {
                fp.push_back(static_cast<float>(P[3 * (k - 1) + a] + f * (P[3 * k + a] - P[3 * (k - 1) + a])));
            }
        }
    }
    const int nc = (int)(fp.size() / 3);
    if (nc == 0) {
        return cudaSuccess;
    }
    // the directions round a candidate: 14 axis / diagonal, 128 on a golden spiral
    std::vector<float> dirs = { 1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1,
                                .577f, .577f, .577f, -.577f, .577f, .577f, .577f, -.577f, .577f, .577f, .577f, -.577f,
                                -.577f, -.577f, .577f, -.577f, .577f, -.577f, .577f, -.577f, -.577f, -.577f, -.577f, -.577f };
    for (int i = 0; i < 128; ++i) {
        const double zc = 1 - (2 * i + 1) / 128.0, rr = std::sqrt(std::max(0.0, 1 - zc * zc)), ph = 2.39996322972865 * i;
        dirs.push_back(static_cast<float>(rr * std::cos(ph)));
        dirs.push_back(static_cast<float>(rr * std::sin(ph)));
        dirs.push_back(static_cast<float>(zc));
    }
    const int ndir = (int)(dirs.size() / 3);
    float* dD = (float*)alloc(sizeof(float) * dirs.size());
    float* dF = (float*)alloc(sizeof(float) * fp.size());
    int4* dL = (int4*)alloc(sizeof(int4) * (size_t)nc);
    int* dN = (int*)alloc(sizeof(int) * (size_t)nc);
    float* dHx = (float*)alloc(sizeof(float) * (size_t)nc);
    if (!dD || !dF || !dL || !dN || !dHx) {
        return cudaErrorMemoryAllocation;
    }
    cudaMemcpyAsync(dD, dirs.data(), sizeof(float) * dirs.size(), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dF, fp.data(), sizeof(float) * fp.size(), cudaMemcpyHostToDevice, s);
    k_feat_classify<kShape><<<(unsigned)std::min<int64_t>((nc + kFeatWarps - 1) / kFeatWarps, (int64_t)A.sms * 16),
                              32 * kFeatWarps, 0, s>>>(g, nc, dF, dD, ndir, dL, dN, dHx);
    std::vector<int4> ls((size_t)nc);
    std::vector<int> nls((size_t)nc);
    std::vector<float> hx((size_t)nc);
    cudaMemcpyAsync(ls.data(), dL, sizeof(int4) * (size_t)nc, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(nls.data(), dN, sizeof(int) * (size_t)nc, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hx.data(), dHx, sizeof(float) * (size_t)nc, cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
        return e;
    }
    // one kept per 0.3 h, in candidate order (corners first)
    std::vector<float> keepP;
    std::vector<int4> keepL;
    std::vector<int> keepN;
    for (int c = 0; c < nc; ++c) {
        if (nls[c] < 2) {
            continue;
        }
        const float* x = &fp[3 * (size_t)c];
        const float r = 0.3f * hx[c];
        bool near = false;
        for (size_t k = 0; k < keepP.size() / 3 && !near; ++k) {
            const float dx = keepP[3 * k] - x[0], dy = keepP[3 * k + 1] - x[1], dz = keepP[3 * k + 2] - x[2];
            near = dx * dx + dy * dy + dz * dz < r * r;
        }
        if (!near) {
            keepP.insert(keepP.end(), x, x + 3);
            keepL.push_back(ls[c]);
            keepN.push_back(nls[c]);
        }
    }
    const int nk = (int)keepN.size();
    if (nk == 0) {
        return cudaSuccess;
    }
    // the kept nodes' cells (the reference's hash cells: side 0.4 hmax), sorted
    const float cell = 0.4f * A.hmax > 0 ? 0.4f * A.hmax : 1.0f;
    std::vector<std::pair<unsigned long long, int>> kc((size_t)nk);
    for (int k = 0; k < nk; ++k) {
        unsigned long long key = 0;
        if (!feat_cell_key(static_cast<long long>(std::floor(keepP[3 * (size_t)k] / cell)),
                           static_cast<long long>(std::floor(keepP[3 * (size_t)k + 1] / cell)),
                           static_cast<long long>(std::floor(keepP[3 * (size_t)k + 2] / cell)), &key)) {
            err = "a feature node lies beyond the drop hash's range";
            return cudaErrorInvalidValue;
        }
        kc[(size_t)k] = { key, k };
    }
    std::stable_sort(kc.begin(), kc.end(), [](const std::pair<unsigned long long, int>& a,
                                              const std::pair<unsigned long long, int>& b) { return a.first < b.first; });
    std::vector<unsigned long long> keys((size_t)nk);
    std::vector<int> kidx((size_t)nk);
    for (int k = 0; k < nk; ++k) {
        keys[(size_t)k] = kc[(size_t)k].first;
        kidx[(size_t)k] = kc[(size_t)k].second;
    }
    auto* dK = (unsigned long long*)alloc(8 * (size_t)nk);
    int* dKi = (int*)alloc(sizeof(int) * (size_t)nk);
    float* dKp = (float*)alloc(sizeof(float) * 3 * (size_t)nk);
    int4* dKl = (int4*)alloc(sizeof(int4) * (size_t)nk);
    int* dKn = (int*)alloc(sizeof(int) * (size_t)nk);
    const int n0 = B.n;
    int* keep = (int*)alloc(sizeof(int) * (size_t)(n0 + 1));
    if (!dK || !dKi || !dKp || !dKl || !dKn || !keep) {
        return cudaErrorMemoryAllocation;
    }
    cudaMemcpyAsync(dK, keys.data(), 8 * (size_t)nk, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dKi, kidx.data(), sizeof(int) * (size_t)nk, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dKp, keepP.data(), sizeof(float) * 3 * (size_t)nk, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dKl, keepL.data(), sizeof(int4) * (size_t)nk, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dKn, keepN.data(), sizeof(int) * (size_t)nk, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(keep, 0, sizeof(int), s);
    if (n0 > 0) {
        k_feat_drop<<<gs_blocks(n0, A.sms), kSeedThreads, 0, s>>>(g, n0, B.P, cell, nk, dK, dKi, dKp, keep);
        if ((e = scan_counts(sc, keep, n0)) != cudaSuccess) {
            return e;
        }
    }
    int nkeep = 0;
    cudaMemcpyAsync(&nkeep, keep + n0, sizeof(int), cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
        return e;
    }
    const int n2 = nkeep + nk;
    float* P2 = (float*)alloc(sizeof(float) * 3 * (size_t)n2);
    uint16_t* lab2 = (uint16_t*)alloc(sizeof(uint16_t) * (size_t)n2);
    uint8_t* typ2 = (uint8_t*)alloc((size_t)n2);
    uint16_t* part2 = (uint16_t*)alloc(sizeof(uint16_t) * 2 * (size_t)n2);
    uint16_t* part32 = (uint16_t*)alloc(sizeof(uint16_t) * (size_t)n2);
    if (!P2 || !lab2 || !typ2 || !part2 || !part32) {
        return cudaErrorMemoryAllocation;
    }
    k_feat_compact<<<gs_blocks(n0 + nk, A.sms), kSeedThreads, 0, s>>>(n0, keep, B.P, B.lab, B.typ, B.part, B.part3, nk,
                                                                     dKp, dKl, dKn, P2, lab2, typ2, part2, part32);
    B.P = P2;
    B.lab = lab2;
    B.typ = typ2;
    B.part = part2;
    B.part3 = part32;
    B.n = n2;
    return cudaGetLastError();
}

// ---- host side: the stages in order ----------------------------------------------------
template <bool kShape>
cudaError_t seed_stages(const SeedArgs& A, SeedBuffers& B, std::string& err) {
    const DGrid& g = A.g;
    cudaStream_t s = A.stream;
    Scratch sc{ s };
    auto alloc = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (pool_malloc(&p, std::max<size_t>(bytes, 16), s) != cudaSuccess) {
            return nullptr;
        }
        B.tmp.push_back(p);
        return p;
    };
    auto total_of = [&](const int* cnt, int64_t n, int* out) -> cudaError_t {
        cudaError_t e = cudaMemcpyAsync(out, cnt + n, sizeof(int), cudaMemcpyDeviceToHost, s);
        return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
    };
    cudaError_t e;
    // 1. the lattice: count -> scan -> fill over voxels
    const int64_t nv = (int64_t)g.nx * g.ny * g.nz;
    int* cnt = (int*)alloc(sizeof(int) * (size_t)(nv + 1));
    if (!cnt) {
        return cudaErrorMemoryAllocation;
    }
    cudaMemsetAsync(cnt, 0, sizeof(int), s);
    k_seed_voxels<kShape><<<gs_blocks(nv, A.sms), kSeedThreads, 0, s>>>(g, A.grade, A.spacing, A.nseed, A.voxmode, cnt, 0,
                                                                        nullptr, nullptr);
    if ((e = scan_counts(sc, cnt, nv)) != cudaSuccess) {
        return e;
    }
    int n = 0;
    if ((e = total_of(cnt, nv, &n)) != cudaSuccess) {
        return e;
    }
    float* P = (float*)alloc(sizeof(float) * 3 * (size_t)n);
    uint16_t* lab = (uint16_t*)alloc(sizeof(uint16_t) * (size_t)n);
    uint8_t* typ = (uint8_t*)alloc((size_t)n);
    uint16_t* part = (uint16_t*)alloc(sizeof(uint16_t) * 2 * (size_t)n);
    if (!P || !lab || !typ || !part) {
        return cudaErrorMemoryAllocation;
    }
    if (n > 0) {
        k_seed_voxels<kShape><<<gs_blocks(nv, A.sms), kSeedThreads, 0, s>>>(g, A.grade, A.spacing, A.nseed, A.voxmode,
                                                                            cnt, 1, P, lab);
        // 2. classification
        k_seed_classify<kShape><<<gs_blocks(n, A.sms), kSeedThreads, 0, s>>>(g, n, P, lab, typ, part);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) {
        return e;
    }
    const int64_t nvert = (int64_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    // 3. junction-line seeds: candidates at the 3-label vertices, one per key
    // (the first in (key, vertex) order), the lattice nodes near them dropped
    if (A.jseed > 0.0f) {
        int* jc = (int*)alloc(sizeof(int) * (size_t)(nvert + 1));
        int* jerr = (int*)alloc(sizeof(int));
        if (!jc || !jerr) {
            return cudaErrorMemoryAllocation;
        }
        cudaMemsetAsync(jc, 0, sizeof(int), s);
        cudaMemsetAsync(jerr, 0, sizeof(int), s);
        k_seed_junctions<kShape><<<gs_blocks(nvert, A.sms), kSeedThreads, 0, s>>>(
            g, A.grade, A.spacing, A.nseed, A.jseed, jc, 0, nullptr, nullptr, nullptr, nullptr, jerr);
        if ((e = scan_counts(sc, jc, nvert)) != cudaSuccess) {
            return e;
        }
        int m = 0;
        if ((e = total_of(jc, nvert, &m)) != cudaSuccess) {
            return e;
        }
        if (m > 0) {
            float* cx = (float*)alloc(sizeof(float) * 3 * (size_t)m);
            int* clab = (int*)alloc(sizeof(int) * 3 * (size_t)m);
            auto* khi = (unsigned long long*)alloc(8 * (size_t)m);
            auto* klo = (unsigned long long*)alloc(8 * (size_t)m);
            auto* lo_s = (unsigned long long*)alloc(8 * (size_t)m);
            auto* hi_p = (unsigned long long*)alloc(8 * (size_t)m);
            auto* hi_s = (unsigned long long*)alloc(8 * (size_t)m);
            auto* lo_f = (unsigned long long*)alloc(8 * (size_t)m);
            int* iota = (int*)alloc(4 * (size_t)m);
            int* perm1 = (int*)alloc(4 * (size_t)m);
            int* perm2 = (int*)alloc(4 * (size_t)m);
            int* flag = (int*)alloc(4 * (size_t)(m + 1));
            if (!cx || !clab || !khi || !klo || !lo_s || !hi_p || !hi_s || !lo_f || !iota || !perm1 || !perm2 || !flag) {
                return cudaErrorMemoryAllocation;
            }
            k_seed_junctions<kShape><<<gs_blocks(nvert, A.sms), kSeedThreads, 0, s>>>(
                g, A.grade, A.spacing, A.nseed, A.jseed, jc, 1, cx, clab, khi, klo, jerr);
            int herr = 0;
            cudaMemcpyAsync(&herr, jerr, sizeof(int), cudaMemcpyDeviceToHost, s);
            if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
                return e;
            }
            if (herr) {
                err = "a junction seed's cell index is beyond the sort key's range";
                return cudaErrorInvalidValue;
            }
            // stable LSD order: by the sorted label triple, then by level and cell;
            // ties keep the vertex order the candidates were written in
            k_iota<<<gs_blocks(m, A.sms), kSeedThreads, 0, s>>>(m, iota);
            size_t b1 = 0, b2 = 0;
            cub::DeviceRadixSort::SortPairs(nullptr, b1, klo, lo_s, iota, perm1, m, 0, 48, s);
            cub::DeviceRadixSort::SortPairs(nullptr, b2, hi_p, hi_s, perm1, perm2, m, 0, 64, s);
            b1 = std::max(b1, b2);
            if ((e = sc.need(b1)) != cudaSuccess) {
                return e;
            }
            b2 = b1;
            if ((e = cub::DeviceRadixSort::SortPairs(sc.p, b1, klo, lo_s, iota, perm1, m, 0, 48, s)) != cudaSuccess) {
                return e;
            }
            k_gather_u64<<<gs_blocks(m, A.sms), kSeedThreads, 0, s>>>(m, perm1, khi, hi_p);
            if ((e = cub::DeviceRadixSort::SortPairs(sc.p, b2, hi_p, hi_s, perm1, perm2, m, 0, 64, s)) != cudaSuccess) {
                return e;
            }
            k_gather_u64<<<gs_blocks(m, A.sms), kSeedThreads, 0, s>>>(m, perm2, klo, lo_f);
            cudaMemsetAsync(flag, 0, sizeof(int), s);
            k_seed_jfirst<<<gs_blocks(m, A.sms), kSeedThreads, 0, s>>>(m, hi_s, lo_f, flag);
            if ((e = scan_counts(sc, flag, m)) != cudaSuccess) {
                return e;
            }
            int ns = 0;
            if ((e = total_of(flag, m, &ns)) != cudaSuccess) {
                return e;
            }
            DropHash H;
            H.cell = 0.4f * A.hmax;
            H.vs[0] = g.vx;
            H.vs[1] = g.vy;
            H.vs[2] = g.vz;
            const float ext[3] = { (g.nx + 1) * g.vx, (g.ny + 1) * g.vy, (g.nz + 1) * g.vz };
            for (int a = 0; a < 3; ++a) {
                H.hd[a] = static_cast<int>(ext[a] / H.cell) + 2;
            }
            float* sx = (float*)alloc(sizeof(float) * 3 * (size_t)ns);
            int* slab = (int*)alloc(sizeof(int) * 3 * (size_t)ns);
            long long* bkey = (long long*)alloc(8 * (size_t)ns);
            long long* bkey_s = (long long*)alloc(8 * (size_t)ns);
            int* bidx = (int*)alloc(4 * (size_t)ns);
            int* bidx_s = (int*)alloc(4 * (size_t)ns);
            int* keep = (int*)alloc(4 * (size_t)(n + 1));
            if (!sx || !slab || !bkey || !bkey_s || !bidx || !bidx_s || !keep) {
                return cudaErrorMemoryAllocation;
            }
            k_seed_jkeep<<<gs_blocks(m, A.sms), kSeedThreads, 0, s>>>(m, perm2, flag, cx, clab, H, sx, slab, bkey, bidx);
            size_t b3 = 0;
            cub::DeviceRadixSort::SortPairs(nullptr, b3, (unsigned long long*)bkey, (unsigned long long*)bkey_s, bidx,
                                            bidx_s, ns, 0, 64, s);
            if ((e = sc.need(b3)) != cudaSuccess) {
                return e;
            }
            b3 = sc.bytes;
            if ((e = cub::DeviceRadixSort::SortPairs(sc.p, b3, (unsigned long long*)bkey, (unsigned long long*)bkey_s,
                                                     bidx, bidx_s, ns, 0, 64, s)) != cudaSuccess) {
                return e;
            }
            cudaMemsetAsync(keep, 0, sizeof(int), s);
            if (n > 0) {
                k_seed_jdrop<<<gs_blocks(n, A.sms), kSeedThreads, 0, s>>>(g, n, P, typ, H, ns, bkey_s, bidx_s, sx, keep);
                if ((e = scan_counts(sc, keep, n)) != cudaSuccess) {
                    return e;
                }
            }
            int nk = 0;
            if ((e = total_of(keep, n, &nk)) != cudaSuccess) {
                return e;
            }
            const int n2 = nk + ns;
            float* P2 = (float*)alloc(sizeof(float) * 3 * (size_t)n2);
            uint16_t* lab2 = (uint16_t*)alloc(sizeof(uint16_t) * (size_t)n2);
            uint8_t* typ2 = (uint8_t*)alloc((size_t)n2);
            uint16_t* part2 = (uint16_t*)alloc(sizeof(uint16_t) * 2 * (size_t)n2);
            if (!P2 || !lab2 || !typ2 || !part2) {
                return cudaErrorMemoryAllocation;
            }
            k_seed_jcompact<<<gs_blocks(n + ns, A.sms), kSeedThreads, 0, s>>>(n, keep, P, lab, typ, part, ns, sx, slab,
                                                                             P2, lab2, typ2, part2);
            P = P2;
            lab = lab2;
            typ = typ2;
            part = part2;
            n = n2;
        }
    }
    // 4. corner nodes, appended: count -> scan -> fill over the grid vertices
    int nc = 0;
    int* cc = nullptr;
    if (A.corners) {
        cc = (int*)alloc(sizeof(int) * (size_t)(nvert + 1));
        if (!cc) {
            return cudaErrorMemoryAllocation;
        }
        cudaMemsetAsync(cc, 0, sizeof(int), s);
        k_seed_corners<kShape><<<gs_blocks(nvert, A.sms), kSeedThreads, 0, s>>>(g, cc, 0, 0, nullptr, nullptr, nullptr,
                                                                                nullptr, nullptr);
        if ((e = scan_counts(sc, cc, nvert)) != cudaSuccess) {
            return e;
        }
        if ((e = total_of(cc, nvert, &nc)) != cudaSuccess) {
            return e;
        }
    }
    const int nt = n + nc;
    B.P = (float*)alloc(sizeof(float) * 3 * (size_t)nt);
    B.lab = (uint16_t*)alloc(sizeof(uint16_t) * (size_t)nt);
    B.typ = (uint8_t*)alloc((size_t)nt);
    B.part = (uint16_t*)alloc(sizeof(uint16_t) * 2 * (size_t)nt);
    B.part3 = (uint16_t*)alloc(sizeof(uint16_t) * (size_t)nt);
    if (!B.P || !B.lab || !B.typ || !B.part || !B.part3) {
        return cudaErrorMemoryAllocation;
    }
    if (n > 0) {
        cudaMemcpyAsync(B.P, P, sizeof(float) * 3 * (size_t)n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(B.lab, lab, sizeof(uint16_t) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(B.typ, typ, (size_t)n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(B.part, part, sizeof(uint16_t) * 2 * (size_t)n, cudaMemcpyDeviceToDevice, s);
        cudaMemsetAsync(B.part3, 0xFF, sizeof(uint16_t) * (size_t)n, s);
    }
    if (nc > 0) {
        k_seed_corners<kShape><<<gs_blocks(nvert, A.sms), kSeedThreads, 0, s>>>(g, cc, 1, n, B.P, B.lab, B.typ, B.part,
                                                                                B.part3);
    }
    B.n = nt;
    if ((e = cudaGetLastError()) != cudaSuccess) {
        return e;
    }
    // 5. shape input: nodes pinned on the sharp features
    if (A.feat && A.nfeat > 0) {
        if ((e = feature_pass<kShape>(A, B, sc, alloc, err)) != cudaSuccess) {
            return e;
        }
    }
    return cudaStreamSynchronize(s);
}

cudaError_t seed_run(const SeedArgs& A, SeedBuffers& B, std::string& err) {
    return A.g.gm < 0 ? seed_stages<true>(A, B, err) : seed_stages<false>(A, B, err);
}

}  // namespace v2m
