// v2m_kernels.cu -- the relaxation's kernels for sm_100a (B200).
//
// One launch per stage covers every volume of a session; a thread (or warp)
// finds its volume through nodevol[] (node stages) or the 1024-aligned bin
// ranges (scan stages), and a volume whose loop has finished, or that does not
// rebuild this iteration, makes its threads return at once. Nothing waits on
// another block: no spin loops, no grid-wide barriers, so every launch ends.
//
// Stage map (fangq/trussnet reference in brackets):
//   k_keys        bin key of each node + bin counts          [k_keys, src/opencl/v2m_kernels.cl:106-120]
//   k_scan_*      exclusive scan of the bin counts            [k_scan_block / k_scan_add :46-103]
//   k_scatter     node ids into their bins                    [k_scatter :122-128]
//   k_binsort     ascending ids within each bin + bin-order   [src/v2m_particles.cpp:791-806; k_gather :131-142]
//                 positions/sizes (the CPU's stable order)
//   k_neighbors   K-nearest truss of each node, one warp each [v2m_neighbors, src/opencl/v2m_particle_body.cl:73-151]
//   k_force       bar forces, each node's bars summed in list [v2m_force :161-184]
//                 order (an ordered fold: no float atomics)
//   k_move        FIRE/Jacobi step + trapped move + the        [v2m_move :844-935; k_stats :196-267]
//                 iteration's reductions (log2 histogram, max,
//                 half-skin count, FIRE power per block)
//   k_control     FIRE update, p99, stop test, rebuild trigger [src/v2m_particles.cpp:849-946; FireCtl src/v2m_particles.h:47-76]
//   k_refresh     lists of nodes past a full skin rebuilt     [src/v2m_particles.cpp:917-937]
#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "v2m_binsort.cuh"
#include "v2m_field.cuh"
#include "v2m_kernels.h"

namespace v2m {

__device__ __forceinline__ void raise_error(Global* G, int code, int info) {
    if (atomicCAS(&G->err, 0, code) == 0) {
        G->err_info = info;
    }
}

// ---- hash geometry (src/opencl/v2m_particle_body.cl:38-58) -----------------------
__device__ __forceinline__ int level_of(const DHash& H, float R) {
    int L = 0;
    while (L + 1 < H.nlev && H.b0 * (float)(1 << L) < R) {
        ++L;
    }
    return L;
}

__device__ __forceinline__ int bin_coord(const DHash& H, int L, float x, float o, int ax) {
    const int c = (int)floorf((x - o) / (H.b0 * (float)(1 << L)));
    const int n = H.dim[L][ax];
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

// bin_coord with a reciprocal of the bin side instead of the division: within
// a few 1e-5 of a bin of it, for search boxes that are widened by more than that
__device__ __forceinline__ int bin_coord_near(const DHash& H, int L, float x, float o, int ax, float inv) {
    const int c = (int)floorf((x - o) * inv);
    const int n = H.dim[L][ax];
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

__device__ __forceinline__ int bin_key(const DHash& H, int L, float px, float py, float pz) {
    const int cx = bin_coord(H, L, px, H.ox, 0), cy = bin_coord(H, L, py, H.oy, 1), cz = bin_coord(H, L, pz, H.oz, 2);
    return H.off[L] + cx + H.dim[L][0] * (cy + H.dim[L][1] * cz);
}

// Position + signed size: the sign bit of w marks a non-INTERIOR node.
__device__ __forceinline__ float pack_h(float h, int ty) {
    return ty != V2M_INTERIOR ? -h : h;
}

// ---- keys + counts ---------------------------------------------------------------
__global__ void k_keys(const DVol* __restrict__ vols, const VolCtl* __restrict__ ctl, const uint16_t* __restrict__ nodevol,
                       const float4* __restrict__ Pq, int* __restrict__ key, int* __restrict__ cnt,
                       float4* __restrict__ P0, int64_t N, Global* G) {
    if (!*((volatile int*)&G->rebuild_any)) {
        return;
    }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int v = nodevol[i];
        if (v == 0xFFFF || !ctl[v].rebuild) {
            continue;
        }
        const DVol& V = vols[v];
        const float4 p = Pq[i];
        const float hh = size_at(V.g, V.hmode, p.x, p.y, p.z);
        const int k = bin_key(V.H, level_of(V.H, (V.t + V.skin) * hh), p.x, p.y, p.z);
        if (k < 0 || k >= V.nkeys) {
            raise_error(G, 1, (int)i);
            continue;
        }
        key[i] = k;
        atomicAdd(cnt + V.kofs + k, 1);
        P0[i] = make_float4(p.x, p.y, p.z, 0.0f);
    }
}

// ---- exclusive scan of the bin counts, per volume, based at the volume's first node --
// Bin entries are tiled by kScanTile; every tile lies in one volume (1024-aligned).
__global__ void k_scan_tiles(const DVol* __restrict__ vols, const VolCtl* __restrict__ ctl,
                             const int16_t* __restrict__ tilevol, const int* __restrict__ cnt, int* __restrict__ tilesum,
                             int64_t KT) {
    const int t = blockIdx.x;
    const int v = tilevol[t];
    if (v < 0 || !ctl[v].rebuild) {
        return;
    }
    const DVol& V = vols[v];
    const int64_t base = (int64_t)t * kScanTile;
    const int64_t end = V.kofs + V.nkeys + 1;
    int s = 0;
    for (int q = threadIdx.x; q < kScanTile; q += blockDim.x) {
        const int64_t e = base + q;
        if (e < end && e >= V.kofs) {
            s += cnt[e];
        }
    }
    __shared__ int red[32];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = s;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_down_sync(0xffffffffu, s, o);
        }
        if (threadIdx.x == 0) {
            tilesum[t] = s;
        }
    }
}

// One block per volume: exclusive scan over its tiles' sums, starting at nofs.
__global__ void k_scan_vol(const DVol* __restrict__ vols, const VolCtl* __restrict__ ctl, const int* __restrict__ tilesum,
                           int* __restrict__ tileofs) {
    const int v = blockIdx.x;
    if (!ctl[v].rebuild) {
        return;
    }
    const DVol& V = vols[v];
    const int t0 = V.tofs_key, nt = V.ntile_key;
    __shared__ int carry;
    if (threadIdx.x == 0) {
        carry = (int)V.nofs;
    }
    __syncthreads();
    for (int b = 0; b < nt; b += blockDim.x) {
        const int t = b + threadIdx.x;
        int x = t < nt ? tilesum[t0 + t] : 0;
        // block inclusive scan
        int incl = x;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if ((threadIdx.x & 31) >= o) {
                incl += y;
            }
        }
        __shared__ int wsum[32];
        if ((threadIdx.x & 31) == 31) {
            wsum[threadIdx.x >> 5] = incl;
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            int w = threadIdx.x < (blockDim.x >> 5) ? wsum[threadIdx.x] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (threadIdx.x >= o) {
                    w += y;
                }
            }
            wsum[threadIdx.x] = w;
        }
        __syncthreads();
        const int wp = (threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1] : 0;
        if (t < nt) {
            tileofs[t0 + t] = carry + wp + incl - x;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            carry += wsum[(blockDim.x >> 5) - 1];
        }
        __syncthreads();
    }
}

// Per tile: cstart = tile offset + exclusive scan of the counts; the scatter's
// cursors start there; the counts are cleared for the next rebuild.
__global__ void k_scan_apply(const DVol* __restrict__ vols, const VolCtl* __restrict__ ctl,
                             const int16_t* __restrict__ tilevol, int* __restrict__ cnt, const int* __restrict__ tileofs,
                             int* __restrict__ cstart, int* __restrict__ cursor) {
    const int t = blockIdx.x;
    const int v = tilevol[t];
    if (v < 0 || !ctl[v].rebuild) {
        return;
    }
    const DVol& V = vols[v];
    const int64_t base = (int64_t)t * kScanTile;
    const int64_t end = V.kofs + V.nkeys + 1;
    constexpr int PER = kScanTile / kScanThreads;
    int x[PER];
    int s = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int64_t e = base + threadIdx.x * PER + q;
        x[q] = (e < end && e >= V.kofs) ? cnt[e] : 0;
        s += x[q];
    }
    int incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if ((threadIdx.x & 31) >= o) {
            incl += y;
        }
    }
    __shared__ int wsum[kScanThreads / 32];
    if ((threadIdx.x & 31) == 31) {
        wsum[threadIdx.x >> 5] = incl;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        int w = threadIdx.x < kScanThreads / 32 ? wsum[threadIdx.x] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (threadIdx.x >= o) {
                w += y;
            }
        }
        if (threadIdx.x < kScanThreads / 32) {
            wsum[threadIdx.x] = w;
        }
    }
    __syncthreads();
    int run = tileofs[t] + ((threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1] : 0) + incl - s;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int64_t e = base + threadIdx.x * PER + q;
        if (e < end && e >= V.kofs) {
            cstart[e] = run;
            cursor[e] = run;
            cnt[e] = 0;
        }
        run += x[q];
    }
}

// ---- scatter and in-bin order ------------------------------------------------------
__global__ void k_scatter(const VolCtl* __restrict__ ctl, const DVol* __restrict__ vols, const uint16_t* __restrict__ nodevol,
                          const int* __restrict__ key, int* __restrict__ cursor, int* __restrict__ sorted, int64_t N,
                          Global* G) {
    if (!*((volatile int*)&G->rebuild_any)) {
        return;
    }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int v = nodevol[i];
        if (v == 0xFFFF || !ctl[v].rebuild) {
            continue;
        }
        const DVol& V = vols[v];
        const int pos = atomicAdd(cursor + V.kofs + key[i], 1);
        if (pos < V.nofs || pos >= V.nofs + V.n) {
            raise_error(G, 2, (int)i);
            continue;
        }
        sorted[pos] = (int)i;
    }
}

// The label test of a candidate, taken in bin order with its id: the label in
// the low 16 bits, bit 16 set for an INTERIOR node.
__device__ __forceinline__ int snap_info(int ty, int lb) {
    return lb | (ty == V2M_INTERIOR ? 0x10000 : 0);
}

// One thread per bin: the bin's ids ascending (the CPU's stable counting sort,
// src/v2m_particles.cpp:791-795), then their positions and sizes in bin order,
// and beside them (Js) each slot's id and label test (snap_info) as they are at
// this build, for the full list build that follows.
// A bin of more than kSmallBin ids is handed to the whole block
// (block_bin_sort, over `tmp` at the same offsets), so the work stays linear in
// the bin's size: clustered or coincident nodes cannot stall one thread.
__global__ void __launch_bounds__(kBinSortThreads) k_binsort(const DVol* __restrict__ vols, const VolCtl* __restrict__ ctl,
                                                          const int16_t* __restrict__ tilevol,
                                                          const int* __restrict__ cstart, int* __restrict__ sorted,
                                                          int* __restrict__ tmp, const float4* __restrict__ Pq,
                                                          const uint8_t* __restrict__ typ, const uint16_t* __restrict__ lab,
                                                          float4* __restrict__ Ps, int2* __restrict__ Js, int64_t KT,
                                                          const Global* G) {
    __shared__ BinSortSmem sm;
    __shared__ int64_t big[kBinSortThreads];
    __shared__ int nbig;
    if (!*((volatile const int*)&G->rebuild_any)) {
        return;
    }
    for (int64_t base = blockIdx.x * (int64_t)kBinSortThreads; base < KT; base += (int64_t)gridDim.x * kBinSortThreads) {
        if (threadIdx.x == 0) {
            nbig = 0;
        }
        __syncthreads();
        const int64_t e = base + threadIdx.x;
        if (e < KT) {
            const int v = tilevol[e / kScanTile];
            if (v >= 0 && ctl[v].rebuild && e >= vols[v].kofs && e < vols[v].kofs + vols[v].nkeys) {
                const int s0 = cstart[e], s1 = cstart[e + 1];
                if (s1 - s0 <= kSmallBin) {
                    small_bin_sort(sorted + s0, s1 - s0);
                    for (int s = s0; s < s1; ++s) {
                        const int j = sorted[s];
                        const float4 p = Pq[j];
                        Ps[s] = make_float4(p.x, p.y, p.z, fabsf(p.w));
                        Js[s] = make_int2(j, snap_info(typ[j], lab[j]));
                    }
                } else {
                    big[atomicAdd(&nbig, 1)] = e;
                }
            }
        }
        __syncthreads();
        const int nb = nbig;
        for (int q = 0; q < nb; ++q) {
            const int s0 = cstart[big[q]], s1 = cstart[big[q] + 1];
            block_bin_sort(sorted + s0, tmp + s0, s1 - s0, sm);
            for (int s = s0 + threadIdx.x; s < s1; s += kBinSortThreads) {
                const int j = sorted[s];
                const float4 p = Pq[j];
                Ps[s] = make_float4(p.x, p.y, p.z, fabsf(p.w));
                Js[s] = make_int2(j, snap_info(typ[j], lab[j]));
            }
            __syncthreads();
        }
    }
}


// ---- K-nearest truss lists ----------------------------------------------------------
// One warp per node. The accepted candidates (distance and label tests of
// src/opencl/v2m_particle_body.cl:104-123) gather in a per-warp shared buffer;
// the list is the K smallest by (distance, id) -- the reference's insertion
// order is a total order, so its list is exactly these K, whatever the scan
// order. Node ids are flat; within a volume they order like the reference's.
constexpr int kCap = 64;

struct NbrWarpSmem {
    float d[kCap];
    int id[kCap];
    int rs0[32], rc[32];   // the non-empty rows of a batch, compacted
};

__device__ __forceinline__ bool pair_less(float da, int ia, float db, int ib) {
    return da < db || (da == db && ia < ib);
}

// Keep the K smallest of buf[0..m) in rank order; returns the new count.
__device__ __forceinline__ int warp_prune(NbrWarpSmem& sm, int m, int lane) {
    float dd[2];
    int ii[2], rk[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int e = lane + 32 * r;
        rk[r] = kCap;
        if (e < m) {
            dd[r] = sm.d[e];
            ii[r] = sm.id[e];
            int c = 0;
            for (int f = 0; f < m; ++f) {
                c += pair_less(sm.d[f], sm.id[f], dd[r], ii[r]);
            }
            rk[r] = c;
        }
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        if (rk[r] < V2M_K) {
            sm.d[rk[r]] = dd[r];
            sm.id[rk[r]] = ii[r];
        }
    }
    __syncwarp();
    return m < V2M_K ? m : V2M_K;
}

// Buffer entries of the candidate scan come in two forms: accepted ones,
// (distance, id); and raw ones, appended by the scan as (squared distance,
// -(bin-order index + 1)), which passed the distance test only. Before a prune
// (and at the end) the raw ones are checked -- node i itself and the
// interior-across-labels test of src/opencl/v2m_particle_body.cl:104-123 -- and
// given their distance, all in one pass over the buffer, instead of inside the
// scan's batches. Returns the number of accepted entries, packed to the front.
__device__ __forceinline__ int warp_validate(NbrWarpSmem& sm, int m, int lane, int64_t i, int ti_int, int li,
                                             const int* __restrict__ sorted, const uint8_t* __restrict__ typ,
                                             const uint16_t* __restrict__ lab) {
    float dd[2];
    int ii[2];
    bool keep[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int e = lane + 32 * r;
        keep[r] = false;
        dd[r] = 0.0f;
        ii[r] = 0;
        if (e < m) {
            dd[r] = sm.d[e];
            ii[r] = sm.id[e];
            keep[r] = true;
            if (ii[r] < 0) {
                const int j = sorted[-ii[r] - 1];
                keep[r] = j != (int)i && !(ti_int && typ[j] == V2M_INTERIOR && lab[j] != li);
                ii[r] = j;
                dd[r] = sqrtf(dd[r]);
            }
        }
    }
    __syncwarp();
    int out = 0;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const unsigned mk = __ballot_sync(0xffffffffu, keep[r]);
        if (keep[r]) {
            const int slot = out + __popc(mk & ((1u << lane) - 1u));
            sm.d[slot] = dd[r];
            sm.id[slot] = ii[r];
        }
        out += __popc(mk);
    }
    __syncwarp();
    return out;
}

// Distance from p to the bin interval [o + c b, o + (c + 1) b) along one axis;
// the edge bins reach to infinity (bin_coord clamps nodes outside the hash
// grid into them).
__device__ __forceinline__ float axis_gap(float p, int c, float o, float b, int n) {
    if (c > 0) {
        const float lo = o + (float)c * b;
        if (p < lo) {
            return lo - p;
        }
    }
    if (c < n - 1) {
        const float hi = o + (float)(c + 1) * b;
        if (p > hi) {
            return p - hi;
        }
    }
    return 0.0f;
}

// kSnap: the full list build, right after the hash build: each candidate's id
// and label test come from the build's bin-order snapshot (Js) in the same
// coalesced load round as its position, and are applied in the scan, so the
// buffer holds accepted entries only. Otherwise (the self-refresh between
// builds, where types may have changed since the snapshot) the scan appends
// distance-tested candidates and warp_validate checks them against the
// current typ / lab arrays.
template <bool kSnap>
__device__ void warp_neighbors(const DVol& V, int64_t i, int lane, NbrWarpSmem& sm, const float4* __restrict__ Pq,
                               const uint8_t* __restrict__ typ, const uint16_t* __restrict__ lab,
                               const int* __restrict__ cstart, const int* __restrict__ sorted,
                               const float4* __restrict__ Ps, const int2* __restrict__ Js, int* __restrict__ nbr,
                               uint8_t* __restrict__ nnb, int64_t N) {
    const DHash& H = V.H;
    const float4 pi = Pq[i];
    const float px = pi.x, py = pi.y, pz = pi.z;
    const float hi = fabsf(pi.w);
    const float ts = V.t + V.skin;
    const float Ri = ts * hi;
    const int ti_int = typ[i] == V2M_INTERIOR;
    const int li = lab[i];
    const int Li = level_of(H, Ri);
    const int* cs = cstart + V.kofs;
    // The bins of a level inside the search box form rows along x with
    // consecutive keys, so a row's candidates are one contiguous range of the
    // sorted ids: the lanes take rows (of all three levels), not bins.
    // Below the top level every node has ts h_j <= the level's bin side b, so a
    // candidate is accepted only within r = (Ri + b) / 2 of node i (the box's
    // half-width): rows and the ends of rows wholly farther than r (with a
    // margin of 1e-3 b for rounding) hold only rejected candidates and are
    // skipped. The top level also holds larger nodes: it is scanned whole.
    // (below the top level the box is widened by 1e-3 b and found with a
    // reciprocal: it still holds every bin within r; the top level's box is
    // the reference's, from the same divisions)
    // Lane q < 3 computes the box of level Li - 1 + q; a row takes its
    // level's box from that lane by shuffle.
    int bx0 = 0, bx1 = 0, by0 = 0, bz0 = 0, bny = 1, bkey = 0, bnr = 0;
    float binv = 0.0f;
    {
        const int L = Li - 1 + lane;
        if (lane < 3 && L >= 0 && L < H.nlev) {
            const float bL = H.b0 * (float)(1 << L);
            const float r = 0.5f * (Ri + bL);
            int y1, z1;
            if (L < H.nlev - 1) {
                const float inv = 1.0f / bL, rw = r + 1e-3f * bL;
                binv = inv;
                bx0 = bin_coord_near(H, L, px - rw, H.ox, 0, inv);
                bx1 = bin_coord_near(H, L, px + rw, H.ox, 0, inv);
                by0 = bin_coord_near(H, L, py - rw, H.oy, 1, inv);
                y1 = bin_coord_near(H, L, py + rw, H.oy, 1, inv);
                bz0 = bin_coord_near(H, L, pz - rw, H.oz, 2, inv);
                z1 = bin_coord_near(H, L, pz + rw, H.oz, 2, inv);
            } else {
                bx0 = bin_coord(H, L, px - r, H.ox, 0);
                bx1 = bin_coord(H, L, px + r, H.ox, 0);
                by0 = bin_coord(H, L, py - r, H.oy, 1);
                y1 = bin_coord(H, L, py + r, H.oy, 1);
                bz0 = bin_coord(H, L, pz - r, H.oz, 2);
                z1 = bin_coord(H, L, pz + r, H.oz, 2);
            }
            bny = y1 - by0 + 1;
            bnr = bny * (z1 - bz0 + 1);
            bkey = H.off[L] + bx0;
        }
    }
    const int row1 = __shfl_sync(0xffffffffu, bnr, 0);
    const int row2 = row1 + __shfl_sync(0xffffffffu, bnr, 1);
    const int nrows = row2 + __shfl_sync(0xffffffffu, bnr, 2);
    int m = 0;
    // once the buffer holds K entries, the K-th smallest distance so far (after a
    // prune, entry K-1): a candidate whose squared distance is above bd2 =
    // (1.0001 bd)^2 is farther than it, whatever the rounding, and can never
    // make the list
    float bd2 = __int_as_float(0x7f800000);
    for (int rb = 0; rb < nrows; rb += 32) {
        const int r = rb + lane;
        const int q = r < row1 ? 0 : (r < row2 ? 1 : 2);
        const int qx0 = __shfl_sync(0xffffffffu, bx0, q);
        const int qx1 = __shfl_sync(0xffffffffu, bx1, q);
        const int qy0 = __shfl_sync(0xffffffffu, by0, q);
        const int qz0 = __shfl_sync(0xffffffffu, bz0, q);
        const int qny = __shfl_sync(0xffffffffu, bny, q);
        const int qkey = __shfl_sync(0xffffffffu, bkey, q);
        const float qinv = __shfl_sync(0xffffffffu, binv, q);
        int s0 = 0, c = 0;
        if (r < nrows) {
            const int L = Li - 1 + q;
            const int rr = r - (q == 0 ? 0 : (q == 1 ? row1 : row2));
            const int zz = rr / qny;
            const int cy = qy0 + (rr - zz * qny), cz = qz0 + zz;
            int xa = qx0, xb = qx1;
            bool skip = false;
            if (L < H.nlev - 1) {
                const float bL = H.b0 * (float)(1 << L);
                const float m = 1e-3f * bL;
                const float rad = 0.5f * (Ri + bL) + m;
                const float dy = axis_gap(py, cy, H.oy, bL, H.dim[L][1]);
                const float dz = axis_gap(pz, cz, H.oz, bL, H.dim[L][2]);
                const float rem = rad * rad - dy * dy - dz * dz;
                if (rem < 0.0f) {
                    skip = true;
                } else {
                    const float w = sqrtf(rem) + m;
                    xa = max(xa, bin_coord_near(H, L, px - w, H.ox, 0, qinv));
                    xb = min(xb, bin_coord_near(H, L, px + w, H.ox, 0, qinv));
                    skip = xa > xb;
                }
            }
            if (!skip) {
                const int key0 = qkey + (xa - qx0) + H.dim[L][0] * (cy + H.dim[L][1] * cz);
                if (kChecked && (key0 < 0 || key0 + (xb - xa) + 1 > V.nkeys)) {
                    check_fail(V.g.chk, 22, i);   // a search row beyond the volume's bins
                    skip = true;
                } else {
                    s0 = cs[key0];
                    c = cs[key0 + (xb - xa) + 1] - s0;
                    if (kChecked && (c < 0 || s0 < V.nofs || s0 + c > V.nofs + V.n)) {
                        check_fail(V.g.chk, 23, i);   // bin starts outside the volume's nodes
                        c = 0;
                    }
                }
            }
        }
        // compact the non-empty rows to the first lanes (so that row ends are
        // distinct), then an inclusive prefix sum of their counts
        {
            const unsigned ne = __ballot_sync(0xffffffffu, c > 0);
            if (c > 0) {
                const int rk = __popc(ne & ((1u << lane) - 1u));
                sm.rs0[rk] = s0;
                sm.rc[rk] = c;
            }
            __syncwarp();
            const int nne = __popc(ne);
            s0 = lane < nne ? sm.rs0[lane] : 0;
            c = lane < nne ? sm.rc[lane] : 0;
            __syncwarp();
        }
        int incl = c;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) {
                incl += y;
            }
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        for (int cb = 0; cb < total; cb += 32) {
            const int q = cb + lane;
            // row of candidate q: the rows ending at or before q (row ends are
            // distinct: a bit each for those inside this batch of 32)
            const int before = __popc(__ballot_sync(0xffffffffu, c > 0 && incl <= cb));
            const unsigned ends = __reduce_or_sync(
                0xffffffffu, (c > 0 && incl > cb && incl < cb + 32) ? (1u << (incl - cb)) : 0u);
            const int lo = before + __popc(ends & ((2u << lane) - 1u));
            const int bs0 = __shfl_sync(0xffffffffu, s0, lo & 31);
            const int bexc = __shfl_sync(0xffffffffu, incl - c, lo & 31);
            // kSnap: every test here; else the distance test only, the rest
            // waits for warp_validate
            bool ok = false;
            float d2 = 0.0f;
            int sidx = 0, jid = 0;
            if (q < total) {
                sidx = bs0 + (q - bexc);
                const float4 ps = Ps[sidx];
                int2 js = make_int2(0, 0);
                if (kSnap) {
                    js = Js[sidx];
                }
                const float ex = ps.x - px, ey = ps.y - py, ez = ps.z - pz;
                d2 = ex * ex + ey * ey + ez * ez;
                const float rj = ts * 0.5f * (hi + ps.w);
                ok = !(d2 >= rj * rj) && !(d2 > bd2);   // (a NaN distance is kept, as before)
                if (kSnap) {
                    jid = js.x;
                    ok = ok && jid != (int)i &&
                         !(ti_int && (js.y & 0x10000) && (js.y & 0xFFFF) != li);
                }
            }
            const unsigned mask = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const int slot = m + __popc(mask & ((1u << lane) - 1u));
                sm.d[slot] = kSnap ? sqrtf(d2) : d2;
                sm.id[slot] = kSnap ? jid : -sidx - 1;
            }
            m += __popc(mask);
            __syncwarp();
            if (m > kCap - 32) {
                if (!kSnap) {
                    m = warp_validate(sm, m, lane, i, ti_int, li, sorted, typ, lab);
                }
                m = warp_prune(sm, m, lane);
                if (m == V2M_K) {
                    const float bd = sm.d[V2M_K - 1] * 1.0001f;
                    bd2 = bd * bd;
                }
            }
        }
    }
    // final ranks
    if (!kSnap) {
        m = warp_validate(sm, m, lane, i, ti_int, li, sorted, typ, lab);
    }
    m = warp_prune(sm, m, lane);
    // slots past m hold the node's own id (k_force loads whole batches of slots)
    if (lane < V2M_K) {
        nbr[(int64_t)lane * N + i] = lane < m ? sm.id[lane] : (int)i;
    }
    if (lane == 0) {
        nnb[i] = (uint8_t)m;
    }
    __syncwarp();
}

// 64 registers (32 resident warps per multiprocessor): faster than the
// uncapped 71-register build, whose occupancy is lower.
__global__ void __launch_bounds__(kNbrMaxThreads, 4) k_neighbors(const DVol* __restrict__ vols, const VolCtl* __restrict__ ctl,
                                                           const uint16_t* __restrict__ nodevol, const float4* __restrict__ Pq,
                                                           const uint8_t* __restrict__ typ, const uint16_t* __restrict__ lab,
                                                           const int* __restrict__ cstart, const int* __restrict__ sorted,
                                                           const float4* __restrict__ Ps, const int2* __restrict__ Js,
                                                           int* __restrict__ nbr, uint8_t* __restrict__ nnb, int64_t N,
                                                           const Global* G) {
    __shared__ NbrWarpSmem sm[kNbrMaxThreads / 32];
    if (!*((volatile const int*)&G->rebuild_any)) {
        return;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x / 32);
    for (int64_t i = blockIdx.x * (int64_t)(blockDim.x / 32) + w; i < N; i += nwarps) {
        const int v = nodevol[i];
        if (v == 0xFFFF || !ctl[v].rebuild) {
            continue;
        }
        warp_neighbors<true>(vols[v], i, lane, sm[w], Pq, typ, lab, cstart, sorted, Ps, Js, nbr, nnb, N);
    }
}

// The self-refresh of the nodes past a full skin (list filled by k_move), one
// warp per entry, except in a volume that rebuilds this iteration; the last
// block to finish empties the list.
__global__ void __launch_bounds__(kNbrMaxThreads, 4) k_refresh(const DVol* __restrict__ vols, const VolCtl* __restrict__ ctl,
                                                         const uint16_t* __restrict__ nodevol, const float4* __restrict__ Pq,
                                                         const uint8_t* __restrict__ typ, const uint16_t* __restrict__ lab,
                                                         const int* __restrict__ cstart, const int* __restrict__ sorted,
                                                         const float4* __restrict__ Ps, int* __restrict__ nbr,
                                                         uint8_t* __restrict__ nnb, float4* __restrict__ P0,
                                                         const int* __restrict__ rlist, Global* G, int64_t N) {
    __shared__ NbrWarpSmem sm[kNbrMaxThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int cnt = *((volatile int*)&G->nrefresh);
    const int wpb = blockDim.x / 32;
    const int nw = gridDim.x * wpb;
    for (int e = blockIdx.x * wpb + w; e < cnt; e += nw) {
        const int64_t i = rlist[e];
        if (kChecked && (i < 0 || i >= N || cnt > N)) {
            if (lane == 0) {
                raise_error(G, 25, e);   // a refresh entry beyond the nodes
            }
            continue;
        }
        const int v = nodevol[i];
        // a volume that rebuilds this iteration rebuilds every list and sets every
        // build position next (src/v2m_particles.cpp:771-820): its refreshes would
        // be overwritten unread
        if (ctl[v].done || ctl[v].rebuild) {
            continue;
        }
        warp_neighbors<false>(vols[v], i, lane, sm[w], Pq, typ, lab, cstart, sorted, Ps, nullptr, nbr, nnb, N);
        if (lane == 0) {
            const float4 p = Pq[i];
            P0[i] = make_float4(p.x, p.y, p.z, 0.0f);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const int d = atomicAdd(&G->blocks_done, 1);
        if (d == (int)gridDim.x - 1) {
            G->nrefresh = 0;
            G->qtrap_last = G->qtrap + G->qjun;
            G->qint_last = G->qint;
            G->qtrap = 0;
            G->qint = 0;
            G->qjun = 0;
            G->qdef = 0;
            G->blocks_done = 0;
            __threadfence();
        }
    }
}

// ---- bar forces ----------------------------------------------------------------
constexpr int kForceBatch = 4;

// One thread per node; the lists are slot-major (nbr[k*N + i]) so a warp's k-th
// entries are one coalesced 128-byte row; neighbour position + signed size is
// one 16-byte gather. Bars are added in list order, as v2m_force does: the
// deterministic ordered fold of the node's CSR row (no float atomics).
//
// The kernel is bound by those gathers: a warp's request for the k-th
// neighbours of its 32 nodes touches ~29 distinct 32-byte sectors, and the L1's
// per-request wavefronts, not DRAM (whose traffic equals the algorithmic bytes),
// set its time. It therefore keeps its own instructions and registers low:
//   - the ids arrive in batches of kForceBatch, the next batch's ids loaded
//     while the current batch's positions are in flight (no id array held in
//     registers: 48 registers, 5 blocks of 256 per multiprocessor);
//   - list slots past nnb hold the node's own id (every list writer pads them),
//     so the loads need no per-slot predicate; a padded bar is excluded from
//     the fold by its slot index, exactly as the reference's loop bound does;
//   - the size factor of a bar is (node factor if the neighbour is
//     non-interior, else fscale / 2), the node factor being fsurf / 2 for a
//     non-interior node and fscale / 2 otherwise: the same products as
//     ((both non-interior) ? fsurf : fscale) * 0.5f, since halving is exact.
// A list id outside the node's volume (a corrupted list) is clamped into it, so
// that no gather leaves the volume's nodes, and reported after the fold through
// the largest offset seen: the check feeds neither the loop nor the addresses.
__global__ void __launch_bounds__(256, 5) k_force(const DVol* __restrict__ vols, const VolCtl* __restrict__ ctl,
                                               const uint16_t* __restrict__ nodevol, const float4* __restrict__ Pq,
                                               const int* __restrict__ nbr, const uint8_t* __restrict__ nnb,
                                               float4* __restrict__ F, int64_t N, Global* G) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) {
        return;
    }
    const int v = nodevol[i];
    if (v == 0xFFFF) {
        return;
    }
    const VolCtl& c = ctl[v];
    const DVol& V = vols[v];
    if (c.done || c.it >= V.max_iters) {
        return;
    }
    const float fsh = V.fscale * 0.5f, fuh = V.fsurf * 0.5f;
    const float4 p = Pq[i];
    const float hi = fabsf(p.w);
    const float cneg = signbit(p.w) ? fuh : fsh;
    const int n = nnb[i];
    const unsigned lo = (unsigned)V.nofs, top = (unsigned)V.n - 1u;
    const float4* __restrict__ Pv = Pq + lo;
    const int* row = nbr + i;
    float fx = 0.0f, fy = 0.0f, fz = 0.0f, fa = 0.0f;
    unsigned mx = 0u;
    int jn[kForceBatch];
#pragma unroll
    for (int u = 0; u < kForceBatch; ++u) {
        jn[u] = __ldg(row + (int64_t)u * N);
    }
#pragma unroll
    for (int k0 = 0; k0 < V2M_K; k0 += kForceBatch) {
        if (k0 >= n) {
            break;
        }
        float4 qq[kForceBatch];
#pragma unroll
        for (int u = 0; u < kForceBatch; ++u) {
            const unsigned r = (unsigned)jn[u] - lo;
            mx = max(mx, r);
            qq[u] = __ldg(Pv + min(r, top));
        }
        if (k0 + kForceBatch < V2M_K) {
#pragma unroll
            for (int u = 0; u < kForceBatch; ++u) {
                jn[u] = __ldg(row + (int64_t)(k0 + kForceBatch + u) * N);
            }
        }
#pragma unroll
        for (int u = 0; u < kForceBatch; ++u) {
            const float4 q = qq[u];
            const float ex = p.x - q.x, ey = p.y - q.y, ez = p.z - q.z;
            const float l = sqrtf(ex * ex + ey * ey + ez * ez);
            const float l0 = (__float_as_int(q.w) < 0 ? cneg : fsh) * (hi + fabsf(q.w));
            if (k0 + u >= n || l >= l0 || l <= 0.0f) {
                continue;
            }
            const float f = (l0 - l) / l;
            fx += f * ex;
            fy += f * ey;
            fz += f * ez;
            fa += 1.0f;
        }
    }
    F[i] = make_float4(fx, fy, fz, fa);
    if (mx > top) {
        raise_error(G, 3, (int)i);
    }
}

// ---- move + per-iteration reductions ------------------------------------------------
// bin of |dp|/h in the log2 histogram: floor(log2(m)) of the correctly rounded
// float log2 (computed in double and rounded once), as glibc's log2f gives
__device__ __forceinline__ int hist_bin(float m) {
    if (!(m > 0.0f)) {
        return 0;
    }
    const float lf = (float)log2((double)m);
    int b = 20 + (int)floorf(lf);
    return b < 0 ? 0 : (b > 31 ? 31 : b);
}

// The iteration's reductions of one finished node (its |dp|/h, position, size):
// log2 histogram, max, Verlet half-skin count or self-refresh request
// (src/v2m_particles.cpp:874-937; src/opencl/v2m_kernels.cl:196-249). `shared`
// accumulates into the block's counters when every node of the block belongs to
// volume `v` (then flushed once), else straight into the volume's counters.
struct TailAcc {
    int hist[32];
    unsigned maxbits, maxd;
    int half;
};

__device__ __forceinline__ void node_tail(const DVol& Vd, VolCtl* ctl, int v, int64_t i, float m, float px, float py,
                                          float pz, float hh, const float4* __restrict__ P0, int* __restrict__ rlist,
                                          Global* G, TailAcc* sh) {
    const float4 q0 = P0[i];
    const float ex = px - q0.x, ey = py - q0.y, ez = pz - q0.z;
    const float m2 = ex * ex + ey * ey + ez * ez, s2 = Vd.skin * Vd.skin * hh * hh;
    const int b = hist_bin(m);
    VolCtl* cv = ctl + v;
    if (sh) {
        atomicAdd(&sh->hist[b], 1);
        atomicMax(&sh->maxbits, __float_as_uint(m));
        if (Vd.policy == 1) {
            atomicMax(&sh->maxd, __float_as_uint(sqrtf(m2) / hh));
        }
    } else {
        atomicAdd(&cv->hist[b], 1);
        atomicMax(&cv->maxbits, __float_as_uint(m));
        if (Vd.policy == 1) {
            atomicMax(reinterpret_cast<unsigned*>(&cv->pad1), __float_as_uint(sqrtf(m2) / hh));
        }
    }
    if (m2 > s2 && Vd.policy != 2) {
        const int e = atomicAdd(&G->nrefresh, 1);
        rlist[e] = (int)i;
        atomicAdd(&cv->nrefresh, 1);
    } else if (m2 > 0.25f * s2) {
        if (sh) {
            atomicAdd(&sh->half, 1);
        } else {
            atomicAdd(&cv->nhalf, 1);
        }
    }
}

__device__ __forceinline__ void tail_init(TailAcc& a) {
    if (threadIdx.x < 32) {
        a.hist[threadIdx.x] = 0;
    }
    if (threadIdx.x == 0) {
        a.maxbits = 0u;
        a.maxd = 0u;
        a.half = 0;
    }
}

__device__ __forceinline__ void tail_flush(TailAcc& a, VolCtl* cv) {
    if (threadIdx.x < 32 && a.hist[threadIdx.x]) {
        atomicAdd(&cv->hist[threadIdx.x], a.hist[threadIdx.x]);
    }
    if (threadIdx.x == 0) {
        if (a.maxbits) {
            atomicMax(&cv->maxbits, a.maxbits);
        }
        if (a.maxd) {
            atomicMax(reinterpret_cast<unsigned*>(&cv->pad1), a.maxd);
        }
        if (a.half) {
            atomicAdd(&cv->nhalf, a.half);
        }
    }
}

// First half of v2m_move (src/opencl/v2m_particle_body.cl:844-921), every node in
// node order: FIRE velocity update and power, the step, the settle test and the
// step cap. Corners and settled nodes finish here; the others are queued with
// their step (S = s, h): other trapped nodes at the front of the queue and
// INTERIOR ones at its back, JUNCTION ones in queue[N, 2N); k_move_int and
// k_move_main take them by kind. The FIRE power of the block is summed here, in
// node order (a fixed-shape double tree: deterministic whatever the queue order).
__global__ void __launch_bounds__(kMoveThreads, 5) k_move_pre(const DVol* __restrict__ vols, VolCtl* __restrict__ ctl,
                                                          const uint16_t* __restrict__ nodevol,
                                                          const float4* __restrict__ Pq, const float4* __restrict__ F,
                                                          float4* __restrict__ Vel, const uint8_t* __restrict__ typ,
                                                          float* __restrict__ mvout, float* __restrict__ pwout,
                                                          const float4* __restrict__ P0, float4* __restrict__ S,
                                                          int* __restrict__ queue, double2* __restrict__ psum,
                                                          int* __restrict__ rlist, Global* G, int64_t N) {
    __shared__ TailAcc acc;
    __shared__ int sh_vol;
    __shared__ double sh_pw[kMoveThreads / 32], sh_pa[kMoveThreads / 32];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    tail_init(acc);
    if (threadIdx.x == 0) {
        sh_vol = -1;
        if (blockIdx.x == 0) {
            G->rebuild_any = 0;   // the last iteration's rebuild stages are done
        }
    }
    __syncthreads();
    const int v = i < N ? nodevol[i] : 0xFFFF;
    bool active = v != 0xFFFF;
    float pwv = 0.0f;
    int qkind = -1;   // 0: trapped queue, 1: interior queue
    if (active) {
        const DVol& Vd = vols[v];
        const VolCtl& c = ctl[v];
        if (c.done || c.it >= Vd.max_iters) {
            active = false;
        } else {
            if (threadIdx.x == 0) {
                sh_vol = v;
            }
            const int fire = Vd.fire;
            const float fdt = c.fdt, falpha = c.falpha;
            const float4 pq = Pq[i];
            const int ty0 = typ[i];
            // the node's force and velocity read with its record, ahead of the
            // branches that use them (one round of loads; a CORNER node's or a
            // zeroed velocity's values go unused)
            const float4 f4pre = F[i];
            const float4 v4pre = Vel[i];
            // h at the node's position (v2m_move's v2m_h_at), which the stored size is unless a caller
            // overwrote positions or sizes
            const float h = Vd.hn_exact ? fabsf(pq.w) : size_at(Vd.g, Vd.hmode, pq.x, pq.y, pq.z);
            bool finished = true;
            if (ty0 != V2M_CORNER) {
                const float4 f4 = f4pre;
                const float stiff = f4.w > 1.0f ? f4.w : 1.0f;
                const float ac[3] = { f4.x / stiff, f4.y / stiff, f4.z / stiff };
                float s[3];
                if (fire) {
                    float vv[3] = { 0.0f, 0.0f, 0.0f };
                    if (!c.vzero) {
                        const float4 v4 = v4pre;
                        vv[0] = v4.x;
                        vv[1] = v4.y;
                        vv[2] = v4.z;
                    }
                    const float pv = ac[0] * vv[0] + ac[1] * vv[1] + ac[2] * vv[2];
                    pwv = pv;
                    if (pv < 0.0f) {
                        vv[0] = vv[1] = vv[2] = 0.0f;
                    } else {
                        const float vn = sqrtf(vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]);
                        const float an = sqrtf(ac[0] * ac[0] + ac[1] * ac[1] + ac[2] * ac[2]);
                        if (an > 0.0f) {
                            for (int k = 0; k < 3; ++k) {
                                vv[k] = (1.0f - falpha) * vv[k] + falpha * vn * ac[k] / an;
                            }
                        }
                    }
                    for (int k = 0; k < 3; ++k) {
                        vv[k] += fdt * ac[k];
                        s[k] = fdt * vv[k];
                    }
                } else {
                    for (int k = 0; k < 3; ++k) {
                        s[k] = Vd.dt * ac[k];
                    }
                }
                const float sl = sqrtf(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
                if (!(sl < 5e-4f * h)) {
                    if (sl > Vd.maxstep * h) {
                        for (int k = 0; k < 3; ++k) {
                            s[k] *= Vd.maxstep * h / sl;
                        }
                    }
                    S[i] = make_float4(s[0], s[1], s[2], h);
                    finished = false;
                    qkind = ty0 == V2M_INTERIOR ? 1 : (ty0 == V2M_JUNCTION ? 2 : 0);
                }
            }
            if (fire) {
                pwout[i] = pwv;
            }
            if (finished) {
                if (fire) {
                    Vel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                }
                mvout[i] = 0.0f;
                node_tail(Vd, ctl, v, i, 0.0f, pq.x, pq.y, pq.z, fabsf(pq.w), P0, rlist, G, &acc);
            }
        }
    }
    // queue the moving nodes, one atomic per block and kind: INTERFACE (and other
    // non-junction trapped) nodes from the front of queue[0, N), INTERIOR ones
    // from its back, JUNCTION ones from the front of queue[N, 2N)
    __shared__ int sh_cnt[3][kMoveThreads / 32];
    __shared__ int sh_base[3];
    const unsigned lane = threadIdx.x & 31u;
    const int wid = threadIdx.x >> 5;
    unsigned km[3];
#pragma unroll
    for (int kind = 0; kind < 3; ++kind) {
        km[kind] = __ballot_sync(0xffffffffu, qkind == kind);
        if (lane == 0) {
            sh_cnt[kind][wid] = __popc(km[kind]);
        }
    }
    // the block's FIRE power and the sum of its magnitudes (the latter bounds
    // the rounding error of any order of summation: k_control)
    double pd = active ? (double)pwv : 0.0;
    double pa = fabs(pd);
    for (int o = 16; o > 0; o >>= 1) {
        pd += __shfl_down_sync(0xffffffffu, pd, o);
        pa += __shfl_down_sync(0xffffffffu, pa, o);
    }
    if (lane == 0) {
        sh_pw[wid] = pd;
        sh_pa[wid] = pa;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int kind = threadIdx.x;
        int tot = 0;
        for (int w = 0; w < kMoveThreads / 32; ++w) {
            tot += sh_cnt[kind][w];
        }
        sh_base[kind] = tot ? atomicAdd(kind == 0 ? &G->qtrap : (kind == 1 ? &G->qint : &G->qjun), tot) : 0;
    }
    __syncthreads();
    if (qkind >= 0) {
        const unsigned mk = qkind == 0 ? km[0] : (qkind == 1 ? km[1] : km[2]);   // (no local-memory array)
        int slot = sh_base[qkind] + __popc(mk & ((1u << lane) - 1u));
        for (int w = 0; w < wid; ++w) {
            slot += sh_cnt[qkind][w];
        }
        queue[qkind == 0 ? (int64_t)slot : (qkind == 1 ? N - 1 - slot : N + slot)] = (int)i;
    }
    const int bv = sh_vol;
    if (bv < 0) {
        return;
    }
    if (threadIdx.x == 0) {
        double t = 0.0, ta = 0.0;
        for (int w = 0; w < kMoveThreads / 32; ++w) {
            t += sh_pw[w];
            ta += sh_pa[w];
        }
        psum[blockIdx.x] = make_double2(t, ta);
    }
    tail_flush(acc, ctl + bv);
}

// The iteration's reductions of the nodes a warp finished (the lanes of `act`,
// this lane among them), combined with warp votes: log2 histogram, max |dp|/h,
// half-skin count, max displacement (one lane per volume and bin), and the
// refresh list with one atomic per warp (src/v2m_particles.cpp:874-937).
__device__ __forceinline__ void warp_tail(const DVol& Vd, VolCtl* cv, int v, int64_t i, unsigned act, unsigned lane,
                                          float m, float px, float py, float pz, float hh,
                                          const float4* __restrict__ P0, int* __restrict__ rlist, Global* G) {
    const float4 q0 = P0[i];
    const float ex = px - q0.x, ey = py - q0.y, ez = pz - q0.z;
    const float m2 = ex * ex + ey * ey + ez * ez, s2 = Vd.skin * Vd.skin * hh * hh;
    const int b = hist_bin(m);
    const unsigned gb = __match_any_sync(act, (unsigned)(v << 5) | (unsigned)b);
    if (lane == (unsigned)(__ffs(gb) - 1)) {
        atomicAdd(&cv->hist[b], __popc(gb));
    }
    const unsigned gvol = __match_any_sync(act, (unsigned)v);
    const unsigned leader = (unsigned)(__ffs(gvol) - 1);
    const unsigned mx = __reduce_max_sync(gvol, __float_as_uint(m));
    const bool refresh = m2 > s2 && Vd.policy != 2;   // (policy 2: the first build's lists for the whole run)
    const bool half = !refresh && m2 > 0.25f * s2;
    const unsigned nh = __popc(__ballot_sync(act, half) & gvol);
    unsigned md = 0u;
    if (Vd.policy == 1) {
        md = __reduce_max_sync(gvol, __float_as_uint(sqrtf(m2) / hh));
    }
    const int slot = blockIdx.x & (kCtlSlots - 1);
    if (lane == leader) {
        if (mx) {
            atomicMax(&cv->maxbits_p[slot], mx);
        }
        if (nh) {
            atomicAdd(&cv->nhalf_p[slot], (int)nh);
        }
        if (md) {
            atomicMax(&cv->maxd_p[slot], md);
        }
    }
    const unsigned rm = __ballot_sync(act, refresh);
    if (rm) {
        const unsigned first = (unsigned)(__ffs(rm) - 1);
        int base = 0;
        if (lane == first) {
            base = atomicAdd(&G->nrefresh, __popc(rm));
        }
        base = __shfl_sync(act, base, first);
        if (refresh) {
            rlist[base + __popc(rm & ((1u << lane) - 1u))] = (int)i;
        }
        const unsigned rv = rm & gvol;
        if (lane == leader && rv) {
            atomicAdd(&cv->nrefresh, __popc(rv));
        }
    }
}

// Second half of v2m_move for the queued INTERIOR nodes whose move stays
// INTERIOR (label fields, smooth mode): v2m_move_step's owner ranking at
// q = p + s and its snap test (src/opencl/v2m_particle_body.cl:659-700), then
// the node's velocity, |dp|/h, size and the iteration's reductions. This is
// the common case of the move (most queued nodes) and needs none of the
// trapped move's projections, so it runs as its own kernel with no
// out-of-line calls: the ranking reads the bricks' corner tables only, and
// its warps do not share blocks with the long trapped moves. A node whose
// move may leave INTERIOR -- its owner label changes, or the snap test's
// distance estimate is within reach -- or whose step trips the safety net,
// or whose cell needs the per-corner path, and every node of a volume with
// analytic shape fields, gray fields or voxel mode, is handed to k_move_main
// unchanged (appended behind the JUNCTION queue): nothing of it is written
// here, and k_move_main's move_step takes it from the start, so every node's
// result is move_step's.
#ifndef V2M_INT_MIN_BLOCKS
#define V2M_INT_MIN_BLOCKS 8   // resident blocks of k_move_int per multiprocessor (8 x 128 threads: 64 registers)
#endif
__global__ void __launch_bounds__(kMainThreads, V2M_INT_MIN_BLOCKS) k_move_int(const DVol* __restrict__ vols, VolCtl* __restrict__ ctl,
                                                         const uint16_t* __restrict__ nodevol, float4* __restrict__ Pq,
                                                         float4* __restrict__ Vel, const uint16_t* __restrict__ lab,
                                                         float* __restrict__ mvout, const float4* __restrict__ P0,
                                                         const float4* __restrict__ S, int* __restrict__ queue,
                                                         int* __restrict__ rlist, Global* G, int64_t N) {
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int qb = *((volatile int*)&G->qint), qj = *((volatile int*)&G->qjun);
    if (blockIdx.x * (int64_t)blockDim.x >= qb) {
        return;
    }
    const unsigned lane = threadIdx.x & 31u;
    int64_t i = q < qb ? queue[N - 1 - q] : -1;
    if (kChecked && (i < -1 || i >= N)) {
        raise_error(G, 24, (int)q);   // a move queue entry beyond the nodes
        i = -1;
    }
    const int v = i >= 0 ? nodevol[i] : -1;
    bool fin = false, defer = false;
    float m = 0.0f, qx = 0.0f, qy = 0.0f, qz = 0.0f, hn = 0.0f;
    if (v >= 0) {
        const DVol& Vd = vols[v];
        const DGrid& g = Vd.g;
        if (g.gm != 0 || Vd.voxmode) {
            defer = true;
        } else {
            const float4 pq = Pq[i];
            const float4 s4 = S[i];
            const int a = lab[i];
            const float h = s4.w;
            qx = pq.x + s4.x;
            qy = pq.y + s4.y;
            qz = pq.z + s4.z;
            // owner_on_cell's ranking at q, on the brick's corner tables only
            LabList ll;
            const int n = labels_near(g, qx, qy, qz, ll);
            if (n == 1) {
                defer = ll.get(0) != a;
            } else {
                Cell cl;
                cell_at(g, qx, qy, qz, cl);
                defer = !cl.fast;   // the per-corner path (a cell based outside the grid, or among > 16 labels)
                if (!defer) {
                    int best = ll.get(0), sec = V2M_NOLAB;
                    float pb = -1.0f, ps = pb;
#pragma unroll 1
                    for (int t = 0; t < n; t += 2) {
                        const int l0 = ll.get(t);
                        const bool two = t + 1 < n;
                        const int l1 = two ? ll.get(t + 1) : l0;
                        float c0[8], c1[8];
                        table_corners(g, cl, l0, c0);
                        table_corners(g, cl, l1, c1);
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
                    defer = best != a;
                    if (!defer && sec != V2M_NOLAB && Vd.snap > 0.0f) {
                        // psi_grad_on(a, sec) on the ranked cell, as move_step
                        float c[8], e[8];
                        table_corners(g, cl, a, c);
                        table_corners(g, cl, sec, e);
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            c[k] -= e[k];
                        }
                        const float4 r = psi_grad_diff(g, c, cl.fx, cl.fy, cl.fz);
                        const float gn = sqrtf(r.x * r.x + r.y * r.y + r.z * r.z);
                        defer = gn > 1e-9f && r.w / gn < Vd.snap * h;
                    }
                }
            }
            if (!defer) {
                const float lim = (Vd.maxstep + fmaxf(Vd.snap, 0.5f)) * h;
                const float m2 = (qx - pq.x) * (qx - pq.x) + (qy - pq.y) * (qy - pq.y) + (qz - pq.z) * (qz - pq.z);
                if (!(m2 <= lim * lim)) {
                    defer = true;
                } else {
                    m = sqrtf(m2) / h;
                    hn = size_at(g, Vd.hmode, qx, qy, qz);
                    fin = true;
                    if (Vd.fire) {
                        const float fdt = ctl[v].fdt;
                        Vel[i] = m > 0.0f ? make_float4((qx - pq.x) / fdt, (qy - pq.y) / fdt, (qz - pq.z) / fdt, 0.0f)
                                          : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    }
                    mvout[i] = m;
                    Pq[i] = make_float4(qx, qy, qz, pack_h(hn, V2M_INTERIOR));
                    // (typ and part stay as they are: an INTERIOR node keeps both)
                }
            }
        }
    }
    const unsigned fm = __ballot_sync(0xffffffffu, fin);
    if (fin) {
        warp_tail(vols[v], ctl + v, v, i, fm, lane, m, qx, qy, qz, hn, P0, rlist, G);
    }
    const unsigned dm = __ballot_sync(0xffffffffu, defer);
    if (dm) {
        const unsigned first = (unsigned)(__ffs(dm) - 1);
        int base = 0;
        if (lane == first) {
            base = atomicAdd(&G->qdef, __popc(dm));
        }
        base = __shfl_sync(0xffffffffu, base, first);
        if (defer) {
            queue[N + qj + base + __popc(dm & ((1u << lane) - 1u))] = (int)i;
        }
    }
}

// Second half of v2m_move: the trapped move (v2m_move_step) of every queued
// trapped node and of the INTERIOR nodes k_move_int handed over, then its
// velocity, |dp|/h and the iteration's reductions. Blocks of kMainThreads with
// no block-wide barrier: a warp's statistics are combined with warp votes and
// flushed by one lane per (volume, bin), so a finished warp never waits for a
// slower one.
// Two instances: kShape = false moves the nodes of volumes with sampled fields,
// kShape = true (launched only when some volume has them) those with analytic
// shape fields; with both present each skips the other's nodes.
#ifndef V2M_MOVE_MIN_BLOCKS
#define V2M_MOVE_MIN_BLOCKS 8   // resident blocks of k_move_main per multiprocessor (8 x 128 threads: 64 registers)
#endif
template <bool kShape>
__global__ void __launch_bounds__(kMainThreads, V2M_MOVE_MIN_BLOCKS) k_move_main(const DVol* __restrict__ vols, VolCtl* __restrict__ ctl,
                                                           const uint16_t* __restrict__ nodevol, float4* __restrict__ Pq,
                                                           float4* __restrict__ Vel, uint8_t* __restrict__ typ,
                                                           const uint16_t* __restrict__ lab, uint32_t* __restrict__ part,
                                                           float* __restrict__ mvout, const float4* __restrict__ P0,
                                                           const float4* __restrict__ S, const int* __restrict__ queue,
                                                           int* __restrict__ rlist, Global* G, int64_t N,
                                                           int shape_any) {
    // the queues laid end to end -- junction and handed-over INTERIOR moves
    // [0, qj+qd) (queue[N, N+qj+qd)), then the other trapped ones [qj+qd, tot)
    // -- over at most N threads: a warp holds nodes of one kind, save the warps
    // at the seams, and the longest moves (junctions) start first
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int qa = *((volatile int*)&G->qtrap), qj = *((volatile int*)&G->qjun), qd = *((volatile int*)&G->qdef);
    const int64_t qjd = (int64_t)qj + qd;
    const int64_t tot = qjd + qa;
    if (blockIdx.x * (int64_t)blockDim.x >= tot) {
        return;
    }
    int64_t i = -1;
    if (q < qjd) {
        i = queue[N + q];
    } else if (q < tot) {
        i = queue[q - qjd];
    }
    if (kChecked && (i < -1 || i >= N || tot > N)) {
        raise_error(G, 24, (int)q);   // a move queue entry (or length) beyond the nodes
        i = -1;
    }
    int v = i >= 0 ? nodevol[i] : -1;
    if (shape_any && v >= 0 && (vols[v].g.gm < 0) != kShape) {
        v = -1;   // the other instance moves it
    }
    const unsigned lane = threadIdx.x & 31u;
    const unsigned act = __ballot_sync(0xffffffffu, v >= 0);
    if (v < 0) {
        return;
    }
    const DVol& Vd = vols[v];
    const VolCtl& c = ctl[v];
    const DGrid& g = Vd.g;
    const float4 pq = Pq[i];
    const float4 s4 = S[i];
    NodeState st;
    st.p[0] = pq.x;
    st.p[1] = pq.y;
    st.p[2] = pq.z;
    st.hn = fabsf(pq.w);
    st.a = lab[i];
    st.ty = typ[i];
    const uint32_t pp = part[i];
    st.pb = (int)(pp & 0xFFFFu);
    st.pc = (int)(pp >> 16);
    const int ty0 = st.ty;
    float s[3] = { s4.x, s4.y, s4.z };
    const float m = move_step<kShape>(g, Vd.hmode, s4.w, s, Vd.maxstep, Vd.snap, Vd.voxmode, st);
    if (Vd.fire) {
        const float fdt = c.fdt;
        Vel[i] = (m > 0.0f && st.ty == ty0)
                     ? make_float4((st.p[0] - pq.x) / fdt, (st.p[1] - pq.y) / fdt, (st.p[2] - pq.z) / fdt, 0.0f)
                     : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    mvout[i] = m;
    Pq[i] = make_float4(st.p[0], st.p[1], st.p[2], pack_h(st.hn, st.ty));
    typ[i] = (uint8_t)st.ty;
    part[i] = (uint32_t)(st.pb & 0xFFFF) | ((uint32_t)(st.pc & 0xFFFF) << 16);
    warp_tail(Vd, ctl + v, v, i, act, lane, m, st.p[0], st.p[1], st.p[2], st.hn, P0, rlist, G);
}

// ---- corner tables (once per session) ----------------------------------------------
// One thread per brick: the labels a cell based in the brick can meet -- the
// brick's own and its + neighbours' listed labels, and label 0 when the
// 9x9x9 region passes the grid's edge (phi_voxel is 1 for label 0 there) --
// and whether the region is one label everywhere (no table needed). More than
// 16 labels: no table (count -1; such cells take the per-corner path). The
// brick's record (DGrid::xbrick) gets the count and the labels; the host fills
// in the first table.
// xn gets the number of tables the brick needs.
__global__ void k_xcount(DGrid g, uint4* __restrict__ xbrick, int* __restrict__ xn, int nb) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) {
        return;
    }
    const int bx = b % g.nbx, by = (b / g.nbx) % g.nby, bz = b / (g.nbx * g.nby);
    uint16_t lst[V2M_BL];
    int n = 0;
    bool over = false;
    const bool outside = bx * 8 + 8 >= g.nx || by * 8 + 8 >= g.ny || bz * 8 + 8 >= g.nz;
    bool uni = !outside;
    int ulab = -1;
    for (int d = 0; d < 8; ++d) {
        const int X = bx + (d & 1), Y = by + ((d >> 1) & 1), Z = bz + (d >> 2);
        if (X >= g.nbx || Y >= g.nby || Z >= g.nbz) {
            continue;   // only voxels past the grid's edge (counted by outside)
        }
        const int nbk = X + g.nbx * (Y + g.nby * Z);
        const int cnt = g.bl_cnt[nbk];
        const int c = cnt < V2M_BL ? cnt : V2M_BL;
        if (!(cnt == 1 && g.bl_slot[nbk] < 0)) {
            uni = false;
        }
        for (int k = 0; k < c; ++k) {
            const int l = g.bl_lab[(size_t)nbk * V2M_BL + k];
            if (ulab < 0) {
                ulab = l;
            } else if (l != ulab) {
                uni = false;
            }
            bool have = false;
            for (int q = 0; q < n; ++q) {
                have |= lst[q] == l;
            }
            if (!have) {
                if (n < V2M_BL) {
                    lst[n++] = (uint16_t)l;
                } else {
                    over = true;
                }
            }
        }
    }
    if (outside) {
        bool have = false;
        for (int q = 0; q < n; ++q) {
            have |= lst[q] == 0;
        }
        if (!have) {
            if (n < V2M_BL) {
                lst[n++] = 0;
            } else {
                over = true;
            }
        }
    }
    if (uni && ulab >= 0) {
        // a uniform region must hold its label in every voxel (phi_voxel reads L there)
        for (int e = 0; e < 729 && uni; ++e) {
            const int i = bx * 8 + e % 9, j = by * 8 + (e / 9) % 9, k = bz * 8 + e / 81;
            uni = g.L[i + (size_t)g.nx * (j + (size_t)g.ny * k)] == ulab;
        }
    } else {
        uni = false;
    }
    int cnt;
    if (over) {
        cnt = -1;
        xn[b] = 0;
    } else if (uni) {
        lst[0] = (uint16_t)ulab;
        n = 1;
        cnt = 1;
        xn[b] = 0;
    } else {
        cnt = n;
        xn[b] = n;
    }
    uint32_t w[8];
    for (int q = 0; q < 8; ++q) {
        const uint32_t lo = 2 * q < n ? lst[2 * q] : 0u, hi = 2 * q + 1 < n ? lst[2 * q + 1] : 0u;
        w[q] = lo | (hi << 16);
    }
    uint4* r = xbrick + (size_t)3 * b;
    r[0] = make_uint4((uint32_t)cnt, 0xFFFFFFFFu, w[0], w[1]);
    r[1] = make_uint4(w[2], w[3], w[4], w[5]);
    r[2] = make_uint4(w[6], w[7], 0u, 0u);
}

// One block per table (brick, label): its 729 voxel values by phi_voxel.
__global__ void k_xfill(DGrid g, const int2* __restrict__ tabs, float* __restrict__ xphi) {
    const int t = blockIdx.x;
    const int2 bl = tabs[t];
    const int bx = bl.x % g.nbx, by = (bl.x / g.nbx) % g.nby, bz = bl.x / (g.nbx * g.nby);
    for (int e = threadIdx.x; e < 729; e += blockDim.x) {
        xphi[(size_t)t * 729 + e] = phi_voxel(g, bl.y, bx * 8 + e % 9, by * 8 + (e / 9) % 9, bz * 8 + e / 81);
    }
}

// The FIRE power in the CPU's order (src/v2m_particles.cpp:849-859: node 0
// first, one double accumulator), on one thread.
__device__ __noinline__ double serial_power(const float* __restrict__ pw, int64_t nofs, int n) {
    double t = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        t += (double)pw[nofs + i];
    }
    return t;
}

// Serial FIRE power of every iteration (V2M_CUDA_SERIAL_POWER=1); one thread per
// volume.
__global__ void k_power_serial(const DVol* __restrict__ vols, const VolCtl* __restrict__ ctl, const float* __restrict__ pw,
                               double* __restrict__ pser, int nvol) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvol) {
        return;
    }
    const DVol& V = vols[v];
    if (!V.fire || ctl[v].done || ctl[v].it >= V.max_iters) {
        return;
    }
    pser[v] = serial_power(pw, V.nofs, V.n);
}

// ---- the loop's control (one block per volume) ---------------------------------------
// Only the sign of the FIRE power matters (FireCtl::update, src/v2m_particles.h:58-73),
// and relax_cpu takes it from a serial double sum of the float powers. The
// block sums summed in a fixed tree give a sum P and a sum A of magnitudes.
// Every summation order of the n terms, the serial one and this tree alike, is
// within gamma_(n+64) A of the exact sum S (recursive summation error bound,
// gamma_k = k u / (1 - k u), u = 2^-53; no term passes through more than n + 64
// additions in either). So when |P| > kPowerGuard (n + 64) u A, S and the serial
// sum both have P's sign and P decides exactly as relax_cpu would. Otherwise
// (a sum within rounding of zero) the serial sum is taken on one thread. A = 0
// means every term is zero: every sum is +0.
constexpr double kPowerGuard = 2.5;   // 2 gamma_(n+64) A <= 2.0001 (n + 64) u A' for n < 2^31, with margin

__global__ void k_control(const DVol* __restrict__ vols, VolCtl* __restrict__ ctl, const double2* __restrict__ psum,
                          const double* __restrict__ pser, const float* __restrict__ pw, int serial, int move_threads,
                          Global* G) {
    const int v = blockIdx.x;
    const DVol& V = vols[v];
    VolCtl& c = ctl[v];
    __shared__ double red[kCtlThreads], reda[kCtlThreads];
    __shared__ int s_skip;
    if (threadIdx.x == 0) {
        s_skip = c.done || c.it >= V.max_iters;
        if (s_skip) {
            c.rebuild = 0;
        }
    }
    __syncthreads();
    if (s_skip) {
        return;
    }
    double P = 0.0, A = 0.0;
    if (V.fire && !serial) {
        const int b0 = (int)(V.nofs / move_threads);
        const int nb = (V.n + move_threads - 1) / move_threads;
        double t = 0.0, ta = 0.0;
        for (int b = threadIdx.x; b < nb; b += kCtlThreads) {
            const double2 q = psum[b0 + b];
            t += q.x;
            ta += q.y;
        }
        red[threadIdx.x] = t;
        reda[threadIdx.x] = ta;
        __syncthreads();
        for (int w = kCtlThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) {
                red[threadIdx.x] += red[threadIdx.x + w];
                reda[threadIdx.x] += reda[threadIdx.x + w];
            }
            __syncthreads();
        }
        P = red[0];
        A = reda[0];
    } else if (V.fire) {
        P = pser[v];
    }
    if (threadIdx.x != 0) {
        return;
    }
    if (V.fire && !serial) {
        if (A == 0.0) {
            P = 0.0;
        } else if (!(fabs(P) > kPowerGuard * ((double)V.n + 64.0) * 0x1p-53 * A)) {
            P = serial_power(pw, V.nofs, V.n);   // within rounding of zero: the CPU's own order
            ++c.serial_sums;
        }
    }
    const int it = c.it;
    if (V.fire) {
        c.power = P;
        if (P >= 0.0) {
            if (++c.npos > 5) {
                c.fdt = fminf(c.fdt * 1.1f, V.fire_dtmax);
                c.falpha *= 0.99f;
            }
            c.vzero = 0;
        } else {
            c.npos = 0;
            c.fdt = fmaxf(c.fdt * 0.5f, 0.05f * V.fire_dt0);
            c.falpha = 0.1f;
            ++c.resets;
            c.vzero = 1;
        }
    }
    c.iters = it + 1;
    // fold the move kernel's slots
    for (int k = 0; k < kCtlSlots; ++k) {
        c.maxbits = c.maxbits > c.maxbits_p[k] ? c.maxbits : c.maxbits_p[k];
        c.nhalf += c.nhalf_p[k];
        c.pad1 = (unsigned)c.pad1 > c.maxd_p[k] ? c.pad1 : (int)c.maxd_p[k];
        c.maxbits_p[k] = 0u;
        c.nhalf_p[k] = 0;
        c.maxd_p[k] = 0u;
    }
    c.last_move = __uint_as_float(c.maxbits);
    int acc = 0, b99 = 31;
    for (int b = 0; b < 32; ++b) {
        acc += c.hist[b];
        if ((double)acc >= 0.99 * (double)V.n) {
            b99 = b;
            break;
        }
    }
    const float p99 = ldexpf(1.0f, b99 - 20 + 1);
    c.last_p99 = p99;
    c.nhalf_last = c.nhalf;
    c.nrefresh_last = c.nrefresh;
    const float maxd = __uint_as_float((unsigned)c.pad1);
    for (int b = 0; b < 32; ++b) {
        c.hist[b] = 0;
    }
    c.maxbits = 0u;
    c.nhalf = 0;
    c.nrefresh = 0;
    c.pad1 = 0;
    c.it = it + 1;
    if (p99 < V.dptol && (!V.fire || c.fdt >= 0.25f * V.fire_dt0)) {
        c.done = 1;
        c.rebuild = 0;
        c.stop_reason = 1;
        return;
    }
    int reb;
    if (V.policy == 1) {
        reb = maxd > 0.1f;
    } else if (V.policy == 2) {
        reb = 0;
    } else {
        const bool endgame = it >= V.max_iters * 4 / 5 || p99 < 4.0f * V.dptol;
        const int div = endgame ? (V.rebuild_div > 1000 ? V.rebuild_div : 1000) : V.rebuild_div;
        reb = c.nhalf_last > V.n / div;
    }
    c.rebuild = reb;
    if (reb) {
        ++c.rebuilds;
        G->rebuild_any = 1;
    }
}

// ---- small utilities -----------------------------------------------------------------
__global__ void k_set_rebuild(VolCtl* ctl, int nvol, int val, Global* G) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v == 0) {
        G->rebuild_any = val;
    }
    if (v < nvol && !ctl[v].done) {
        ctl[v].rebuild = val;
        if (val) {
            ++ctl[v].rebuilds;
        }
    }
}

// The constraint direction of each node of one volume at its current position,
// for the differentiable unroll's trapped steps: an INTERFACE node's unit normal
// of psi_(own, partner) (it glides in the tangent plane), a JUNCTION node's unit
// junction-line direction, normal_(own, partner 1) x normal_(own, partner 2)
// (it moves along the line); zero for the others or where a gradient vanishes.
template <bool kShape>
__global__ void k_constraint_dirs(const DVol* __restrict__ vols, int v, const float4* __restrict__ Pq,
                                  const uint8_t* __restrict__ typ, const uint16_t* __restrict__ lab,
                                  const uint32_t* __restrict__ part, float* __restrict__ out) {
    const DVol& V = vols[v];
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= V.n) {
        return;
    }
    const int64_t i = V.nofs + t;
    const int ty = typ[i];
    float d[3] = { 0.0f, 0.0f, 0.0f };
    if (ty == V2M_INTERFACE || ty == V2M_JUNCTION) {
        const float4 p = Pq[i];
        const int a = lab[i], b = (int)(part[i] & 0xFFFFu), c = (int)(part[i] >> 16);
        const float4 g1 = psi_grad4<kShape>(V.g, a, b, p.x, p.y, p.z);
        float u[3] = { g1.x, g1.y, g1.z };
        if (ty == V2M_JUNCTION) {
            const float4 g2 = psi_grad4<kShape>(V.g, a, c, p.x, p.y, p.z);
            u[0] = g1.y * g2.z - g1.z * g2.y;
            u[1] = g1.z * g2.x - g1.x * g2.z;
            u[2] = g1.x * g2.y - g1.y * g2.x;
        }
        const float un = sqrtf(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        if (un > 0.0f) {
            d[0] = u[0] / un;
            d[1] = u[1] / un;
            d[2] = u[2] / un;
        }
    }
    out[3 * t] = d[0];
    out[3 * t + 1] = d[1];
    out[3 * t + 2] = d[2];
}

// Every list slot holds the node's own id until a list build writes it (the
// force kernel loads whole batches of slots, padding included).
__global__ void k_lists_init(int* __restrict__ nbr, int64_t N) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < N * V2M_K) {
        nbr[t] = (int)(t % N);
    }
}

// Row-major copy of the slot-major lists of one volume (for checks and read-back).
__global__ void k_lists_rowmajor(const int* __restrict__ nbr, const uint8_t* __restrict__ nnb, int64_t nofs, int n,
                                 int64_t N, int* __restrict__ out, int* __restrict__ nout) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * V2M_K) {
        return;
    }
    const int64_t i = t / V2M_K;
    const int k = (int)(t % V2M_K);
    const int c = nnb[nofs + i];
    out[t] = k < c ? nbr[(int64_t)k * N + nofs + i] - (int)nofs : 0;
    if (k == 0) {
        nout[i] = c;
    }
}

// The inverse: row-major host lists (local ids) into the slot-major store.
__global__ void k_lists_from_rowmajor(int* __restrict__ nbr, uint8_t* __restrict__ nnb, int64_t nofs, int n, int64_t N,
                                      const int* __restrict__ in, const int* __restrict__ nin) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * V2M_K) {
        return;
    }
    const int64_t i = t / V2M_K;
    const int k = (int)(t % V2M_K);
    const int c = nin[i];
    nbr[(int64_t)k * N + nofs + i] = k < c ? in[t] + (int)nofs : (int)(nofs + i);   // padded with the node's own id
    if (k == 0) {
        nnb[nofs + i] = (uint8_t)c;
    }
}

// Positions / types / sizes between the reference's layout and the packed one.
__global__ void k_pack_nodes(const float* __restrict__ P, const uint8_t* __restrict__ typ, const DVol* __restrict__ vols,
                             int v, float4* __restrict__ Pq) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const DVol& V = vols[v];
    if (t >= V.n) {
        return;
    }
    const float x = P[3 * t], y = P[3 * t + 1], z = P[3 * t + 2];
    const float h = size_at(V.g, V.hmode, x, y, z);
    Pq[V.nofs + t] = make_float4(x, y, z, pack_h(h, typ[V.nofs + t]));
}

__global__ void k_unpack_P(const float4* __restrict__ Pq, int64_t nofs, int n, float* __restrict__ P) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) {
        return;
    }
    const float4 p = Pq[nofs + t];
    P[3 * t] = p.x;
    P[3 * t + 1] = p.y;
    P[3 * t + 2] = p.z;
}

__global__ void k_hn(const float4* __restrict__ Pq, int64_t nofs, int n, float* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        out[t] = fabsf(Pq[nofs + t].w);
    }
}

__global__ void k_set_hn(float4* __restrict__ Pq, int64_t nofs, int n, const float* __restrict__ in,
                         const uint8_t* __restrict__ typ) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        const float4 p = Pq[nofs + t];
        Pq[nofs + t] = make_float4(p.x, p.y, p.z, pack_h(in[t], typ[nofs + t]));
    }
}

// Re-sign w after a host write of the types.
__global__ void k_resign(float4* __restrict__ Pq, const uint8_t* __restrict__ typ, int64_t nofs, int n) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        const float4 p = Pq[nofs + t];
        Pq[nofs + t] = make_float4(p.x, p.y, p.z, pack_h(fabsf(p.w), typ[nofs + t]));
    }
}

__global__ void k_float4_to3(const float4* __restrict__ a, int64_t nofs, int n, float* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        const float4 p = a[nofs + t];
        out[3 * t] = p.x;
        out[3 * t + 1] = p.y;
        out[3 * t + 2] = p.z;
    }
}

__global__ void k_float3_to4(const float* __restrict__ in, int64_t nofs, int n, float4* __restrict__ a) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        a[nofs + t] = make_float4(in[3 * t], in[3 * t + 1], in[3 * t + 2], 0.0f);
    }
}

// Local ids of a volume's bin-sorted node list.
__global__ void k_local_ids(const int* __restrict__ a, int64_t nofs, int n, int* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        out[t] = a[nofs + t] - (int)nofs;
    }
}

__global__ void k_local_cstart(const int* __restrict__ a, int64_t kofs, int cnt, int64_t nofs, int* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < cnt) {
        out[t] = a[kofs + t] - (int)nofs;
    }
}

// ---- launchers -----------------------------------------------------------------------
static inline unsigned nblk(int64_t n, int b) {
    return (unsigned)((n + b - 1) / b);
}

// grid of a grid-stride kernel: enough blocks to fill the GPU, no more
static inline unsigned gsblocks(const Dev& d, int64_t items, int per_block) {
    const int64_t need = (items + per_block - 1) / per_block;
    const int64_t cap = (int64_t)d.sms * 8;
    return (unsigned)std::max<int64_t>(1, std::min(need, cap));
}

void launch_keys(cudaStream_t s, const Dev& d) {
    k_keys<<<gsblocks(d, d.N, 256), 256, 0, s>>>(d.vols, d.ctl, d.nodevol, d.Pq, d.key, d.cnt, d.P0, d.N, d.G);
}

void launch_scan(cudaStream_t s, const Dev& d) {
    k_scan_tiles<<<d.ntile_key, kScanThreads, 0, s>>>(d.vols, d.ctl, d.tilevol, d.cnt, d.tilesum, d.KT);
    k_scan_vol<<<d.nvol, 1024, 0, s>>>(d.vols, d.ctl, d.tilesum, d.tileofs);
    k_scan_apply<<<d.ntile_key, kScanThreads, 0, s>>>(d.vols, d.ctl, d.tilevol, d.cnt, d.tileofs, d.cstart, d.cursor);
}

void launch_scatter(cudaStream_t s, const Dev& d) {
    k_scatter<<<gsblocks(d, d.N, 256), 256, 0, s>>>(d.ctl, d.vols, d.nodevol, d.key, d.cursor, d.sorted, d.N, d.G);
    k_binsort<<<gsblocks(d, d.KT, kBinSortThreads), kBinSortThreads, 0, s>>>(d.vols, d.ctl, d.tilevol, d.cstart,
                                                                             d.sorted, d.sort_tmp, d.Pq, d.typ, d.lab,
                                                                             d.Ps, d.Js, d.KT, d.G);
}

void launch_neighbors(cudaStream_t s, const Dev& d, int threads) {
    k_neighbors<<<gsblocks(d, d.N, threads / 32) * 2, threads, 0, s>>>(d.vols, d.ctl, d.nodevol, d.Pq, d.typ, d.lab,
                                                                        d.cstart, d.sorted, d.Ps, d.Js, d.nbr, d.nnb,
                                                                        d.N, d.G);
}

void launch_force(cudaStream_t s, const Dev& d, int threads) {
    k_force<<<nblk(d.N, threads), threads, 0, s>>>(d.vols, d.ctl, d.nodevol, d.Pq, d.nbr, d.nnb, d.F, d.N, d.G);
}

void launch_move(cudaStream_t s, const Dev& d) {
    k_move_pre<<<nblk(d.N, kMoveThreads), kMoveThreads, 0, s>>>(d.vols, d.ctl, d.nodevol, d.Pq, d.F, d.Vel, d.typ,
                                                                d.mv, d.pw, d.P0, d.S, d.queue, d.psum, d.rlist, d.G,
                                                                d.N);
    k_move_int<<<nblk(d.N, kMainThreads), kMainThreads, 0, s>>>(d.vols, d.ctl, d.nodevol, d.Pq, d.Vel, d.lab, d.mv,
                                                                d.P0, d.S, d.queue, d.rlist, d.G, d.N);
    k_move_main<false><<<nblk(d.N, kMainThreads), kMainThreads, 0, s>>>(
        d.vols, d.ctl, d.nodevol, d.Pq, d.Vel, d.typ, d.lab, d.part, d.mv, d.P0, d.S, d.queue, d.rlist, d.G, d.N,
        d.shape_any);
    if (d.shape_any) {
        k_move_main<true><<<nblk(d.N, kMainThreads), kMainThreads, 0, s>>>(
            d.vols, d.ctl, d.nodevol, d.Pq, d.Vel, d.typ, d.lab, d.part, d.mv, d.P0, d.S, d.queue, d.rlist, d.G, d.N,
            d.shape_any);
    }
}

void launch_xcount(cudaStream_t s, const DGrid& g, uint4* xbrick, int* xn, int nb) {
    k_xcount<<<nblk(nb, 128), 128, 0, s>>>(g, xbrick, xn, nb);
}

void launch_xfill(cudaStream_t s, const DGrid& g, const int2* tabs, float* xphi, int ntab) {
    if (ntab > 0) {
        k_xfill<<<ntab, 256, 0, s>>>(g, tabs, xphi);
    }
}

void launch_control(cudaStream_t s, const Dev& d, int serial) {
    if (serial) {
        k_power_serial<<<nblk(d.nvol, 32), 32, 0, s>>>(d.vols, d.ctl, d.pw, d.pser, d.nvol);
    }
    k_control<<<d.nvol, kCtlThreads, 0, s>>>(d.vols, d.ctl, d.psum, d.pser, d.pw, serial, kMoveThreads, d.G);
}

void launch_refresh(cudaStream_t s, const Dev& d, int blocks) {
    k_refresh<<<blocks, kNbrMaxThreads / 2, 0, s>>>(d.vols, d.ctl, d.nodevol, d.Pq, d.typ, d.lab, d.cstart, d.sorted, d.Ps,
                                              d.nbr, d.nnb, d.P0, d.rlist, d.G, d.N);
}

void launch_set_rebuild(cudaStream_t s, const Dev& d, int val) {
    k_set_rebuild<<<nblk(d.nvol, 128), 128, 0, s>>>(d.ctl, d.nvol, val, d.G);
}

void launch_constraint_dirs(cudaStream_t s, const Dev& d, int v, int n, bool shape, float* out) {
    if (shape) {
        k_constraint_dirs<true><<<nblk(n, 256), 256, 0, s>>>(d.vols, v, d.Pq, d.typ, d.lab, d.part, out);
    } else {
        k_constraint_dirs<false><<<nblk(n, 256), 256, 0, s>>>(d.vols, v, d.Pq, d.typ, d.lab, d.part, out);
    }
}

void launch_lists_init(cudaStream_t s, const Dev& d) {
    k_lists_init<<<nblk(d.N * V2M_K, 256), 256, 0, s>>>(d.nbr, d.N);
}

void launch_lists_rowmajor(cudaStream_t s, const Dev& d, int64_t nofs, int n, int* out, int* nout) {
    k_lists_rowmajor<<<nblk((int64_t)n * V2M_K, 256), 256, 0, s>>>(d.nbr, d.nnb, nofs, n, d.N, out, nout);
}

void launch_lists_from_rowmajor(cudaStream_t s, const Dev& d, int64_t nofs, int n, const int* in, const int* nin) {
    k_lists_from_rowmajor<<<nblk((int64_t)n * V2M_K, 256), 256, 0, s>>>(d.nbr, d.nnb, nofs, n, d.N, in, nin);
}

void launch_pack_nodes(cudaStream_t s, const Dev& d, int v, int n, const float* P, const uint8_t* typ_all) {
    k_pack_nodes<<<nblk(n, 256), 256, 0, s>>>(P, typ_all, d.vols, v, d.Pq);
}

void launch_unpack_P(cudaStream_t s, const Dev& d, int64_t nofs, int n, float* P) {
    k_unpack_P<<<nblk(n, 256), 256, 0, s>>>(d.Pq, nofs, n, P);
}

void launch_hn(cudaStream_t s, const Dev& d, int64_t nofs, int n, float* out) {
    k_hn<<<nblk(n, 256), 256, 0, s>>>(d.Pq, nofs, n, out);
}

void launch_set_hn(cudaStream_t s, const Dev& d, int64_t nofs, int n, const float* in) {
    k_set_hn<<<nblk(n, 256), 256, 0, s>>>(d.Pq, nofs, n, in, d.typ);
}

void launch_resign(cudaStream_t s, const Dev& d, int64_t nofs, int n) {
    k_resign<<<nblk(n, 256), 256, 0, s>>>(d.Pq, d.typ, nofs, n);
}

void launch_float4_to3(cudaStream_t s, const float4* a, int64_t nofs, int n, float* out) {
    k_float4_to3<<<nblk(n, 256), 256, 0, s>>>(a, nofs, n, out);
}

void launch_float3_to4(cudaStream_t s, const float* in, int64_t nofs, int n, float4* a) {
    k_float3_to4<<<nblk(n, 256), 256, 0, s>>>(in, nofs, n, a);
}

void launch_local_ids(cudaStream_t s, const int* a, int64_t nofs, int n, int* out) {
    k_local_ids<<<nblk(n, 256), 256, 0, s>>>(a, nofs, n, out);
}

void launch_local_cstart(cudaStream_t s, const int* a, int64_t kofs, int cnt, int64_t nofs, int* out) {
    k_local_cstart<<<nblk(cnt, 256), 256, 0, s>>>(a, kofs, cnt, nofs, out);
}

}  // namespace v2m
