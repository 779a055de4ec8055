// v2m_types.cuh -- the device-side descriptors of the relaxation (host and device).
//
// A launch covers every volume of a session at once: node, bin and tile indices
// are flat over the volumes, and each thread block works inside one volume (its
// tile), whose descriptor (DVol) and mutable control block (VolCtl) it reads.
#pragma once

#include <cstdint>

#ifndef V2M_K
#define V2M_K 24
#define V2M_MAXLEV 8
#define V2M_BS 8
#define V2M_SLOT 512
#define V2M_BL 16
#define V2M_INTERIOR 0
#define V2M_INTERFACE 1
#define V2M_JUNCTION 2
#define V2M_CORNER 3
#define V2M_NOLAB 0xFFFF
#endif

namespace v2m {

// The read-only fields of one volume (tn::Grid, src/v2m_grid.h:45-81), device pointers.
struct DGrid {
    int nx, ny, nz, nbx, nby, nbz;
    float vx, vy, vz;
    const uint16_t* L;
    const int* bl_cnt;
    const uint16_t* bl_lab;
    const int* bl_slot;
    const float* phi;
    const float* hvox;
    const float* gI;
    const float* gTW;       // gray: thresholds and widths; gm < 0: the analytic shape program
    int gm;
    int64_t ntw;            // floats in gTW
    // Corner tables (built once per session): for every brick, the labels met by
    // a trilinear cell based in it (its own, its + neighbours' and, past the
    // grid's edge, label 0) and, per label, the 9x9x9 voxel values of the brick
    // plus a one-voxel halo on the + sides, each the reference's per-voxel phi.
    // Any cell based inside the grid then reads its 8 corners from one table.
    // A brick's record is 48 bytes, read as three 16-byte loads issued together:
    // int count (labels listed; -1: no table, the per-corner path), int first
    // table (-1: uniform, the first label is 1 at every corner), 16 u16 labels,
    // 8 bytes of padding.
    const uint4* xbrick;    // 3 per brick
    const float* xphi;      // 729 floats per table, x fastest
    int64_t nslots;         // phi slots (512 floats each)
    int64_t ntab;           // corner tables (729 floats each)
    // The checked build (V2M_CHECK) records its first failed bounds check here
    // (code, index) and skips the access; the host reads it after each run.
    int* chk;
};

// V2M_CHECK: the build with device bounds checks on the lookups whose ranges
// hold by construction (the sanitizer substitute: a failed check records an
// error code and its index, skips the access, and the call returns
// V2M_ERR_KERNEL; nothing traps). Without it the checks compile away.
#ifdef V2M_CHECK
constexpr bool kChecked = true;
#else
constexpr bool kChecked = false;
#endif

__device__ __forceinline__ void check_fail(int* chk, int code, long long info) {
    if (chk && atomicCAS(chk, 0, code) == 0) {
        chk[1] = (int)info;
    }
}

// Multi-level hash geometry (V2mHash, src/opencl/v2m_particle_body.cl:21-27).
struct DHash {
    float b0;
    int nlev;
    float ox, oy, oz;
    int dim[V2M_MAXLEV][3];
    int off[V2M_MAXLEV];
};

// One volume: fields, hash, where its nodes / bins / tiles live, its parameters.
struct DVol {
    DGrid g;
    DHash H;
    int64_t nofs;      // first node (flat)
    int n;             // nodes
    int64_t kofs;      // first bin-start entry (flat; the volume owns nkeys + 1 entries)
    int nkeys;
    // tiles: [tofs_node, +ntile_node) node tiles, [tofs_key, +ntile_key) bin tiles
    int tofs_node, ntile_node, tofs_key, ntile_key;
    // parameters (tn::RelaxParams)
    float t, skin, fscale, fsurf, dt, maxstep, snap, dptol;
    int voxmode, fire, max_iters, rebuild_div, hmode, policy;
    float fire_dt0, fire_dtmax;
    // 1: every node's stored size (|Pq.w|) is the size field at its position --
    // true from the seeds on (the pack and every move set it so); 0 after a
    // caller wrote positions or sizes directly, until the next reset
    int hn_exact;
};

// Mutable per-volume loop state (relax_cpu's locals, src/v2m_particles.cpp:822-946).
struct VolCtl {
    int it;            // iterations done
    int done;          // 1: converged or max_iters reached (every later stage is a no-op)
    int rebuild;       // 1: the rebuild stages run at the end of this iteration
    int vzero;         // 1: FIRE reset: the next move starts from zero velocities
    float fdt, falpha; // FIRE time step and steering
    int npos, resets;
    int rebuilds;      // lists built so far
    int iters;         // RelaxStats.iters
    float last_move, last_p99;
    double power;      // last FIRE power sum
    int nhalf_last, nrefresh_last, stop_reason;
    int serial_sums;   // iterations whose FIRE power was within rounding of zero (summed serially)
    // accumulators of the current iteration (cleared by the control stage)
    int hist[32];
    unsigned int maxbits;
    int nhalf;
    int nrefresh;
    int pad1;
    // the move kernel's partial max / half-skin count / max displacement, spread
    // over kCtlSlots slots (by block) to keep its atomics off one address; the
    // control stage folds them into maxbits, nhalf and pad1
    unsigned int maxbits_p[16];
    int nhalf_p[16];
    unsigned int maxd_p[16];
};

constexpr int kCtlSlots = 16;

// Session-wide counters and the self-refresh work list.
struct Global {
    int nrefresh;        // entries in the refresh list
    int blocks_done;     // last-block-done counter of the refresh kernel
    int err;             // kernel error flag (first error code)
    int err_info;
    int qtrap, qint;     // move queue lengths: trapped non-junction nodes (front), interior nodes (back)
    int qtrap_last, qint_last;   // the last iteration's queue lengths (trapped: junctions included)
    int rebuild_any;     // some volume rebuilds this iteration (the rebuild stages return at once otherwise)
    int qjun;            // junction moves (queue[N, N + qjun))
    int qdef;            // INTERIOR moves k_move_int hands to k_move_main (queue[N + qjun, N + qjun + qdef))
};

constexpr int kMaxVol = 1024;

}  // namespace v2m
