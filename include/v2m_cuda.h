/*
 * v2m_cuda.h -- C ABI of the B200 (sm_100a) relaxation library libv2m_cuda.so.
 *
 * The library replaces v2mesh's OpenCL relaxation, tn::relax_cl
 * (src/v2m_gpu.h:16-18 in fangq/trussnet), behind plain C: POD views of the
 * reference's Grid / RelaxParams / Nodes / RelaxStats, host pointers and sizes,
 * an int status (0 = ok, < 0 = error) and a thread-local error text. The C++
 * shim libv2m_relax_cl.so builds tn::relax_cl with the reference's exact
 * signature on top of these entry points, so the reference's v2m_core links
 * against it unchanged (the pipeline's CPU fallback still catches its
 * std::runtime_error).
 *
 * Nothing here falls back to the CPU: without a usable CUDA device every entry
 * point returns V2M_ERR_CUDA.
 */
#ifndef V2M_CUDA_H
#define V2M_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define V2M_CUDA_ABI_VERSION 1

/* status codes */
#define V2M_OK 0
#define V2M_ERR_ARG (-1)      /* invalid argument (sizes, null pointers, limits) */
#define V2M_ERR_CUDA (-2)     /* a CUDA runtime call failed (no device, out of memory, launch) */
#define V2M_ERR_KERNEL (-3)   /* a kernel raised its error flag (index out of range, bounded wait) */
#define V2M_ERR_STATE (-4)    /* call out of order (e.g. force before the first rebuild) */

/* node types (src/opencl/v2m_seed_body.cl:15-19) */
#define V2M_INTERIOR 0
#define V2M_INTERFACE 1
#define V2M_JUNCTION 2
#define V2M_CORNER 3
#define V2M_NOLAB 0xFFFF

#define V2M_K 24        /* truss neighbours per node (src/opencl/v2m_particle_body.cl:18) */
#define V2M_MAXLEV 8    /* hash levels (src/opencl/v2m_particle_body.cl:19) */
#define V2M_BS 8        /* brick side (src/opencl/v2m_grid_body.cl:20) */
#define V2M_SLOT 512    /* phi values per (brick, label) slot (src/opencl/v2m_grid_body.cl:21) */
#define V2M_BL 16       /* labels per brick (src/opencl/v2m_grid_body.cl:22) */

/*
 * The read-only fields the relaxation samples: tn::Grid (src/v2m_grid.h:45-81),
 * the members relax_cl reads. Every array is caller-owned host memory, x-fastest
 * (index i + nx*(j + ny*k)); bricks are 8^3 voxels, nb = nbx*nby*nbz.
 */
typedef struct {
    int32_t nx, ny, nz;          /* voxels */
    int32_t nbx, nby, nbz;       /* bricks: ceil(n / 8) per axis */
    float vs[3];                 /* voxel size (mm) */
    const uint16_t* L;           /* labels, nx*ny*nz */
    const int32_t* bl_cnt;       /* nb: labels within R of each brick (V2M_BL+1 = overflow) */
    const uint16_t* bl_lab;      /* V2M_BL*nb: those labels, ascending, 0xFFFF padded */
    const int32_t* bl_slot;      /* nb: first slot of each mixed brick, -1 = uniform */
    const float* phi;            /* V2M_SLOT*nslots smoothed indicators */
    int64_t nslots;
    const float* h;              /* nx*ny*nz target size (mm) */
    float hmin, hmax;            /* range of h (mm): the hash geometry */
    const float* gI;             /* gray-scale intensity nx*ny*nz (gm > 0), else NULL */
    const float* gTW;            /* gray-scale [t_0..t_{m-1}, W_0..W_{m-1}] (gm > 0); the labels' compiled
                                    analytic fields (gm < 0, the layout of src/opencl/v2m_sdf_body.cl:9-21);
                                    else NULL */
    int32_t gm;                  /* number of gray thresholds; 0 = label volume; < 0 = analytic shape fields */
    int64_t ngTW;                /* floats in gTW (tn::Grid::gTW.size()); 0 = 2 gm (gray-scale) */
    const uint8_t* grade;        /* nx*ny*nz size grades (tn::Grid::grade): seeding only, may be NULL */
    const float* feat;           /* shape input's sharp features (tn::Grid::feat, grid mm, the layout of
                                    src/v2m_sdfshape.h ShapeScene::feat): seeding pins nodes on them; may be NULL */
    int64_t nfeat;               /* floats in feat */
} v2m_grid_view;

/*
 * tn::RelaxParams (src/v2m_particles.h:21-41), same names and meaning, plus
 * three extensions (0 keeps the reference's behaviour).
 */
typedef struct {
    int32_t nseed;
    float t, skin, fscale, fsurf, dt, maxstep, snap;
    int32_t max_iters;
    float dptol, jseed;
    int32_t corners, voxel_trap;
    float thin;
    int32_t fire;
    float fire_dtmax;
    int32_t verbose;
    /* extensions */
    int32_t h_mode;          /* 0: h at the nearest voxel (reference); 1: trilinear h */
    int32_t rebuild_div;     /* Verlet trigger divisor; 0: V2M_REBUILD_DIV or 300 (src/v2m_gpu.cpp:119) */
    int32_t rebuild_policy;  /* 0: reference Verlet trigger; 1: rebuild when max |dp| since the build > 0.1 h;
                                2: fixed lists -- the first build's lists for the whole run (no rebuild, no
                                self-refresh) */
} v2m_relax_params;

/* tn::Nodes (src/v2m_particles.h:78-87): the node arrays, caller-owned host memory. */
typedef struct {
    int64_t n;
    float* P;              /* 3n positions (grid mm), in/out */
    const uint16_t* lab;   /* n own labels */
    uint8_t* typ;          /* n types, in/out */
    uint16_t* part;        /* 2n partner labels, in/out */
} v2m_nodes_view;

/* tn::RelaxStats (src/v2m_particles.h:89-96). */
typedef struct {
    int32_t iters, rebuilds;
    float last_move, last_p99;
    int32_t fire_resets;
    float fire_dt;
    int64_t n_interior, n_interface, n_junction, n_corner;
    double ms_seed, ms_hash, ms_force, ms_move;
} v2m_relax_stats;

/* The reference's RelaxParams defaults (src/v2m_particles.h:22-40). */
void v2m_relax_params_default(v2m_relax_params* p);

/* Text of the last error on this thread ("" if none). */
const char* v2m_cuda_last_error(void);

/* Number of CUDA devices (0 when none or the driver is missing). */
int v2m_cuda_device_count(void);

/*
 * Relax the nodes on CUDA device `device` (-1 = device 0). Same contract as
 * tn::relax_cl (src/v2m_gpu.cpp:116-553) and tn::relax_cpu
 * (src/v2m_particles.cpp:728-976): positions, types and partner labels are
 * updated in place, the node count and order are unchanged. Host buffers in,
 * host buffers out; the grid is uploaded on every call.
 */
int v2m_relax_cuda(const v2m_grid_view* g, const v2m_relax_params* prm, v2m_nodes_view* nd, v2m_relax_stats* st,
                   int device);

/*
 * Seeding on CUDA device `device` (-1 = device 0): tn::seed_cpu
 * (src/v2m_particles.cpp:625-726) -- the graded HCP lattice of the grid's size
 * grades (g->grade is required), each node classified onto its interface or
 * junction curve, the junction-line seeds (params->jseed > 0) with the lattice
 * nodes near them dropped, the CORNER nodes (params->corners), and, for shape
 * input with features (g->feat, read on the host), the feature pass
 * (add_feature_nodes, :304-623: CORNER nodes pinned on the sharp features, the
 * seeds within 0.4 h of them dropped), in the reference's order and bit for bit. Uses
 * nseed, jseed, corners and voxel_trap of the parameters. *n receives the node
 * count and *out a result to copy out (v2m_seed_copy: P 3n floats, lab n,
 * typ n, part 2n, part3 n or NULL) and free (v2m_seed_free).
 */
typedef struct v2m_seed_result v2m_seed_result;
int v2m_seed_cuda(const v2m_grid_view* g, const v2m_relax_params* prm, int device, v2m_seed_result** out,
                  int64_t* n);
int v2m_seed_copy(const v2m_seed_result* r, float* P, uint16_t* lab, uint8_t* typ, uint16_t* part, uint16_t* part3);
void v2m_seed_free(v2m_seed_result* r);

/*
 * tn::GridParams (src/v2m_grid.h:21-43) for the device grid build, same names
 * and meaning; label input only: no interface sizes, no user sizing field.
 */
typedef struct {
    float sigma, sigma_thin, thin_lo, thin_hi, thick, thin_floor, preserve, sigma_curv, hbase, hmin, hmax, K, g;
    const float* hlab;   /* per-label size (mm), index = label, 0 = hbase; NULL (nhlab = 0): none */
    int32_t nhlab;
} v2m_grid_params;

/* The reference's GridParams defaults (src/v2m_grid.h:22-37). */
void v2m_grid_params_default(v2m_grid_params* p);

/*
 * The relaxation's fields built on CUDA device `device` (-1 = device 0) from a
 * label volume: tn::build_grid_cpu (src/v2m_grid.cpp:47-722) for label input,
 * bit for bit -- the labels within R of each brick, one slot per (mixed brick,
 * label), the smoothed indicators (sigma, blended with sigma_thin by the local
 * thickness), the sizing field (label sizes, curvature bound, gradient limit)
 * and the size grades. L: nx*ny*nz labels (host, x fastest); vs: voxel size
 * (mm). *out receives the grid, read through v2m_grid_result_view (host arrays
 * owned by the result; the view's L is the result's copy of the labels) and
 * freed by v2m_grid_free. The steps that call the C library's logf in the
 * reference (the thickness's erfinv, the grades) evaluate it on the host.
 */
typedef struct v2m_grid_result v2m_grid_result;
int v2m_grid_build_cuda(const uint16_t* L, int32_t nx, int32_t ny, int32_t nz, const float* vs,
                        const v2m_grid_params* p, int device, v2m_grid_result** out);
int v2m_grid_result_view(const v2m_grid_result* r, v2m_grid_view* g);
/* hbase (mm), the brick label radius R, the slot count and the gradient-limit sweeps of a built grid */
int v2m_grid_result_info(const v2m_grid_result* r, float* hbase, int32_t* R, int64_t* nslots, int32_t* limit_sweeps);
void v2m_grid_free(v2m_grid_result* r);

/*
 * The pipeline's points mode on the device (run_pipeline with stop_after_relax,
 * src/v2m_pipeline.cpp:424-565; `v2mesh --mode points`): the label volume is
 * uploaded once, its grid built (v2m_grid_build_cuda), seeded (v2m_seed_cuda)
 * and relaxed (v2m_relax_cuda) with every stage reading the previous one's
 * device arrays, and the relaxed nodes are copied back once: *n nodes in *out
 * (read with v2m_seed_copy: P, lab, typ, part, part3; freed with
 * v2m_seed_free), bit for bit build_grid_cpu -> seed_cpu -> relax_cpu. st may
 * be NULL.
 */
int v2m_points_cuda(const uint16_t* L, int32_t nx, int32_t ny, int32_t nz, const float* vs, const v2m_grid_params* gp,
                    const v2m_relax_params* prm, int device, v2m_seed_result** out, int64_t* n, v2m_relax_stats* st);

/*
 * Many independent volumes in one set of launches (one per stage for all of
 * them), the iteration loop captured in a CUDA graph. Each volume keeps its own
 * hash, lists, FIRE state and stop / rebuild decisions, so volume v's result is
 * the one v2m_relax_cuda gives for it alone. No counterpart in the reference,
 * which relaxes one volume per call (src/v2m_pipeline.cpp:492-536).
 */
int v2m_relax_cuda_batch(int nvol, const v2m_grid_view* g, const v2m_relax_params* prm, v2m_nodes_view* nd,
                         v2m_relax_stats* st, int device);

/*
 * Sessions: the relaxation state kept on the device between calls, for step-wise
 * use (the stages of relax_cl one at a time), repeated runs from the same seeds,
 * and batches. A session owns device copies of the grids and of the seeds.
 */
typedef struct v2m_session v2m_session;

int v2m_session_create(int nvol, const v2m_grid_view* g, const v2m_relax_params* prm, const v2m_nodes_view* nd,
                       int device, v2m_session** out);
int v2m_session_destroy(v2m_session* s);
/* Back to the seeds: positions, types, partners, velocities, FIRE state, counters. */
int v2m_session_reset(v2m_session* s);
/* relax_cl's rebuild (src/v2m_gpu.cpp:259-277): keys, stable counting sort, bin-order gather, K-nearest lists. */
int v2m_session_rebuild(v2m_session* s);
/* k_force (src/opencl/v2m_kernels.cl:159-169) for every node. */
int v2m_session_force(v2m_session* s);
/*
 * The rest of one iteration (src/v2m_particles.cpp:838-946): move, FIRE update,
 * histogram / p99, stop test, Verlet self-refresh and rebuild trigger (the
 * rebuild itself included when it fires).
 */
int v2m_session_step_tail(v2m_session* s);
/* Up to `iters` whole iterations (force + tail); graph != 0 replays a captured CUDA graph. */
int v2m_session_iterate(v2m_session* s, int iters, int graph);
/* A whole relaxation from the current state: first rebuild, then the loop to max_iters or convergence. */
int v2m_session_run(v2m_session* s, int graph);
int v2m_session_synchronize(v2m_session* s);
/* Write the current nodes (P, typ, part) of volume `vol` into nd (host). */
int v2m_session_read_nodes(v2m_session* s, int vol, v2m_nodes_view* nd);
int v2m_session_stats(v2m_session* s, int vol, v2m_relax_stats* st);

/* Internal arrays of volume `vol` copied to host memory, for parity checks. */
#define V2M_ARR_KEY 1        /* int32 [n]   bin key of each node (level offset + bin) */
#define V2M_ARR_SORTED 2     /* int32 [n]   node ids in (key, id) order */
#define V2M_ARR_CSTART 3     /* int32 [nkeys+1] bin starts */
#define V2M_ARR_PS 4         /* float [4n]  positions + h in bin order */
#define V2M_ARR_NBR 5        /* int32 [K*n] truss lists, row-major nbr[i*K+k] as the reference */
#define V2M_ARR_NNB 6        /* int32 [n]   list lengths */
#define V2M_ARR_F 7          /* float [4n]  force + active bars */
#define V2M_ARR_HN 8         /* float [n]   h at each node */
#define V2M_ARR_MV 9         /* float [n]   |dp| / h of the last move */
#define V2M_ARR_V 10         /* float [3n]  FIRE velocities */
#define V2M_ARR_PW 11        /* float [n]   FIRE power a.v of the last move */
#define V2M_ARR_P0 12        /* float [3n]  positions at the last list build */
#define V2M_ARR_HIST 13      /* int32 [34]  log2 histogram, max |dp|/h bits, half-skin count */
#define V2M_ARR_SERIAL_SUMS 14 /* int32 [1] iterations whose FIRE power was within rounding of zero, so that
                                  its sign was taken from relax_cpu's serial order */
#define V2M_ARR_DIRS 15      /* float [3n]  each node's constraint direction at its position (read only): an
                                  INTERFACE node's unit normal of psi_(own, partner), a JUNCTION node's unit
                                  junction-line direction, zero otherwise -- v2m_unroll_set_constraints' input */
int v2m_session_read_array(v2m_session* s, int vol, int what, void* host, int64_t bytes);
/* Overwrite an internal array of volume `vol` from host memory (P, typ, part, nbr, nnb, V, hn). */
int v2m_session_write_array(v2m_session* s, int vol, int what, const void* host, int64_t bytes);
/* Overwrite the truss lists of volume `vol` (row-major nbr[i*K+k], local ids, and nnb). */
int v2m_session_write_lists(v2m_session* s, int vol, const int32_t* nbr, const int32_t* nnb);
#define V2M_ARR_P 20         /* float [3n]  positions */
#define V2M_ARR_TYP 21       /* uint8 [n]   types */
#define V2M_ARR_PART 22      /* uint16 [2n] partner labels */

/* Sizes of volume `vol`: n nodes, nkeys bins, hash levels. */
int v2m_session_info(v2m_session* s, int vol, int64_t* n, int64_t* nkeys, int32_t* nlev);

/*
 * Kernel launches issued so far by the session (all kernels of this library),
 * and the device time of the force kernel's launches (CUDA events), for the
 * roofline figures of the benchmark.
 */
int v2m_session_counters(v2m_session* s, int64_t* launches, int64_t* force_launches, double* force_ms);

/*
 * Benchmark helper: `runs` whole relaxations from the seeds (reset, first
 * rebuild, loop), bracketed by CUDA events on the session's stream; the elapsed
 * device time in *ms. time_force != 0 also records events around every force
 * launch (read back with v2m_session_counters).
 */
int v2m_session_timed_runs(v2m_session* s, int runs, int graph, int time_force, float* ms);

/*
 * Autotuner: times the launch shapes that cannot change a result (the force
 * kernel's block, the list kernel's warps per block) on the session's own
 * lists, keeps the fastest, appends it to the tuning cache
 * (V2M_CUDA_TUNE_CACHE, default $HOME/.cache/v2m_cuda_tune.txt) and resets the
 * session to its seeds. A session created with V2M_CUDA_AUTOTUNE=1 uses the
 * cached shapes or tunes once. `report` (may be NULL) receives the timings.
 */
int v2m_session_autotune(v2m_session* s, int reps, char* report, int64_t report_len);
int v2m_session_shapes(v2m_session* s, int32_t* force_threads, int32_t* nbr_threads);
int v2m_session_clear_counters(v2m_session* s);
/*
 * Per-stage device milliseconds over `iters` iterations from the current state,
 * plain launches with CUDA events between the stages: ms[0] force, ms[1] move,
 * ms[2] control + self-refresh, ms[3] the rebuild stages, ms[4] the iterations.
 */
int v2m_session_profile_stages(v2m_session* s, int iters, double* ms);
/* Nodes the last iteration's move handed to the trapped-move stage: non-INTERIOR and INTERIOR ones. */
int v2m_session_queue_sizes(v2m_session* s, int32_t* trapped, int32_t* interior);

/*
 * The differentiable relaxation unroll and its adjoint (no counterpart in the
 * reference). K Jacobi relaxation steps on frozen lists (row-major nbr[i*K+k],
 * local ids, as v2m_session_read_array returns them), the target size h(x)
 * interpolated trilinearly in a sizing grid G of m[0] x m[1] x m[2] values
 * (x fastest) at x = (a cs[0], b cs[1], c cs[2]); the active bars of each step
 * are taped by the forward pass and replayed by the backward pass; checkpoints
 * every `ckpt` steps. Loss = sum over the list entries of (l_ij / h_ij - 1)^2.
 * Position, gradient and grid arrays are DEVICE pointers (float, x/y/z
 * interleaved per node); the calls synchronize before returning. At most 2^29
 * nodes, and no node in more than 255 lists.
 */
typedef struct v2m_unroll v2m_unroll;
int v2m_unroll_create(int64_t n, const int32_t* nbr, const int32_t* nnb, const uint8_t* typ, const int32_t* m,
                      const float* cs, float fscale, float fsurf, float dt, int K, int ckpt, int device,
                      v2m_unroll** out);
int v2m_unroll_destroy(v2m_unroll* u);
/* K steps from x0 into xK; replay != 0 reuses the tape of the last recording forward pass */
int v2m_unroll_forward(v2m_unroll* u, const float* x0, const float* G, float* xK, int replay);
/* loss at x (host double) */
int v2m_unroll_loss(v2m_unroll* u, const float* x, const float* G, double* loss);
/* gx = gscale dLoss/dx at x; gG = gscale dLoss/dG (accumulate != 0: added to the internal grid accumulator) */
int v2m_unroll_loss_backward(v2m_unroll* u, const float* x, const float* G, float gscale, float* gx, float* gG,
                             int accumulate);
/* reverse of the last forward pass: gx0 = dL/dx0 and gG = dL/dG (+ gG_in if not NULL) from gxK = dL/dxK */
int v2m_unroll_backward(v2m_unroll* u, const float* G, const float* gxK, float* gx0, float* gG, const float* gG_in);
/* Taped constraints, the trapped move frozen like the active bars: with dirs (HOST float [3n], x/y/z per
 * node) each INTERFACE node's step is projected onto the plane normal to its direction (it glides in its
 * interface's tangent plane) and each JUNCTION node's onto its direction (it moves along the junction
 * line); other types and zero directions are unconstrained (CORNER nodes stay, as always). The
 * directions are normalised and stay fixed over the unroll; V2M_ARR_DIRS of a session gives them at the
 * session's positions. dirs = NULL removes the constraints. Either way the next forward pass records a
 * new tape (replay before it is an error). */
int v2m_unroll_set_constraints(v2m_unroll* u, const float* dirs);
/* the tape (K x n active-bar masks) to host memory */
int v2m_unroll_tape(v2m_unroll* u, uint32_t* host, int64_t count);
/* device milliseconds of the last forward (K steps) and backward passes */
int v2m_unroll_timing(v2m_unroll* u, float* ms_forward, float* ms_backward);
const char* v2m_unroll_last_error(void);

/*
 * Host-side check of truss lists (no device is used): row-major nbr[i*V2M_K+k]
 * (local ids) and nnb[i] of n nodes, held to the rules of the reference's list
 * build (v2m_neighbors, src/opencl/v2m_particle_body.cl:73-151): 0 <= nnb <=
 * V2M_K, ids in [0, n), no self-edge, no repeated id, and entries in strictly
 * ascending (distance, id) order, the distance recomputed with the list build's
 * float expression from the positions the lists were built from -- pi (3n
 * floats): each node's position at its last build (V2M_ARR_P0); pj (3n floats):
 * each node's position in the bin-order snapshot of the last full build (Ps by
 * way of the sorted ids). Returns V2M_OK, or V2M_ERR_KERNEL with the first
 * violation in `report` (and v2m_cuda_last_error). No counterpart in the
 * reference, which has no list checker.
 */
int v2m_validate_lists(int64_t n, const int32_t* nbr, const int32_t* nnb, const float* pi, const float* pj,
                       char* report, int64_t report_len);

/*
 * The hash's stable counting sort with no device allocation, for callers that
 * cannot call cudaMalloc: a process whose GPU memory belongs to its own pool (a
 * framework's caching allocator, a host application that reserved most of the
 * device), where a library allocation can fail or fragment the pool and
 * cudaFree would synchronize the whole device. No counterpart in the
 * reference.
 *
 * key: DEVICE int32[n], each in [0, nbins); outputs, DEVICE buffers of the
 * caller: sorted int32[n] (node ids by (key, id)) and cstart int32[nbins + 1]
 * (bin starts) -- what the hash build produces (v2m_session_read_array's
 * V2M_ARR_SORTED / V2M_ARR_CSTART). stream: a cudaStream_t, NULL for the legacy
 * default stream. The call is synchronous: it waits on `stream` and returns
 * when the sort is done. A key outside [0, nbins) returns V2M_ERR_ARG.
 *
 * Scratch is a fixed array in the library's device memory (about 24 MB, on every
 * GPU that loads the library, until exit): nbins is limited to
 * V2M_NOALLOC_MAX_BINS and n to V2M_NOALLOC_MAX_KEYS, larger requests return
 * V2M_ERR_ARG. Its device address is looked up on the first call made on each
 * device; a cudaDeviceReset of that device makes it stale (do not call again on
 * that device in the same process). Calls share the array: calls that overlap
 * on the GPU race. Bins of any size cost work linear in their size.
 */
#define V2M_NOALLOC_MAX_BINS (1 << 20)
#define V2M_NOALLOC_MAX_KEYS (1 << 22)
int v2m_bin_sort_noalloc(const int32_t* key, int64_t n, int64_t nbins, int32_t* sorted, int32_t* cstart,
                         void* stream);
const char* v2m_bin_sort_noalloc_error(void);

#ifdef __cplusplus
}
#endif

#endif /* V2M_CUDA_H */
