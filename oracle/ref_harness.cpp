// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY. A C-ABI harness around the
// reference's own CPU relaxation, compiled from fangq/trussnet's sources where
// they lie (oracle/Makefile) into oracle/_ref/libv2m_ref.so. Only the tests,
// the smoke check and the benchmark's CPU-baseline leg load it, as the checker;
// the CUDA library never does.
//
// What it exposes:
//   ref_relax_cpu      tn::relax_cpu itself (src/v2m_particles.cpp:728-976)
//   ref_grid_build     tn::build_grid_cpu (src/v2m_grid.cpp) on a label volume
//   ref_shape_grid     shape input: the reference's shape compiler
//                      (src/v2m_sdfshape.cpp) on a JSON scene, its raster's argmax
//                      labels through build_grid_cpu, and the grid's fields set to
//                      the compiled program (gm = -1), as src/v2m_grid.cpp:350-353
//   ref_seed           tn::seed_cpu (src/v2m_particles.cpp:624-635)
//   ref_state_*        relax_cpu's loop split into its stages (rebuild / force /
//                      the rest of an iteration) over the reference's own bodies
//                      (v2m_bin_key, v2m_neighbors, v2m_force, v2m_move from
//                      src/opencl/v2m_particle_body.cl), so a device stage can be
//                      compared with the reference stage on identical inputs.
//                      ref_state_run replays the whole loop; a test checks that it
//                      equals ref_relax_cpu bit for bit.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "v2m_grid.h"
#include "v2m_omp.h"
#include "v2m_particles.h"
#include "v2m_sdfshape.h"
#include "v2m_volume.h"

#include "../include/v2m_cuda.h"

namespace refbody {
using std::ceil;
using std::exp;
using std::fabs;
using std::floor;
using std::fmax;
using std::fmin;
using std::log;
using std::pow;
using std::sqrt;
typedef uint8_t uchar;
typedef uint16_t ushort;
#undef V2M_K
#undef V2M_MAXLEV
#undef V2M_BS
#undef V2M_SLOT
#undef V2M_BL
#undef V2M_INTERIOR
#undef V2M_INTERFACE
#undef V2M_JUNCTION
#undef V2M_CORNER
#undef V2M_NOLAB
#define V2M_G
#include "opencl/v2m_grid_body.cl"
#include "opencl/v2m_sdf_body.cl"
#include "opencl/v2m_seed_body.cl"
#include "opencl/v2m_particle_body.cl"
#undef V2M_G
}  // namespace refbody

using namespace refbody;

namespace {

thread_local std::string g_err;

// A tn::Grid that owns copies of a v2m_grid_view's arrays.
struct OwnedGrid {
    tn::Grid g;
    std::vector<uint16_t> L;
    std::vector<float> gI;
};

void grid_from_view(const v2m_grid_view* v, OwnedGrid& o) {
    const size_t nv = static_cast<size_t>(v->nx) * v->ny * v->nz;
    const size_t nb = static_cast<size_t>(v->nbx) * v->nby * v->nbz;
    tn::Grid& g = o.g;
    g.nx = v->nx;
    g.ny = v->ny;
    g.nz = v->nz;
    g.nbx = v->nbx;
    g.nby = v->nby;
    g.nbz = v->nbz;
    g.vs[0] = v->vs[0];
    g.vs[1] = v->vs[1];
    g.vs[2] = v->vs[2];
    o.L.assign(v->L, v->L + nv);
    g.L = &o.L;
    g.bl_cnt.assign(v->bl_cnt, v->bl_cnt + nb);
    g.bl_lab.assign(v->bl_lab, v->bl_lab + nb * V2M_BL);
    g.bl_slot.assign(v->bl_slot, v->bl_slot + nb);
    g.phi.assign(v->phi, v->phi + static_cast<size_t>(v->nslots) * V2M_SLOT);
    g.h.assign(v->h, v->h + nv);
    g.hmin = v->hmin;
    g.hmax = v->hmax;
    g.gm = v->gm;

    if (v->gm > 0) {
        o.gI.assign(v->gI, v->gI + nv);
        g.gI = o.gI.data();
        g.gTW.assign(v->gTW, v->gTW + 2 * v->gm);
    } else if (v->gm < 0) {   // the analytic shape program
        g.gI = nullptr;
        g.gTW.assign(v->gTW, v->gTW + v->ngTW);
    } else {
        g.gI = nullptr;
        g.gTW.assign(1, 0.0f);
    }
    if (v->grade) {
        g.grade.assign(v->grade, v->grade + nv);
    }
}

tn::RelaxParams params_from(const v2m_relax_params* p) {
    tn::RelaxParams r;
    r.nseed = p->nseed;
    r.t = p->t;
    r.skin = p->skin;
    r.fscale = p->fscale;
    r.fsurf = p->fsurf;
    r.dt = p->dt;
    r.maxstep = p->maxstep;
    r.snap = p->snap;
    r.max_iters = p->max_iters;
    r.dptol = p->dptol;
    r.jseed = p->jseed;
    r.corners = p->corners != 0;
    r.voxel_trap = p->voxel_trap != 0;
    r.thin = p->thin;
    r.fire = p->fire != 0;
    r.fire_dtmax = p->fire_dtmax;
    r.verbose = p->verbose != 0;
    return r;
}

void nodes_from(const v2m_nodes_view* v, tn::Nodes& nd) {
    const size_t n = static_cast<size_t>(v->n);
    nd.P.assign(v->P, v->P + 3 * n);
    nd.lab.assign(v->lab, v->lab + n);
    nd.typ.assign(v->typ, v->typ + n);
    nd.part.assign(v->part, v->part + 2 * n);
    nd.part3.assign(n, 0xFFFF);
}

void nodes_to(const tn::Nodes& nd, v2m_nodes_view* v) {
    std::memcpy(v->P, nd.P.data(), nd.P.size() * 4);
    std::memcpy(v->typ, nd.typ.data(), nd.typ.size());
    std::memcpy(v->part, nd.part.data(), nd.part.size() * 2);
}

void stats_to(const tn::RelaxStats& s, v2m_relax_stats* o) {
    o->iters = s.iters;
    o->rebuilds = s.rebuilds;
    o->last_move = s.last_move;
    o->last_p99 = s.last_p99;
    o->fire_resets = s.fire_resets;
    o->fire_dt = s.fire_dt;
    o->n_interior = static_cast<int64_t>(s.n_interior);
    o->n_interface = static_cast<int64_t>(s.n_interface);
    o->n_junction = static_cast<int64_t>(s.n_junction);
    o->n_corner = static_cast<int64_t>(s.n_corner);
    o->ms_seed = s.ms_seed;
    o->ms_hash = s.ms_hash;
    o->ms_force = s.ms_force;
    o->ms_move = s.ms_move;
}

V2mDims dims_of(const tn::Grid& g) {
    V2mDims d;
    d.nx = g.nx;
    d.ny = g.ny;
    d.nz = g.nz;
    d.nbx = g.nbx;
    d.nby = g.nby;
    d.nbz = g.nbz;
    d.vx = g.vs[0];
    d.vy = g.vs[1];
    d.vz = g.vs[2];
    return d;
}

}  // namespace

#define GRID_FIELD d, g.L->data(), g.bl_cnt.data(), g.bl_lab.data(), g.bl_slot.data(), g.phi.data(), g.gI, g.gTW.data(), g.gm

// relax_cpu's loop state, stage by stage (src/v2m_particles.cpp:728-946).
struct RefState {
    OwnedGrid og;
    tn::RelaxParams prm;
    tn::Nodes nd;
    V2mHash H;
    V2mDims d;
    int n = 0, nkeys = 0, fire = 0, rebuild_div = 300;
    std::vector<int> key, cstart, sorted, nbr, nnb;
    std::vector<float> F, P0, mv, hn, Ps, V, pw;
    tn::FireCtl fc{ tn::RelaxParams() };
    tn::RelaxStats st;
    int it = 0, stopped = 0, hist[32] = { 0 }, nhalf = 0, nrefresh = 0;
    float mmax = 0.0f;
    double last_power = 0.0;
};

extern "C" {

const char* ref_last_error(void) {
    return g_err.c_str();
}

int ref_relax_cpu(const v2m_grid_view* gv, const v2m_relax_params* pv, v2m_nodes_view* nv, v2m_relax_stats* sv) {
    try {
        OwnedGrid og;
        grid_from_view(gv, og);
        tn::Nodes nd;
        nodes_from(nv, nd);
        tn::RelaxStats st;
        tn::relax_cpu(og.g, params_from(pv), nd, st);
        nodes_to(nd, nv);

        if (sv) {
            stats_to(st, sv);
        }

        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// ---- the reference grid build and seeding, for realistic test inputs ----------
struct RefGrid {
    tn::LabelVolume lv;
    tn::Grid g;
};

void* ref_grid_build(const uint16_t* labels, int nx, int ny, int nz, const float* vs, float sigma, float hbase,
                     float hmin, float hmax) {
    try {
        RefGrid* r = new RefGrid();
        r->lv.nx = nx;
        r->lv.ny = ny;
        r->lv.nz = nz;
        r->lv.voxelsize = { { vs[0], vs[1], vs[2] } };
        r->lv.data.assign(labels, labels + static_cast<size_t>(nx) * ny * nz);
        int m = 0;

        for (uint16_t l : r->lv.data) {
            m = std::max<int>(m, l);
        }

        r->lv.maxlabel = m;
        tn::GridParams gp;
        gp.sigma = sigma;
        gp.hbase = hbase;
        gp.hmin = hmin;
        gp.hmax = hmax;
        tn::build_grid_cpu(r->lv, gp, r->g);
        return r;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

// Shape input. The scene is compiled (with the overlap rule) and its program completed as the
// reference's shape front end does (src/v2m_modes.cpp:508-546: the gap-closing
// radius gap and the cull margin, then the per-brick programs when bricks != 0,
// then the raster that sets the field width, origin and blend radius). The
// label volume is the raster's per-voxel argmax (the lowest label on a tie);
// the grid is built from it (sigma, hbase, hmin, hmax as in ref_grid_build) and
// then takes the program as its fields: gm = -1, gTW = the program.
void* ref_shape_grid(const char* json, const char* overlap, double voxel, double gap, double margin, int bricks,
                     float sigma, float hbase, float hmin, float hmax, int feat) {
    try {
        tn::ShapeScene sc = tn::load_shapes(std::string(json), true, std::string(overlap));
        const size_t N = static_cast<size_t>(sc.nlab);
        sc.prog[6 + N] = static_cast<float>(gap);
        sc.prog[7 + N] = static_cast<float>(margin);
        if (bricks) {
            tn::build_brick_programs(sc, voxel);
        }
        const tn::Tpm t = tn::rasterize_scene(sc, voxel);
        RefGrid* r = new RefGrid();
        r->lv.nx = t.nx;
        r->lv.ny = t.ny;
        r->lv.nz = t.nz;
        r->lv.voxelsize = { { static_cast<float>(voxel), static_cast<float>(voxel), static_cast<float>(voxel) } };
        const size_t nv = t.nv();
        r->lv.data.assign(nv, 0);
        int m = 0;
        for (size_t v = 0; v < nv; ++v) {
            int best = 0;
            for (int l = 1; l < t.C; ++l) {
                if (t.p[static_cast<size_t>(l) * nv + v] > t.p[static_cast<size_t>(best) * nv + v]) {
                    best = l;
                }
            }
            r->lv.data[v] = static_cast<uint16_t>(best);
            m = std::max(m, best);
        }
        r->lv.maxlabel = m;
        tn::GridParams gp;
        gp.sigma = sigma;
        gp.hbase = hbase;
        gp.hmin = hmin;
        gp.hmax = hmax;
        if (feat) {
            // the shape front end's hand-off (src/v2m_modes.cpp:543-544): the grid
            // build takes the program and the features from the volume, shifts
            // the features into grid mm and refines the sizing near them
            // (src/v2m_grid.cpp:350-371, 560-600); seed_cpu then pins nodes on them
            r->lv.sdf = sc.prog;
            r->lv.sdf_feat = sc.feat;
        }
        tn::build_grid_cpu(r->lv, gp, r->g);
        r->g.gm = -1;
        r->g.gTW = sc.prog;
        return r;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

// Pointers into the reference grid (valid until ref_grid_free).
// tn::build_grid_cpu with every GridParams field of the C ABI's v2m_grid_params
// (the device grid build's parameters), hlab included.
void* ref_grid_build_p(const uint16_t* labels, int nx, int ny, int nz, const float* vs, const v2m_grid_params* p) {
    try {
        RefGrid* r = new RefGrid();
        r->lv.nx = nx;
        r->lv.ny = ny;
        r->lv.nz = nz;
        r->lv.voxelsize = { { vs[0], vs[1], vs[2] } };
        r->lv.data.assign(labels, labels + static_cast<size_t>(nx) * ny * nz);
        int m = 0;
        for (uint16_t l : r->lv.data) {
            m = std::max<int>(m, l);
        }
        r->lv.maxlabel = m;
        tn::GridParams gp;
        gp.sigma = p->sigma;
        gp.sigma_thin = p->sigma_thin;
        gp.thin_lo = p->thin_lo;
        gp.thin_hi = p->thin_hi;
        gp.thick = p->thick;
        gp.thin_floor = p->thin_floor;
        gp.preserve = p->preserve;
        gp.sigma_curv = p->sigma_curv;
        gp.hbase = p->hbase;
        gp.hmin = p->hmin;
        gp.hmax = p->hmax;
        gp.K = p->K;
        gp.g = p->g;
        if (p->nhlab > 0) {
            gp.hlab.assign(p->hlab, p->hlab + p->nhlab);
        }
        tn::build_grid_cpu(r->lv, gp, r->g);
        return r;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

int ref_grid_view(void* h, v2m_grid_view* v) {
    RefGrid* r = static_cast<RefGrid*>(h);
    tn::Grid& g = r->g;
    v->nx = g.nx;
    v->ny = g.ny;
    v->nz = g.nz;
    v->nbx = g.nbx;
    v->nby = g.nby;
    v->nbz = g.nbz;
    v->vs[0] = g.vs[0];
    v->vs[1] = g.vs[1];
    v->vs[2] = g.vs[2];
    v->L = g.L->data();
    v->bl_cnt = g.bl_cnt.data();
    v->bl_lab = g.bl_lab.data();
    v->bl_slot = g.bl_slot.data();
    v->phi = g.phi.data();
    v->nslots = static_cast<int64_t>(g.phi.size() / V2M_SLOT);
    v->h = g.h.data();
    v->hmin = g.hmin;
    v->hmax = g.hmax;
    v->gI = g.gI;
    v->gTW = g.gTW.empty() ? nullptr : g.gTW.data();
    v->gm = g.gm;
    v->ngTW = static_cast<int64_t>(g.gTW.size());
    v->grade = g.grade.empty() ? nullptr : g.grade.data();
    v->feat = g.feat.empty() ? nullptr : g.feat.data();
    v->nfeat = static_cast<int64_t>(g.feat.size());
    return 0;
}

void ref_grid_free(void* h) {
    delete static_cast<RefGrid*>(h);
}

// Seeds of the reference (seed_cpu); returns a handle, the count in *n.
void* ref_seed(void* gh, const v2m_relax_params* pv, int64_t* n) {
    try {
        RefGrid* r = static_cast<RefGrid*>(gh);
        tn::Nodes* nd = new tn::Nodes();
        tn::seed_cpu(r->g, params_from(pv), *nd);
        *n = static_cast<int64_t>(nd->size());
        return nd;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

int ref_seed_copy(void* h, float* P, uint16_t* lab, uint8_t* typ, uint16_t* part) {
    tn::Nodes* nd = static_cast<tn::Nodes*>(h);
    std::memcpy(P, nd->P.data(), nd->P.size() * 4);
    std::memcpy(lab, nd->lab.data(), nd->lab.size() * 2);
    std::memcpy(typ, nd->typ.data(), nd->typ.size());
    std::memcpy(part, nd->part.data(), nd->part.size() * 2);
    return 0;
}

// seed_cpu on a grid given as a view (its grade array required); a handle for
// ref_seed_copy / ref_seed_part3 / ref_seed_free.
void* ref_seed_view(const v2m_grid_view* gv, const v2m_relax_params* pv, int64_t* n) {
    try {
        if (!gv->grade) {
            throw std::runtime_error("seed_cpu needs the grid's size grades");
        }
        OwnedGrid og;
        grid_from_view(gv, og);
        tn::Nodes* nd = new tn::Nodes();
        tn::seed_cpu(og.g, params_from(pv), *nd);
        *n = static_cast<int64_t>(nd->size());
        return nd;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

// The seeds' third partner labels (part3: a CORNER node's fourth label).
int ref_seed_part3(void* h, uint16_t* part3) {
    tn::Nodes* nd = static_cast<tn::Nodes*>(h);
    std::memcpy(part3, nd->part3.data(), nd->part3.size() * 2);
    return 0;
}

void ref_seed_free(void* h) {
    delete static_cast<tn::Nodes*>(h);
}

// ---- relax_cpu, stage by stage -------------------------------------------------
void* ref_state_create(const v2m_grid_view* gv, const v2m_relax_params* pv, const v2m_nodes_view* nv) {
    try {
        RefState* s = new RefState();
        grid_from_view(gv, s->og);
        s->prm = params_from(pv);
        nodes_from(nv, s->nd);
        const tn::Grid& g = s->og.g;
        const tn::RelaxParams& prm = s->prm;
        s->d = dims_of(g);
        s->n = static_cast<int>(s->nd.size());
        s->rebuild_div = pv->rebuild_div > 0 ? pv->rebuild_div
                         : (std::getenv("V2M_REBUILD_DIV") ? std::atoi(std::getenv("V2M_REBUILD_DIV")) : 300);
        // hash geometry (src/v2m_particles.cpp:737-761)
        V2mHash& H = s->H;
        std::memset(&H, 0, sizeof(H));
        H.b0 = (prm.t + prm.skin) * g.hmin;
        H.ox = -0.5f * g.vs[0];
        H.oy = -0.5f * g.vs[1];
        H.oz = -0.5f * g.vs[2];
        const float ext[3] = { g.nx * g.vs[0], g.ny * g.vs[1], g.nz * g.vs[2] };
        H.nlev = 1;

        while (H.nlev < V2M_MAXLEV && H.b0 * static_cast<float>(1 << (H.nlev - 1)) < (prm.t + prm.skin) * g.hmax) {
            ++H.nlev;
        }

        int nkeys = 0;

        for (int L = 0; L < H.nlev; ++L) {
            H.off[L] = nkeys;
            const float bL = H.b0 * static_cast<float>(1 << L);

            for (int a = 0; a < 3; ++a) {
                H.dim[L][a] = std::max(1, static_cast<int>(std::ceil(ext[a] / bL)));
            }

            nkeys += H.dim[L][0] * H.dim[L][1] * H.dim[L][2];
        }

        s->nkeys = nkeys;
        const int n = s->n;
        s->key.assign(n, 0);
        s->cstart.assign(static_cast<size_t>(nkeys) + 1, 0);
        s->sorted.assign(n, 0);
        s->nbr.assign(static_cast<size_t>(n) * V2M_K, 0);
        s->nnb.assign(n, 0);
        s->F.assign(static_cast<size_t>(n) * 4, 0.0f);
        s->P0 = s->nd.P;
        s->mv.assign(n, 0.0f);
        s->hn.assign(n, 0.0f);

        for (int i = 0; i < n; ++i) {
            s->hn[i] = v2m_h_at(s->d, g.h.data(), s->nd.P[3 * i], s->nd.P[3 * i + 1], s->nd.P[3 * i + 2]);
        }

        s->fire = prm.fire && !prm.voxel_trap ? 1 : 0;
        s->V.assign(s->fire ? static_cast<size_t>(n) * 3 : 1, 0.0f);
        s->pw.assign(s->fire ? n : 1, 0.0f);
        s->fc = tn::FireCtl(prm);
        return s;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_state_free(void* h) {
    delete static_cast<RefState*>(h);
}

int ref_state_info(void* h, int64_t* nkeys, int32_t* nlev, float* b0) {
    RefState* s = static_cast<RefState*>(h);
    *nkeys = s->nkeys;
    *nlev = s->H.nlev;
    *b0 = s->H.b0;
    return 0;
}

// relax_cpu's rebuild lambda (src/v2m_particles.cpp:771-820)
int ref_state_rebuild(void* h) {
    RefState* s = static_cast<RefState*>(h);
    const tn::Grid& g = s->og.g;
    const tn::RelaxParams& prm = s->prm;
    tn::Nodes& nd = s->nd;
    const int n = s->n;
    tn::OmpThreadCap cap;
    #pragma omp parallel for

    for (int i = 0; i < n; ++i) {
        const float hh = v2m_h_at(s->d, g.h.data(), nd.P[3 * i], nd.P[3 * i + 1], nd.P[3 * i + 2]);
        s->key[i] = v2m_bin_key(&s->H, v2m_level_of(&s->H, (prm.t + prm.skin) * hh), nd.P[3 * i], nd.P[3 * i + 1],
                                nd.P[3 * i + 2]);
    }

    std::fill(s->cstart.begin(), s->cstart.end(), 0);

    for (int i = 0; i < n; ++i) {
        ++s->cstart[s->key[i] + 1];
    }

    for (int k = 0; k < s->nkeys; ++k) {
        s->cstart[k + 1] += s->cstart[k];
    }

    std::vector<int> cur(s->cstart.begin(), s->cstart.end() - 1);

    for (int i = 0; i < n; ++i) {
        s->sorted[cur[s->key[i]]++] = i;
    }

    s->Ps.resize(static_cast<size_t>(n) * 4);

    for (int s2 = 0; s2 < n; ++s2) {
        const int j = s->sorted[s2];
        s->Ps[4 * s2] = nd.P[3 * j];
        s->Ps[4 * s2 + 1] = nd.P[3 * j + 1];
        s->Ps[4 * s2 + 2] = nd.P[3 * j + 2];
        s->Ps[4 * s2 + 3] = s->hn[j];
    }

    #pragma omp parallel for schedule(dynamic, 256)

    for (int i = 0; i < n; ++i) {
        float kds[V2M_K];
        int kids[V2M_K];
        v2m_neighbors(&s->H, s->hn.data(), nd.P.data(), nd.lab.data(), nd.typ.data(), s->cstart.data(), s->sorted.data(),
                      s->Ps.data(), prm.t, prm.skin, i, s->nbr.data(), s->nnb.data(), kds, kids, 1);
    }

    s->P0 = nd.P;
    ++s->st.rebuilds;
    return 0;
}

// src/v2m_particles.cpp:828-836
int ref_state_force(void* h) {
    RefState* s = static_cast<RefState*>(h);
    tn::Nodes& nd = s->nd;
    tn::OmpThreadCap cap;
    #pragma omp parallel for schedule(dynamic, 1024)

    for (int i = 0; i < s->n; ++i) {
        v2m_force(s->hn.data(), nd.P.data(), nd.typ.data(), s->nbr.data(), s->nnb.data(), s->prm.fscale, s->prm.fsurf, i,
                  &s->F[4 * i]);
    }

    return 0;
}

// The move of every node only (src/v2m_particles.cpp:838-847), no bookkeeping.
int ref_state_move_only(void* h) {
    RefState* s = static_cast<RefState*>(h);
    const tn::Grid& g = s->og.g;
    const tn::RelaxParams& prm = s->prm;
    tn::Nodes& nd = s->nd;
    const V2mDims d = s->d;
    float mmax = 0.0f;
    tn::OmpThreadCap cap;
    #pragma omp parallel for schedule(dynamic, 1024) reduction(max : mmax)

    for (int i = 0; i < s->n; ++i) {
        s->mv[i] = v2m_move(GRID_FIELD, g.h.data(), s->F.data(), prm.dt, prm.maxstep, prm.snap, prm.voxel_trap ? 1 : 0, i,
                            nd.P.data(), nd.lab.data(), nd.typ.data(), nd.part.data(), s->hn.data(), s->fire, s->V.data(),
                            s->fc.dt, s->fc.alpha, s->pw.data());
        mmax = std::max(mmax, s->mv[i]);
    }

    s->mmax = mmax;
    return 0;
}

// The rest of iteration `it` after the force (src/v2m_particles.cpp:838-946).
// Returns 1 when the loop stops (convergence), 0 to go on.
int ref_state_tail(void* h) {
    RefState* s = static_cast<RefState*>(h);
    const tn::Grid& g = s->og.g;
    const tn::RelaxParams& prm = s->prm;
    tn::Nodes& nd = s->nd;
    const int n = s->n;
    const int it = s->it;
    ref_state_move_only(h);

    if (s->fire) {
        double pt = 0.0;

        for (int i = 0; i < n; ++i) {
            pt += s->pw[i];
        }

        s->last_power = pt;

        if (s->fc.update(pt)) {
            std::fill(s->V.begin(), s->V.end(), 0.0f);
        }
    }

    s->st.iters = it + 1;
    s->st.last_move = s->mmax;
    s->st.fire_resets = s->fc.resets;
    s->st.fire_dt = s->fire ? s->fc.dt : 0.0f;
    int hist[32] = { 0 };

    for (int i = 0; i < n; ++i) {
        const float m = s->mv[i];
        const int b = m > 0.0f ? std::min(31, std::max(0, 20 + static_cast<int>(std::floor(std::log2(m))))) : 0;
        ++hist[b];
    }

    std::memcpy(s->hist, hist, sizeof(hist));
    int acc = 0, b99 = 31;

    for (int b = 0; b < 32; ++b) {
        acc += hist[b];

        if (acc >= 0.99 * n) {
            b99 = b;
            break;
        }
    }

    const float p99 = std::ldexp(1.0f, b99 - 20 + 1);
    s->st.last_p99 = p99;
    s->it = it + 1;

    if (p99 < prm.dptol && (!s->fire || s->fc.may_stop())) {
        s->stopped = 1;
        return 1;
    }

    int nhalf = 0, nref = 0;

    for (int i = 0; i < n; ++i) {
        const float ex = nd.P[3 * i] - s->P0[3 * i], ey = nd.P[3 * i + 1] - s->P0[3 * i + 1],
                    ez = nd.P[3 * i + 2] - s->P0[3 * i + 2];
        const float hh = v2m_h_at(s->d, g.h.data(), nd.P[3 * i], nd.P[3 * i + 1], nd.P[3 * i + 2]);
        const float m2 = ex * ex + ey * ey + ez * ez, s2 = prm.skin * prm.skin * hh * hh;

        if (m2 > s2) {
            float kds[V2M_K];
            int kids[V2M_K];
            v2m_neighbors(&s->H, s->hn.data(), nd.P.data(), nd.lab.data(), nd.typ.data(), s->cstart.data(),
                          s->sorted.data(), s->Ps.data(), prm.t, prm.skin, i, s->nbr.data(), s->nnb.data(), kds, kids, 1);
            s->P0[3 * i] = nd.P[3 * i];
            s->P0[3 * i + 1] = nd.P[3 * i + 1];
            s->P0[3 * i + 2] = nd.P[3 * i + 2];
            ++nref;
        } else {
            nhalf += m2 > 0.25f * s2;
        }
    }

    s->nhalf = nhalf;
    s->nrefresh = nref;
    const bool endgame = it >= prm.max_iters * 4 / 5 || p99 < 4.0f * prm.dptol;

    if (nhalf > n / (endgame ? std::max(s->rebuild_div, 1000) : s->rebuild_div)) {
        ref_state_rebuild(h);
    }

    return 0;
}

// The whole relax_cpu loop from the current state (first rebuild included).
int ref_state_run(void* h) {
    RefState* s = static_cast<RefState*>(h);
    ref_state_rebuild(h);

    for (int it = s->it; it < s->prm.max_iters; ++it) {
        ref_state_force(h);

        if (ref_state_tail(h)) {
            break;
        }
    }

    return 0;
}

int ref_state_counts(void* h, int32_t* it, int32_t* stopped, int32_t* nhalf, int32_t* nrefresh, int32_t* rebuilds,
                     int32_t* fire_resets, float* fire_dt, float* fire_alpha, double* power, float* mmax, float* p99) {
    RefState* s = static_cast<RefState*>(h);
    *it = s->it;
    *stopped = s->stopped;
    *nhalf = s->nhalf;
    *nrefresh = s->nrefresh;
    *rebuilds = s->st.rebuilds;
    *fire_resets = s->fc.resets;
    *fire_dt = s->fc.dt;
    *fire_alpha = s->fc.alpha;
    *power = s->last_power;
    *mmax = s->mmax;
    *p99 = s->st.last_p99;
    return 0;
}

// Copy an internal array out (the V2M_ARR_* codes of v2m_cuda.h).
int64_t ref_state_read(void* h, int what, void* out, int64_t bytes) {
    RefState* s = static_cast<RefState*>(h);
    const void* src = nullptr;
    int64_t nb = 0;
    std::vector<int> hist34;

    switch (what) {
    case V2M_ARR_KEY: src = s->key.data(); nb = 4LL * s->key.size(); break;
    case V2M_ARR_SORTED: src = s->sorted.data(); nb = 4LL * s->sorted.size(); break;
    case V2M_ARR_CSTART: src = s->cstart.data(); nb = 4LL * s->cstart.size(); break;
    case V2M_ARR_PS: src = s->Ps.data(); nb = 4LL * s->Ps.size(); break;
    case V2M_ARR_NBR: src = s->nbr.data(); nb = 4LL * s->nbr.size(); break;
    case V2M_ARR_NNB: src = s->nnb.data(); nb = 4LL * s->nnb.size(); break;
    case V2M_ARR_F: src = s->F.data(); nb = 4LL * s->F.size(); break;
    case V2M_ARR_HN: src = s->hn.data(); nb = 4LL * s->hn.size(); break;
    case V2M_ARR_MV: src = s->mv.data(); nb = 4LL * s->mv.size(); break;
    case V2M_ARR_V: src = s->V.data(); nb = 4LL * s->V.size(); break;
    case V2M_ARR_PW: src = s->pw.data(); nb = 4LL * s->pw.size(); break;
    case V2M_ARR_P0: src = s->P0.data(); nb = 4LL * s->P0.size(); break;
    case V2M_ARR_P: src = s->nd.P.data(); nb = 4LL * s->nd.P.size(); break;
    case V2M_ARR_TYP: src = s->nd.typ.data(); nb = static_cast<int64_t>(s->nd.typ.size()); break;
    case V2M_ARR_PART: src = s->nd.part.data(); nb = 2LL * s->nd.part.size(); break;
    case V2M_ARR_HIST: {
        hist34.assign(s->hist, s->hist + 32);
        int mb;
        std::memcpy(&mb, &s->mmax, 4);
        hist34.push_back(mb);
        hist34.push_back(s->nhalf);
        src = hist34.data();
        nb = 4LL * 34;
        break;
    }
    default: g_err = "unknown array"; return -1;
    }

    if (bytes < nb) {
        g_err = "buffer too small";
        return -1;
    }

    std::memcpy(out, src, static_cast<size_t>(nb));
    return nb;
}

// Overwrite node state (P, typ, part, hn, V, nbr, nnb) so that a stage can be
// compared from an arbitrary state.
int ref_state_write(void* h, int what, const void* in, int64_t bytes) {
    RefState* s = static_cast<RefState*>(h);
    void* dst = nullptr;
    int64_t nb = 0;

    switch (what) {
    case V2M_ARR_P: dst = s->nd.P.data(); nb = 4LL * s->nd.P.size(); break;
    case V2M_ARR_TYP: dst = s->nd.typ.data(); nb = static_cast<int64_t>(s->nd.typ.size()); break;
    case V2M_ARR_PART: dst = s->nd.part.data(); nb = 2LL * s->nd.part.size(); break;
    case V2M_ARR_HN: dst = s->hn.data(); nb = 4LL * s->hn.size(); break;
    case V2M_ARR_V: dst = s->V.data(); nb = 4LL * s->V.size(); break;
    case V2M_ARR_NBR: dst = s->nbr.data(); nb = 4LL * s->nbr.size(); break;
    case V2M_ARR_NNB: dst = s->nnb.data(); nb = 4LL * s->nnb.size(); break;
    default: g_err = "unknown array"; return -1;
    }

    if (bytes != nb) {
        g_err = "size mismatch";
        return -1;
    }

    std::memcpy(dst, in, static_cast<size_t>(nb));
    return 0;
}

}  // extern "C"
