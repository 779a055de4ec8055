// relax_cl_shim.cpp -- the drop-in for v2mesh's OpenCL relaxation: tn::relax_cl
// with the reference's exact signature (src/v2m_gpu.h:16-18 of fangq/trussnet),
// implemented over the C ABI of libv2m_cuda.so (include/v2m_cuda.h).
//
// Build it against the reference's headers (src/v2m_grid.h, src/v2m_particles.h,
// src/v2m_gpu.h, src/v2m_gdel.h) and link v2m_core with it in place of
// src/v2m_gpu.cpp, src/v2m_gdel.cpp and src/opencl/v2m_cl_*.cpp; the pipeline's
// call site (src/v2m_pipeline.cpp:492-536) is unchanged: a failure here throws
// std::runtime_error, which it catches, restoring the seeds and running
// relax_cpu. The library itself never falls back to the CPU.
//
// The GPU Delaunay (tn::gdel_tetrahedrize) is not part of this library: its
// stub returns false, which its contract (src/v2m_gdel.h:30-33) defines as
// "device path unavailable", so the exact CPU Delaunay runs.
#include <cstdint>
#include <stdexcept>
#include <string>

#include "v2m_cuda.h"
#include "v2m_gdel.h"
#include "v2m_gpu.h"

namespace tn {

void relax_cl(const Grid& g, const RelaxParams& prm, Nodes& nd, RelaxStats& st, int device) {
    if (!g.L) {
        throw std::runtime_error("relax_cl: grid without labels");
    }
    v2m_grid_view gv{};
    gv.nx = g.nx;
    gv.ny = g.ny;
    gv.nz = g.nz;
    gv.nbx = g.nbx;
    gv.nby = g.nby;
    gv.nbz = g.nbz;
    gv.vs[0] = g.vs[0];
    gv.vs[1] = g.vs[1];
    gv.vs[2] = g.vs[2];
    gv.L = g.L->data();
    gv.bl_cnt = g.bl_cnt.data();
    gv.bl_lab = g.bl_lab.data();
    gv.bl_slot = g.bl_slot.data();
    gv.phi = g.phi.data();
    gv.nslots = static_cast<int64_t>(g.phi.size() / V2M_SLOT);
    gv.h = g.h.data();
    gv.hmin = g.hmin;
    gv.hmax = g.hmax;
    gv.gI = g.gI;
    gv.gTW = g.gTW.empty() ? nullptr : g.gTW.data();
    gv.gm = g.gm;
    gv.ngTW = static_cast<int64_t>(g.gTW.size());
    gv.feat = g.feat.empty() ? nullptr : g.feat.data();
    gv.nfeat = static_cast<int64_t>(g.feat.size());

    v2m_relax_params pv;
    v2m_relax_params_default(&pv);
    pv.nseed = prm.nseed;
    pv.t = prm.t;
    pv.skin = prm.skin;
    pv.fscale = prm.fscale;
    pv.fsurf = prm.fsurf;
    pv.dt = prm.dt;
    pv.maxstep = prm.maxstep;
    pv.snap = prm.snap;
    pv.max_iters = prm.max_iters;
    pv.dptol = prm.dptol;
    pv.jseed = prm.jseed;
    pv.corners = prm.corners ? 1 : 0;
    pv.voxel_trap = prm.voxel_trap ? 1 : 0;
    pv.thin = prm.thin;
    pv.fire = prm.fire ? 1 : 0;
    pv.fire_dtmax = prm.fire_dtmax;
    pv.verbose = prm.verbose ? 1 : 0;

    v2m_nodes_view nv{};
    nv.n = static_cast<int64_t>(nd.size());
    if (nd.P.size() != 3 * nd.size() || nd.typ.size() != nd.size() || nd.part.size() != 2 * nd.size()) {
        throw std::runtime_error("relax_cl: inconsistent node arrays");
    }
    nv.P = nd.P.data();
    nv.lab = nd.lab.data();
    nv.typ = nd.typ.data();
    nv.part = nd.part.data();

    v2m_relax_stats sv{};
    const int rc = v2m_relax_cuda(&gv, &pv, &nv, &sv, device);
    if (rc != V2M_OK) {
        throw std::runtime_error(std::string("relax_cl: CUDA relaxation failed (") + std::to_string(rc) +
                                 "): " + v2m_cuda_last_error());
    }
    st.iters = sv.iters;
    st.rebuilds = sv.rebuilds;
    st.last_move = sv.last_move;
    st.last_p99 = sv.last_p99;
    st.fire_resets = sv.fire_resets;
    st.fire_dt = sv.fire_dt;
    st.n_interior = static_cast<size_t>(sv.n_interior);
    st.n_interface = static_cast<size_t>(sv.n_interface);
    st.n_junction = static_cast<size_t>(sv.n_junction);
    st.n_corner = static_cast<size_t>(sv.n_corner);
    st.ms_hash += sv.ms_hash;
    st.ms_force += sv.ms_force;
    st.ms_move += sv.ms_move;
}

bool gdel_tetrahedrize(const double*, uint32_t, ::TetMesh&, GdelStats&, int) {
    return false;
}

}  // namespace tn
