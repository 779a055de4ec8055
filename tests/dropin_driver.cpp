// dropin_driver.cpp -- the reference pipeline's relaxation dispatch
// (src/v2m_pipeline.cpp:492-526 of fangq/trussnet) over the reference's own
// types, linked against the drop-in tn::relax_cl (libv2m_relax_cl.so) and the
// reference's CPU path (oracle/_ref/libv2m_ref.so: build_grid_cpu, seed_cpu,
// relax_cpu). It builds a three-label phantom, seeds it with the reference,
// then:
//   1. relax_cl in try; on std::runtime_error restore the seeds and relax_cpu
//      (exactly the pipeline's fallback), printing which path ran;
//   2. relax_cpu on the same seeds;
//   3. prints whether positions, types and partners are bit-identical.
// Output: one line "path=<cuda|cpu-fallback> nodes=N identical=<0|1> iters=I".
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include "v2m_gpu.h"
#include "v2m_grid.h"
#include "v2m_particles.h"
#include "v2m_volume.h"

int main(int argc, char** argv) {
    const int dim = argc > 1 ? std::atoi(argv[1]) : 40;
    const int iters = argc > 2 ? std::atoi(argv[2]) : 30;
    tn::LabelVolume lv;
    lv.nx = lv.ny = lv.nz = dim;
    lv.data.assign(static_cast<size_t>(dim) * dim * dim, 0);
    const float c = 0.5f * (dim - 1);
    for (int k = 0; k < dim; ++k)
        for (int j = 0; j < dim; ++j)
            for (int i = 0; i < dim; ++i) {
                const float r2 = (i - c) * (i - c) + (j - c) * (j - c) + (k - c) * (k - c);
                uint16_t l = 0;
                if (r2 < (0.45f * dim) * (0.45f * dim)) l = i > c + 2 ? 3 : 1;
                if (r2 < (0.28f * dim) * (0.28f * dim)) l = 2;
                lv.data[i + static_cast<size_t>(dim) * (j + static_cast<size_t>(dim) * k)] = l;
            }
    lv.maxlabel = 3;
    tn::GridParams gp;
    gp.hbase = 2.5f;
    gp.hmin = 1.5f;
    gp.hmax = 3.0f;
    tn::Grid g;
    tn::build_grid_cpu(lv, gp, g);
    tn::RelaxParams prm;
    prm.max_iters = iters;
    tn::Nodes seeds;
    tn::seed_cpu(g, prm, seeds);

    // the pipeline's dispatch
    tn::Nodes a = seeds;
    tn::RelaxStats sa;
    const char* path = "cuda";
    try {
        tn::relax_cl(g, prm, a, sa, -1);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "relax_cl failed (%s); running on the CPU\n", e.what());
        a = seeds;
        tn::relax_cpu(g, prm, a, sa);
        path = "cpu-fallback";
    }
    tn::Nodes b = seeds;
    tn::RelaxStats sb;
    tn::relax_cpu(g, prm, b, sb);
    const bool same = a.P.size() == b.P.size() && std::memcmp(a.P.data(), b.P.data(), a.P.size() * 4) == 0 &&
                      a.typ == b.typ && a.part == b.part;
    std::printf("path=%s nodes=%zu identical=%d iters=%d/%d rebuilds=%d/%d\n", path, seeds.size(), same ? 1 : 0,
                sa.iters, sb.iters, sa.rebuilds, sb.rebuilds);
    return 0;
}
