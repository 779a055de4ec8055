// v2m_grid.h -- the device grid build's interface to the host code (v2m_grid.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace v2m {

// tn::GridParams (src/v2m_grid.h:21-43 of fangq/trussnet), label input: no
// interface sizes, no user sizing field.
struct GridParamsH {
    float sigma = 1.0f, sigma_thin = 0.35f, thin_lo = 2.0f, thin_hi = 4.0f, thick = 0.0f, thin_floor = 0.5f;
    float preserve = 0.0f, sigma_curv = 2.0f, hbase = 0.0f, hmin = 0.0f, hmax = 0.0f, K = 3.0f, g = 0.3f;
    std::vector<float> hlab;
};

struct GridBuildArgs {
    const uint16_t* L = nullptr;   // host labels, x fastest
    int nx = 0, ny = 0, nz = 0;
    float vs[3] = { 1.0f, 1.0f, 1.0f };
    GridParamsH prm;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::function<void(const char*)> lap;   // stage timing hook (may be empty)
};

// Device arrays (in `tmp`, freed by the caller) and the derived sizes.
struct GridBuildOut {
    std::vector<void*> tmp;
    uint16_t* L = nullptr;
    int* bl_cnt = nullptr;
    uint16_t* bl_lab = nullptr;
    int* bl_slot = nullptr;
    float* phi = nullptr;
    float* h = nullptr;
    uint8_t* grade = nullptr;
    int64_t nslots = 0;
    int nlab = 0, R = 0, limit_sweeps = 0, overflow_bricks = 0;
    float hbase = 0.0f, hmin = 0.0f, hmax = 0.0f;
};

cudaError_t grid_build(const GridBuildArgs& A, GridBuildOut& O, std::string& err);

}  // namespace v2m
