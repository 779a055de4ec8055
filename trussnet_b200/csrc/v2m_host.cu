// v2m_host.cu -- host side of libv2m_cuda.so: sessions, the iteration loop
// (plain launches or a captured CUDA graph) and the C ABI of include/v2m_cuda.h.
//
// The loop mirrors relax_cl / relax_cpu (src/v2m_gpu.cpp:116-553,
// src/v2m_particles.cpp:728-976 of fangq/trussnet) with one difference of
// structure: the per-iteration decisions (FIRE step, convergence, Verlet
// rebuild) are taken on the device by k_control, so an iteration needs no host
// round trip and a run of iterations replays as one graph. The host reads the
// per-volume control blocks only between graph replays, to stop early.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <sys/mman.h>

#include <algorithm>
#include <climits>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <sys/stat.h>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/v2m_cuda.h"
#include "v2m_grid.h"
#include "v2m_kernels.h"

using namespace v2m;

namespace {

thread_local std::string g_err;

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct ArgError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct KernelError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Host-side fault injection, for the callers' recovery paths (the pipeline's
// CPU fallback, src/v2m_pipeline.cpp:497-526 of fangq/trussnet): with
// V2M_CUDA_FAIL_AT=<stage>[:<k>] the host code fails at that point as if a CUDA
// call had, with "injected fault at <stage>" -- nothing is done to the GPU.
// Stages: create (before the first allocation), rebuild (the first list build),
// iterate:<k> (the first host check at or after iteration k), readback (after
// the positions have been written into the caller's arrays, before the types
// and partners: the caller's nodes are left half-updated).
void inject(const char* stage, int it = -1) {
    const char* e = std::getenv("V2M_CUDA_FAIL_AT");
    if (!e || !*e) {
        return;
    }
    const std::string spec(e);
    const size_t colon = spec.find(':');
    const std::string name = spec.substr(0, colon);
    if (name != stage) {
        return;
    }
    if (it >= 0 && colon != std::string::npos && it < std::atoi(spec.c_str() + colon + 1)) {
        return;
    }
    throw CudaError(std::string("injected fault at ") + stage + (it >= 0 ? " (iteration " + std::to_string(it) + ")" : ""));
}

// Host-side stage timing of a call (V2M_CUDA_PROFILE=1, the counterpart of the
// reference's V2M_CL_PROFILE, src/v2m_gpu.cpp:250-258): each stage's wall time
// after synchronizing the stream, printed to stderr when the call ends.
struct StageClock {
    bool on = false;
    cudaStream_t stream = nullptr;
    std::chrono::steady_clock::time_point t0;
    std::string out;
    explicit StageClock(const char* what) : on(std::getenv("V2M_CUDA_PROFILE") != nullptr) {
        if (on) {
            out = std::string("[v2m_cuda] ") + what;
            t0 = std::chrono::steady_clock::now();
        }
    }
    void lap(const char* stage) {
        if (!on) {
            return;
        }
        if (stream) {
            cudaStreamSynchronize(stream);
        }
        const auto t = std::chrono::steady_clock::now();
        char buf[96];
        std::snprintf(buf, sizeof(buf), " %s %.2f ms", stage, std::chrono::duration<double, std::milli>(t - t0).count());
        out += buf;
        t0 = t;
    }
    ~StageClock() {
        if (on) {
            std::fprintf(stderr, "%s\n", out.c_str());
        }
    }
};
thread_local StageClock* g_clock = nullptr;

// Tracing: an NVTX range over every call of the C ABI, and an NVTX mark at each
// stage a call passes (lap), so a profiler's timeline (Nsight Systems, ncu's
// NVTX filters) shows the library's calls and their stages beside the kernels.
// NVTX is header-only here: without a tool attached each call costs a branch.
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

void lap(const char* stage) {
    nvtxMarkA(stage);
    if (g_clock) {
        g_clock->lap(stage);
    }
}

void ck(cudaError_t e, const char* where) {
    if (e != cudaSuccess) {
        throw CudaError(std::string(where) + ": CUDA error " + std::to_string((int)e) + " (" + cudaGetErrorString(e) + ")");
    }
}

int64_t align_up(int64_t x, int64_t a) {
    return (x + a - 1) / a * a;
}

void mkdir_p(const std::string& dir) {
    for (size_t i = 1; i <= dir.size(); ++i) {
        if (i == dir.size() || dir[i] == '/') {
            mkdir(dir.substr(0, i).c_str(), 0755);
        }
    }
}

int env_int(const char* name, int dflt) {
    const char* e = std::getenv(name);
    return e ? std::atoi(e) : dflt;
}


// Per-volume host bookkeeping.
struct VolInfo {
    int n = 0, nkeys = 0;
    int64_t nofs = 0, kofs = 0;
    int max_iters = 0;
    int hmode = 0;
};

}  // namespace

namespace v2m {

cudaMemPool_t library_pool(int device) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    if (device < 0 || device >= 64) {
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[device]) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        if (cudaMemPoolCreate(&pools[device], &props) != cudaSuccess) {
            cudaGetLastError();
            pools[device] = nullptr;
            return nullptr;
        }
        const char* e = std::getenv("V2M_CUDA_POOL_KEEP_MB");
        uint64_t keep = (uint64_t)(e ? std::max(0, std::atoi(e)) : 16384) << 20;
        cudaMemPoolSetAttribute(pools[device], cudaMemPoolAttrReleaseThreshold, &keep);
    }
    return pools[device];
}

namespace {

constexpr size_t kStageBytes = (size_t)32 << 20;

// memcpy split over up to 8 host threads in 1 MB-aligned slices
void parallel_copy(void* dst, const void* src, size_t len) {
    const size_t slice = (size_t)1 << 20;
    const unsigned nth = (unsigned)std::min<size_t>(std::max(1u, std::min(8u, std::thread::hardware_concurrency())),
                                                    (len + slice - 1) / slice);
    if (nth <= 1) {
        std::memcpy(dst, src, len);
        return;
    }
    std::vector<std::thread> pool;
    const size_t per = (len / nth + slice - 1) / slice * slice;
    for (unsigned q = 0; q < nth; ++q) {
        const size_t a = std::min(len, q * per), b = std::min(len, a + per);
        if (a < b) {
            pool.emplace_back([=] { std::memcpy((char*)dst + a, (const char*)src + a, b - a); });
        }
    }
    for (auto& t : pool) {
        t.join();
    }
}

struct Staging {
    std::mutex mu;
    void* buf[2] = { nullptr, nullptr };
    cudaEvent_t ev[2] = { nullptr, nullptr };
};

Staging& staging() {
    static Staging st;
    return st;
}

cudaError_t staging_ready(Staging& S) {
    for (int q = 0; q < 2; ++q) {
        if (!S.buf[q]) {
            cudaError_t e = cudaMallocHost(&S.buf[q], kStageBytes);
            if (e != cudaSuccess) {
                S.buf[q] = nullptr;
                return e;
            }
        }
        if (!S.ev[q]) {
            cudaError_t e = cudaEventCreateWithFlags(&S.ev[q], cudaEventDisableTiming);
            if (e != cudaSuccess) {
                S.ev[q] = nullptr;
                return e;
            }
        }
    }
    return cudaSuccess;
}

}  // namespace

cudaError_t staged_map(void* dst, const void* src, size_t bytes, cudaStream_t s,
                       const std::function<void(void*, size_t, size_t)>& fn) {
    Staging& S = staging();
    std::lock_guard<std::mutex> lk(S.mu);
    cudaError_t e = staging_ready(S);
    if (e != cudaSuccess) {
        return e;
    }
    const size_t nchunk = (bytes + kStageBytes - 1) / kStageBytes;
    // chunk c goes device -> buf[c % 2] (event), host fn, then buf -> dst (event);
    // the buffer is reused two chunks later, after its copy back has completed
    for (size_t c = 0; c < nchunk; ++c) {
        const int q = (int)(c & 1);
        const size_t off = c * kStageBytes, len = std::min(kStageBytes, bytes - off);
        if ((e = cudaEventSynchronize(S.ev[q])) != cudaSuccess) {
            return e;
        }
        if ((e = cudaMemcpyAsync(S.buf[q], (const char*)src + off, len, cudaMemcpyDeviceToHost, s)) != cudaSuccess) {
            return e;
        }
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
            return e;
        }
        fn(S.buf[q], len, off);
        if (dst) {
            if ((e = cudaMemcpyAsync((char*)dst + off, S.buf[q], len, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
                return e;
            }
            if ((e = cudaEventRecord(S.ev[q], s)) != cudaSuccess) {
                return e;
            }
        }
    }
    return cudaStreamSynchronize(s);
}

cudaError_t staged_d2h(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    Staging& S = staging();
    std::lock_guard<std::mutex> lk(S.mu);
    cudaError_t e = staging_ready(S);
    if (e != cudaSuccess) {
        return e;
    }
    const size_t nchunk = (bytes + kStageBytes - 1) / kStageBytes;
    for (size_t c = 0; c < nchunk + 1; ++c) {
        if (c < nchunk) {   // the DMA of chunk c ...
            const size_t off = c * kStageBytes, len = std::min(kStageBytes, bytes - off);
            if ((e = cudaMemcpyAsync(S.buf[c & 1], (const char*)src + off, len, cudaMemcpyDeviceToHost, s)) !=
                    cudaSuccess ||
                (e = cudaEventRecord(S.ev[c & 1], s)) != cudaSuccess) {
                return e;
            }
        }
        if (c > 0) {   // ... while the host copies chunk c - 1 out (over several threads: a fresh
                       // destination's first-touch page faults are the cost, and they run in parallel)
            const size_t p = c - 1, off = p * kStageBytes, len = std::min(kStageBytes, bytes - off);
            if ((e = cudaEventSynchronize(S.ev[p & 1])) != cudaSuccess) {
                return e;
            }
            parallel_copy((char*)dst + off, S.buf[p & 1], len);
        }
    }
    return cudaSuccess;
}

}  // namespace v2m

struct v2m_session {
    int device = 0;
    int* chk = nullptr;   // the checked build's bounds-check word (device, 2 ints)
    cudaStream_t stream = nullptr;
    int nvol = 0;
    std::vector<DVol> hvols;
    std::vector<VolInfo> info;
    std::vector<v2m_relax_params> prm;
    Dev d;
    std::vector<void*> allocs;
    float4* Pq0 = nullptr;
    uint8_t* typ0 = nullptr;
    uint32_t* part0 = nullptr;
    VolCtl* ctl_init = nullptr;
    int serial_power = 0;
    int force_threads = 256;
    int nbr_threads = 128;
    int refresh_blocks = 0;
    int max_iters = 0;
    int graph_iters = 10;
    cudaGraphExec_t gexec = nullptr;
    std::vector<cudaEvent_t> gev;   // force start/stop events recorded inside the graph
    int64_t launches = 0, force_launches = 0;
    double force_ms = 0.0;
    int time_force = 0;
    double ms_hash = 0.0, ms_loop = 0.0;

    template <typename T>
    T* alloc(size_t count) {
        void* p = nullptr;
        const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
        ck(pool_malloc(&p, bytes, stream), "device allocation");
        allocs.push_back(p);
        return static_cast<T*>(p);
    }

    ~v2m_session() {
        if (gexec) {
            cudaGraphExecDestroy(gexec);
        }
        for (cudaEvent_t e : gev) {
            cudaEventDestroy(e);
        }
        for (void* p : allocs) {
            cudaFreeAsync(p, stream);   // (back to the library's pool)
        }
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }
};

namespace {

bool tune_lookup(v2m_session* s);
void tune_store(v2m_session* s);
std::string do_autotune(v2m_session* s, int reps);

// The checked build's bounds-check word of the session's grids (code, index).
void check_bounds_word(v2m_session* s) {
    if (!s->chk) {
        return;
    }
    int w[2] = { 0, 0 };
    ck(cudaMemcpyAsync(w, s->chk, sizeof(w), cudaMemcpyDeviceToHost, s->stream), "read bounds checks");
    ck(cudaStreamSynchronize(s->stream), "synchronize");
    if (w[0]) {
        throw KernelError("bounds check " + std::to_string(w[0]) + " failed at index " + std::to_string(w[1]));
    }
}

void check_kernel_error(v2m_session* s) {
    Global g;
    ck(cudaMemcpyAsync(&g, s->d.G, sizeof(Global), cudaMemcpyDeviceToHost, s->stream), "read error flag");
    ck(cudaStreamSynchronize(s->stream), "synchronize");
    if (g.err) {
        throw KernelError("kernel error " + std::to_string(g.err) + " at index " + std::to_string(g.err_info));
    }
    check_bounds_word(s);
}

// True when p is device memory (not readable by the host): views may carry
// arrays already on the device (the device grid build and seeding hand theirs
// on without a host round trip).
bool on_device(const void* p) {
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice;
}

void validate(const v2m_grid_view* g, const v2m_relax_params* p, const v2m_nodes_view* nd) {
    if (!g || !p || !nd) {
        throw ArgError("null argument");
    }
    if (g->nx < 1 || g->ny < 1 || g->nz < 1) {
        throw ArgError("grid dimensions must be positive");
    }
    if (g->nbx != (g->nx + 7) / 8 || g->nby != (g->ny + 7) / 8 || g->nbz != (g->nz + 7) / 8) {
        throw ArgError("brick counts must be ceil(n / 8) per axis");
    }
    if (!(g->vs[0] > 0.0f && g->vs[1] > 0.0f && g->vs[2] > 0.0f)) {
        throw ArgError("voxel sizes must be positive");
    }
    if (!g->L || !g->bl_cnt || !g->bl_lab || !g->bl_slot || !g->h || (g->nslots > 0 && !g->phi)) {
        throw ArgError("grid array missing");
    }
    if (g->gm < 0) {
        // the analytic shape program: its header and code offsets (the device
        // also bounds-checks every read of it)
        if (!g->gTW || g->ngTW < 9 || g->ngTW > (int64_t)INT_MAX) {
            throw ArgError("analytic shape fields need the program gTW and its length ngTW");
        }
        const float nf = g->gTW[0];
        if (!(nf >= 1.0f && nf <= 65535.0f)) {
            throw ArgError("shape program: label count out of range");
        }
        const int nl = (int)nf;
        if ((int64_t)9 + nl > g->ngTW) {
            throw ArgError("shape program shorter than its header");
        }
        if (!(g->gTW[1] > 0.0f)) {
            throw ArgError("shape program: the field width must be positive");
        }
        for (int l = 0; l < nl; ++l) {
            const float o = g->gTW[5 + l];
            if (!(o >= 0.0f && o < (float)g->ngTW)) {
                throw ArgError("shape program: code offset out of range");
            }
        }
        const float T = g->gTW[8 + nl];
        if (!(T == 0.0f || (T > 0.0f && (int64_t)T + 4 <= g->ngTW))) {
            throw ArgError("shape program: brick table out of range");
        }
    }
    if (g->gm > 0 && (!g->gI || !g->gTW || (g->ngTW != 0 && g->ngTW < 2 * (int64_t)g->gm))) {
        throw ArgError("gray-scale fields need gI and gTW (2 gm floats)");
    }
    if (!(g->hmin > 0.0f) || !(g->hmax >= g->hmin)) {
        throw ArgError("need 0 < hmin <= hmax");
    }
    if (nd->n < 0 || nd->n > (int64_t)0x7FFFFFFF / 2) {
        throw ArgError("node count out of range");
    }
    if (nd->n > 0 && (!nd->P || !nd->lab || !nd->typ || !nd->part)) {
        throw ArgError("node array missing");
    }
    if (p->max_iters < 0) {
        throw ArgError("max_iters must be >= 0");
    }
    // brick tables: every slot a lookup can reach must exist (host arrays;
    // device-resident ones come from this library's own grid build)
    const int64_t nb = on_device(g->bl_cnt) ? 0 : (int64_t)g->nbx * g->nby * g->nbz;
    for (int64_t b = 0; b < nb; ++b) {
        const int c = g->bl_cnt[b];
        if (c < 0 || c > V2M_BL + 1) {
            throw ArgError("brick label count out of range");
        }
        const int s = g->bl_slot[b];
        if (s >= 0 && (int64_t)s + std::min(c, V2M_BL) > g->nslots) {
            throw ArgError("brick slot beyond the phi array");
        }
    }
    for (int64_t i = 0, nn = on_device(nd->typ) ? 0 : nd->n; i < nn; ++i) {
        if (nd->typ[i] > V2M_CORNER) {
            throw ArgError("node type out of range");
        }
        if (g->gm > 0 && nd->lab[i] > g->gm) {
            throw ArgError("gray-scale node label above the threshold count");
        }
    }
    if (!(p->t + p->skin > 0.0f)) {
        throw ArgError("t + skin must be positive");
    }
}

// Hash geometry of relax_cpu (src/v2m_particles.cpp:737-761), same float operations.
DHash hash_geometry(const v2m_grid_view* g, const v2m_relax_params* p, int* nkeys) {
    DHash H;
    std::memset(&H, 0, sizeof(H));
    H.b0 = (p->t + p->skin) * g->hmin;
    H.ox = -0.5f * g->vs[0];
    H.oy = -0.5f * g->vs[1];
    H.oz = -0.5f * g->vs[2];
    const float ext[3] = { g->nx * g->vs[0], g->ny * g->vs[1], g->nz * g->vs[2] };
    H.nlev = 1;
    while (H.nlev < V2M_MAXLEV && H.b0 * static_cast<float>(1 << (H.nlev - 1)) < (p->t + p->skin) * g->hmax) {
        ++H.nlev;
    }
    int64_t nk = 0;
    for (int L = 0; L < H.nlev; ++L) {
        H.off[L] = (int)nk;
        const float bL = H.b0 * static_cast<float>(1 << L);
        for (int a = 0; a < 3; ++a) {
            H.dim[L][a] = std::max(1, static_cast<int>(std::ceil(ext[a] / bL)));
        }
        nk += (int64_t)H.dim[L][0] * H.dim[L][1] * H.dim[L][2];
    }
    if (nk > 0x3FFFFFFF) {
        throw ArgError("too many hash bins (hmin too small for the grid)");
    }
    *nkeys = (int)nk;
    return H;
}

template <typename T>
T* upload(v2m_session* s, const T* host, size_t count) {
    T* d = s->alloc<T>(count);
    if (count) {
        ck(cudaMemcpyAsync(d, host, count * sizeof(T), cudaMemcpyDefault, s->stream), "upload");
    }
    return d;
}

// The corner tables of one volume's grid (DGrid::xbrick, xphi), built on the
// device from the uploaded grid; the table list is laid out on the host.
void build_corner_tables(v2m_session* s, DGrid& g, size_t nb) {
    uint4* xbrick = s->alloc<uint4>(3 * nb);
    int* xn = nullptr;
    ck(pool_malloc((void**)&xn, 4 * std::max<size_t>(nb, 1), s->stream), "cudaMallocAsync");
    launch_xcount(s->stream, g, xbrick, xn, (int)nb);
    ck(cudaGetLastError(), "corner tables");
    std::vector<int> hn(nb);
    std::vector<uint4> rec(3 * nb);
    ck(cudaMemcpyAsync(hn.data(), xn, 4 * nb, cudaMemcpyDeviceToHost, s->stream), "corner tables");
    ck(cudaMemcpyAsync(rec.data(), xbrick, sizeof(uint4) * 3 * nb, cudaMemcpyDeviceToHost, s->stream), "corner tables");
    ck(cudaFreeAsync(xn, s->stream), "cudaFreeAsync");
    ck(cudaStreamSynchronize(s->stream), "synchronize");
    std::vector<int2> tabs;
    for (size_t b = 0; b < nb; ++b) {
        if (hn[b] > 0) {
            if (tabs.size() + hn[b] > (size_t)0x7FFFFFFF) {
                throw ArgError("too many corner tables");
            }
            rec[3 * b].y = (uint32_t)tabs.size();   // the first table
            const uint32_t w[8] = { rec[3 * b].z, rec[3 * b].w, rec[3 * b + 1].x, rec[3 * b + 1].y,
                                    rec[3 * b + 1].z, rec[3 * b + 1].w, rec[3 * b + 2].x, rec[3 * b + 2].y };
            for (int q = 0; q < hn[b]; ++q) {
                tabs.push_back(make_int2((int)b, (int)((w[q >> 1] >> (16 * (q & 1))) & 0xFFFFu)));
            }
        }
    }
    const int2* dtabs = upload(s, tabs.data(), tabs.size());
    ck(cudaMemcpyAsync(xbrick, rec.data(), sizeof(uint4) * 3 * nb, cudaMemcpyHostToDevice, s->stream), "corner tables");
    float* xphi = s->alloc<float>(tabs.size() * 729);
    launch_xfill(s->stream, g, dtabs, xphi, (int)tabs.size());
    ck(cudaGetLastError(), "corner tables");
    ck(cudaStreamSynchronize(s->stream), "synchronize");   // (tabs and rec are host vectors)
    g.xbrick = xbrick;
    g.xphi = xphi;
    g.ntab = (int64_t)tabs.size();
}

// One volume's fields on the device: the caller's arrays uploaded, and the
// corner tables built from them.
DGrid upload_grid(v2m_session* s, const v2m_grid_view* g) {
    DGrid G;
    std::memset(&G, 0, sizeof(G));
    const size_t nvox = (size_t)g->nx * g->ny * g->nz;
    const size_t nb = (size_t)g->nbx * g->nby * g->nbz;
    G.nx = g->nx;
    G.ny = g->ny;
    G.nz = g->nz;
    G.nbx = g->nbx;
    G.nby = g->nby;
    G.nbz = g->nbz;
    G.vx = g->vs[0];
    G.vy = g->vs[1];
    G.vz = g->vs[2];
    G.L = upload(s, g->L, nvox);
    G.bl_cnt = upload(s, g->bl_cnt, nb);
    G.bl_lab = upload(s, g->bl_lab, nb * V2M_BL);
    G.bl_slot = upload(s, g->bl_slot, nb);
    G.phi = upload(s, g->phi, (size_t)g->nslots * V2M_SLOT);
    G.nslots = g->nslots;
    G.hvox = upload(s, g->h, nvox);
    if (kChecked) {   // one bounds-check word per session, shared by its grids
        if (!s->chk) {
            s->chk = s->alloc<int>(2);
            ck(cudaMemsetAsync(s->chk, 0, 2 * sizeof(int), s->stream), "memset");
        }
        G.chk = s->chk;
    }
    G.gm = g->gm;
    if (g->gm > 0) {
        G.gI = upload(s, g->gI, nvox);
        G.gTW = upload(s, g->gTW, 2 * (size_t)g->gm);
        G.ntw = 2 * (int64_t)g->gm;
    } else if (g->gm < 0) {
        G.gI = nullptr;
        G.gTW = upload(s, g->gTW, (size_t)g->ngTW);
        G.ntw = g->ngTW;
    } else {
        G.gI = nullptr;
        G.gTW = s->alloc<float>(4);
        G.ntw = 0;
    }
    build_corner_tables(s, G, nb);
    return G;
}

void init_ctl(v2m_session* s) {
    std::vector<VolCtl> c(s->nvol);
    for (int v = 0; v < s->nvol; ++v) {
        std::memset(&c[v], 0, sizeof(VolCtl));
        c[v].fdt = s->hvols[v].fire_dt0;
        c[v].falpha = 0.1f;
    }
    ck(cudaMemcpyAsync(s->d.ctl, c.data(), sizeof(VolCtl) * s->nvol, cudaMemcpyHostToDevice, s->stream), "ctl");
    ck(cudaStreamSynchronize(s->stream), "synchronize");
}

void upload_vols(v2m_session* s) {
    ck(cudaMemcpyAsync(s->d.vols, s->hvols.data(), sizeof(DVol) * s->nvol, cudaMemcpyHostToDevice, s->stream), "vols");
}

void do_reset(v2m_session* s) {
    const Dev& d = s->d;
    for (DVol& V : s->hvols) {
        V.hn_exact = 1;   // the seeds' sizes are packed from their positions
    }
    upload_vols(s);
    ck(cudaMemcpyAsync(d.Pq, s->Pq0, sizeof(float4) * d.N, cudaMemcpyDeviceToDevice, s->stream), "reset P");
    ck(cudaMemcpyAsync(d.typ, s->typ0, d.N, cudaMemcpyDeviceToDevice, s->stream), "reset typ");
    ck(cudaMemcpyAsync(d.part, s->part0, sizeof(uint32_t) * d.N, cudaMemcpyDeviceToDevice, s->stream), "reset part");
    ck(cudaMemsetAsync(d.Vel, 0, sizeof(float4) * d.N, s->stream), "reset V");
    ck(cudaMemsetAsync(d.F, 0, sizeof(float4) * d.N, s->stream), "reset F");
    ck(cudaMemsetAsync(d.mv, 0, sizeof(float) * d.N, s->stream), "reset mv");
    ck(cudaMemsetAsync(d.pw, 0, sizeof(float) * d.N, s->stream), "reset pw");
    ck(cudaMemsetAsync(d.cnt, 0, sizeof(int) * d.KT, s->stream), "reset cnt");
    ck(cudaMemsetAsync(d.G, 0, sizeof(Global), s->stream), "reset G");
    init_ctl(s);
    s->ms_hash = s->ms_loop = 0.0;
}

v2m_session* create(int nvol, const v2m_grid_view* gv, const v2m_relax_params* pv, const v2m_nodes_view* nv, int device) {
    if (nvol < 1 || nvol > kMaxVol) {
        throw ArgError("volume count must be in [1, 1024]");
    }
    for (int v = 0; v < nvol; ++v) {
        validate(gv + v, pv + v, nv + v);
    }
    lap("checks");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        throw CudaError("no CUDA device available");
    }
    const int dev = device < 0 ? 0 : device;
    if (dev >= ndev) {
        throw ArgError("device index out of range");
    }
    ck(cudaSetDevice(dev), "cudaSetDevice");
    inject("create");
    v2m_session* s = new v2m_session();
    try {
        s->device = dev;
        s->nvol = nvol;
        ck(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        if (g_clock) {
            g_clock->stream = s->stream;
        }
        s->serial_power = env_int("V2M_CUDA_SERIAL_POWER", 0);
        s->force_threads = env_int("V2M_CUDA_FORCE_THREADS", 256);
        if (s->force_threads != 64 && s->force_threads != 128 && s->force_threads != 256) {
            s->force_threads = 256;
        }
        s->graph_iters = std::max(1, env_int("V2M_CUDA_GRAPH_ITERS", 10));
        s->time_force = env_int("V2M_CUDA_TIME_FORCE", 0);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        s->refresh_blocks = sms * 4;
        s->d.sms = sms;
        s->d.shape_any = 0;
        for (int v = 0; v < nvol; ++v) {
            s->d.shape_any |= gv[v].gm < 0;
        }
        static const int env_div = std::getenv("V2M_REBUILD_DIV") ? std::atoi(std::getenv("V2M_REBUILD_DIV")) : 300;
        // layout
        int64_t N = 0, KT = 0;
        s->hvols.resize(nvol);
        s->info.resize(nvol);
        s->prm.assign(pv, pv + nvol);
        for (int v = 0; v < nvol; ++v) {
            DVol& V = s->hvols[v];
            std::memset(&V, 0, sizeof(DVol));
            VolInfo& I = s->info[v];
            I.n = (int)nv[v].n;
            V.H = hash_geometry(gv + v, pv + v, &I.nkeys);
            I.nofs = N;
            N += align_up(std::max<int64_t>(I.n, 1), kNodeAlign);
            I.kofs = KT;
            KT += align_up((int64_t)I.nkeys + 1, kScanTile);
            I.max_iters = pv[v].max_iters;
            I.hmode = pv[v].h_mode;
            s->max_iters = std::max(s->max_iters, I.max_iters);
        }
        if (N > 0x7FFFFFFF) {
            throw ArgError("too many nodes in the session");
        }
        Dev& d = s->d;
        d.nvol = nvol;
        d.N = N;
        d.KT = KT;
        d.ntile_key = (int)(KT / kScanTile);
        d.vols = s->alloc<DVol>(nvol);
        d.ctl = s->alloc<VolCtl>(nvol);
        d.G = s->alloc<Global>(1);
        d.nodevol = s->alloc<uint16_t>(N);
        d.tilevol = s->alloc<int16_t>(d.ntile_key);
        d.Pq = s->alloc<float4>(N);
        d.F = s->alloc<float4>(N);
        d.Vel = s->alloc<float4>(N);
        d.P0 = s->alloc<float4>(N);
        d.Ps = s->alloc<float4>(N);
        d.Js = s->alloc<int2>(N);
        d.typ = s->alloc<uint8_t>(N);
        d.lab = s->alloc<uint16_t>(N);
        d.part = s->alloc<uint32_t>(N);
        d.mv = s->alloc<float>(N);
        d.pw = s->alloc<float>(N);
        d.key = s->alloc<int>(N);
        d.sorted = s->alloc<int>(N);
        d.sort_tmp = s->alloc<int>(N);
        d.nbr = s->alloc<int>((size_t)N * V2M_K);
        d.nnb = s->alloc<uint8_t>(N);
        d.rlist = s->alloc<int>(N);
        d.S = s->alloc<float4>(N);
        d.queue = s->alloc<int>(2 * N);
        d.cnt = s->alloc<int>(KT);
        d.cstart = s->alloc<int>(KT);
        d.cursor = s->alloc<int>(KT);
        d.tilesum = s->alloc<int>(d.ntile_key);
        d.tileofs = s->alloc<int>(d.ntile_key);
        d.psum = s->alloc<double2>(N / kMoveThreads + 1);
        d.pser = s->alloc<double>(nvol);
        s->Pq0 = s->alloc<float4>(N);
        s->typ0 = s->alloc<uint8_t>(N);
        s->part0 = s->alloc<uint32_t>(N);
        ck(cudaMemsetAsync(d.nnb, 0, N, s->stream), "memset");
        launch_lists_init(s->stream, d);
        ck(cudaGetLastError(), "list init");
        ck(cudaMemsetAsync(d.Pq, 0, sizeof(float4) * N, s->stream), "memset");
        ck(cudaMemsetAsync(d.P0, 0, sizeof(float4) * N, s->stream), "memset");
        ck(cudaMemsetAsync(d.Ps, 0, sizeof(float4) * N, s->stream), "memset");
        ck(cudaMemsetAsync(d.typ, 0, N, s->stream), "memset");
        ck(cudaMemsetAsync(d.lab, 0, 2 * N, s->stream), "memset");
        ck(cudaMemsetAsync(d.part, 0xFF, 4 * N, s->stream), "memset");
        ck(cudaMemsetAsync(d.key, 0, 4 * N, s->stream), "memset");
        ck(cudaMemsetAsync(d.sorted, 0, 4 * N, s->stream), "memset");
        ck(cudaMemsetAsync(d.cstart, 0, 4 * KT, s->stream), "memset");
        lap("allocate");
        std::vector<uint16_t> nodevol(N, 0xFFFF);
        std::vector<int16_t> tilevol(d.ntile_key, -1);
        for (int v = 0; v < nvol; ++v) {
            const VolInfo& I = s->info[v];
            const v2m_grid_view* g = gv + v;
            const v2m_relax_params* p = pv + v;
            DVol& V = s->hvols[v];
            V.g = upload_grid(s, g);
            V.nofs = I.nofs;
            V.n = I.n;
            V.kofs = I.kofs;
            V.nkeys = I.nkeys;
            V.tofs_key = (int)(I.kofs / kScanTile);
            V.ntile_key = (int)(align_up((int64_t)I.nkeys + 1, kScanTile) / kScanTile);
            V.tofs_node = (int)(I.nofs / kMoveThreads);
            V.ntile_node = (int)((I.n + kMoveThreads - 1) / kMoveThreads);
            V.t = p->t;
            V.skin = p->skin;
            V.fscale = p->fscale;
            V.fsurf = p->fsurf;
            V.dt = p->dt;
            V.maxstep = p->maxstep;
            V.snap = p->snap;
            V.dptol = p->dptol;
            V.voxmode = p->voxel_trap ? 1 : 0;
            V.fire = (p->fire && !p->voxel_trap) ? 1 : 0;
            V.max_iters = p->max_iters;
            V.rebuild_div = p->rebuild_div > 0 ? p->rebuild_div : (env_div > 0 ? env_div : 1);
            V.hmode = p->h_mode;
            V.policy = p->rebuild_policy;
            V.hn_exact = 1;
            V.fire_dt0 = std::sqrt(p->dt);
            V.fire_dtmax = p->fire_dtmax * V.fire_dt0;
            std::fill(nodevol.begin() + I.nofs, nodevol.begin() + I.nofs + I.n, (uint16_t)v);
            for (int t = 0; t < V.ntile_key; ++t) {
                tilevol[V.tofs_key + t] = (int16_t)v;
            }
            if (I.n > 0) {
                ck(cudaMemcpyAsync(d.lab + I.nofs, nv[v].lab, 2 * (size_t)I.n, cudaMemcpyDefault, s->stream), "lab");
                ck(cudaMemcpyAsync(d.typ + I.nofs, nv[v].typ, (size_t)I.n, cudaMemcpyDefault, s->stream), "typ");
                ck(cudaMemcpyAsync(d.part + I.nofs, nv[v].part, 4 * (size_t)I.n, cudaMemcpyDefault, s->stream), "part");
            }
        }
        lap("grid upload + corner tables");
        ck(cudaMemcpyAsync(d.vols, s->hvols.data(), sizeof(DVol) * nvol, cudaMemcpyHostToDevice, s->stream), "vols");
        ck(cudaMemcpyAsync(d.nodevol, nodevol.data(), 2 * N, cudaMemcpyHostToDevice, s->stream), "nodevol");
        ck(cudaMemcpyAsync(d.tilevol, tilevol.data(), 2 * (size_t)d.ntile_key, cudaMemcpyHostToDevice, s->stream), "tilevol");
        // positions: staged as float[3n] then packed with the size and type sign
        for (int v = 0; v < nvol; ++v) {
            const VolInfo& I = s->info[v];
            if (I.n == 0) {
                continue;
            }
            float* tmp = nullptr;
            ck(pool_malloc((void**)&tmp, 12 * (size_t)I.n, s->stream), "cudaMallocAsync");
            ck(cudaMemcpyAsync(tmp, nv[v].P, 12 * (size_t)I.n, cudaMemcpyDefault, s->stream), "P");
            launch_pack_nodes(s->stream, d, v, I.n, tmp, d.typ);
            ck(cudaFreeAsync(tmp, s->stream), "cudaFreeAsync");
        }
        ck(cudaGetLastError(), "pack");
        ck(cudaMemcpyAsync(s->Pq0, d.Pq, sizeof(float4) * N, cudaMemcpyDeviceToDevice, s->stream), "seed P");
        ck(cudaMemcpyAsync(s->typ0, d.typ, N, cudaMemcpyDeviceToDevice, s->stream), "seed typ");
        ck(cudaMemcpyAsync(s->part0, d.part, 4 * N, cudaMemcpyDeviceToDevice, s->stream), "seed part");
        do_reset(s);
        lap("node upload");
        s->nbr_threads = env_int("V2M_CUDA_NBR_THREADS", 128);
        if (s->nbr_threads != 64 && s->nbr_threads != 128 && s->nbr_threads != 256) {
            s->nbr_threads = 128;
        }
        if (env_int("V2M_CUDA_AUTOTUNE", 0) && !tune_lookup(s)) {
            do_autotune(s, 20);
            tune_store(s);
        }
        return s;
    } catch (...) {
        delete s;
        throw;
    }
}

// relax_cl's rebuild (src/v2m_gpu.cpp:259-277) for the volumes whose rebuild flag is set.
void enqueue_rebuild(v2m_session* s) {
    const Dev& d = s->d;
    launch_keys(s->stream, d);
    launch_scan(s->stream, d);
    launch_scatter(s->stream, d);
    launch_neighbors(s->stream, d, s->nbr_threads);
    s->launches += 7;
}

// (inside a stream capture an event record only becomes a graph node with
// cudaEventRecordExternal; without it the event is a capture dependency only)
void record(v2m_session* s, cudaEvent_t e) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    ck(cudaStreamIsCapturing(s->stream, &cs), "capture status");
    ck(cudaEventRecordWithFlags(e, s->stream, cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : 0),
       "event");
}

void enqueue_force(v2m_session* s, cudaEvent_t e0, cudaEvent_t e1) {
    if (e0) {
        record(s, e0);
    }
    launch_force(s->stream, s->d, s->force_threads);
    if (e1) {
        record(s, e1);
    }
    s->launches += 1;
    s->force_launches += 1;
}

// The rest of an iteration: move + reductions, control, self-refresh, rebuild.
void enqueue_tail(v2m_session* s) {
    const Dev& d = s->d;
    launch_move(s->stream, d);
    launch_control(s->stream, d, s->serial_power);
    launch_refresh(s->stream, d, s->refresh_blocks);
    // k_move_pre, k_move_int, k_move_main (and its shape instance), control, refresh
    s->launches += 5 + (d.shape_any ? 1 : 0) + (s->serial_power ? 1 : 0);
    enqueue_rebuild(s);
}

void read_ctl(v2m_session* s, std::vector<VolCtl>& c) {
    c.resize(s->nvol);
    ck(cudaMemcpyAsync(c.data(), s->d.ctl, sizeof(VolCtl) * s->nvol, cudaMemcpyDeviceToHost, s->stream), "read ctl");
    ck(cudaStreamSynchronize(s->stream), "synchronize");
}

bool all_done(v2m_session* s, const std::vector<VolCtl>& c) {
    for (int v = 0; v < s->nvol; ++v) {
        if (!c[v].done && c[v].it < s->info[v].max_iters) {
            return false;
        }
    }
    return true;
}

void build_graph(v2m_session* s) {
    if (s->gexec) {
        return;
    }
    const int G = s->graph_iters;
    s->gev.assign(2 * G, nullptr);
    for (auto& e : s->gev) {
        ck(cudaEventCreate(&e), "cudaEventCreate");
    }
    cudaGraph_t graph = nullptr;
    const int64_t l0 = s->launches, f0 = s->force_launches;
    ck(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        for (int k = 0; k < G; ++k) {
            enqueue_force(s, s->gev[2 * k], s->gev[2 * k + 1]);
            enqueue_tail(s);
        }
    } catch (...) {
        cudaStreamEndCapture(s->stream, &graph);
        if (graph) {
            cudaGraphDestroy(graph);
        }
        throw;
    }
    ck(cudaStreamEndCapture(s->stream, &graph), "end capture");
    s->launches = l0;
    s->force_launches = f0;
    cudaError_t e = cudaGraphInstantiate(&s->gexec, graph, 0);
    cudaGraphDestroy(graph);
    ck(e, "cudaGraphInstantiate");
}

// Up to `iters` iterations of every volume still running.
void do_iterate(v2m_session* s, int iters, int graph) {
    std::vector<VolCtl> c;
    read_ctl(s, c);
    if (all_done(s, c)) {
        return;
    }
    const auto t0 = std::chrono::steady_clock::now();
    if (graph) {
        build_graph(s);
        lap("graph capture");
        const int G = s->graph_iters;
        int done_it = 0;
        // per-iteration launches inside the graph: force + tail
        const int per_it = 1 + 4 + (s->serial_power ? 1 : 0) + 7;
        while (done_it < iters) {
            ck(cudaGraphLaunch(s->gexec, s->stream), "cudaGraphLaunch");
            s->launches += (int64_t)G * per_it;
            s->force_launches += G;
            done_it += G;
            read_ctl(s, c);
            inject("iterate", c[0].it);
            if (s->time_force) {
                for (int k = 0; k < G; ++k) {
                    float ms = 0.0f;
                    ck(cudaEventElapsedTime(&ms, s->gev[2 * k], s->gev[2 * k + 1]), "force event time");
                    s->force_ms += ms;
                }
            }
            if (all_done(s, c)) {
                break;
            }
        }
    } else {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (s->time_force) {
            ck(cudaEventCreate(&e0), "event");
            ck(cudaEventCreate(&e1), "event");
        }
        // the host reads the control blocks every `every` iterations (25; 1 is the
        // reference's relax_cl, which blocks on a read-back every iteration,
        // src/v2m_gpu.cpp:348)
        const int every = std::max(1, env_int("V2M_CUDA_HOST_CHECK", 25));
        for (int k = 0; k < iters; ++k) {
            enqueue_force(s, e0, e1);
            enqueue_tail(s);
            ck(cudaGetLastError(), "launch");
            if (s->time_force) {
                ck(cudaEventSynchronize(e1), "event sync");
                float ms = 0.0f;
                ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
                s->force_ms += ms;
            }
            if ((k + 1) % every == 0 || k + 1 == iters) {
                read_ctl(s, c);
                inject("iterate", c[0].it);
                if (all_done(s, c)) {
                    break;
                }
            }
        }
        if (e0) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
        }
    }
    ck(cudaGetLastError(), "launch");
    check_kernel_error(s);
    s->ms_loop += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void do_rebuild(v2m_session* s) {
    inject("rebuild");
    const auto t0 = std::chrono::steady_clock::now();
    launch_set_rebuild(s->stream, s->d, 1);
    s->launches += 1;
    enqueue_rebuild(s);
    launch_set_rebuild(s->stream, s->d, 0);
    s->launches += 1;
    ck(cudaGetLastError(), "launch");
    check_kernel_error(s);
    s->ms_hash += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void fill_stats(v2m_session* s, int v, v2m_relax_stats* st) {
    std::vector<VolCtl> c;
    read_ctl(s, c);
    const VolInfo& I = s->info[v];
    std::memset(st, 0, sizeof(*st));
    st->iters = c[v].iters;
    st->rebuilds = c[v].rebuilds;
    st->last_move = c[v].last_move;
    st->last_p99 = c[v].last_p99;
    st->fire_resets = c[v].resets;
    st->fire_dt = s->hvols[v].fire ? c[v].fdt : 0.0f;
    if (I.n > 0) {
        std::vector<uint8_t> t(I.n);
        ck(cudaMemcpyAsync(t.data(), s->d.typ + I.nofs, I.n, cudaMemcpyDeviceToHost, s->stream), "typ");
        ck(cudaStreamSynchronize(s->stream), "synchronize");
        for (uint8_t x : t) {
            st->n_interior += x == V2M_INTERIOR;
            st->n_interface += x == V2M_INTERFACE;
            st->n_junction += x == V2M_JUNCTION;
            st->n_corner += x == V2M_CORNER;
        }
    }
    st->ms_hash = s->ms_hash;
    st->ms_move = s->ms_loop;
    st->ms_force = s->force_ms;
}

void read_nodes(v2m_session* s, int v, v2m_nodes_view* nd) {
    const VolInfo& I = s->info[v];
    if (!nd || nd->n != I.n) {
        throw ArgError("node view does not match the volume");
    }
    if (I.n == 0) {
        return;
    }
    float* tmp = nullptr;
    ck(pool_malloc((void**)&tmp, 12 * (size_t)I.n, s->stream), "cudaMallocAsync");
    launch_unpack_P(s->stream, s->d, I.nofs, I.n, tmp);
    ck(cudaMemcpyAsync(nd->P, tmp, 12 * (size_t)I.n, cudaMemcpyDeviceToHost, s->stream), "P");
    if (std::getenv("V2M_CUDA_FAIL_AT")) {
        ck(cudaStreamSynchronize(s->stream), "synchronize");   // (the positions are in the caller's arrays)
        try {
            inject("readback");
        } catch (...) {
            cudaFreeAsync(tmp, s->stream);
            throw;
        }
    }
    ck(cudaMemcpyAsync(nd->typ, s->d.typ + I.nofs, I.n, cudaMemcpyDeviceToHost, s->stream), "typ");
    ck(cudaMemcpyAsync(nd->part, s->d.part + I.nofs, 4 * (size_t)I.n, cudaMemcpyDeviceToHost, s->stream), "part");
    ck(cudaFreeAsync(tmp, s->stream), "cudaFreeAsync");
    ck(cudaStreamSynchronize(s->stream), "synchronize");
}

template <typename F>
int guard(F&& f) {
    try {
        f();
        g_err.clear();
        return V2M_OK;
    } catch (const ArgError& e) {
        g_err = e.what();
        return V2M_ERR_ARG;
    } catch (const KernelError& e) {
        g_err = e.what();
        return V2M_ERR_KERNEL;
    } catch (const CudaError& e) {
        g_err = e.what();
        return V2M_ERR_CUDA;
    } catch (const std::exception& e) {
        g_err = e.what();
        return V2M_ERR_CUDA;
    }
}

// tn::seed_cpu's spacing of seed level L (src/opencl/v2m_seed_body.cl:441-443),
// with the same float operations and the host's float pow
float seed_spacing(int L, int nseed, float hmin, float hmax) {
    return nseed <= 1 ? hmin : hmin * std::pow(hmax / hmin, (float)L / (float)(nseed - 1));
}

}  // namespace

// A host array left uninitialized (the device copy writes every element).
template <typename T>
struct HostArray {
    // plain memory (T is an arithmetic type); large arrays 2 MB aligned and
    // marked for transparent huge pages, which halves their first-touch cost
    // when the device copies land in them
    struct Free {
        void operator()(T* q) const {
            std::free(q);
        }
    };
    std::unique_ptr<T, Free> p;
    size_t n = 0;
    void resize(size_t count) {
        static_assert(std::is_arithmetic<T>::value, "HostArray holds plain numbers");
        constexpr size_t kHuge = (size_t)2 << 20;
        const size_t bytes = count * sizeof(T);
        void* q = nullptr;
        if (bytes >= 2 * kHuge) {
            q = std::aligned_alloc(kHuge, (bytes + kHuge - 1) / kHuge * kHuge);
            if (q) {
                madvise(q, bytes, MADV_HUGEPAGE);   // advice only: ignored where unsupported
            }
        } else if (bytes) {
            q = std::malloc(bytes);
        }
        if (bytes && !q) {
            throw std::bad_alloc();
        }
        p.reset(static_cast<T*>(q));
        n = count;
    }
    T* data() const {
        return p.get();
    }
    size_t size() const {
        return n;
    }
};

// A grid built on the device, held on the host (tn::Grid's arrays).
struct v2m_grid_result {
    int32_t nx = 0, ny = 0, nz = 0;
    float vs[3] = { 1, 1, 1 };
    HostArray<uint16_t> L, bl_lab;
    HostArray<int32_t> bl_cnt, bl_slot;
    HostArray<float> phi, h;
    HostArray<uint8_t> grade;
    int64_t nslots = 0;
    float hbase = 0, hmin = 0, hmax = 0;
    int32_t R = 0, limit_sweeps = 0;
};

// Seeds made on the device, held on the host until copied out.
struct v2m_seed_result {
    std::vector<float> P;
    std::vector<uint16_t> lab;
    std::vector<uint8_t> typ;
    std::vector<uint16_t> part, part3;
};

namespace {

int pick_device(int device) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        throw CudaError("no CUDA device available");
    }
    const int dev = device < 0 ? 0 : device;
    if (dev >= ndev) {
        throw ArgError("device index out of range");
    }
    ck(cudaSetDevice(dev), "cudaSetDevice");
    return dev;
}

void release_seeds(SeedBuffers& B, cudaStream_t st) {
    for (void* p : B.tmp) {
        cudaFreeAsync(p, st);
    }
    B.tmp.clear();
    cudaStreamSynchronize(st);
}

// The seeding's own argument checks (before any device is touched).
void check_seed_args(const v2m_grid_view* g, const v2m_relax_params* prm) {
    if (!g->grade) {
        throw ArgError("seeding needs the grid's size grades (grade)");
    }
    if (prm->nseed < 1 || prm->nseed > 256) {
        throw ArgError("nseed must be in [1, 256]");
    }
    if (g->nfeat < 0 || (g->nfeat > 0 && !g->feat)) {
        throw ArgError("feat: nfeat floats needed");
    }
    {
        // the counts and offsets are int32, as the reference's: bound the
        // lattice points of the finest level (spacing hmin) over all voxels,
        // and the grid vertices
        const double s0 = seed_spacing(0, prm->nseed, g->hmin, g->hmax);
        const double per = (g->vs[0] / s0 + 2.0) * (g->vs[1] / (0.8660254 * s0) + 2.0) *
                           (g->vs[2] / (0.8164966 * s0) + 2.0);
        const double nvox = (double)g->nx * g->ny * g->nz;
        const double nvert = (double)(g->nx + 1) * (g->ny + 1) * (g->nz + 1);
        if (!(s0 > 0.0) || per * nvox >= 2147483647.0 || nvert >= 2147483647.0) {
            throw ArgError("seeding: the grid could hold more seeds than int32 counts allow");
        }
    }
}

// Seeding of grid g (a view of host or device arrays, g->grade required) on
// device dev, into B (device arrays; release_seeds frees them). `tmp` holds the
// grid's device copy and its corner tables.
void seed_on(v2m_session& tmp, const v2m_grid_view* g, const v2m_relax_params* prm, int dev, SeedBuffers& B) {
    check_seed_args(g, prm);
    SeedArgs A;
    A.g = upload_grid(&tmp, g);
    const size_t nvox = (size_t)g->nx * g->ny * g->nz;
    A.grade = upload(&tmp, g->grade, nvox);
    std::vector<float> sp(prm->nseed);
    for (int L = 0; L < prm->nseed; ++L) {
        sp[L] = seed_spacing(L, prm->nseed, g->hmin, g->hmax);
    }
    A.spacing = upload(&tmp, sp.data(), sp.size());
    A.nseed = prm->nseed;
    A.voxmode = prm->voxel_trap ? 1 : 0;
    A.jseed = prm->jseed;
    A.corners = prm->corners ? 1 : 0;
    A.hmax = g->hmax;
    A.feat = g->feat;
    A.nfeat = g->feat ? g->nfeat : 0;
    cudaDeviceGetAttribute(&A.sms, cudaDevAttrMultiProcessorCount, dev);
    A.stream = tmp.stream;
    std::string err;
    cudaError_t e = seed_run(A, B, err);
    if (e == cudaSuccess) {
        try {
            check_bounds_word(&tmp);
        } catch (...) {
            release_seeds(B, tmp.stream);
            throw;
        }
    }
    if (e != cudaSuccess) {
        release_seeds(B, tmp.stream);
        cudaGetLastError();
        if (!err.empty()) {
            throw ArgError("seeding: " + err);
        }
        throw CudaError(std::string("seeding: ") + cudaGetErrorString(e));
    }
}

void seeds_to_host(const SeedBuffers& B, cudaStream_t st, v2m_seed_result& r) {
    const size_t m = (size_t)B.n;
    r.P.resize(3 * m);
    r.lab.resize(m);
    r.typ.resize(m);
    r.part.resize(2 * m);
    r.part3.resize(m);
    if (m) {
        ck(cudaMemcpyAsync(r.P.data(), B.P, 12 * m, cudaMemcpyDeviceToHost, st), "seeds");
        ck(cudaMemcpyAsync(r.lab.data(), B.lab, 2 * m, cudaMemcpyDeviceToHost, st), "seeds");
        ck(cudaMemcpyAsync(r.typ.data(), B.typ, m, cudaMemcpyDeviceToHost, st), "seeds");
        ck(cudaMemcpyAsync(r.part.data(), B.part, 4 * m, cudaMemcpyDeviceToHost, st), "seeds");
        ck(cudaMemcpyAsync(r.part3.data(), B.part3, 2 * m, cudaMemcpyDeviceToHost, st), "seeds");
    }
    ck(cudaStreamSynchronize(st), "synchronize");
}

// The device grid build's arguments from the C ABI's, checked.
GridBuildArgs grid_args(const uint16_t* L, int32_t nx, int32_t ny, int32_t nz, const float* vs,
                        const v2m_grid_params* p) {
    if (!L || !vs || !p) {
        throw ArgError("null argument");
    }
    if (nx < 1 || ny < 1 || nz < 1 || (int64_t)nx * ny * nz > (int64_t)0x7FFFFFFF) {
        throw ArgError("grid dimensions must be positive, at most 2^31 voxels");
    }
    if (!(vs[0] > 0.0f && vs[1] > 0.0f && vs[2] > 0.0f)) {
        throw ArgError("voxel sizes must be positive");
    }
    if (!(p->sigma > 0.0f) || !(p->sigma_curv > 0.0f) || p->sigma_thin < 0.0f || !(p->g >= 0.0f) ||
        !(p->K > 0.0f) || (p->nhlab > 0 && !p->hlab) || p->nhlab < 0) {
        throw ArgError("grid parameters out of range (sigma, sigma_curv > 0; sigma_thin, g >= 0; K > 0)");
    }
    GridBuildArgs A;
    A.L = L;
    A.nx = nx;
    A.ny = ny;
    A.nz = nz;
    A.vs[0] = vs[0];
    A.vs[1] = vs[1];
    A.vs[2] = vs[2];
    GridParamsH& q = A.prm;
    q.sigma = p->sigma;
    q.sigma_thin = p->sigma_thin;
    q.thin_lo = p->thin_lo;
    q.thin_hi = p->thin_hi;
    q.thick = p->thick;
    q.thin_floor = p->thin_floor;
    q.preserve = p->preserve;
    q.sigma_curv = p->sigma_curv;
    q.hbase = p->hbase;
    q.hmin = p->hmin;
    q.hmax = p->hmax;
    q.K = p->K;
    q.g = p->g;
    if (p->nhlab > 0) {
        q.hlab.assign(p->hlab, p->hlab + p->nhlab);
    }
    return A;
}

// A view of the device grid build's output (device arrays).
v2m_grid_view device_view(const GridBuildArgs& A, const GridBuildOut& O) {
    v2m_grid_view g{};
    g.nx = A.nx;
    g.ny = A.ny;
    g.nz = A.nz;
    g.nbx = (A.nx + 7) / 8;
    g.nby = (A.ny + 7) / 8;
    g.nbz = (A.nz + 7) / 8;
    g.vs[0] = A.vs[0];
    g.vs[1] = A.vs[1];
    g.vs[2] = A.vs[2];
    g.L = O.L;
    g.bl_cnt = O.bl_cnt;
    g.bl_lab = O.bl_lab;
    g.bl_slot = O.bl_slot;
    g.phi = O.phi;
    g.nslots = O.nslots;
    g.h = O.h;
    g.hmin = O.hmin;
    g.hmax = O.hmax;
    g.gm = 0;
    g.grade = O.grade;
    return g;
}

}  // namespace

extern "C" {

void v2m_relax_params_default(v2m_relax_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->nseed = 8;
    p->t = 1.3f;
    p->skin = 0.3f;
    p->fscale = 1.2f;
    p->fsurf = 1.0f;
    p->dt = 0.5f;
    p->maxstep = 0.2f;
    p->snap = 0.5f;
    p->max_iters = 500;
    p->dptol = 2e-3f;
    p->jseed = 0.8f;
    p->corners = 1;
    p->voxel_trap = 0;
    p->thin = 0.0f;
    p->fire = 1;
    p->fire_dtmax = 2.0f;
    p->verbose = 0;
}

const char* v2m_cuda_last_error(void) {
    return g_err.c_str();
}

int v2m_cuda_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int v2m_session_create(int nvol, const v2m_grid_view* g, const v2m_relax_params* prm, const v2m_nodes_view* nd,
                       int device, v2m_session** out) {
    Trace trace("v2m_session_create");
    return guard([&] {
        if (!out) {
            throw ArgError("null output");
        }
        *out = create(nvol, g, prm, nd, device);
    });
}

int v2m_session_destroy(v2m_session* s) {
    return guard([&] {
        if (s) {
            cudaSetDevice(s->device);
            cudaStreamSynchronize(s->stream);
            delete s;
        }
    });
}

int v2m_session_reset(v2m_session* s) {
    return guard([&] {
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        do_reset(s);
    });
}

int v2m_session_rebuild(v2m_session* s) {
    Trace trace("v2m_session_rebuild");
    return guard([&] {
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        do_rebuild(s);
    });
}

int v2m_session_force(v2m_session* s) {
    Trace trace("v2m_session_force");
    return guard([&] {
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        enqueue_force(s, nullptr, nullptr);
        ck(cudaGetLastError(), "launch");
        check_kernel_error(s);
    });
}

int v2m_session_step_tail(v2m_session* s) {
    Trace trace("v2m_session_step_tail");
    return guard([&] {
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        enqueue_tail(s);
        ck(cudaGetLastError(), "launch");
        check_kernel_error(s);
    });
}

int v2m_session_iterate(v2m_session* s, int iters, int graph) {
    Trace trace("v2m_session_iterate");
    return guard([&] {
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        do_iterate(s, iters, graph);
    });
}

int v2m_session_run(v2m_session* s, int graph) {
    Trace trace("v2m_session_run");
    return guard([&] {
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        do_rebuild(s);
        do_iterate(s, s->max_iters, graph);
    });
}

int v2m_session_synchronize(v2m_session* s) {
    return guard([&] {
        ck(cudaStreamSynchronize(s->stream), "synchronize");
        check_kernel_error(s);
    });
}

int v2m_session_read_nodes(v2m_session* s, int vol, v2m_nodes_view* nd) {
    return guard([&] {
        if (vol < 0 || vol >= s->nvol) {
            throw ArgError("volume index out of range");
        }
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        read_nodes(s, vol, nd);
    });
}

int v2m_session_stats(v2m_session* s, int vol, v2m_relax_stats* st) {
    return guard([&] {
        if (vol < 0 || vol >= s->nvol || !st) {
            throw ArgError("bad argument");
        }
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        fill_stats(s, vol, st);
    });
}

int v2m_session_info(v2m_session* s, int vol, int64_t* n, int64_t* nkeys, int32_t* nlev) {
    return guard([&] {
        if (vol < 0 || vol >= s->nvol) {
            throw ArgError("volume index out of range");
        }
        if (n) {
            *n = s->info[vol].n;
        }
        if (nkeys) {
            *nkeys = s->info[vol].nkeys;
        }
        if (nlev) {
            *nlev = s->hvols[vol].H.nlev;
        }
    });
}

int v2m_session_counters(v2m_session* s, int64_t* launches, int64_t* force_launches, double* force_ms) {
    return guard([&] {
        if (launches) {
            *launches = s->launches;
        }
        if (force_launches) {
            *force_launches = s->force_launches;
        }
        if (force_ms) {
            *force_ms = s->force_ms;
        }
    });
}

int v2m_session_read_array(v2m_session* s, int vol, int what, void* host, int64_t bytes) {
    return guard([&] {
        if (vol < 0 || vol >= s->nvol || !host) {
            throw ArgError("bad argument");
        }
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        const VolInfo& I = s->info[vol];
        const Dev& d = s->d;
        const int n = I.n;
        auto need = [&](int64_t b) {
            if (bytes < b) {
                throw ArgError("host buffer too small");
            }
        };
        auto d2h = [&](const void* src, int64_t b) {
            need(b);
            if (b) {
                ck(cudaMemcpyAsync(host, src, (size_t)b, cudaMemcpyDeviceToHost, s->stream), "read");
            }
        };
        void* tmp = nullptr;
        auto scratch = [&](size_t b) {
            ck(pool_malloc(&tmp, std::max<size_t>(b, 16), s->stream), "cudaMallocAsync");
            return tmp;
        };
        switch (what) {
        case V2M_ARR_KEY: d2h(d.key + I.nofs, 4LL * n); break;
        case V2M_ARR_SORTED: {
            need(4LL * n);
            int* t = (int*)scratch(4 * (size_t)n);
            launch_local_ids(s->stream, d.sorted, I.nofs, n, t);
            d2h(t, 4LL * n);
            break;
        }
        case V2M_ARR_CSTART: {
            need(4LL * (I.nkeys + 1));
            int* t = (int*)scratch(4 * (size_t)(I.nkeys + 1));
            launch_local_cstart(s->stream, d.cstart, I.kofs, I.nkeys + 1, I.nofs, t);
            d2h(t, 4LL * (I.nkeys + 1));
            break;
        }
        case V2M_ARR_PS: d2h(d.Ps + I.nofs, 16LL * n); break;
        case V2M_ARR_NBR:
        case V2M_ARR_NNB: {
            int* t = (int*)scratch(4 * ((size_t)n * V2M_K + n));
            launch_lists_rowmajor(s->stream, d, I.nofs, n, t, t + (size_t)n * V2M_K);
            if (what == V2M_ARR_NBR) {
                d2h(t, 4LL * n * V2M_K);
            } else {
                d2h(t + (size_t)n * V2M_K, 4LL * n);
            }
            break;
        }
        case V2M_ARR_F: d2h(d.F + I.nofs, 16LL * n); break;
        case V2M_ARR_HN: {
            need(4LL * n);
            float* t = (float*)scratch(4 * (size_t)n);
            launch_hn(s->stream, d, I.nofs, n, t);
            d2h(t, 4LL * n);
            break;
        }
        case V2M_ARR_MV: d2h(d.mv + I.nofs, 4LL * n); break;
        case V2M_ARR_PW: d2h(d.pw + I.nofs, 4LL * n); break;
        case V2M_ARR_V:
        case V2M_ARR_P0: {
            need(12LL * n);
            std::vector<VolCtl> c;
            read_ctl(s, c);
            if (what == V2M_ARR_V && c[vol].vzero) {   // a FIRE reset zeroed every velocity
                std::memset(host, 0, 12 * (size_t)n);
                break;
            }
            float* t = (float*)scratch(12 * (size_t)n);
            launch_float4_to3(s->stream, what == V2M_ARR_V ? d.Vel : d.P0, I.nofs, n, t);
            d2h(t, 12LL * n);
            break;
        }
        case V2M_ARR_P: {
            need(12LL * n);
            float* t = (float*)scratch(12 * (size_t)n);
            launch_unpack_P(s->stream, d, I.nofs, n, t);
            d2h(t, 12LL * n);
            break;
        }
        case V2M_ARR_TYP: d2h(d.typ + I.nofs, n); break;
        case V2M_ARR_PART: d2h(d.part + I.nofs, 4LL * n); break;
        case V2M_ARR_HIST: {
            need(4LL * 34);
            std::vector<VolCtl> c;
            read_ctl(s, c);
            int* h = (int*)host;
            std::memcpy(h, c[vol].hist, 32 * 4);
            std::memcpy(h + 32, &c[vol].maxbits, 4);
            h[33] = c[vol].nhalf;
            break;
        }
        case V2M_ARR_DIRS: {
            need(12LL * n);
            float* t = (float*)scratch(12 * (size_t)n);
            launch_constraint_dirs(s->stream, d, vol, n, s->hvols[vol].g.gm < 0, t);
            d2h(t, 12LL * n);
            break;
        }
        case V2M_ARR_SERIAL_SUMS: {
            need(4);
            std::vector<VolCtl> c;
            read_ctl(s, c);
            *(int*)host = c[vol].serial_sums;
            break;
        }
        default: throw ArgError("unknown array");
        }
        if (tmp) {
            ck(cudaFreeAsync(tmp, s->stream), "cudaFreeAsync");
        }
        ck(cudaStreamSynchronize(s->stream), "synchronize");
    });
}

int v2m_session_write_array(v2m_session* s, int vol, int what, const void* host, int64_t bytes) {
    return guard([&] {
        if (vol < 0 || vol >= s->nvol || !host) {
            throw ArgError("bad argument");
        }
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        const VolInfo& I = s->info[vol];
        const Dev& d = s->d;
        const int n = I.n;
        auto exact = [&](int64_t b) {
            if (bytes != b) {
                throw ArgError("size mismatch");
            }
        };
        void* tmp = nullptr;
        auto staged = [&](int64_t b) {
            ck(pool_malloc(&tmp, std::max<size_t>((size_t)b, 16), s->stream), "cudaMallocAsync");
            ck(cudaMemcpyAsync(tmp, host, (size_t)b, cudaMemcpyHostToDevice, s->stream), "write");
            return tmp;
        };
        if (what == V2M_ARR_P || what == V2M_ARR_HN) {
            s->hvols[vol].hn_exact = 0;   // the move reads h from the size field from now on
            upload_vols(s);
        }
        switch (what) {
        case V2M_ARR_P: {
            exact(12LL * n);
            // keep the stored size: positions only
            float* t = (float*)staged(12LL * n);
            std::vector<float> hn(n);
            float* hd = nullptr;
            ck(pool_malloc((void**)&hd, 4 * (size_t)n + 16, s->stream), "cudaMallocAsync");
            launch_hn(s->stream, d, I.nofs, n, hd);
            launch_float3_to4(s->stream, t, I.nofs, n, d.Pq);
            launch_set_hn(s->stream, d, I.nofs, n, hd);
            ck(cudaFreeAsync(hd, s->stream), "cudaFreeAsync");
            break;
        }
        case V2M_ARR_TYP:
            exact(n);
            ck(cudaMemcpyAsync(d.typ + I.nofs, host, n, cudaMemcpyHostToDevice, s->stream), "write");
            launch_resign(s->stream, d, I.nofs, n);
            break;
        case V2M_ARR_PART:
            exact(4LL * n);
            ck(cudaMemcpyAsync(d.part + I.nofs, host, 4 * (size_t)n, cudaMemcpyHostToDevice, s->stream), "write");
            break;
        case V2M_ARR_HN: {
            exact(4LL * n);
            float* t = (float*)staged(4LL * n);
            launch_set_hn(s->stream, d, I.nofs, n, t);
            break;
        }
        case V2M_ARR_V: {
            exact(12LL * n);
            float* t = (float*)staged(12LL * n);
            launch_float3_to4(s->stream, t, I.nofs, n, d.Vel);
            break;
        }
        default: throw ArgError("array not writable");
        }
        if (tmp) {
            ck(cudaFreeAsync(tmp, s->stream), "cudaFreeAsync");
        }
        ck(cudaGetLastError(), "launch");
        ck(cudaStreamSynchronize(s->stream), "synchronize");
    });
}

int v2m_session_write_lists(v2m_session* s, int vol, const int32_t* nbr, const int32_t* nnb) {
    return guard([&] {
        if (vol < 0 || vol >= s->nvol || !nbr || !nnb) {
            throw ArgError("bad argument");
        }
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        const VolInfo& I = s->info[vol];
        const int n = I.n;
        for (int i = 0; i < n; ++i) {
            if (nnb[i] < 0 || nnb[i] > V2M_K) {
                throw ArgError("list length out of range");
            }
            for (int k = 0; k < nnb[i]; ++k) {
                const int j = nbr[(size_t)i * V2M_K + k];
                if (j < 0 || j >= n) {
                    throw ArgError("neighbour id out of range");
                }
            }
        }
        int* t = nullptr;
        ck(pool_malloc((void**)&t, 4 * ((size_t)n * V2M_K + n) + 16, s->stream), "cudaMallocAsync");
        ck(cudaMemcpyAsync(t, nbr, 4 * (size_t)n * V2M_K, cudaMemcpyHostToDevice, s->stream), "write");
        ck(cudaMemcpyAsync(t + (size_t)n * V2M_K, nnb, 4 * (size_t)n, cudaMemcpyHostToDevice, s->stream), "write");
        launch_lists_from_rowmajor(s->stream, s->d, I.nofs, n, t, t + (size_t)n * V2M_K);
        ck(cudaFreeAsync(t, s->stream), "cudaFreeAsync");
        ck(cudaGetLastError(), "launch");
        ck(cudaStreamSynchronize(s->stream), "synchronize");
    });
}

}  // extern "C"

// ---- autotuner ---------------------------------------------------------------------
// Launch shapes that cannot change a result: the force kernel's block (one node
// per thread, a pure function of the state) and the list kernel's warps per
// block (one node per warp). The move block is not tuned: it fixes the shape of
// the FIRE power's summation tree. Each candidate is timed with CUDA events on
// the session's own lists; the choice is cached per (device, node-count octave,
// volume count) in V2M_CUDA_TUNE_CACHE (default $HOME/.cache/v2m_cuda_tune.txt).
namespace {

std::string tune_key(v2m_session* s) {
    cudaDeviceProp p;
    cudaGetDeviceProperties(&p, s->device);
    int oct = 0;
    while ((int64_t(1) << (oct + 1)) <= s->d.N) {
        ++oct;
    }
    std::string name = p.name;
    for (char& c : name) {
        if (c == ' ') {
            c = '_';
        }
    }
    return name + "|n2^" + std::to_string(oct) + "|v" + std::to_string(s->nvol);
}

std::string tune_path() {
    if (const char* e = std::getenv("V2M_CUDA_TUNE_CACHE")) {
        return e;
    }
    const char* home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/v2m_cuda_tune.txt";
}

bool tune_lookup(v2m_session* s) {
    FILE* f = std::fopen(tune_path().c_str(), "r");
    if (!f) {
        return false;
    }
    char key[512];
    int ft = 0, nt = 0;
    bool hit = false;
    const std::string want = tune_key(s);
    while (std::fscanf(f, "%511s %d %d", key, &ft, &nt) == 3) {
        // (entries with shapes outside the kernels' launch bounds are ignored)
        if (want == key && (ft == 64 || ft == 128 || ft == 256) && (nt == 64 || nt == 128 || nt == 256)) {
            s->force_threads = ft;
            s->nbr_threads = nt;
            hit = true;
        }
    }
    std::fclose(f);
    return hit;
}

void tune_store(v2m_session* s) {
    const std::string path = tune_path();
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) {
        std::string dir = path.substr(0, slash);
        mkdir_p(dir);
    }
    FILE* f = std::fopen(path.c_str(), "a");
    if (f) {
        std::fprintf(f, "%s %d %d\n", tune_key(s).c_str(), s->force_threads, s->nbr_threads);
        std::fclose(f);
    }
}

float time_launches(v2m_session* s, int reps, const std::function<void()>& launch) {
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    launch();   // warm
    ck(cudaEventRecord(e0, s->stream), "event");
    for (int r = 0; r < reps; ++r) {
        launch();
    }
    ck(cudaEventRecord(e1, s->stream), "event");
    ck(cudaEventSynchronize(e1), "event sync");
    float ms = 0.0f;
    ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ck(cudaGetLastError(), "launch");
    return ms / reps;
}

std::string do_autotune(v2m_session* s, int reps) {
    do_reset(s);
    do_rebuild(s);
    std::string rep;
    float best = 1e30f;
    int bf = s->force_threads;
    for (int t : { 64, 128, 256 }) {   // k_force's launch bound is 256
        const float ms = time_launches(s, reps, [&] { launch_force(s->stream, s->d, t); });
        rep += "force " + std::to_string(t) + " " + std::to_string(ms) + " ms\n";
        if (ms < best) {
            best = ms;
            bf = t;
        }
    }
    launch_set_rebuild(s->stream, s->d, 1);
    best = 1e30f;
    int bn = s->nbr_threads;
    for (int t : { 64, 128, 256 }) {
        const float ms = time_launches(s, reps, [&] { launch_neighbors(s->stream, s->d, t); });
        rep += "neighbors " + std::to_string(t) + " " + std::to_string(ms) + " ms\n";
        if (ms < best) {
            best = ms;
            bn = t;
        }
    }
    s->force_threads = bf;
    s->nbr_threads = bn;
    if (s->gexec) {   // the graph holds the old shapes
        cudaGraphExecDestroy(s->gexec);
        s->gexec = nullptr;
    }
    do_reset(s);
    rep += "chosen force " + std::to_string(bf) + " neighbors " + std::to_string(bn) + "\n";
    return rep;
}

}  // namespace

extern "C" {

int v2m_session_autotune(v2m_session* s, int reps, char* report, int64_t report_len) {
    return guard([&] {
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        const std::string r = do_autotune(s, reps > 0 ? reps : 20);
        tune_store(s);
        if (report && report_len > 0) {
            std::snprintf(report, (size_t)report_len, "%s", r.c_str());
        }
    });
}

int v2m_session_shapes(v2m_session* s, int32_t* force_threads, int32_t* nbr_threads) {
    return guard([&] {
        if (force_threads) {
            *force_threads = s->force_threads;
        }
        if (nbr_threads) {
            *nbr_threads = s->nbr_threads;
        }
    });
}

// Per-stage device time over `iters` iterations run as plain launches with
// CUDA events between the stages: ms[0] force, [1] move (pre + main),
// [2] control + refresh, [3] rebuild stages (keys, scan, scatter, in-bin order,
// lists; no-ops unless a volume rebuilds), [4] whole iterations.
int v2m_session_profile_stages(v2m_session* s, int iters, double* ms) {
    return guard([&] {
        if (iters < 1 || !ms) {
            throw ArgError("bad argument");
        }
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        cudaEvent_t ev[6];
        for (auto& e : ev) {
            ck(cudaEventCreate(&e), "event");
        }
        for (int k = 0; k < 5; ++k) {
            ms[k] = 0.0;
        }
        const Dev& d = s->d;
        for (int it = 0; it < iters; ++it) {
            ck(cudaEventRecord(ev[0], s->stream), "event");
            launch_force(s->stream, d, s->force_threads);
            ck(cudaEventRecord(ev[1], s->stream), "event");
            launch_move(s->stream, d);
            ck(cudaEventRecord(ev[2], s->stream), "event");
            launch_control(s->stream, d, s->serial_power);
            launch_refresh(s->stream, d, s->refresh_blocks);
            ck(cudaEventRecord(ev[3], s->stream), "event");
            enqueue_rebuild(s);
            ck(cudaEventRecord(ev[4], s->stream), "event");
            ck(cudaEventSynchronize(ev[4]), "event sync");
            for (int k = 0; k < 4; ++k) {
                float t = 0.0f;
                ck(cudaEventElapsedTime(&t, ev[k], ev[k + 1]), "elapsed");
                ms[k] += t;
            }
            float t = 0.0f;
            ck(cudaEventElapsedTime(&t, ev[0], ev[4]), "elapsed");
            ms[4] += t;
        }
        for (auto& e : ev) {
            cudaEventDestroy(e);
        }
        check_kernel_error(s);
    });
}

int v2m_session_queue_sizes(v2m_session* s, int32_t* trapped, int32_t* interior) {
    return guard([&] {
        Global g;
        ck(cudaMemcpyAsync(&g, s->d.G, sizeof(Global), cudaMemcpyDeviceToHost, s->stream), "read");
        ck(cudaStreamSynchronize(s->stream), "synchronize");
        if (trapped) {
            *trapped = g.qtrap_last;
        }
        if (interior) {
            *interior = g.qint_last;
        }
    });
}

int v2m_session_timed_runs(v2m_session* s, int runs, int graph, int time_force, float* ms) {
    return guard([&] {
        if (runs < 1 || !ms) {
            throw ArgError("bad argument");
        }
        ck(cudaSetDevice(s->device), "cudaSetDevice");
        s->time_force = time_force;
        cudaEvent_t e0, e1;
        ck(cudaEventCreate(&e0), "event");
        ck(cudaEventCreate(&e1), "event");
        ck(cudaStreamSynchronize(s->stream), "synchronize");
        ck(cudaEventRecord(e0, s->stream), "event");
        for (int r = 0; r < runs; ++r) {
            do_reset(s);
            do_rebuild(s);
            do_iterate(s, s->max_iters, graph);
        }
        ck(cudaEventRecord(e1, s->stream), "event");
        ck(cudaEventSynchronize(e1), "event sync");
        ck(cudaEventElapsedTime(ms, e0, e1), "elapsed");
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    });
}

int v2m_session_clear_counters(v2m_session* s) {
    return guard([&] {
        s->launches = 0;
        s->force_launches = 0;
        s->force_ms = 0.0;
    });
}

int v2m_seed_cuda(const v2m_grid_view* g, const v2m_relax_params* prm, int device, v2m_seed_result** out,
                  int64_t* n) {
    Trace trace("v2m_seed_cuda");
    return guard([&] {
        if (!out || !n) {
            throw ArgError("null argument");
        }
        *out = nullptr;
        *n = 0;
        v2m_nodes_view none{};
        validate(g, prm, &none);
        check_seed_args(g, prm);
        const int dev = pick_device(device);
        v2m_session tmp;   // (an allocation context: the grid's device copy)
        tmp.device = dev;
        ck(cudaStreamCreateWithFlags(&tmp.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        SeedBuffers B;
        seed_on(tmp, g, prm, dev, B);
        std::unique_ptr<v2m_seed_result> r(new v2m_seed_result());
        try {
            seeds_to_host(B, tmp.stream, *r);
        } catch (...) {
            release_seeds(B, tmp.stream);
            throw;
        }
        release_seeds(B, tmp.stream);
        *n = (int64_t)r->lab.size();
        *out = r.release();
    });
}

int v2m_seed_copy(const v2m_seed_result* r, float* P, uint16_t* lab, uint8_t* typ, uint16_t* part, uint16_t* part3) {
    return guard([&] {
        if (!r) {
            throw ArgError("null argument");
        }
        const size_t m = r->lab.size();
        if (m && (!P || !lab || !typ || !part)) {
            throw ArgError("null output array");
        }
        if (m) {
            std::memcpy(P, r->P.data(), 12 * m);
            std::memcpy(lab, r->lab.data(), 2 * m);
            std::memcpy(typ, r->typ.data(), m);
            std::memcpy(part, r->part.data(), 4 * m);
            if (part3) {
                std::memcpy(part3, r->part3.data(), 2 * m);
            }
        }
    });
}

void v2m_seed_free(v2m_seed_result* r) {
    delete r;
}

void v2m_grid_params_default(v2m_grid_params* p) {
    std::memset(p, 0, sizeof(*p));
    const GridParamsH d;
    p->sigma = d.sigma;
    p->sigma_thin = d.sigma_thin;
    p->thin_lo = d.thin_lo;
    p->thin_hi = d.thin_hi;
    p->thick = d.thick;
    p->thin_floor = d.thin_floor;
    p->preserve = d.preserve;
    p->sigma_curv = d.sigma_curv;
    p->hbase = d.hbase;
    p->hmin = d.hmin;
    p->hmax = d.hmax;
    p->K = d.K;
    p->g = d.g;
}

int v2m_grid_build_cuda(const uint16_t* L, int32_t nx, int32_t ny, int32_t nz, const float* vs,
                        const v2m_grid_params* p, int device, v2m_grid_result** out) {
    Trace trace("v2m_grid_build_cuda");
    return guard([&] {
        if (!out) {
            throw ArgError("null argument");
        }
        *out = nullptr;
        GridBuildArgs A = grid_args(L, nx, ny, nz, vs, p);
        const int dev = pick_device(device);
        A.device = dev;
        cudaStream_t st = nullptr;
        ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
        A.stream = st;
        StageClock clock("grid build:");
        clock.stream = st;
        A.lap = [&](const char* w) { clock.lap(w); };
        GridBuildOut O;
        std::string err;
        auto release = [&] {
            for (void* x : O.tmp) {
                cudaFreeAsync(x, st);
            }
            O.tmp.clear();
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        };
        const cudaError_t e = grid_build(A, O, err);
        if (e != cudaSuccess) {
            release();
            cudaGetLastError();
            throw CudaError(std::string("grid build: ") + cudaGetErrorString(e));
        }
        std::unique_ptr<v2m_grid_result> r(new v2m_grid_result());
        const size_t nv = (size_t)nx * ny * nz;
        const size_t nb = (size_t)((nx + 7) / 8) * ((ny + 7) / 8) * ((nz + 7) / 8);
        r->nx = nx;
        r->ny = ny;
        r->nz = nz;
        r->vs[0] = vs[0];
        r->vs[1] = vs[1];
        r->vs[2] = vs[2];
        r->L.resize(nv);
        parallel_copy(r->L.data(), L, 2 * nv);
        r->bl_cnt.resize(nb);
        r->bl_lab.resize(nb * V2M_BL);
        r->bl_slot.resize(nb);
        r->phi.resize((size_t)O.nslots * V2M_SLOT);
        r->h.resize(nv);
        r->grade.resize(nv);
        auto d2h = [&](void* dst, const void* src, size_t bytes) {
            if (bytes) {
                ck(staged_d2h(dst, src, bytes, st), "grid read-back");
            }
        };
        try {
            d2h(r->bl_cnt.data(), O.bl_cnt, 4 * nb);
            d2h(r->bl_lab.data(), O.bl_lab, 2 * nb * V2M_BL);
            d2h(r->bl_slot.data(), O.bl_slot, 4 * nb);
            d2h(r->phi.data(), O.phi, 4 * r->phi.size());
            d2h(r->h.data(), O.h, 4 * nv);
            d2h(r->grade.data(), O.grade, nv);
            ck(cudaStreamSynchronize(st), "synchronize");
            clock.lap("read-back");
        } catch (...) {
            release();
            throw;
        }
        release();
        r->nslots = O.nslots;
        r->hbase = O.hbase;
        r->hmin = O.hmin;
        r->hmax = O.hmax;
        r->R = O.R;
        r->limit_sweeps = O.limit_sweeps;
        *out = r.release();
    });
}

int v2m_points_cuda(const uint16_t* L, int32_t nx, int32_t ny, int32_t nz, const float* vs, const v2m_grid_params* gp,
                    const v2m_relax_params* prm, int device, v2m_seed_result** out, int64_t* n, v2m_relax_stats* st) {
    Trace trace("v2m_points_cuda");
    v2m_session* s = nullptr;
    v2m_session tmp;   // (the allocation context of the grid build and the seeding)
    GridBuildOut O;
    SeedBuffers B;
    const int rc = guard([&] {
        if (!out || !n || !prm) {
            throw ArgError("null argument");
        }
        *out = nullptr;
        *n = 0;
        GridBuildArgs A = grid_args(L, nx, ny, nz, vs, gp);
        const int dev = pick_device(device);
        tmp.device = dev;
        ck(cudaStreamCreateWithFlags(&tmp.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        A.device = dev;
        A.stream = tmp.stream;
        std::string err;
        const cudaError_t e = grid_build(A, O, err);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw CudaError(std::string("grid build: ") + cudaGetErrorString(e));
        }
        // the stages hand their device arrays on: grid -> seeds -> session
        const v2m_grid_view gv = device_view(A, O);
        v2m_nodes_view none{};
        validate(&gv, prm, &none);
        seed_on(tmp, &gv, prm, dev, B);
        ck(cudaStreamSynchronize(tmp.stream), "synchronize");   // (the session reads them on its own stream)
        v2m_nodes_view nv{};
        nv.n = B.n;
        nv.P = B.P;
        nv.lab = B.lab;
        nv.typ = B.typ;
        nv.part = B.part;
        s = create(1, &gv, prm, &nv, dev);
        do_rebuild(s);
        do_iterate(s, s->max_iters, env_int("V2M_CUDA_GRAPH", 1));
        std::unique_ptr<v2m_seed_result> r(new v2m_seed_result());
        seeds_to_host(B, tmp.stream, *r);   // (lab and part3 stay the seeds')
        v2m_nodes_view hv{};
        hv.n = B.n;
        hv.P = r->P.data();
        hv.lab = r->lab.data();
        hv.typ = r->typ.data();
        hv.part = r->part.data();
        read_nodes(s, 0, &hv);
        if (st) {
            fill_stats(s, 0, st);
        }
        *n = B.n;
        *out = r.release();
    });
    const std::string keep = g_err;
    if (s) {
        cudaStreamSynchronize(s->stream);
        delete s;
    }
    if (tmp.stream) {
        release_seeds(B, tmp.stream);
        for (void* x : O.tmp) {
            cudaFreeAsync(x, tmp.stream);
        }
        O.tmp.clear();
        cudaStreamSynchronize(tmp.stream);
    }
    g_err = keep;
    return rc;
}

int v2m_grid_result_view(const v2m_grid_result* r, v2m_grid_view* g) {
    return guard([&] {
        if (!r || !g) {
            throw ArgError("null argument");
        }
        std::memset(g, 0, sizeof(*g));
        g->nx = r->nx;
        g->ny = r->ny;
        g->nz = r->nz;
        g->nbx = (r->nx + 7) / 8;
        g->nby = (r->ny + 7) / 8;
        g->nbz = (r->nz + 7) / 8;
        g->vs[0] = r->vs[0];
        g->vs[1] = r->vs[1];
        g->vs[2] = r->vs[2];
        g->L = r->L.data();
        g->bl_cnt = r->bl_cnt.data();
        g->bl_lab = r->bl_lab.data();
        g->bl_slot = r->bl_slot.data();
        g->phi = r->phi.data();
        g->nslots = r->nslots;
        g->h = r->h.data();
        g->hmin = r->hmin;
        g->hmax = r->hmax;
        g->gm = 0;
        g->grade = r->grade.data();
    });
}

int v2m_grid_result_info(const v2m_grid_result* r, float* hbase, int32_t* R, int64_t* nslots, int32_t* limit_sweeps) {
    return guard([&] {
        if (!r) {
            throw ArgError("null argument");
        }
        if (hbase) {
            *hbase = r->hbase;
        }
        if (R) {
            *R = r->R;
        }
        if (nslots) {
            *nslots = r->nslots;
        }
        if (limit_sweeps) {
            *limit_sweeps = r->limit_sweeps;
        }
    });
}

void v2m_grid_free(v2m_grid_result* r) {
    delete r;
}

int v2m_validate_lists(int64_t n, const int32_t* nbr, const int32_t* nnb, const float* pi, const float* pj,
                       char* report, int64_t report_len) {
    std::string msg;
    const int rc = guard([&] {
        if (n < 0 || (n > 0 && (!nbr || !nnb || !pi || !pj))) {
            throw ArgError("v2m_validate_lists: null array");
        }
        auto fail = [&](int64_t i, int k, const std::string& what) {
            msg = "node " + std::to_string(i) + (k >= 0 ? ", entry " + std::to_string(k) : "") + ": " + what;
            throw KernelError("truss lists invalid: " + msg);
        };
        for (int64_t i = 0; i < n; ++i) {
            const int c = nnb[i];
            if (c < 0 || c > V2M_K) {
                fail(i, -1, "length " + std::to_string(c) + " outside [0, " + std::to_string(V2M_K) + "]");
            }
            const float px = pi[3 * i], py = pi[3 * i + 1], pz = pi[3 * i + 2];
            float dprev = 0.0f;
            int jprev = -1;
            for (int k = 0; k < c; ++k) {
                const int j = nbr[i * V2M_K + k];
                if (j < 0 || j >= n) {
                    fail(i, k, "id " + std::to_string(j) + " outside [0, n)");
                }
                if (j == i) {
                    fail(i, k, "self-edge");
                }
                for (int q = 0; q < k; ++q) {
                    if (nbr[i * V2M_K + q] == j) {
                        fail(i, k, "id " + std::to_string(j) + " repeated");
                    }
                }
                // the distance as v2m_neighbors computes it (src/opencl/v2m_particle_body.cl:104-123)
                const float ex = pj[3 * (int64_t)j] - px, ey = pj[3 * (int64_t)j + 1] - py,
                            ez = pj[3 * (int64_t)j + 2] - pz;
                const float d = std::sqrt(ex * ex + ey * ey + ez * ez);
                if (k > 0 && !(dprev < d || (dprev == d && jprev < j))) {
                    fail(i, k, "not after the previous entry in (distance, id) order");
                }
                dprev = d;
                jprev = j;
            }
        }
    });
    if (report && report_len > 0) {
        std::snprintf(report, (size_t)report_len, "%s", rc == V2M_OK ? "" : g_err.c_str());
    }
    return rc;
}

int v2m_relax_cuda(const v2m_grid_view* g, const v2m_relax_params* prm, v2m_nodes_view* nd, v2m_relax_stats* st,
                   int device) {
    return v2m_relax_cuda_batch(1, g, prm, nd, st, device);
}

int v2m_relax_cuda_batch(int nvol, const v2m_grid_view* g, const v2m_relax_params* prm, v2m_nodes_view* nd,
                         v2m_relax_stats* st, int device) {
    Trace trace("v2m_relax_cuda_batch");
    v2m_session* s = nullptr;
    StageClock clock("relax_cl:");
    g_clock = &clock;
    const int rc = guard([&] {
        s = create(nvol, g, prm, nd, device);
        do_rebuild(s);
        lap("first list build");
        do_iterate(s, s->max_iters, env_int("V2M_CUDA_GRAPH", 1));
        lap("loop");
        for (int v = 0; v < nvol; ++v) {
            read_nodes(s, v, nd + v);
            if (st) {
                fill_stats(s, v, st + v);
            }
        }
        lap("read-back");
    });
    if (s) {
        const std::string keep = g_err;
        cudaStreamSynchronize(s->stream);
        delete s;
        g_err = keep;
        clock.stream = nullptr;
        lap("release");
    }
    g_clock = nullptr;
    return rc;
}

}  // extern "C"
