// Batched 2D scenes: C ABI (include/mpm/mpm.h, mpm_batch_*), class assignment
// by cluster size, CUDA-graph capture of the per-class persistent launches,
// and the autotuner. Kernels: mpm_batch.cuh.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "mpm/mpm.h"
#include "mpm_batch.cuh"
#include "mpm_host.h"

using namespace mpm;

namespace {

constexpr int kClusterSizes[4] = {1, 2, 4, 8};

struct BatchClass {
    int cl = 0;        // CTAs per cluster
    int cap = 0;       // nodes per accumulator array per CTA
    int count = 0;     // scenes
    int first = 0;     // offset into the order array
    int clusters = 0;  // persistent clusters launched
};

}  // namespace

struct mpm_batch {
    int device = 0;
    int nscenes = 0;
    long long N = 0;
    std::vector<long long> p0;
    std::vector<int> counts;
    std::vector<BatchScene> scenes;  // host copy (cl, rows follow the configuration)
    BatchBuffers buf[2] = {};
    BatchScene* d_scenes = nullptr;
    BatchSceneState* d_state = nullptr;
    int* d_order = nullptr;
    int* d_queue = nullptr;
    int* d_needs_affine = nullptr;
    unsigned* d_status = nullptr;
    unsigned long long* d_stamps = nullptr;
    size_t stamps_cap = 0;
    int last_steps = 0;
    cudaStream_t stream = nullptr, own_stream = nullptr;
    cudaStream_t aux[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[4] = {nullptr, nullptr, nullptr, nullptr};
    mpm_batch_config cfg{};
    BatchClass cls[4];
    int smem_max = 0;  // dynamic shared memory opt-in per CTA, bytes
    int cap_max = 0;   // nodes per accumulator array that fit in it
    cudaGraphExec_t graph = nullptr;
    int graph_steps = -1;
    bool use_graphs = true;
    std::string err;
};

namespace {

mpm_status bfail(mpm_batch* b, mpm_status code, const std::string& what) {
    if (b) b->err = what;
    return code;
}

#define BATCH_CUDA(b, call)                                                                                \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) {                                                                           \
            cudaGetLastError();                                                                            \
            return bfail((b), e_ == cudaErrorMemoryAllocation ? MPM_ERR_OUT_OF_MEMORY : MPM_ERR_CUDA,      \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                              \
        }                                                                                                  \
    } while (0)

template <typename T> cudaError_t balloc(T** p, size_t count) {
    *p = nullptr;
    return cudaMalloc(reinterpret_cast<void**>(p), (count ? count : 1) * sizeof(T));
}

void drop_graph(mpm_batch* b) {
    if (b->graph) {
        cudaStreamSynchronize(b->stream);
        cudaGraphExecDestroy(b->graph);
    }
    b->graph = nullptr;
    b->graph_steps = -1;
}

void release(mpm_batch* b) {
    drop_graph(b);
    for (BatchBuffers& f : b->buf) {
        float* fl[] = {f.x, f.v, f.B, f.Fe, f.Jp, f.A, f.mass, f.vol};
        for (float* p : fl)
            if (p) cudaFree(p);
        if (f.id) cudaFree(f.id);
    }
    if (b->d_scenes) cudaFree(b->d_scenes);
    if (b->d_state) cudaFree(b->d_state);
    if (b->d_order) cudaFree(b->d_order);
    if (b->d_queue) cudaFree(b->d_queue);
    if (b->d_needs_affine) cudaFree(b->d_needs_affine);
    if (b->d_status) cudaFree(b->d_status);
    if (b->d_stamps) cudaFree(b->d_stamps);
    for (int c = 0; c < 4; ++c) {
        if (b->aux[c]) cudaStreamDestroy(b->aux[c]);
        if (b->join[c]) cudaEventDestroy(b->join[c]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
}

using BatchKernel = void (*)(BatchParticles, BatchRun);

BatchKernel kernel_for(int threads) {
    return threads == 1024 ? k_batch_run<1024> : threads == 512 ? k_batch_run<512> : k_batch_run<256>;
}

BatchParticles particles(const mpm_batch* b) { return BatchParticles{{b->buf[0], b->buf[1]}, b->N}; }

// Where each scene's particles are now (buffer parity) and their slot order.
mpm_status scene_states(mpm_batch* b, std::vector<BatchSceneState>& st) {
    st.resize(b->nscenes);
    BATCH_CUDA(b, cudaMemcpyAsync(st.data(), b->d_state, sizeof(BatchSceneState) * st.size(), cudaMemcpyDeviceToHost,
                                  b->stream));
    BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
    return MPM_OK;
}

// Forget every scene's bands (they belong to a cluster size): the next step
// of each multi-CTA scene starts with a sort.
mpm_status invalidate_bands(mpm_batch* b) {
    std::vector<BatchSceneState> st;
    mpm_status r = scene_states(b, st);
    if (r != MPM_OK) return r;
    for (auto& x : st) x.sorted = 0;
    BATCH_CUDA(b, cudaMemcpy(b->d_state, st.data(), sizeof(BatchSceneState) * st.size(), cudaMemcpyHostToDevice));
    return MPM_OK;
}

cudaLaunchConfig_t launch_config(const mpm_batch* b, const BatchClass& k, cudaLaunchAttribute* attr, int clusters) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)(clusters * k.cl));
    lc.blockDim = dim3((unsigned)b->cfg.threads);
    lc.dynamicSmemBytes = (size_t)kBatchAccs * sizeof(unsigned long long) * (size_t)k.cap;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)k.cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return lc;
}

// Cluster size and node band of every scene under b->cfg; scenes grouped by
// cluster size, most particles per CTA first; persistent cluster counts.
mpm_status configure(mpm_batch* b, const mpm_batch_config& cfg) {
    if (cfg.threads != 256 && cfg.threads != 512 && cfg.threads != 1024)
        return bfail(b, MPM_ERR_INVALID_ARGUMENT, "threads must be 256, 512 or 1024");
    if (cfg.max_cluster != 1 && cfg.max_cluster != 2 && cfg.max_cluster != 4 && cfg.max_cluster != 8)
        return bfail(b, MPM_ERR_INVALID_ARGUMENT, "max_cluster must be 1, 2, 4 or 8");
    if (cfg.particles_per_cta < 0) return bfail(b, MPM_ERR_INVALID_ARGUMENT, "particles_per_cta must be >= 0");
    if (cfg.sort_period < 0) return bfail(b, MPM_ERR_INVALID_ARGUMENT, "sort_period must be >= 0");
    std::vector<BatchScene> sc = b->scenes;
    std::vector<std::vector<int>> members(4);
    for (int s = 0; s < b->nscenes; ++s) {
        const int nx = sc[s].C.nx, ny = sc[s].C.ny;
        int ci = -1;
        for (int c = 0; c < 4 && kClusterSizes[c] <= cfg.max_cluster; ++c) {
            const long long rows = (ny + kClusterSizes[c] - 1) / kClusterSizes[c];
            if (rows * nx <= b->cap_max) { ci = c; break; }
        }
        if (ci < 0)
            return bfail(b, MPM_ERR_CAPACITY,
                         "scene " + std::to_string(s) + ": its grid of " + std::to_string((long long)nx * ny) +
                             " nodes does not fit in the shared memory of a cluster of " +
                             std::to_string(cfg.max_cluster) + " CTAs");
        if (cfg.particles_per_cta > 0)
            while (ci < 3 && kClusterSizes[ci + 1] <= cfg.max_cluster &&
                   (long long)sc[s].n > (long long)cfg.particles_per_cta * kClusterSizes[ci])
                ++ci;
        sc[s].cl = kClusterSizes[ci];
        // a multi-CTA scene may give any CTA up to its full capacity in rows
        sc[s].rows = sc[s].cl == 1 ? ny : b->cap_max / nx;
        if (sc[s].n > 0) members[ci].push_back(s);
    }
    std::vector<int> order;
    BatchClass cls[4];
    for (int c = 0; c < 4; ++c) {
        std::sort(members[c].begin(), members[c].end(), [&](int a, int d) {
            const long long wa = (long long)sc[a].n + (long long)sc[a].C.nodes;
            const long long wd = (long long)sc[d].n + (long long)sc[d].C.nodes;
            return wa != wd ? wa > wd : a < d;
        });
        cls[c].cl = kClusterSizes[c];
        cls[c].first = (int)order.size();
        cls[c].count = (int)members[c].size();
        for (int s : members[c]) {
            cls[c].cap = std::max(cls[c].cap, sc[s].rows * sc[s].C.nx);
            order.push_back(s);
        }
        if (cls[c].cl > 1 && cls[c].count > 0) cls[c].cap = b->cap_max;
    }
    // Shared-memory opt-in and persistent cluster counts.
    b->cfg = cfg;
    BatchKernel kern = kernel_for(cfg.threads);
    BATCH_CUDA(b, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, b->smem_max));
    BATCH_CUDA(b, cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 0));
    for (int c = 0; c < 4; ++c) {
        if (cls[c].count == 0) continue;
        cudaLaunchAttribute attr[1];
        cudaLaunchConfig_t lc = launch_config(b, cls[c], attr, 1);
        int active = 0;
        BATCH_CUDA(b, cudaOccupancyMaxActiveClusters(&active, kern, &lc));
        if (active < 1)
            return bfail(b, MPM_ERR_UNSUPPORTED,
                         "a cluster of " + std::to_string(cls[c].cl) + " CTAs x " + std::to_string(cfg.threads) +
                             " threads cannot be resident on this device");
        cls[c].clusters = std::min(cls[c].count, active);
    }
    drop_graph(b);
    b->scenes = sc;
    for (int c = 0; c < 4; ++c) b->cls[c] = cls[c];
    BATCH_CUDA(b, cudaMemcpy(b->d_scenes, sc.data(), sizeof(BatchScene) * sc.size(), cudaMemcpyHostToDevice));
    if (!order.empty())
        BATCH_CUDA(b, cudaMemcpy(b->d_order, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice));
    // bands of the old cluster sizes are void: each scene re-sorts on its next step
    return invalidate_bands(b);
}

// Enqueue one call: zero the queues, then every class's persistent launch on
// its own stream (fork / join around the batch's stream).
cudaError_t enqueue(mpm_batch* b, int nsteps) {
    cudaError_t e = cudaMemsetAsync(b->d_queue, 0, sizeof(int) * 4, b->stream);
    if (e != cudaSuccess) return e;
    if ((e = cudaEventRecord(b->fork, b->stream)) != cudaSuccess) return e;
    const BatchParticles P = particles(b);
    BatchKernel kern = kernel_for(b->cfg.threads);
    for (int c = 0; c < 4; ++c) {
        const BatchClass& k = b->cls[c];
        if (k.count == 0) continue;
        if ((e = cudaStreamWaitEvent(b->aux[c], b->fork, 0)) != cudaSuccess) return e;
        BatchRun R{b->d_scenes, b->d_state, b->d_order + k.first, k.count, k.cap, b->d_queue + c,
                   b->d_needs_affine, b->d_status, b->d_stamps, nsteps,
                   b->cfg.sort_period > 0 ? b->cfg.sort_period : 16};
        cudaLaunchAttribute attr[1];
        cudaLaunchConfig_t lc = launch_config(b, k, attr, k.clusters);
        lc.stream = b->aux[c];
        if ((e = cudaLaunchKernelEx(&lc, kern, P, R)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(b->join[c], b->aux[c])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(b->stream, b->join[c], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Scene slice of one field in creation order (slots hold particles id[slot]).
mpm_status copy_slice_out(mpm_batch* b, int field, int comps, int scene, float* host) {
    const int n = b->counts[scene];
    if (n == 0) return MPM_OK;
    std::vector<BatchSceneState> st;
    mpm_status r = scene_states(b, st);
    if (r != MPM_OK) return r;
    const BatchBuffers& F = b->buf[st[scene].parity & 1];
    const float* soa[] = {F.x, F.v, F.B, F.Fe, F.Jp};
    std::vector<float> tmp((size_t)n * comps);
    std::vector<int> id(n);
    for (int c = 0; c < comps; ++c)
        BATCH_CUDA(b, cudaMemcpyAsync(tmp.data() + (size_t)c * n, soa[field] + (size_t)c * b->N + b->p0[scene],
                                      sizeof(float) * n, cudaMemcpyDeviceToHost, b->stream));
    BATCH_CUDA(b, cudaMemcpyAsync(id.data(), F.id + b->p0[scene], sizeof(int) * n, cudaMemcpyDeviceToHost, b->stream));
    BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
    for (int j = 0; j < n; ++j) {
        const int i = id[j];
        if (i < 0 || i >= n) return bfail(b, MPM_ERR_CUDA, "corrupt particle order");
        for (int c = 0; c < comps; ++c) host[(size_t)i * comps + c] = tmp[(size_t)c * n + j];
    }
    return MPM_OK;
}

bool valid_scene(const mpm_batch* b, int32_t s) { return b && s >= 0 && s < b->nscenes; }

enum { kFieldX = 0, kFieldV = 1, kFieldB = 2, kFieldFe = 3, kFieldJp = 4 };

}  // namespace

extern "C" {

mpm_status mpm_batch_create(const mpm_params* params, const mpm_particles_init* init, int32_t nscenes,
                            mpm_batch** out) {
    if (!out) return MPM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!params || !init || nscenes < 1) return MPM_ERR_INVALID_ARGUMENT;
    long long N = 0;
    for (int s = 0; s < nscenes; ++s) {
        std::string why;
        mpm_status st = validate_params(&params[s], why);
        if (st != MPM_OK) return st;
        if (params[s].dim != 2 || params[s].formulation != MPM_FORMULATION_MLS) return MPM_ERR_UNSUPPORTED;
        if (params[s].height + 1 > kBatchMaxRows) return MPM_ERR_CAPACITY;
        if (init[s].count < 0 || init[s].count > 0x7fffffff) return MPM_ERR_INVALID_ARGUMENT;
        if (init[s].count > 0 && (!init[s].position || !init[s].volume)) return MPM_ERR_INVALID_ARGUMENT;
        N += init[s].count;
    }
    if (N > 0x7fffffffLL) return MPM_ERR_INVALID_ARGUMENT;
    int ndev = 0, dev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return MPM_ERR_NO_DEVICE; }
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return MPM_ERR_NO_DEVICE; }
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_batch_run<256>) != cudaSuccess) { cudaGetLastError(); return MPM_ERR_NO_DEVICE; }

    mpm_batch* b = new mpm_batch();
    auto bail = [&](mpm_status code) { release(b); delete b; return code; };
    b->device = dev;
    b->nscenes = nscenes;
    b->N = N;
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return bail(MPM_ERR_CUDA);
    b->smem_max = optin - (int)std::max(fa.sharedSizeBytes, (size_t)0) - 1024;
    b->smem_max -= b->smem_max % 256;
    b->cap_max = b->smem_max / (int)(kBatchAccs * sizeof(unsigned long long));

    // Per-scene constants and fixed-point scales, as mpm_create chooses them.
    b->p0.resize(nscenes);
    b->counts.resize(nscenes);
    b->scenes.resize(nscenes);
    std::vector<float> massv((size_t)N), volv((size_t)N);
    long long off = 0;
    for (int s = 0; s < nscenes; ++s) {
        const int n = (int)init[s].count;
        double total_mass = 0.0;
        for (int i = 0; i < n; ++i) {
            const float vol = init[s].volume[i];
            const float m = init[s].mass ? init[s].mass[i] : (vol * params[s].rho) / 100.f;
            if (!std::isfinite(vol) || !std::isfinite(m)) return bail(MPM_ERR_INVALID_ARGUMENT);
            volv[off + i] = vol;
            massv[off + i] = m;
            total_mass += m;
        }
        for (long long i = 0; i < 2LL * n; ++i)
            if (!std::isfinite(init[s].position[i]) || (init[s].velocity && !std::isfinite(init[s].velocity[i])))
                return bail(MPM_ERR_INVALID_ARGUMENT);
        BatchScene& S = b->scenes[s];
        S.C = step_consts(params[s], 2);
        int l2[3];
        fixed_point_scales(params[s], total_mass, S.C, l2);
        S.p0 = off;
        S.n = n;
        b->p0[s] = off;
        b->counts[s] = n;
        off += n;
    }

    if (cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking) != cudaSuccess) return bail(MPM_ERR_CUDA);
    b->stream = b->own_stream;
    for (int c = 0; c < 4; ++c)
        if (cudaStreamCreateWithFlags(&b->aux[c], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->join[c], cudaEventDisableTiming) != cudaSuccess)
            return bail(MPM_ERR_CUDA);
    if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) return bail(MPM_ERR_CUDA);
    const size_t n = (size_t)N;
    bool alloc_ok = true;
    for (BatchBuffers& f : b->buf)
        alloc_ok = alloc_ok && !balloc(&f.x, n * 2) && !balloc(&f.v, n * 2) && !balloc(&f.B, n * 4) &&
                   !balloc(&f.Fe, n * 4) && !balloc(&f.Jp, n) && !balloc(&f.A, n * 4) && !balloc(&f.mass, n) &&
                   !balloc(&f.vol, n) && !balloc(&f.id, n);
    if (!alloc_ok || balloc(&b->d_scenes, (size_t)nscenes) || balloc(&b->d_state, (size_t)nscenes) ||
        balloc(&b->d_order, (size_t)nscenes) || balloc(&b->d_queue, 4) ||
        balloc(&b->d_needs_affine, (size_t)nscenes) || balloc(&b->d_status, (size_t)nscenes)) {
        cudaGetLastError();
        return bail(MPM_ERR_OUT_OF_MEMORY);
    }
    // SoA upload into buffer 0: F_E = I, B = 0, J_p = 1 (Particle ctor,
    // src/cpu/Particles.cpp:7-19); slot order = creation order.
    const BatchBuffers& F = b->buf[0];
    std::vector<float> soa(n * 4, 0.f);
    bool ok = true;
    auto up = [&](float* dst, size_t count) {
        return cudaMemcpy(dst, soa.data(), sizeof(float) * count, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    for (int s = 0; s < nscenes; ++s)
        for (int i = 0; i < b->counts[s]; ++i)
            for (int k = 0; k < 2; ++k) soa[(size_t)k * n + b->p0[s] + i] = init[s].position[(size_t)i * 2 + k];
    ok = ok && up(F.x, n * 2);
    for (int s = 0; s < nscenes; ++s)
        for (int i = 0; i < b->counts[s]; ++i)
            for (int k = 0; k < 2; ++k)
                soa[(size_t)k * n + b->p0[s] + i] = init[s].velocity ? init[s].velocity[(size_t)i * 2 + k] : 0.f;
    ok = ok && up(F.v, n * 2);
    std::fill(soa.begin(), soa.end(), 0.f);
    ok = ok && up(F.B, n * 4) && up(F.A, n * 4);
    for (int k = 0; k < 4; ++k)
        for (size_t i = 0; i < n; ++i) soa[(size_t)k * n + i] = (k % 3 == 0) ? 1.f : 0.f;
    ok = ok && up(F.Fe, n * 4);
    std::fill(soa.begin(), soa.begin() + n, 1.f);
    ok = ok && up(F.Jp, n);
    ok = ok && cudaMemcpy(F.mass, massv.data(), sizeof(float) * n, cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(F.vol, volv.data(), sizeof(float) * n, cudaMemcpyHostToDevice) == cudaSuccess;
    std::vector<int> ids(n);
    for (int s = 0; s < nscenes; ++s)
        for (int i = 0; i < b->counts[s]; ++i) ids[b->p0[s] + i] = i;
    ok = ok && cudaMemcpy(F.id, ids.data(), sizeof(int) * n, cudaMemcpyHostToDevice) == cudaSuccess;
    std::vector<BatchSceneState> st0(nscenes);
    std::memset(st0.data(), 0, sizeof(BatchSceneState) * nscenes);
    ok = ok && cudaMemcpy(b->d_state, st0.data(), sizeof(BatchSceneState) * nscenes, cudaMemcpyHostToDevice) == cudaSuccess;
    std::vector<int> ones(nscenes, 1);
    ok = ok && cudaMemcpy(b->d_needs_affine, ones.data(), sizeof(int) * nscenes, cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemset(b->d_status, 0, sizeof(unsigned) * nscenes) == cudaSuccess;
    if (!ok) { cudaGetLastError(); return bail(MPM_ERR_CUDA); }
    mpm_batch_config cfg{};
    cfg.threads = 512;
    cfg.particles_per_cta = 8192;
    cfg.max_cluster = kBatchMaxCluster;
    cfg.sort_period = 16;
    mpm_status st = configure(b, cfg);
    if (st != MPM_OK) return bail(st);
    *out = b;
    return MPM_OK;
}

mpm_status mpm_batch_destroy(mpm_batch* b) {
    if (!b) return MPM_ERR_INVALID_ARGUMENT;
    if (b->stream) cudaStreamSynchronize(b->stream);
    release(b);
    delete b;
    return MPM_OK;
}

const char* mpm_batch_last_error(const mpm_batch* b) { return b ? b->err.c_str() : "null batch"; }

mpm_status mpm_batch_info(const mpm_batch* b, int32_t* nscenes, int64_t* total) {
    if (!b) return MPM_ERR_INVALID_ARGUMENT;
    if (nscenes) *nscenes = b->nscenes;
    if (total) *total = b->N;
    return MPM_OK;
}

mpm_status mpm_batch_step(mpm_batch* b, int32_t nsteps) {
    if (!b || nsteps < 0) return MPM_ERR_INVALID_ARGUMENT;
    if (nsteps == 0) return MPM_OK;
    const size_t need = (size_t)b->nscenes * (size_t)(nsteps + 1);
    if (need > b->stamps_cap) {
        drop_graph(b);
        BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
        if (b->d_stamps) cudaFree(b->d_stamps);
        b->d_stamps = nullptr;
        b->stamps_cap = 0;
        BATCH_CUDA(b, balloc(&b->d_stamps, need));
        b->stamps_cap = need;
    }
    b->last_steps = nsteps;
    if (b->use_graphs && b->graph_steps != nsteps) {
        drop_graph(b);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t e1 = enqueue(b, nsteps);
            cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
            e = e1 != cudaSuccess ? e1 : e2;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            // fall back to direct launches for the life of the batch
            cudaGetLastError();
            b->graph = nullptr;
            b->use_graphs = false;
        } else {
            b->graph_steps = nsteps;
        }
    }
    if (b->graph) BATCH_CUDA(b, cudaGraphLaunch(b->graph, b->stream));
    else BATCH_CUDA(b, enqueue(b, nsteps));
    return MPM_OK;
}

mpm_status mpm_batch_set_stream(mpm_batch* b, void* stream) {
    if (!b) return MPM_ERR_INVALID_ARGUMENT;
    BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
    drop_graph(b);
    b->stream = stream ? (cudaStream_t)stream : b->own_stream;
    return MPM_OK;
}

mpm_status mpm_batch_get_state(mpm_batch* b, int32_t scene, mpm_state_host* st) {
    if (!valid_scene(b, scene) || !st || st->count != b->counts[scene]) return MPM_ERR_INVALID_ARGUMENT;
    mpm_status r = MPM_OK;
    if (st->position && (r = copy_slice_out(b, kFieldX, 2, scene, st->position)) != MPM_OK) return r;
    if (st->velocity && (r = copy_slice_out(b, kFieldV, 2, scene, st->velocity)) != MPM_OK) return r;
    if (st->affine_b && (r = copy_slice_out(b, kFieldB, 4, scene, st->affine_b)) != MPM_OK) return r;
    if (st->elastic_f && (r = copy_slice_out(b, kFieldFe, 4, scene, st->elastic_f)) != MPM_OK) return r;
    if (st->plastic_det && (r = copy_slice_out(b, kFieldJp, 1, scene, st->plastic_det)) != MPM_OK) return r;
    return MPM_OK;
}

// Writes the scene back in creation order (ids reset), so it re-sorts on its
// next step and re-derives its affine matrices. Fields left NULL keep their
// values.
mpm_status mpm_batch_set_state(mpm_batch* b, int32_t scene, const mpm_state_host* st) {
    if (!valid_scene(b, scene) || !st || st->count != b->counts[scene]) return MPM_ERR_INVALID_ARGUMENT;
    const int n = b->counts[scene];
    auto finite = [&](const float* p, size_t k) {
        if (!p) return true;
        for (size_t i = 0; i < k; ++i)
            if (!std::isfinite(p[i])) return false;
        return true;
    };
    if (!finite(st->position, 2 * (size_t)n) || !finite(st->velocity, 2 * (size_t)n) ||
        !finite(st->affine_b, 4 * (size_t)n) || !finite(st->elastic_f, 4 * (size_t)n) ||
        !finite(st->plastic_det, (size_t)n))
        return bfail(b, MPM_ERR_INVALID_ARGUMENT, "state holds non-finite values");
    if (n == 0) return MPM_OK;
    std::vector<BatchSceneState> ss;
    mpm_status r = scene_states(b, ss);
    if (r != MPM_OK) return r;
    const BatchBuffers& F = b->buf[ss[scene].parity & 1];
    // current contents in creation order, overlaid with what the caller gives
    const int comps[] = {2, 2, 4, 4, 1};
    const float* given[] = {st->position, st->velocity, st->affine_b, st->elastic_f, st->plastic_det};
    float* soa[] = {F.x, F.v, F.B, F.Fe, F.Jp};
    std::vector<int> id(n);
    BATCH_CUDA(b, cudaMemcpyAsync(id.data(), F.id + b->p0[scene], sizeof(int) * n, cudaMemcpyDeviceToHost, b->stream));
    std::vector<float> mass(n), vol(n), ms(n), vs(n);
    BATCH_CUDA(b, cudaMemcpyAsync(ms.data(), F.mass + b->p0[scene], sizeof(float) * n, cudaMemcpyDeviceToHost, b->stream));
    BATCH_CUDA(b, cudaMemcpyAsync(vs.data(), F.vol + b->p0[scene], sizeof(float) * n, cudaMemcpyDeviceToHost, b->stream));
    BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
    for (int j = 0; j < n; ++j) {
        if (id[j] < 0 || id[j] >= n) return bfail(b, MPM_ERR_CUDA, "corrupt particle order");
        mass[id[j]] = ms[j];
        vol[id[j]] = vs[j];
    }
    for (int f = 0; f < 5; ++f) {
        std::vector<float> host((size_t)n * comps[f]);
        if (given[f]) std::memcpy(host.data(), given[f], sizeof(float) * host.size());
        else if ((r = copy_slice_out(b, f, comps[f], scene, host.data())) != MPM_OK) return r;
        std::vector<float> tmp(host.size());
        for (int i = 0; i < n; ++i)
            for (int c = 0; c < comps[f]; ++c) tmp[(size_t)c * n + i] = host[(size_t)i * comps[f] + c];
        for (int c = 0; c < comps[f]; ++c)
            BATCH_CUDA(b, cudaMemcpyAsync(soa[f] + (size_t)c * b->N + b->p0[scene], tmp.data() + (size_t)c * n,
                                          sizeof(float) * n, cudaMemcpyHostToDevice, b->stream));
        BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
    }
    for (int i = 0; i < n; ++i) id[i] = i;
    BATCH_CUDA(b, cudaMemcpy(F.mass + b->p0[scene], mass.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    BATCH_CUDA(b, cudaMemcpy(F.vol + b->p0[scene], vol.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    BATCH_CUDA(b, cudaMemcpy(F.id + b->p0[scene], id.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    ss[scene].sorted = 0;
    ss[scene].step = 0;
    BATCH_CUDA(b, cudaMemcpy(b->d_state + scene, &ss[scene], sizeof(BatchSceneState), cudaMemcpyHostToDevice));
    const int one = 1;
    BATCH_CUDA(b, cudaMemcpy(b->d_needs_affine + scene, &one, sizeof(int), cudaMemcpyHostToDevice));
    return MPM_OK;
}

mpm_status mpm_batch_get_positions(mpm_batch* b, int32_t scene, float* out, size_t cap_floats) {
    if (!valid_scene(b, scene) || (!out && b->counts[scene] > 0)) return MPM_ERR_INVALID_ARGUMENT;
    if (cap_floats < (size_t)b->counts[scene] * 2) return bfail(b, MPM_ERR_CAPACITY, "output buffer too small");
    return copy_slice_out(b, kFieldX, 2, scene, out);
}

mpm_status mpm_batch_get_status(mpm_batch* b, int32_t scene, uint32_t* flags) {
    if (!valid_scene(b, scene) || !flags) return MPM_ERR_INVALID_ARGUMENT;
    unsigned f = 0;
    BATCH_CUDA(b, cudaMemcpyAsync(&f, b->d_status + scene, sizeof(f), cudaMemcpyDeviceToHost, b->stream));
    BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
    *flags = f;
    return MPM_OK;
}

mpm_status mpm_batch_step_times(mpm_batch* b, uint64_t* out, size_t cap, int32_t* nsteps) {
    if (!b || !nsteps) return MPM_ERR_INVALID_ARGUMENT;
    *nsteps = b->last_steps;
    const size_t need = (size_t)b->nscenes * (size_t)(b->last_steps + 1);
    if (b->last_steps == 0) return MPM_OK;
    if (!out || cap < need) return bfail(b, MPM_ERR_CAPACITY, "output buffer too small");
    BATCH_CUDA(b, cudaMemcpyAsync(out, b->d_stamps, sizeof(uint64_t) * need, cudaMemcpyDeviceToHost, b->stream));
    BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
    return MPM_OK;
}

mpm_status mpm_batch_get_config(const mpm_batch* b, mpm_batch_config* cfg) {
    if (!b || !cfg) return MPM_ERR_INVALID_ARGUMENT;
    *cfg = b->cfg;
    return MPM_OK;
}

mpm_status mpm_batch_set_config(mpm_batch* b, const mpm_batch_config* cfg) {
    if (!b || !cfg) return MPM_ERR_INVALID_ARGUMENT;
    BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
    const mpm_batch_config old = b->cfg;
    mpm_status st = configure(b, *cfg);
    if (st != MPM_OK) {
        const std::string why = b->err;
        configure(b, old);
        b->err = why;
    }
    return st;
}

mpm_status mpm_batch_tune(mpm_batch* b, int32_t trial_steps, mpm_batch_config* chosen, double* best_ms) {
    if (!b || trial_steps < 1) return MPM_ERR_INVALID_ARGUMENT;
    BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
    const size_t n = (size_t)b->N;
    // Snapshot of everything a step changes: both particle buffers (a sort
    // moves particles between them), per-scene state, flags.
    struct Span { void* p; size_t bytes; };
    std::vector<Span> spans;
    for (BatchBuffers& f : b->buf) {
        spans.push_back({f.x, sizeof(float) * 2 * n});
        spans.push_back({f.v, sizeof(float) * 2 * n});
        spans.push_back({f.B, sizeof(float) * 4 * n});
        spans.push_back({f.Fe, sizeof(float) * 4 * n});
        spans.push_back({f.Jp, sizeof(float) * n});
        spans.push_back({f.A, sizeof(float) * 4 * n});
        spans.push_back({f.mass, sizeof(float) * n});
        spans.push_back({f.vol, sizeof(float) * n});
        spans.push_back({f.id, sizeof(int) * n});
    }
    spans.push_back({b->d_state, sizeof(BatchSceneState) * (size_t)b->nscenes});
    spans.push_back({b->d_needs_affine, sizeof(int) * (size_t)b->nscenes});
    spans.push_back({b->d_status, sizeof(unsigned) * (size_t)b->nscenes});
    size_t total = 0;
    for (const Span& sp : spans) total += (sp.bytes + 255) / 256 * 256;
    unsigned char* snap = nullptr;
    BATCH_CUDA(b, balloc(&snap, total));
    auto copy_all = [&](bool save) {
        size_t o = 0;
        cudaError_t e = cudaSuccess;
        for (const Span& sp : spans) {
            if (e != cudaSuccess) break;
            e = save ? cudaMemcpyAsync(snap + o, sp.p, sp.bytes, cudaMemcpyDeviceToDevice, b->stream)
                     : cudaMemcpyAsync(sp.p, snap + o, sp.bytes, cudaMemcpyDeviceToDevice, b->stream);
            o += (sp.bytes + 255) / 256 * 256;
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        return e;
    };
    const mpm_batch_config start = b->cfg;
    mpm_batch_config best = start;
    double best_t = 1e300;
    mpm_status st = MPM_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t ce = copy_all(true);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
    const int threads_c[3] = {256, 512, 1024};
    const int ppc_c[4] = {0, 16384, 8192, 4096};
    for (int ti = 0; ti < 3 && ce == cudaSuccess && st == MPM_OK; ++ti)
        for (int pi = 0; pi < 4 && ce == cudaSuccess && st == MPM_OK; ++pi) {
            mpm_batch_config cfg = start;
            cfg.threads = threads_c[ti];
            cfg.particles_per_cta = ppc_c[pi];
            if (configure(b, cfg) != MPM_OK) { b->err.clear(); continue; }  // not resident: skip the candidate
            // one untimed call (graph capture, first-touch), then the timed one
            for (int rep = 0; rep < 2 && ce == cudaSuccess && st == MPM_OK; ++rep) {
                if ((ce = copy_all(false)) != cudaSuccess) break;
                if ((st = invalidate_bands(b)) != MPM_OK) break;
                if ((ce = cudaEventRecord(e0, b->stream)) != cudaSuccess) break;
                st = mpm_batch_step(b, trial_steps);
                if (st != MPM_OK) break;
                if ((ce = cudaEventRecord(e1, b->stream)) != cudaSuccess) break;
                if ((ce = cudaEventSynchronize(e1)) != cudaSuccess) break;
            }
            float ms = 0.f;
            if (ce == cudaSuccess && st == MPM_OK && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms < best_t) {
                best_t = ms;
                best = cfg;
            }
        }
    // put the batch back as it was, whatever happened above
    const cudaError_t ce_restore = copy_all(false);
    if (ce == cudaSuccess) ce = ce_restore;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(snap);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        configure(b, start);
        return bfail(b, MPM_ERR_CUDA, std::string("tuner: ") + cudaGetErrorString(ce));
    }
    if (st != MPM_OK) {
        const std::string why = b->err;
        configure(b, start);
        b->err = why;
        return st;
    }
    st = configure(b, best);
    if (st != MPM_OK) return st;
    if (chosen) *chosen = best;
    if (best_ms) *best_ms = best_t;
    return MPM_OK;
}

}  // extern "C"
