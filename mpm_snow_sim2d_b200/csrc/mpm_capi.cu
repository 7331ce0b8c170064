// C ABI of the B200 MLS-MPM solver (include/mpm/mpm.h): device memory, the
// step sequence, state import/export and checkpoints. The product path has no
// CPU fallback: without a usable sm_100 device every create fails.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <random>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "mpm/mpm.h"
#include "mpm_kernels.cuh"
#include "mpm_tiled.cuh"
#include "mpm_fused.cuh"
#include "mpm_mlp.cuh"
#include "mpm_render.cuh"
#include "mpm_host.h"

using namespace mpm;

struct mpm_mlp {
    int device = 0;
    float* w = nullptr;            // fp32 master parameters
    __nv_bfloat16* wbf = nullptr;  // bf16 copy used by the kernels
    float* grad = nullptr;
    float* m1 = nullptr;
    float* m2 = nullptr;
    float* loss = nullptr;         // per training step
    int loss_cap = 0;
    float* pairs = nullptr;        // device training pairs [n][20]
    long long n_pairs = 0;
    long long step = 0;            // AdamW steps taken
    MlpNorm norm{};
    std::string err;
};

struct mpm_solver {
    mpm_params params{};
    int dim = 2, form = kMLS;
    int stencil = 4;  // nodes per axis: 4 cubic (MLS, CLASSIC), 3 quadratic (QUAD)
    int n = 0;
    long long nodes = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    // particles (SoA)
    float *x = nullptr, *v = nullptr, *B = nullptr, *Fe = nullptr, *Jp = nullptr, *A = nullptr;
    float *mass = nullptr, *vol = nullptr;
    float mass_u = 0.f, vol_u = 0.f;
    int* id = nullptr;
    // grid
    unsigned long long* acc = nullptr;
    float4* gv = nullptr;
    unsigned* status = nullptr;
    float* staging = nullptr;
    size_t staging_floats = 0;
    unsigned long long* render_fb = nullptr;  // per-pixel (depth, intensity) words
    unsigned char* render_rgb = nullptr;
    long long render_pixels = 0;
    int log2_sm = 0, log2_sp = 0, log2_sf = 0;
    long long step = 0;
    StepConsts C{};
    std::string err;
    // tiled MLS path
    bool tiled = false;
    bool needs_sort = true;
    int sort_period = 8;
    // sort_period 0 (auto): each period's length follows from the fastest
    // particle two periods earlier (so the host waits for nothing the GPU has
    // not long passed); a function of the state, so runs stay deterministic.
    bool auto_sort = false;
    int cur_K = 16;              // steps of the current period (auto)
    long long next_sort = 0;     // step of the next sort (auto)
    long long sorts_done = 0;    // sorts launched so far
    long long sorted_at = -1;    // step at whose start the last sort ran (no second sort at that step)
    unsigned* vmax_dev = nullptr;   // two slots: largest |v| component over the particles (float bits)
    unsigned* vmax_host = nullptr;  // pinned copies
    cudaEvent_t vmax_event[2] = {nullptr, nullptr};
    struct PeriodPlan { int K; int slot; };  // the length of a coming period: K > 0, or pending in `slot`
    PeriodPlan plan[2] = {};
    int nplan = 0;                  // 0 after creation or a state upload
    int sms = 148;
    TileInfo ti{};
    SortBuffers alt{};
    int p2g_warp_grid = 0;
    // CUDA graphs of one sort period (sort + K steps), per period length K and
    // buffer parity (the sort swaps the particle buffers).
    static constexpr int kMaxPeriod = 64;
    cudaGraphExec_t period_graph[kMaxPeriod + 1][2] = {};
    cudaStream_t graph_stream[2] = {nullptr, nullptr};
    int parity = 0;
    bool use_graphs = true;
    // plasticity: exact return map, or the learned surrogate with exact fallback
    int plasticity = MPM_PLASTIC_EXACT;
    mpm_mlp* mlp = nullptr;
    float mlp_tol = 1e-3f;
    unsigned long long* mlp_counters = nullptr;  // accepted, rejected
    // exact return-map pairs for training
    float* log_data = nullptr;
    unsigned long long* log_n = nullptr;
    long long log_cap = 0;
    bool needs_affine = true; // A must be recomputed from the state before the next P2G
    SlowQueue q{};
    // fused transfer (tiled MLS path): one kernel per step does the G2P of the
    // step and the P2G of the next; `acc_pending` says the grid sums of the
    // current state are already in `acc` (else the next step starts with the
    // P2G-only prologue).
    bool fused = false;
    bool acc_pending = false;
    int fused_grid = 0;
    bool box_tma = false;  // fused step as the TMA box pipeline (MPM_BOX_LOAD=tma) instead of staged boxes
    CUtensorMap gv_map{};  // the node velocities (vf, wall flag) as a [nz][ny][nx][4] float tensor for TMA
};

namespace {

const char* kStatusText[] = {"ok",
                             "invalid argument",
                             "CUDA error",
                             "out of device memory",
                             "particle state became non-finite",
                             "fixed-point grid overflow",
                             "no usable sm_100 CUDA device",
                             "I/O error",
                             "checkpoint does not match this solver",
                             "device-side wait timed out",
                             "unsupported configuration",
                             "capacity too small",
                             "particle stencil outside the grid"};

mpm_status fail(mpm_solver* s, mpm_status code, const std::string& what) {
    if (s) s->err = what;
    return code;
}

mpm_status cuda_fail(mpm_solver* s, cudaError_t e, const char* where) {
    std::string msg = std::string(where) + ": " + cudaGetErrorString(e);
    if (s) s->err = msg;
    return e == cudaErrorMemoryAllocation ? MPM_ERR_OUT_OF_MEMORY : MPM_ERR_CUDA;
}

#define MPM_CUDA(s, call)                                      \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail((s), e_, #call); \
    } while (0)

int nacc(int dim, int form) { return form == kClassic ? 1 + 2 * dim : 1 + dim; }

template <typename T> cudaError_t dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
}

void release(mpm_solver* s) {
    float* fl[] = {s->x, s->v, s->B, s->Fe, s->Jp, s->A, s->mass, s->vol, s->staging};
    for (float* p : fl)
        if (p) cudaFree(p);
    if (s->id) cudaFree(s->id);
    if (s->acc) cudaFree(s->acc);
    if (s->gv) cudaFree(s->gv);
    if (s->status) cudaFree(s->status);
    float* al[] = {s->alt.x, s->alt.v, s->alt.B, s->alt.Fe, s->alt.Jp, s->alt.A, s->alt.mass, s->alt.vol};
    for (float* p : al)
        if (p) cudaFree(p);
    if (s->alt.id) cudaFree(s->alt.id);
    int* ti[] = {s->ti.key,      s->ti.tile_count, s->ti.tile_cursor, s->ti.tile_start, s->ti.mark, s->ti.mark_list,
                 s->ti.n_marked, s->ti.perm,       s->ti.tile_list,   s->ti.n_tile_list, s->ti.sval,
                 s->ti.p2g_next};
    if (s->ti.skey) cudaFree(s->ti.skey);
    for (int* p : ti)
        if (p) cudaFree(p);
    for (auto& row : s->period_graph)
        for (auto& g : row)
            if (g) cudaGraphExecDestroy(g);
    if (s->vmax_dev) cudaFree(s->vmax_dev);
    if (s->vmax_host) cudaFreeHost(s->vmax_host);
    for (auto ev : s->vmax_event)
        if (ev) cudaEventDestroy(ev);
    if (s->mlp_counters) cudaFree(s->mlp_counters);
    if (s->log_data) cudaFree(s->log_data);
    if (s->log_n) cudaFree(s->log_n);
    if (s->q.list) cudaFree(s->q.list);
    if (s->q.count) cudaFree(s->q.count);
    if (s->q.fh) cudaFree(s->q.fh);
    if (s->q.win) cudaFree(s->q.win);
    if (s->ti.tile_len) cudaFree(s->ti.tile_len);
    if (s->ti.fused_next) cudaFree(s->ti.fused_next);
    if (s->own_stream) cudaStreamDestroy(s->own_stream);
}

Particles particle_view(mpm_solver* s) {
    Particles P;
    P.x = s->x; P.v = s->v; P.B = s->B; P.Fe = s->Fe; P.Jp = s->Jp; P.A = s->A;
    P.mass = s->mass; P.vol = s->vol; P.mass_u = s->mass_u; P.vol_u = s->vol_u;
    P.n = s->n;
    return P;
}

template <int D, int FORM> cudaError_t launch_p2g(mpm_solver* s) {
    if (s->n == 0) return cudaSuccess;
    const int threads = 256, blocks = (s->n + threads - 1) / threads;
    k_p2g_simple<D, FORM><<<blocks, threads, 0, s->stream>>>(particle_view(s), s->C, s->acc, s->status);
    return cudaGetLastError();
}

template <int D, int FORM> cudaError_t launch_grid(mpm_solver* s) {
    const int threads = 256;
    const long long blocks = (s->nodes + threads - 1) / threads;
    k_grid_update<D, FORM><<<(unsigned)blocks, threads, 0, s->stream>>>(s->C, s->acc, s->gv, s->status);
    return cudaGetLastError();
}

template <int D, int FORM> cudaError_t launch_g2p(mpm_solver* s) {
    if (s->n == 0) return cudaSuccess;
    const int threads = 256, blocks = (s->n + threads - 1) / threads;
    k_g2p_simple<D, FORM><<<blocks, threads, 0, s->stream>>>(particle_view(s), s->C, s->gv, s->status);
    return cudaGetLastError();
}

// Counting sort of the particle state by cell tile into the alternate
// buffers, then swap. Called every sort_period steps (and after any state
// upload) on the tiled path.
void swap_buffers(mpm_solver* s) {
    std::swap(s->x, s->alt.x);
    std::swap(s->v, s->alt.v);
    std::swap(s->B, s->alt.B);
    std::swap(s->Fe, s->alt.Fe);
    std::swap(s->Jp, s->alt.Jp);
    std::swap(s->A, s->alt.A);
    std::swap(s->id, s->alt.id);
    if (s->mass) std::swap(s->mass, s->alt.mass);
    if (s->vol) std::swap(s->vol, s->alt.vol);
    s->parity ^= 1;
}

// Captured period graphs bake in kernel choices and pointers: drop them when
// the plasticity mode or the pair log changes.
void invalidate_graphs(mpm_solver* s) {
    cudaStreamSynchronize(s->stream);
    for (auto& row : s->period_graph)
        for (auto& g : row)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

template <int D, int S> cudaError_t launch_sort(mpm_solver* s) {
    if (s->n == 0) { s->needs_sort = false; s->next_sort = s->step + s->cur_K; return cudaSuccess; }
    const int threads = 256, blocks = (s->n + threads - 1) / threads;
    k_sort_count<D, S><<<blocks, threads, 0, s->stream>>>(particle_view(s), s->C, s->ti);
    k_sort_scan<<<1, 1024, 0, s->stream>>>(s->ti);
    k_sort_bucket<<<blocks, threads, 0, s->stream>>>(s->n, s->ti);
    SortBuffers dst = s->alt;
    if (s->fused) dst.A = nullptr;  // the fused path keeps A only within a step
    k_tile_sort<D, S><<<s->sms * SortGeom<D>::CTAS_PER_SM, 256, 0, s->stream>>>(particle_view(s), s->id, dst, s->C,
                                                                               s->ti);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    swap_buffers(s);
    s->needs_sort = false;
    s->next_sort = s->step + s->cur_K;
    s->sorted_at = s->step;
    ++s->sorts_done;
    return cudaSuccess;
}

// A sort is due before this step's P2G: after any state upload, at multiples
// of a fixed sort_period, or (auto) when the current period has run out.
bool sort_due(const mpm_solver* s) {
    if (s->needs_sort) return true;
    if (s->auto_sort) return s->step >= s->next_sort;
    return s->sort_period > 0 && s->step % s->sort_period == 0 && s->sorted_at != s->step;
}

// Auto sort period. A period of K steps costs one sort and lets particles
// drift out of the cells they were sorted by, which splits the P2G's
// same-cell runs. K is the longest of {4, 6, 8, 12, 16, 24, 32} steps over
// which the fastest particle moves at most a quarter cell (measured on B200:
// two snowballs colliding at ~0.04 cells/step run 15% faster than with a fixed
// 16-step period; a snowball falling onto a resting slab, ~0.02, is unchanged).
// The maximum is measured at the start of every period and used two periods
// later, read back through pinned memory: the host then waits only for work the
// GPU finished a period ago, and stays ahead of it. The first period after
// creation or a state upload measures its own start (one synchronisation) and
// uses it for the next one as well.
int period_for(const mpm_solver* s, unsigned vmax_bits) {
    float vmax;
    std::memcpy(&vmax, &vmax_bits, sizeof(float));
    const double disp = double(vmax) * double(s->params.delta_time);  // cells per step
#ifndef MPM_AUTO_SORT_CELLS
#define MPM_AUTO_SORT_CELLS 0.25
#endif
    const int choices[] = {32, 24, 16, 12, 8, 6, 4};
    for (int c : choices)
        if (!(disp > 0.0) || disp * c <= MPM_AUTO_SORT_CELLS) return c;
    return 4;
}

cudaError_t measure_vmax(mpm_solver* s, int slot) {
    cudaError_t e = cudaMemsetAsync(s->vmax_dev + slot, 0, sizeof(unsigned), s->stream);
    if (e != cudaSuccess) return e;
    if (s->n > 0) {
        k_max_abs<<<s->sms * 4, 256, 0, s->stream>>>(s->v, (long long)s->n * s->dim, s->vmax_dev + slot);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if ((e = cudaMemcpyAsync(s->vmax_host + slot, s->vmax_dev + slot, sizeof(unsigned), cudaMemcpyDeviceToHost,
                             s->stream)) != cudaSuccess)
        return e;
    return cudaEventRecord(s->vmax_event[slot], s->stream);
}

// Length of a planned period (waits for its measurement when still pending).
cudaError_t resolve_plan(mpm_solver* s, const mpm_solver::PeriodPlan& p, int* K) {
    if (p.K > 0) { *K = p.K; return cudaSuccess; }
    cudaError_t e = cudaEventSynchronize(s->vmax_event[p.slot]);
    if (e == cudaSuccess) *K = period_for(s, s->vmax_host[p.slot]);
    return e;
}

// At the start of a period (auto): take the planned length and measure this
// period's start for the period after next. The first period after creation or
// a state upload measures its own start and uses it for the next one too.
cudaError_t choose_period(mpm_solver* s) {
    if (!s->auto_sort || !sort_due(s)) return cudaSuccess;
    cudaError_t e;
    if (s->nplan == 0) {
        if ((e = measure_vmax(s, 0)) != cudaSuccess || (e = cudaEventSynchronize(s->vmax_event[0])) != cudaSuccess)
            return e;
        s->cur_K = period_for(s, s->vmax_host[0]);
        s->plan[0] = {s->cur_K, 0};
        s->plan[1] = {s->cur_K, 0};
        s->nplan = 2;
        return cudaSuccess;
    }
    const mpm_solver::PeriodPlan front = s->plan[0];
    s->plan[0] = s->plan[1];
    if ((e = resolve_plan(s, front, &s->cur_K)) != cudaSuccess) return e;
    const int slot = s->plan[0].K > 0 ? 0 : 1 - s->plan[0].slot;  // not the slot still pending
    if ((e = measure_vmax(s, slot)) != cudaSuccess) return e;
    s->plan[1] = {0, slot};
    return cudaSuccess;
}

template <int D, int S> cudaError_t launch_p2g_tiled_kernel(mpm_solver* s) {
    if (P2GDynamic<D, S>::value) {
        cudaError_t e = cudaMemsetAsync(s->ti.p2g_next, 0, sizeof(int), s->stream);
        if (e != cudaSuccess) return e;
    }
    k_p2g_warp<D, S><<<s->p2g_warp_grid, kP2GWarps * 32, sizeof(P2GWarpSmem<D, S>), s->stream>>>(
        particle_view(s), s->C, s->ti, s->acc, s->status);
    return cudaGetLastError();
}

// G2P of the tiled MLS path: gather + in-band return map (stage "g2p"), then
// the queued particles' full return map (stage "return_map").
template <int D, int S> cudaError_t launch_g2p_gather(mpm_solver* s) {
    if (s->n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(s->q.count, 0, sizeof(int), s->stream);
    if (e != cudaSuccess) return e;
    const int threads = 256, blocks = (s->n + threads - 1) / threads;
    k_g2p_gather<D, S><<<blocks, threads, 0, s->stream>>>(particle_view(s), s->C, s->gv, s->q, s->status);
    return cudaGetLastError();
}

// The warp-tiled inference kernels use more than the default 48 KB of dynamic
// shared memory; the opt-in is per device and set outside any stream capture.
cudaError_t mlp_kernel_attrs() {
    cudaError_t e = cudaFuncSetAttribute(k_return_map_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(MlpWarpSmem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpWarpSmem));
}

template <int D, int S> cudaError_t launch_return_map(mpm_solver* s) {
    if (s->n == 0) return cudaSuccess;
    PairLog L{s->log_data, s->log_n, s->log_cap};
    if (D == 3 && S == 4 && s->plasticity == MPM_PLASTIC_MLP && s->mlp) {
        MlpParams ML{s->mlp->wbf, s->mlp->w, s->mlp->norm, s->mlp_tol, s->mlp_counters};
        k_return_map_mlp<<<s->sms * 2, kMlpWarps * 32, sizeof(MlpWarpSmem), s->stream>>>(particle_view(s), s->C, s->q,
                                                                                       ML);
        L = PairLog{nullptr, nullptr, 0};
    }
    k_g2p_plastic<D, S><<<s->sms * 4, 256, 0, s->stream>>>(particle_view(s), s->C, s->gv, s->q, L, s->status);
    return cudaGetLastError();
}

template <int D, int S> cudaError_t launch_g2p_split(mpm_solver* s) {
    cudaError_t e = launch_g2p_gather<D, S>(s);
    if (e != cudaSuccess) return e;
    return launch_return_map<D, S>(s);
}

template <int D, int S> cudaError_t prepare_affine(mpm_solver* s) {
    if (!s->needs_affine || s->n == 0) { s->needs_affine = false; return cudaSuccess; }
    const int threads = 256, blocks = (s->n + threads - 1) / threads;
    k_prepare_affine<D, S><<<blocks, threads, 0, s->stream>>>(particle_view(s), s->C);
    s->needs_affine = false;
    return cudaGetLastError();
}

template <int D, int S> cudaError_t launch_p2g_tiled(mpm_solver* s) {
    cudaError_t e0 = prepare_affine<D, S>(s);
    if (e0 != cudaSuccess) return e0;
    if (sort_due(s)) {
        cudaError_t e = launch_sort<D, S>(s);
        if (e != cudaSuccess) return e;
    }
    return launch_p2g_tiled_kernel<D, S>(s);
}

// ---- fused transfer ----

// The fused kernel over the tiles of the last sort: G2P (this step) + P2G (next
// step), or with G2P = false the P2G of the stored state (prologue).
template <int D, int S, bool G2P> cudaError_t launch_fused(mpm_solver* s) {
    cudaError_t e = cudaMemsetAsync(s->ti.fused_next, 0, sizeof(int), s->stream);
    if (e == cudaSuccess && G2P) e = cudaMemsetAsync(s->q.count, 0, 2 * sizeof(int), s->stream);  // count, nwin
    if (e != cudaSuccess) return e;
    if (s->n == 0) return cudaSuccess;
    if (G2P && s->box_tma)
        k_g2p2g_pipe<D, S><<<s->fused_grid, FusedGeom<D>::THREADS, sizeof(PipeSmem<D>), s->stream>>>(
            particle_view(s), s->C, s->ti, s->gv, s->acc, s->q, s->status, s->gv_map);
    else
        k_g2p2g<D, S, G2P><<<s->fused_grid, FusedGeom<D>::THREADS, sizeof(FusedSmem<D>), s->stream>>>(
            particle_view(s), s->C, s->ti, s->gv, s->acc, s->q, s->status);
    return cudaGetLastError();
}

// Queued particles after the G2P part: their return map (learned and/or
// exact), then their P2G for the next step by the windows the fused kernel
// recorded.
template <int D, int S> cudaError_t launch_queued_fused(mpm_solver* s) {
    if (s->n == 0) return cudaSuccess;
    cudaError_t e = launch_return_map<D, S>(s);
    if (e != cudaSuccess) return e;
    k_p2g_windows<D, S><<<s->fused_grid, FusedGeom<D>::THREADS, 0, s->stream>>>(particle_view(s), s->C, s->ti, s->q,
                                                                                s->acc, s->status);
    return cudaGetLastError();
}

// The P2G of the current state when it is not pending yet: the sort first if
// one is due (the kernel works on the tiles of the last sort).
template <int D, int S> cudaError_t fused_prologue(mpm_solver* s) {
    if (s->acc_pending) return cudaSuccess;
    if (sort_due(s)) {
        cudaError_t e = launch_sort<D, S>(s);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = launch_fused<D, S, false>(s);
    if (e != cudaSuccess) return e;
    s->acc_pending = true;
    s->needs_affine = false;
    return cudaSuccess;
}

template <int D> cudaError_t launch_grid_marked(mpm_solver* s) {
    k_grid_marked<D, kMLS><<<s->sms * 8, 256, 0, s->stream>>>(s->C, s->ti, s->acc, s->gv, s->status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaSuccess;
}

// One fused step: [sort] grid update, fused G2P + next P2G, queued particles.
template <int D, int S> cudaError_t step_fused(mpm_solver* s) {
    cudaError_t e = fused_prologue<D, S>(s);
    if (e != cudaSuccess) return e;
    if (sort_due(s) && (e = launch_sort<D, S>(s)) != cudaSuccess) return e;
    if ((e = launch_grid_marked<D>(s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(s->ti.n_marked, 0, sizeof(int), s->stream)) != cudaSuccess) return e;
    if ((e = launch_fused<D, S, true>(s)) != cudaSuccess) return e;
    return launch_queued_fused<D, S>(s);
}

template <int D, int S> cudaError_t step_tiled(mpm_solver* s) {
    if (s->fused) return step_fused<D, S>(s);
    cudaError_t e = launch_p2g_tiled<D, S>(s);
    if (e != cudaSuccess) return e;
    e = launch_grid_marked<D>(s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(s->ti.n_marked, 0, sizeof(int), s->stream);
    if (e != cudaSuccess) return e;
    return launch_g2p_split<D, S>(s);
}

template <int D, int FORM> cudaError_t step_once(mpm_solver* s) {
    cudaError_t e = launch_p2g<D, FORM>(s);
    if (e != cudaSuccess) return e;
    e = launch_grid<D, FORM>(s);
    if (e != cudaSuccess) return e;
    return launch_g2p<D, FORM>(s);
}

cudaError_t dispatch_step(mpm_solver* s) {
    if (s->tiled) {
        if (s->stencil == 3) return s->dim == 2 ? step_tiled<2, 3>(s) : step_tiled<3, 3>(s);
        return s->dim == 2 ? step_tiled<2, 4>(s) : step_tiled<3, 4>(s);
    }
    return step_once<2, kClassic>(s);  // the untiled path: CLASSIC, 2D
}

cudaError_t dispatch_p2g(mpm_solver* s) {
    if (s->tiled && s->fused) {
        if (s->stencil == 3) return s->dim == 2 ? fused_prologue<2, 3>(s) : fused_prologue<3, 3>(s);
        return s->dim == 2 ? fused_prologue<2, 4>(s) : fused_prologue<3, 4>(s);
    }
    if (s->tiled) {
        if (s->stencil == 3) return s->dim == 2 ? launch_p2g_tiled<2, 3>(s) : launch_p2g_tiled<3, 3>(s);
        return s->dim == 2 ? launch_p2g_tiled<2, 4>(s) : launch_p2g_tiled<3, 4>(s);
    }
    return launch_p2g<2, kClassic>(s);
}

// After a P2G-only pass: clear accumulators and node-block marks.
cudaError_t clear_after_p2g(mpm_solver* s) {
    s->acc_pending = false;
    if (s->tiled) {
        cudaError_t e = s->dim == 2 ? launch_grid_marked<2>(s) : launch_grid_marked<3>(s);
        if (e != cudaSuccess) return e;
        return cudaMemsetAsync(s->ti.n_marked, 0, sizeof(int), s->stream);
    }
    return cudaMemsetAsync(s->acc, 0, sizeof(unsigned long long) * nacc(s->dim, s->form) * s->nodes, s->stream);
}


// The tensor map of the TMA pipeline's box loads (k_g2p2g_pipe): gv's first
// half (one float4 per node: (vf, wall flag) in 3D, (vf, vc) in 2D) as a rank
// D+1 FP32 tensor [nz][ny][nx][4], boxes of 4 x BE^D. The encoder comes from the driver through the runtime, so the
// library needs no link to libcuda.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

mpm_status make_box_map(mpm_solver* s) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
        cudaGetLastError();
        return fail(s, MPM_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    }
    const int D = s->dim;
    const cuuint32_t rank = (cuuint32_t)(D + 1);
    cuuint64_t dims[4] = {4, (cuuint64_t)s->C.nx, (cuuint64_t)s->C.ny, (cuuint64_t)s->C.nz};
    cuuint64_t strides[3] = {16, 16ull * (cuuint64_t)s->C.nx, 16ull * (cuuint64_t)s->C.nx * (cuuint64_t)s->C.ny};
    const cuuint32_t be = (cuuint32_t)(D == 3 ? FusedGeom<3>::BE : FusedGeom<2>::BE);
    cuuint32_t box[4] = {4, be, be, be};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = reinterpret_cast<EncodeTiledFn>(fn)(
        &s->gv_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, s->gv, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(s, MPM_ERR_CUDA, "cuTensorMapEncodeTiled failed for the node-velocity box");
    return MPM_OK;
}

// Tiles, node-block marks and the sort's alternate buffers.
mpm_status setup_tiled(mpm_solver* s) {
    const int D = s->dim, n = s->n;
    const int T = D == 3 ? TileGeom<3>::T : TileGeom<2>::T;
    const int ext[3] = {s->C.W, s->C.H, s->C.Dp};
    const int nodes_axis[3] = {s->C.nx, s->C.ny, s->C.nz};
    TileInfo& ti = s->ti;
    ti.n_tiles = 1;
    ti.n_blocks = 1;
    for (int k = 0; k < 3; ++k) {
        ti.tiles[k] = k < D ? (ext[k] + T - 1) / T : 1;
        ti.nblk[k] = k < D ? (nodes_axis[k] + T - 1) / T : 1;
        ti.n_tiles *= ti.tiles[k];
        ti.n_blocks *= ti.nblk[k];
    }
    if (dalloc(&ti.key, (size_t)n) || dalloc(&ti.tile_count, (size_t)ti.n_tiles) ||
        dalloc(&ti.tile_cursor, (size_t)ti.n_tiles) || dalloc(&ti.tile_start, (size_t)ti.n_tiles) ||
        dalloc(&ti.mark, (size_t)ti.n_blocks) || dalloc(&ti.mark_list, (size_t)ti.n_blocks) ||
        dalloc(&ti.n_marked, 1) || dalloc(&ti.p2g_next, 1) ||
        dalloc(&ti.perm, (size_t)n) || dalloc(&ti.tile_list, (size_t)ti.n_tiles) || dalloc(&ti.n_tile_list, 1) ||
        dalloc(&ti.skey, (size_t)n) || dalloc(&ti.sval, (size_t)n) ||
        dalloc(&s->alt.x, (size_t)n * D) || dalloc(&s->alt.v, (size_t)n * D) || dalloc(&s->alt.B, (size_t)n * D * D) ||
        dalloc(&s->alt.Fe, (size_t)n * D * D) || dalloc(&s->alt.Jp, (size_t)n) || dalloc(&s->alt.id, (size_t)n) ||
        dalloc(&s->A, (size_t)n * D * D) || dalloc(&s->alt.A, (size_t)n * D * D)) {
        cudaGetLastError();
        return MPM_ERR_OUT_OF_MEMORY;
    }
    if (s->mass && dalloc(&s->alt.mass, (size_t)n)) return MPM_ERR_OUT_OF_MEMORY;
    if (s->vol && dalloc(&s->alt.vol, (size_t)n)) return MPM_ERR_OUT_OF_MEMORY;
    bool ok = cudaMemset(ti.tile_count, 0, sizeof(int) * ti.n_tiles) == cudaSuccess &&
              cudaMemset(ti.tile_cursor, 0, sizeof(int) * ti.n_tiles) == cudaSuccess &&
              cudaMemset(ti.mark, 0, sizeof(int) * ti.n_blocks) == cudaSuccess &&
              cudaMemset(ti.n_marked, 0, sizeof(int)) == cudaSuccess;
    if (!ok) return MPM_ERR_CUDA;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    s->sms = sms > 0 ? sms : 148;
    {
        const void* kfn;
        size_t wsm;
        if (s->stencil == 3) {
            kfn = D == 3 ? (const void*)k_p2g_warp<3, 3> : (const void*)k_p2g_warp<2, 3>;
            wsm = D == 3 ? sizeof(P2GWarpSmem<3, 3>) : sizeof(P2GWarpSmem<2, 3>);
        } else {
            kfn = D == 3 ? (const void*)k_p2g_warp<3, 4> : (const void*)k_p2g_warp<2, 4>;
            wsm = D == 3 ? sizeof(P2GWarpSmem<3, 4>) : sizeof(P2GWarpSmem<2, 4>);
        }
        cudaError_t ew = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm);
        int per = 0;
        if (ew == cudaSuccess) ew = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kfn, kP2GWarps * 32, wsm);
        if (ew != cudaSuccess || per < 1) return MPM_ERR_CUDA;
        s->p2g_warp_grid = s->sms * per;
    }
    s->q.capacity = n > 0 ? n : 1;
    // windows of a sort: at most ceil(m / 32) per tile of m slots
    s->q.win_capacity = s->q.capacity / 32 + ti.n_tiles + 1;
    if (dalloc(&s->q.list, (size_t)s->q.capacity) || dalloc(&s->q.count, 2) ||
        dalloc(&s->q.fh, (size_t)s->q.capacity * D * D) || dalloc(&s->q.win, (size_t)s->q.win_capacity) ||
        dalloc(&ti.tile_len, (size_t)ti.n_tiles) || dalloc(&ti.fused_next, 1)) {
        cudaGetLastError();
        return MPM_ERR_OUT_OF_MEMORY;
    }
    s->q.nwin = s->q.count + 1;
    {
        // MPM_TRANSFER=split selects the separate P2G / G2P kernels (for comparison)
        const char* tr = std::getenv("MPM_TRANSFER");
        s->fused = !(tr && std::strcmp(tr, "split") == 0);
    }
    if (s->fused) {
        // MPM_BOX_LOAD=tma: node boxes by TMA tensor loads (same results)
        const char* bl = std::getenv("MPM_BOX_LOAD");
        s->box_tma = bl && std::strcmp(bl, "tma") == 0;
        const void* kfn;
        size_t fsm, psm;
        const void* kpro;
        if (D == 3) {
            if (s->box_tma)
                kfn = s->stencil == 3 ? (const void*)k_g2p2g_pipe<3, 3> : (const void*)k_g2p2g_pipe<3, 4>;
            else
                kfn = s->stencil == 3 ? (const void*)k_g2p2g<3, 3, true> : (const void*)k_g2p2g<3, 4, true>;
            kpro = s->stencil == 3 ? (const void*)k_g2p2g<3, 3, false> : (const void*)k_g2p2g<3, 4, false>;
            fsm = s->box_tma ? sizeof(PipeSmem<3>) : sizeof(FusedSmem<3>);
            psm = sizeof(FusedSmem<3>);
        } else {
            if (s->box_tma)
                kfn = s->stencil == 3 ? (const void*)k_g2p2g_pipe<2, 3> : (const void*)k_g2p2g_pipe<2, 4>;
            else
                kfn = s->stencil == 3 ? (const void*)k_g2p2g<2, 3, true> : (const void*)k_g2p2g<2, 4, true>;
            kpro = s->stencil == 3 ? (const void*)k_g2p2g<2, 3, false> : (const void*)k_g2p2g<2, 4, false>;
            fsm = s->box_tma ? sizeof(PipeSmem<2>) : sizeof(FusedSmem<2>);
            psm = sizeof(FusedSmem<2>);
        }
        int per = 0;
        cudaError_t ef = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm);
        if (ef == cudaSuccess) ef = cudaFuncSetAttribute(kpro, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm);
        if (ef == cudaSuccess)
            ef = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kfn, FusedGeom<3>::THREADS, fsm);
        if (ef != cudaSuccess || per < 1) return MPM_ERR_CUDA;
        s->fused_grid = s->sms * per;
        if (s->box_tma) {
            mpm_status em = make_box_map(s);
            if (em != MPM_OK) return em;
        }
    }
    s->sort_period = s->params.sort_period > 0 ? s->params.sort_period : 16;
    s->auto_sort = s->params.sort_period <= 0;
    s->cur_K = s->sort_period;
    s->next_sort = 0;
    if (s->sort_period > mpm_solver::kMaxPeriod) s->use_graphs = false;  // graphs are cached per period up to 64
    if (dalloc(&s->vmax_dev, 2) ||
        cudaHostAlloc(&s->vmax_host, 2 * sizeof(unsigned), cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->vmax_event[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->vmax_event[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return MPM_ERR_OUT_OF_MEMORY;
    }
    s->needs_sort = true;
    return MPM_OK;
}

// Choose power-of-two fixed-point scales so that no node sum can exceed 2^62
// while |node velocity| <= v_cap = 16 cells per step (a blow-up long before
// that point is flagged by the grid pass).
void choose_scales(mpm_solver* s, double total_mass) {
    int l2[3];
    fixed_point_scales(s->params, total_mass, s->C, l2);
    s->log2_sm = l2[0];
    s->log2_sp = l2[1];
    s->log2_sf = l2[2];
}

void fill_consts(mpm_solver* s) { s->C = step_consts(s->params, s->dim); }

mpm_status validate(const mpm_params* p, std::string& why) { return validate_params(p, why); }

mpm_status ensure_staging(mpm_solver* s, size_t floats) {
    if (floats <= s->staging_floats) return MPM_OK;
    if (s->staging) cudaFree(s->staging);
    if (s->render_fb) cudaFree(s->render_fb);
    if (s->render_rgb) cudaFree(s->render_rgb);
    s->staging = nullptr;
    s->staging_floats = 0;
    MPM_CUDA(s, dalloc(&s->staging, floats));
    s->staging_floats = floats;
    return MPM_OK;
}

// Device SoA field -> host interleaved array in creation order.
mpm_status export_field(mpm_solver* s, const float* soa, int comps, float* host) {
    if (s->n == 0) return MPM_OK;
    mpm_status st = ensure_staging(s, (size_t)s->n * comps);
    if (st != MPM_OK) return st;
    const int threads = 256, blocks = (s->n + threads - 1) / threads;
    k_export_soa<<<blocks, threads, 0, s->stream>>>(soa, comps, s->n, s->id, s->staging);
    MPM_CUDA(s, cudaGetLastError());
    MPM_CUDA(s, cudaMemcpyAsync(host, s->staging, sizeof(float) * (size_t)s->n * comps, cudaMemcpyDeviceToHost, s->stream));
    MPM_CUDA(s, cudaStreamSynchronize(s->stream));
    return MPM_OK;
}

mpm_status import_field(mpm_solver* s, float* soa, int comps, const float* host) {
    if (s->n == 0) return MPM_OK;
    mpm_status st = ensure_staging(s, (size_t)s->n * comps);
    if (st != MPM_OK) return st;
    MPM_CUDA(s, cudaMemcpyAsync(s->staging, host, sizeof(float) * (size_t)s->n * comps, cudaMemcpyHostToDevice, s->stream));
    const int threads = 256, blocks = (s->n + threads - 1) / threads;
    k_import_soa<<<blocks, threads, 0, s->stream>>>(soa, comps, s->n, s->id, s->staging);
    MPM_CUDA(s, cudaGetLastError());
    MPM_CUDA(s, cudaStreamSynchronize(s->stream));
    return MPM_OK;
}

uint64_t params_hash(const mpm_params& p) {
    // FNV-1a over the knob bytes (the reserved tail excluded).
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&p);
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < offsetof(mpm_params, reserved); ++i) { h ^= b[i]; h *= 1099511628211ull; }
    return h;
}

}  // namespace

namespace {
const char* kStageNames[] = {"sort", "p2g", "grid_update", "g2p", "return_map"};
constexpr int kStages = 5;

template <int D, int FORM> cudaError_t stage(mpm_solver* s, int k) {
    if (k == 0) return cudaSuccess;
    if (k == 1) return launch_p2g<D, FORM>(s);
    if (k == 2) return launch_grid<D, FORM>(s);
    if (k == 3) return launch_g2p<D, FORM>(s);
    return cudaSuccess;  // the untiled G2P includes its return map
}
template <int D, int S> cudaError_t stage_tiled(mpm_solver* s, int k) {
    if (k == 0) {
        cudaError_t e = prepare_affine<D, S>(s);
        if (e != cudaSuccess) return e;
        if (sort_due(s)) return launch_sort<D, S>(s);
        return cudaSuccess;
    }
    if (k == 1) return launch_p2g_tiled_kernel<D, S>(s);
    if (k == 2) {
        cudaError_t e = launch_grid_marked<D>(s);
        if (e != cudaSuccess) return e;
        return cudaMemsetAsync(s->ti.n_marked, 0, sizeof(int), s->stream);
    }
    if (k == 3) return launch_g2p_gather<D, S>(s);
    return launch_return_map<D, S>(s);
}
template <int D, int S> cudaError_t stage_fused(mpm_solver* s, int k) {
    if (k == 0) return sort_due(s) ? launch_sort<D, S>(s) : cudaSuccess;
    if (k == 1) return fused_prologue<D, S>(s);
    if (k == 2) {
        cudaError_t e = launch_grid_marked<D>(s);
        if (e != cudaSuccess) return e;
        return cudaMemsetAsync(s->ti.n_marked, 0, sizeof(int), s->stream);
    }
    if (k == 3) return launch_fused<D, S, true>(s);
    return launch_queued_fused<D, S>(s);
}
cudaError_t dispatch_stage(mpm_solver* s, int k) {
    if (s->tiled && s->fused) {
        if (s->stencil == 3) return s->dim == 2 ? stage_fused<2, 3>(s, k) : stage_fused<3, 3>(s, k);
        return s->dim == 2 ? stage_fused<2, 4>(s, k) : stage_fused<3, 4>(s, k);
    }
    if (s->tiled) {
        if (s->stencil == 3) return s->dim == 2 ? stage_tiled<2, 3>(s, k) : stage_tiled<3, 3>(s, k);
        return s->dim == 2 ? stage_tiled<2, 4>(s, k) : stage_tiled<3, 4>(s, k);
    }
    return stage<2, kClassic>(s, k);
}
}  // namespace

namespace {
// Replays (capturing on first use) the graph of one sort period: the sort and
// sort_period steps. The captured kernels hold the buffer pointers of the
// current parity; the host-side buffer swap the sort performs is re-applied on
// every replay.
// Returns 1 when the period ran, 0 when graphs are unavailable (the caller then
// steps without them), -1 on a CUDA error (s->err set).
int run_period_graph(mpm_solver* s) {
    const int par = s->parity;
    const int K = s->auto_sort ? s->cur_K : s->sort_period;
    if (K < 1 || K > mpm_solver::kMaxPeriod) return 0;
    cudaGraphExec_t& slot = s->period_graph[K][par];
    if (!slot) {
        cudaStream_t cap = nullptr;
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            s->use_graphs = false;
            return 0;
        }
        cudaStream_t saved = s->stream;
        const long long step0 = s->step, next0 = s->next_sort, sorts0 = s->sorts_done, sorted0 = s->sorted_at;
        const bool ns = s->needs_sort;
        s->stream = cap;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            s->needs_sort = true;  // the period starts with a sort
            for (int k = 0; k < K && e == cudaSuccess; ++k) {
                e = dispatch_step(s);
                ++s->step;
            }
            cudaError_t e2 = cudaStreamEndCapture(cap, &g);
            if (e == cudaSuccess) e = e2;
        }
        // undo the host-side effects of the capture (nothing ran)
        s->stream = saved;
        s->step = step0;
        s->next_sort = next0;
        s->sorts_done = sorts0;
        s->sorted_at = sorted0;
        s->needs_sort = ns;
        if (s->parity != par) swap_buffers(s);
        if (e == cudaSuccess) e = cudaGraphInstantiate(&slot, g, 0);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cap);
        if (e != cudaSuccess) {  // no graph: step without one
            slot = nullptr;
            s->use_graphs = false;
            cudaGetLastError();
            return 0;
        }
    }
    cudaError_t e = cudaGraphLaunch(slot, s->stream);
    if (e != cudaSuccess) { cuda_fail(s, e, "graph launch"); return -1; }
    swap_buffers(s);
    s->needs_sort = false;
    s->next_sort = s->step + K;  // the period's sort ran at its first step
    s->sorted_at = s->step;
    ++s->sorts_done;
    s->step += K;
    return 1;
}
}  // namespace

extern "C" {

void mpm_params_default(mpm_params* out, int32_t dim) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->dim = dim == 3 ? 3 : 2;
    out->width = 200;
    out->height = 100;
    out->depth = 100;
    out->border_margin = 2;
    out->formulation = MPM_FORMULATION_MLS;
    out->boundary = MPM_BOUNDARY_FRICTION;
    out->sort_period = 0;
    out->delta_time = 1e-3f;
    out->gravity = -9.81f;
    out->friction = 0.3f;
    out->theta_c = 2.0e-2f;
    out->theta_s = 6.0e-3f;
    out->xi = 10.f;
    out->nu = 2.0e-1f;
    out->youngs = 1.4e5f;
    out->rho = 400.f;
}

const char* mpm_status_string(mpm_status status) {
    const int i = (int)status;
    if (i < 0 || i >= (int)(sizeof(kStatusText) / sizeof(kStatusText[0]))) return "unknown status";
    return kStatusText[i];
}

mpm_status mpm_create(const mpm_params* params, const mpm_particles_init* init, mpm_solver** out) {
    if (!out) return MPM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    std::string why;
    mpm_status st = validate(params, why);
    if (st != MPM_OK) return st;
    if (!init || init->count < 0 || init->count > 0x7fffffff) return MPM_ERR_INVALID_ARGUMENT;
    if (init->count > 0 && (!init->position || !init->volume)) return MPM_ERR_INVALID_ARGUMENT;

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return MPM_ERR_NO_DEVICE; }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MPM_ERR_NO_DEVICE;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_grid_update<2, kClassic>) != cudaSuccess) { cudaGetLastError(); return MPM_ERR_NO_DEVICE; }

    mpm_solver* s = new mpm_solver();
    s->params = *params;
    s->dim = params->dim;
    s->form = params->formulation;
    s->stencil = stencil_of(s->form);
    s->device = dev;
    s->n = (int)init->count;
    fill_consts(s);
    s->nodes = s->C.nodes;
    const int D = s->dim, n = s->n;

    auto bail = [&](mpm_status code) { release(s); delete s; return code; };
    if (cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking) != cudaSuccess) return bail(MPM_ERR_CUDA);
    s->stream = s->own_stream;
    if (dalloc(&s->x, (size_t)n * D) || dalloc(&s->v, (size_t)n * D) || dalloc(&s->B, (size_t)n * D * D) ||
        dalloc(&s->Fe, (size_t)n * D * D) || dalloc(&s->Jp, (size_t)n) || dalloc(&s->id, (size_t)n) ||
        dalloc(&s->acc, (size_t)nacc(D, s->form) * s->nodes) || dalloc(&s->gv, (size_t)s->nodes * (D == 3 ? 2 : 1)) ||
        dalloc(&s->status, 1)) {
        cudaGetLastError();
        return bail(MPM_ERR_OUT_OF_MEMORY);
    }

    // Host-side preparation: mass = vol * RHO / 100 when not given
    // (src/cpu/Particles.cpp:18, src/gpu/GPUSolver.cpp:119,148).
    std::vector<float> massv(n), volv(n);
    double total_mass = 0.0;
    bool uni_m = true, uni_v = true;
    for (int i = 0; i < n; ++i) {
        volv[i] = init->volume[i];
        massv[i] = init->mass ? init->mass[i] : (init->volume[i] * params->rho) / 100.f;
        if (!std::isfinite(volv[i]) || !std::isfinite(massv[i])) return bail(MPM_ERR_INVALID_ARGUMENT);
        total_mass += massv[i];
        if (massv[i] != massv[0]) uni_m = false;
        if (volv[i] != volv[0]) uni_v = false;
    }
    for (long long i = 0; i < (long long)n * D; ++i)
        if (!std::isfinite(init->position[i]) || (init->velocity && !std::isfinite(init->velocity[i])))
            return bail(MPM_ERR_INVALID_ARGUMENT);
    choose_scales(s, total_mass);
    if (uni_m && n > 0) s->mass_u = massv[0];
    else if (n > 0) {
        if (dalloc(&s->mass, (size_t)n)) return bail(MPM_ERR_OUT_OF_MEMORY);
        if (cudaMemcpy(s->mass, massv.data(), sizeof(float) * n, cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(MPM_ERR_CUDA);
    }
    if (uni_v && n > 0) s->vol_u = volv[0];
    else if (n > 0) {
        if (dalloc(&s->vol, (size_t)n)) return bail(MPM_ERR_OUT_OF_MEMORY);
        if (cudaMemcpy(s->vol, volv.data(), sizeof(float) * n, cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(MPM_ERR_CUDA);
    }

    // SoA upload: F_E = I, B = 0, J_p = 1 (Particle ctor, src/cpu/Particles.cpp:7-19).
    std::vector<float> soa((size_t)n * D * D);
    std::vector<int> ids(n);
    for (int i = 0; i < n; ++i) ids[i] = i;
    auto up = [&](float* dst, size_t count) {
        return cudaMemcpy(dst, soa.data(), sizeof(float) * count, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    bool ok = true;
    for (int k = 0; k < D; ++k)
        for (int i = 0; i < n; ++i) soa[(size_t)k * n + i] = init->position[(size_t)i * D + k];
    ok = ok && up(s->x, (size_t)n * D);
    for (int k = 0; k < D; ++k)
        for (int i = 0; i < n; ++i) soa[(size_t)k * n + i] = init->velocity ? init->velocity[(size_t)i * D + k] : 0.f;
    ok = ok && up(s->v, (size_t)n * D);
    std::fill(soa.begin(), soa.end(), 0.f);
    ok = ok && up(s->B, (size_t)n * D * D);
    for (int k = 0; k < D * D; ++k)
        for (int i = 0; i < n; ++i) soa[(size_t)k * n + i] = (k % (D + 1) == 0) ? 1.f : 0.f;
    ok = ok && up(s->Fe, (size_t)n * D * D);
    for (int i = 0; i < n; ++i) soa[i] = 1.f;
    ok = ok && up(s->Jp, (size_t)n);
    ok = ok && cudaMemcpy(s->id, ids.data(), sizeof(int) * n, cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemset(s->acc, 0, sizeof(unsigned long long) * nacc(D, s->form) * s->nodes) == cudaSuccess;
    ok = ok && cudaMemset(s->gv, 0, sizeof(float4) * s->nodes * (D == 3 ? 2 : 1)) == cudaSuccess;
    ok = ok && cudaMemset(s->status, 0, sizeof(unsigned)) == cudaSuccess;
    ok = ok && cudaDeviceSynchronize() == cudaSuccess;
    if (!ok) { cudaGetLastError(); return bail(MPM_ERR_CUDA); }
    s->tiled = (s->form != kClassic);  // MLS and QUAD
    if (s->tiled) {
        mpm_status ts = setup_tiled(s);
        if (ts != MPM_OK) return bail(ts);
    }
    *out = s;
    return MPM_OK;
}

mpm_status mpm_destroy(mpm_solver* s) {
    if (!s) return MPM_ERR_INVALID_ARGUMENT;
    if (s->stream) cudaStreamSynchronize(s->stream);
    release(s);
    delete s;
    return MPM_OK;
}

mpm_status mpm_step(mpm_solver* s, int32_t nsteps) {
    if (!s || nsteps < 0) return fail(s, MPM_ERR_INVALID_ARGUMENT, "nsteps must be >= 0");
    int32_t k = 0;
    while (k < nsteps) {
        if (s->tiled) {
            cudaError_t ec = choose_period(s);
            if (ec != cudaSuccess) return cuda_fail(s, ec, "sort period");
        }
        const int K = s->auto_sort ? s->cur_K : s->sort_period;
        const bool period_start = s->auto_sort ? s->step >= s->next_sort : (K > 0 && s->step % K == 0);
        if (s->tiled && s->use_graphs && K > 0 && nsteps - k >= K && period_start && !s->needs_sort &&
            !s->needs_affine && (!s->fused || s->acc_pending)) {
            const int r = run_period_graph(s);
            if (r < 0) return MPM_ERR_CUDA;
            if (r > 0) {
                k += K;
                continue;
            }
        }
        cudaError_t e = dispatch_step(s);
        if (e != cudaSuccess) return cuda_fail(s, e, "step launch");
        ++s->step;
        ++k;
    }
    return MPM_OK;
}


int32_t mpm_stage_count(const mpm_solver*) { return kStages; }

const char* mpm_stage_name(const mpm_solver* s, int32_t k) {
    // fused path: "p2g" is the prologue (first step after creation or an
    // upload), "g2p2g" the G2P of each step with the next step's P2G
    if (s && s->tiled && s->fused && k == 3) return "g2p2g";
    return (k >= 0 && k < kStages) ? kStageNames[k] : "";
}

mpm_status mpm_step_profiled(mpm_solver* s, int32_t nsteps, double* stage_ms, int32_t nstages) {
    if (!s || nsteps < 0 || (nstages > 0 && !stage_ms)) return MPM_ERR_INVALID_ARGUMENT;
    cudaEvent_t ev[kStages + 1];
    for (auto& e : ev) MPM_CUDA(s, cudaEventCreate(&e));
    mpm_status st = MPM_OK;
    for (int32_t it = 0; it < nsteps && st == MPM_OK; ++it) {
        if (s->tiled) {
            cudaError_t ec = choose_period(s);
            if (ec != cudaSuccess) { st = cuda_fail(s, ec, "sort period"); break; }
        }
        cudaError_t e = cudaEventRecord(ev[0], s->stream);
        for (int k = 0; k < kStages && e == cudaSuccess; ++k) {
            e = dispatch_stage(s, k);
            if (e == cudaSuccess) e = cudaEventRecord(ev[k + 1], s->stream);
        }
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[kStages]);
        if (e != cudaSuccess) { st = cuda_fail(s, e, "profiled step"); break; }
        ++s->step;
        for (int k = 0; k < kStages && k < nstages; ++k) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
            stage_ms[k] += ms;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return st;
}

mpm_status mpm_get_sort_stats(const mpm_solver* s, int64_t* sorts, int32_t* period) {
    if (!s) return MPM_ERR_INVALID_ARGUMENT;
    if (sorts) *sorts = s->sorts_done;
    if (period) *period = s->auto_sort ? s->cur_K : s->sort_period;
    return MPM_OK;
}

mpm_status mpm_get_info(const mpm_solver* s, int64_t* count, int32_t* dim) {
    if (!s) return MPM_ERR_INVALID_ARGUMENT;
    if (count) *count = s->n;
    if (dim) *dim = s->dim;
    return MPM_OK;
}

mpm_status mpm_get_positions(mpm_solver* s, float* out, size_t cap_floats) {
    if (!s || (!out && s->n > 0)) return fail(s, MPM_ERR_INVALID_ARGUMENT, "out is NULL");
    if (cap_floats < (size_t)s->n * s->dim) return fail(s, MPM_ERR_CAPACITY, "output capacity below count * dim");
    return export_field(s, s->x, s->dim, out);
}

mpm_status mpm_get_state(mpm_solver* s, mpm_state_host* st) {
    if (!s || !st) return MPM_ERR_INVALID_ARGUMENT;
    if (st->count != s->n) return fail(s, MPM_ERR_CAPACITY, "state.count must equal the particle count");
    const int D = s->dim;
    mpm_status r = MPM_OK;
    if (st->position && (r = export_field(s, s->x, D, st->position)) != MPM_OK) return r;
    if (st->velocity && (r = export_field(s, s->v, D, st->velocity)) != MPM_OK) return r;
    if (st->affine_b && (r = export_field(s, s->B, D * D, st->affine_b)) != MPM_OK) return r;
    if (st->elastic_f && (r = export_field(s, s->Fe, D * D, st->elastic_f)) != MPM_OK) return r;
    if (st->plastic_det && (r = export_field(s, s->Jp, 1, st->plastic_det)) != MPM_OK) return r;
    return MPM_OK;
}

mpm_status mpm_set_state(mpm_solver* s, const mpm_state_host* st) {
    if (!s || !st) return MPM_ERR_INVALID_ARGUMENT;
    if (st->count != s->n) return fail(s, MPM_ERR_CAPACITY, "state.count must equal the particle count");
    const int D = s->dim;
    mpm_status r = MPM_OK;
    if (st->position && (r = import_field(s, s->x, D, st->position)) != MPM_OK) return r;
    if (st->velocity && (r = import_field(s, s->v, D, st->velocity)) != MPM_OK) return r;
    if (st->affine_b && (r = import_field(s, s->B, D * D, st->affine_b)) != MPM_OK) return r;
    if (st->elastic_f && (r = import_field(s, s->Fe, D * D, st->elastic_f)) != MPM_OK) return r;
    if (st->plastic_det && (r = import_field(s, s->Jp, 1, st->plastic_det)) != MPM_OK) return r;
    if (s->fused) {
        // the pending grid sums belong to the old state; the next step starts
        // with the P2G-only prologue
        if (s->acc_pending) MPM_CUDA(s, clear_after_p2g(s));
        MPM_CUDA(s, cudaStreamSynchronize(s->stream));
    }
    s->needs_sort = true;
    s->needs_affine = true;
    s->nplan = 0;  // the next period is measured from the uploaded state
    return MPM_OK;
}

mpm_status mpm_rasterize(mpm_solver* s, double* node_mass, double* node_momentum, int64_t* raw, size_t nodes) {
    if (!s) return MPM_ERR_INVALID_ARGUMENT;
    if (nodes != (size_t)s->nodes) return fail(s, MPM_ERR_CAPACITY, "nodes must equal the grid node count");
    const int D = s->dim, NA = nacc(D, s->form);
    cudaError_t e = dispatch_p2g(s);
    if (e != cudaSuccess) return cuda_fail(s, e, "p2g launch");
    std::vector<long long> h((size_t)NA * s->nodes);
    MPM_CUDA(s, cudaMemcpyAsync(h.data(), s->acc, sizeof(long long) * h.size(), cudaMemcpyDeviceToHost, s->stream));
    if (!(s->tiled && s->fused)) MPM_CUDA(s, clear_after_p2g(s));  // fused: these are the next step's sums
    MPM_CUDA(s, cudaStreamSynchronize(s->stream));
    const double ism = std::ldexp(1.0, -s->log2_sm), isp = std::ldexp(1.0, -s->log2_sp),
                 isf = std::ldexp(1.0, -s->log2_sf);
    const long long N = s->nodes;
    for (long long i = 0; i < N; ++i) {
        if (node_mass) node_mass[i] = (double)h[i] * ism;
        for (int k = 0; k < D && node_momentum; ++k) {
            double p = (double)h[(1 + k) * N + i] * isp;
            if (s->form == kClassic) p -= (double)s->params.delta_time * ((double)h[(1 + D + k) * N + i] * isf);
            node_momentum[i * D + k] = p;
        }
    }
    if (raw) std::memcpy(raw, h.data(), sizeof(long long) * (size_t)(1 + D) * N);
    return MPM_OK;
}

mpm_status mpm_get_status(mpm_solver* s, uint32_t* flags) {
    if (!s || !flags) return MPM_ERR_INVALID_ARGUMENT;
    unsigned h = 0;
    MPM_CUDA(s, cudaMemcpyAsync(&h, s->status, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
    MPM_CUDA(s, cudaStreamSynchronize(s->stream));
    *flags = h;
    return MPM_OK;
}

mpm_status mpm_check_status(mpm_solver* s) {
    if (!s) return MPM_ERR_INVALID_ARGUMENT;
    uint32_t f = 0;
    mpm_status r = mpm_get_status(s, &f);
    if (r != MPM_OK) return r;
    std::string names;
    const char* label[] = {"non-finite state", "fixed-point overflow", "stencil outside the grid", "FP64 SVD branch",
                           "device wait timed out"};
    for (int b = 0; b < 5; ++b)
        if (f & (1u << b)) names += std::string(names.empty() ? "" : ", ") + label[b];
    if (f & MPM_FLAG_NAN_STATE) return fail(s, MPM_ERR_NAN_STATE, "status flags: " + names);
    if (f & MPM_FLAG_FIXED_POINT_OVERFLOW) return fail(s, MPM_ERR_FIXED_POINT_OVERFLOW, "status flags: " + names);
    if (f & MPM_FLAG_PARTICLE_OUT_OF_DOMAIN) return fail(s, MPM_ERR_PARTICLE_OUT_OF_DOMAIN, "status flags: " + names);
    if (f & MPM_FLAG_TIMEOUT) return fail(s, MPM_ERR_TIMEOUT, "status flags: " + names);
    return MPM_OK;
}

mpm_status mpm_set_stream(mpm_solver* s, void* stream) {
    if (!s) return MPM_ERR_INVALID_ARGUMENT;
    MPM_CUDA(s, cudaStreamSynchronize(s->stream));
    s->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : s->own_stream;
    return MPM_OK;
}

mpm_status mpm_get_step(const mpm_solver* s, int64_t* step) {
    if (!s || !step) return MPM_ERR_INVALID_ARGUMENT;
    *step = s->step;
    return MPM_OK;
}

const char* mpm_last_error(const mpm_solver* s) { return s ? s->err.c_str() : "null solver"; }

mpm_status mpm_get_fixed_point(const mpm_solver* s, int32_t* lm, int32_t* lp) {
    if (!s) return MPM_ERR_INVALID_ARGUMENT;
    if (lm) *lm = s->log2_sm;
    if (lp) *lp = s->log2_sp;
    return MPM_OK;
}

constexpr int kSchedTag = 0x4B504552;  // extra record: auto sort schedule
constexpr int kTileTag = 0x454C4954;   // extra record: {tag, tile, first slot, particles} of the last sort

// Checkpoint: "MPMS" | u32 version=3 | i32 dim | i64 count | i32 W, H, D |
// u64 params hash | i64 step | f32 x[n*d] v[n*d] B[n*d*d] Fe[n*d*d] Jp[n]
// (creation order) | u32 has_order | [i32 slot_id[n] | i32 n_extra |
// i32x4 extra[n_extra]] | u32 has_sums | [i32 channels | i32 nodes per block
// | i32 nblocks | i32 block[nblocks] | i64 sums[nblocks][channels][nodes]].
// The slot order of the tiled path is saved so that a resumed run groups
// particles exactly as the original did and continues bit-identically.
// `extra` holds tagged records: with the auto sort period, one {kSchedTag,
// period, steps to the next sort, next two periods (8 bits each; 0:
// measure)}; on the fused path one {kTileTag, tile, first slot, count} per
// non-empty tile of the last sort (the particles' tiles at that sort cannot
// be recomputed from their current positions); unknown records are skipped on
// load. On the fused path the grid already holds the next step's P2G sums;
// `sums` keeps them (the node blocks marked for the grid update), so a resumed
// run continues from the very same integers. Version 2 files (no sums
// section) load as well.
mpm_status mpm_save_state(mpm_solver* s, const char* path) {
    if (!s || !path) return MPM_ERR_INVALID_ARGUMENT;
    const int D = s->dim;
    const size_t n = (size_t)s->n;
    std::vector<float> x(n * D), v(n * D), B(n * D * D), Fe(n * D * D), Jp(n);
    mpm_state_host st{(int64_t)n, x.data(), v.data(), B.data(), Fe.data(), Jp.data()};
    mpm_status r = mpm_get_state(s, &st);
    if (r != MPM_OK) return r;
    const uint32_t has_order = (s->tiled && !s->needs_sort) ? 1u : 0u;
    std::vector<int> ids;
    // extra records: the auto sort schedule (period length, steps to the next sort)
    int planned[2] = {0, 0};
    for (int q = 0; s->auto_sort && q < s->nplan; ++q) MPM_CUDA(s, resolve_plan(s, s->plan[q], &planned[q]));
    std::vector<int4> extra;
    if (s->auto_sort)
        extra.push_back(make_int4(kSchedTag, s->cur_K, (int)(s->next_sort - s->step), planned[0] | (planned[1] << 8)));
    if (has_order) {
        ids.resize(n);
        MPM_CUDA(s, cudaMemcpyAsync(ids.data(), s->id, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
        MPM_CUDA(s, cudaStreamSynchronize(s->stream));
    }
    if (has_order && s->fused && n > 0) {
        int ntl = 0;
        MPM_CUDA(s, cudaMemcpy(&ntl, s->ti.n_tile_list, sizeof(int), cudaMemcpyDeviceToHost));
        std::vector<int> tl(ntl), tlen(ntl), tstart(s->ti.n_tiles);
        if (ntl > 0) {
            MPM_CUDA(s, cudaMemcpy(tl.data(), s->ti.tile_list, sizeof(int) * ntl, cudaMemcpyDeviceToHost));
            MPM_CUDA(s, cudaMemcpy(tlen.data(), s->ti.tile_len, sizeof(int) * ntl, cudaMemcpyDeviceToHost));
        }
        MPM_CUDA(s, cudaMemcpy(tstart.data(), s->ti.tile_start, sizeof(int) * s->ti.n_tiles, cudaMemcpyDeviceToHost));
        for (int e = 0; e < ntl; ++e) extra.push_back(make_int4(kTileTag, tl[e], tstart[tl[e]], tlen[e]));
    }
    // the pending grid sums of the fused path, block by block
    uint32_t has_sums = 0;
    int32_t sum_hdr[3] = {nacc(D, s->form), D == 3 ? TileGeom<3>::BN : TileGeom<2>::BN, 0};
    std::vector<int> sum_blocks;
    std::vector<unsigned long long> sums;
    if (has_order && s->fused && s->acc_pending) {
        has_sums = 1;
        MPM_CUDA(s, cudaMemcpy(&sum_hdr[2], s->ti.n_marked, sizeof(int), cudaMemcpyDeviceToHost));
        const int nb = sum_hdr[2];
        sum_blocks.resize(nb);
        sums.resize((size_t)nb * sum_hdr[0] * sum_hdr[1]);
        if (nb > 0) {
            MPM_CUDA(s, cudaMemcpy(sum_blocks.data(), s->ti.mark_list, sizeof(int) * nb, cudaMemcpyDeviceToHost));
            mpm_status es = ensure_staging(s, sums.size() * 2);
            if (es != MPM_OK) return es;
            unsigned long long* dst = reinterpret_cast<unsigned long long*>(s->staging);
            if (D == 3)
                k_pack_marked<3><<<s->sms * 4, 256, 0, s->stream>>>(s->C, s->ti, sum_hdr[0], nb, s->acc, dst);
            else
                k_pack_marked<2><<<s->sms * 4, 256, 0, s->stream>>>(s->C, s->ti, sum_hdr[0], nb, s->acc, dst);
            MPM_CUDA(s, cudaGetLastError());
            MPM_CUDA(s, cudaMemcpyAsync(sums.data(), dst, sizeof(unsigned long long) * sums.size(),
                                        cudaMemcpyDeviceToHost, s->stream));
            MPM_CUDA(s, cudaStreamSynchronize(s->stream));
        }
    }
    const int32_t n_extra = (int32_t)extra.size();
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(s, MPM_ERR_IO, std::string("cannot open ") + path);
    const uint32_t ver = 3;
    const int32_t dim = D, ext[3] = {s->params.width, s->params.height, D == 3 ? s->params.depth : 0};
    const int64_t count = (int64_t)n, step = s->step;
    const uint64_t h = params_hash(s->params);
    bool ok = std::fwrite("MPMS", 1, 4, f) == 4 && std::fwrite(&ver, 4, 1, f) == 1 && std::fwrite(&dim, 4, 1, f) == 1 &&
              std::fwrite(&count, 8, 1, f) == 1 && std::fwrite(ext, 4, 3, f) == 3 && std::fwrite(&h, 8, 1, f) == 1 &&
              std::fwrite(&step, 8, 1, f) == 1;
    for (auto* vec : {&x, &v, &B, &Fe, &Jp})
        ok = ok && std::fwrite(vec->data(), sizeof(float), vec->size(), f) == vec->size();
    ok = ok && std::fwrite(&has_order, 4, 1, f) == 1;
    if (has_order) {
        ok = ok && std::fwrite(ids.data(), sizeof(int), n, f) == n && std::fwrite(&n_extra, 4, 1, f) == 1;
        if (n_extra) ok = ok && std::fwrite(extra.data(), sizeof(int4), extra.size(), f) == extra.size();
    }
    ok = ok && std::fwrite(&has_sums, 4, 1, f) == 1;
    if (has_sums) {
        ok = ok && std::fwrite(sum_hdr, 4, 3, f) == 3 &&
             std::fwrite(sum_blocks.data(), sizeof(int), sum_blocks.size(), f) == sum_blocks.size() &&
             std::fwrite(sums.data(), sizeof(unsigned long long), sums.size(), f) == sums.size();
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? MPM_OK : fail(s, MPM_ERR_IO, "short write");
}

mpm_status mpm_load_state(mpm_solver* s, const char* path) {
    if (!s || !path) return MPM_ERR_INVALID_ARGUMENT;
    // the uploads below replace buffers that work already queued may still read
    MPM_CUDA(s, cudaStreamSynchronize(s->stream));
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(s, MPM_ERR_IO, std::string("cannot open ") + path);
    char magic[4];
    uint32_t ver = 0;
    int32_t dim = 0, ext[3];
    int64_t count = 0, step = 0;
    uint64_t h = 0;
    bool ok = std::fread(magic, 1, 4, f) == 4 && std::fread(&ver, 4, 1, f) == 1 && std::fread(&dim, 4, 1, f) == 1 &&
              std::fread(&count, 8, 1, f) == 1 && std::fread(ext, 4, 3, f) == 3 && std::fread(&h, 8, 1, f) == 1 &&
              std::fread(&step, 8, 1, f) == 1;
    if (!ok || std::memcmp(magic, "MPMS", 4) != 0 || ver < 1 || ver > 3) { std::fclose(f); return fail(s, MPM_ERR_IO, "not a checkpoint"); }
    if (dim != s->dim || count != s->n || ext[0] != s->params.width || ext[1] != s->params.height ||
        (dim == 3 && ext[2] != s->params.depth) || h != params_hash(s->params)) {
        std::fclose(f);
        return fail(s, MPM_ERR_STATE_MISMATCH, "checkpoint was written by a different configuration");
    }
    const int D = s->dim;
    const size_t n = (size_t)count;
    std::vector<float> x(n * D), v(n * D), B(n * D * D), Fe(n * D * D), Jp(n);
    for (auto* vec : {&x, &v, &B, &Fe, &Jp}) ok = ok && std::fread(vec->data(), sizeof(float), vec->size(), f) == vec->size();
    uint32_t has_order = 0;
    std::vector<int> ids;
    int n_extra = 0;
    int sched_K = 0, sched_next = 0, sched_pending = 0;
    std::vector<int4> tiles;                 // {tile, first slot, count} of the last sort (fused path)
    uint32_t has_sums = 0;                   // the pending grid sums (fused path)
    int32_t sum_hdr[3] = {0, 0, 0};
    std::vector<int> sum_blocks;
    std::vector<unsigned long long> sums;
    if (ok && ver >= 2) {
        ok = std::fread(&has_order, 4, 1, f) == 1;
        if (ok && has_order) {
            ids.resize(n);
            ok = std::fread(ids.data(), sizeof(int), n, f) == n && std::fread(&n_extra, 4, 1, f) == 1 && n_extra >= 0 &&
                 (size_t)n_extra <= n + (size_t)s->ti.n_tiles + 1;
            if (ok) {
                std::vector<int4> extra(n_extra);
                ok = std::fread(extra.data(), sizeof(int4), extra.size(), f) == extra.size();
                for (size_t q = 0; ok && q < extra.size(); ++q)
                    if (extra[q].x == kSchedTag && extra[q].y >= 1 && extra[q].y <= mpm_solver::kMaxPeriod &&
                        extra[q].z >= 0 && extra[q].z <= extra[q].y && (extra[q].w & 0xff) <= mpm_solver::kMaxPeriod &&
                        ((extra[q].w >> 8) & 0xff) <= mpm_solver::kMaxPeriod && (extra[q].w >> 16) == 0) {
                        sched_K = extra[q].y;
                        sched_next = extra[q].z;
                        sched_pending = extra[q].w;
                    } else if (extra[q].x == kTileTag) {
                        tiles.push_back(make_int4(extra[q].y, extra[q].z, extra[q].w, 0));
                    }
            }
            // every slot must name a distinct particle
            std::vector<char> seen(ok ? n : 0, 0);
            for (size_t i = 0; ok && i < n; ++i) {
                ok = ids[i] >= 0 && (size_t)ids[i] < n && !seen[ids[i]];
                if (ok) seen[ids[i]] = 1;
            }
        }
    }
    if (ok && ver >= 3) {
        ok = std::fread(&has_sums, 4, 1, f) == 1;
        if (ok && has_sums) {
            const int nb_max = s->ti.n_blocks;
            ok = std::fread(sum_hdr, 4, 3, f) == 3 && sum_hdr[0] == nacc(s->dim, s->form) &&
                 sum_hdr[1] == (s->dim == 3 ? TileGeom<3>::BN : TileGeom<2>::BN) && sum_hdr[2] >= 0 &&
                 sum_hdr[2] <= nb_max;
            if (ok) {
                sum_blocks.resize(sum_hdr[2]);
                sums.resize((size_t)sum_hdr[2] * sum_hdr[0] * sum_hdr[1]);
                ok = std::fread(sum_blocks.data(), sizeof(int), sum_blocks.size(), f) == sum_blocks.size() &&
                     std::fread(sums.data(), sizeof(unsigned long long), sums.size(), f) == sums.size();
                // every block in range and listed once
                std::vector<char> seenb(ok ? (size_t)nb_max : 0, 0);
                for (size_t b = 0; ok && b < sum_blocks.size(); ++b) {
                    ok = sum_blocks[b] >= 0 && sum_blocks[b] < nb_max && !seenb[sum_blocks[b]];
                    if (ok) seenb[sum_blocks[b]] = 1;
                }
            }
        }
    }
    std::fclose(f);
    if (!ok) return fail(s, MPM_ERR_IO, "truncated or corrupt checkpoint");
    const bool restore_order = has_order && s->tiled;
    if (restore_order && n > 0)
        MPM_CUDA(s, cudaMemcpy(s->id, ids.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    mpm_state_host st{(int64_t)n, x.data(), v.data(), B.data(), Fe.data(), Jp.data()};
    mpm_status r = mpm_set_state(s, &st);
    if (r != MPM_OK) return r;
    if (restore_order) {
        s->needs_sort = false;
    }
    if (restore_order && s->fused && n > 0) {
        // the fused kernel walks the tiles of the last sort: restore them when
        // the records are complete (disjoint, in slot order, covering every
        // slot, tiles in range), else sort again (the run then continues
        // correctly but no longer bit-identically)
        std::sort(tiles.begin(), tiles.end(), [](const int4& a, const int4& b) { return a.y < b.y; });
        bool good = !tiles.empty();
        long long next = 0;
        for (size_t e = 0; good && e < tiles.size(); ++e) {
            good = tiles[e].x >= 0 && tiles[e].x < s->ti.n_tiles && tiles[e].y == next && tiles[e].z >= 1 &&
                   (long long)tiles[e].y + tiles[e].z <= (long long)n && (e == 0 || tiles[e].x > tiles[e - 1].x);
            next += tiles[e].z;
        }
        good = good && next == (long long)n;
        if (good) {
            const int ntl = (int)tiles.size();
            std::vector<int> tl(ntl), tlen(ntl), tstart(s->ti.n_tiles, 0);
            for (int e = 0; e < ntl; ++e) { tl[e] = tiles[e].x; tlen[e] = tiles[e].z; tstart[tiles[e].x] = tiles[e].y; }
            // on the solver's stream, after the clear of the flags that mpm_set_state queued there
            cudaStream_t st = s->stream;
            MPM_CUDA(s, cudaMemcpyAsync(s->ti.tile_list, tl.data(), sizeof(int) * ntl, cudaMemcpyHostToDevice, st));
            MPM_CUDA(s, cudaMemcpyAsync(s->ti.tile_len, tlen.data(), sizeof(int) * ntl, cudaMemcpyHostToDevice, st));
            MPM_CUDA(s, cudaMemcpyAsync(s->ti.tile_start, tstart.data(), sizeof(int) * s->ti.n_tiles,
                                        cudaMemcpyHostToDevice, st));
            MPM_CUDA(s, cudaMemcpyAsync(s->ti.n_tile_list, &ntl, sizeof(int), cudaMemcpyHostToDevice, st));
            if (has_sums) {
                // the next step's grid sums as the saved run held them: into the
                // (cleared) accumulators, their blocks marked for the grid update
                const int nb = sum_hdr[2];
                if (nb > 0) {
                    const size_t words = sums.size() + ((size_t)nb + 1) / 2;
                    mpm_status es = ensure_staging(s, words * 2);
                    if (es != MPM_OK) return es;
                    unsigned long long* din = reinterpret_cast<unsigned long long*>(s->staging);
                    int* dblk = reinterpret_cast<int*>(din + sums.size());
                    MPM_CUDA(s, cudaMemcpyAsync(din, sums.data(), sizeof(unsigned long long) * sums.size(),
                                                cudaMemcpyHostToDevice, st));
                    MPM_CUDA(s, cudaMemcpyAsync(dblk, sum_blocks.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, st));
                    if (s->dim == 3)
                        k_unpack_marked<3><<<s->sms * 4, 256, 0, st>>>(s->C, s->ti, sum_hdr[0], nb, dblk, din, s->acc);
                    else
                        k_unpack_marked<2><<<s->sms * 4, 256, 0, st>>>(s->C, s->ti, sum_hdr[0], nb, dblk, din, s->acc);
                    MPM_CUDA(s, cudaGetLastError());
                }
                MPM_CUDA(s, cudaMemcpyAsync(s->ti.n_marked, &sum_hdr[2], sizeof(int), cudaMemcpyHostToDevice, st));
                s->acc_pending = true;
                s->needs_affine = false;
            }
            MPM_CUDA(s, cudaStreamSynchronize(st));
        } else {
            s->needs_sort = true;
        }
    }
    s->step = step;
    if (s->auto_sort) {  // resume the saved sort schedule (else sort at the next step)
        s->cur_K = sched_K > 0 ? sched_K : s->cur_K;
        s->next_sort = sched_K > 0 ? step + sched_next : step;
        const int ka = sched_pending & 0xff, kb = (sched_pending >> 8) & 0xff;
        s->nplan = (sched_K > 0 && ka > 0 && kb > 0) ? 2 : 0;
        s->plan[0] = {ka, 0};
        s->plan[1] = {kb, 0};
    }
    return MPM_OK;
}

// ---------------------------------------------------------------------------
// Learned plasticity surrogate.

int32_t mpm_mlp_param_count(void) { return MlpOff::total; }

}  // extern "C"

namespace {
// The network's buffers live on the device that was current at
// mpm_mlp_create; a kernel launched with another device current would be
// handed pointers it cannot address. Refuse before any copy or launch.
bool mlp_device_current(mpm_mlp* m, const char* who) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        m->err = std::string(who) + ": no usable current device";
        return false;
    }
    if (dev != m->device) {
        m->err = std::string(who) + ": the network lives on device " + std::to_string(m->device) + " but device " +
                 std::to_string(dev) + " is current";
        return false;
    }
    return true;
}
}  // namespace

extern "C" {

mpm_status mpm_mlp_create(uint64_t seed, mpm_mlp** out) {
    if (!out) return MPM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return MPM_ERR_NO_DEVICE; }
    mpm_mlp* m = new mpm_mlp();
    cudaGetDevice(&m->device);
    const int P = MlpOff::total;
    if (dalloc(&m->w, P) || dalloc(&m->wbf, P) || dalloc(&m->grad, P) || dalloc(&m->m1, P) || dalloc(&m->m2, P)) {
        mpm_mlp_destroy(m);
        return MPM_ERR_OUT_OF_MEMORY;
    }
    // uniform initialisation with variance 1/fan_in (output layer x0.1), zero biases and padding
    std::vector<float> w(P, 0.f);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> U(-1.f, 1.f);
    auto fill = [&](int off, int rows, int cols, int used_rows, int used_cols, float gain) {
        const float a = gain * std::sqrt(3.f / float(used_cols));
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c) w[off + r * cols + c] = (r < used_rows && c < used_cols) ? a * U(rng) : 0.f;
    };
    fill(MlpOff::W1, kMlpHid, kMlpInPad, kMlpHid, kMlpIn, 1.f);
    fill(MlpOff::W2, kMlpHid, kMlpHid, kMlpHid, kMlpHid, 1.f);
    fill(MlpOff::W3, kMlpHid, kMlpHid, kMlpHid, kMlpHid, 1.f);
    fill(MlpOff::W4, kMlpOutPad, kMlpHid, kMlpOut, kMlpHid, 0.1f);
    for (int k = 0; k < kMlpIn; ++k) { m->norm.in_mean[k] = 0.f; m->norm.in_std[k] = 1.f; }
    for (int k = 0; k < kMlpOut; ++k) { m->norm.out_mean[k] = 0.f; m->norm.out_std[k] = 1.f; }
    mpm_status st = mpm_mlp_set_params(m, w.data(), (size_t)P);
    if (st != MPM_OK) { mpm_mlp_destroy(m); return st; }
    *out = m;
    return MPM_OK;
}

mpm_status mpm_mlp_destroy(mpm_mlp* m) {
    if (!m) return MPM_ERR_INVALID_ARGUMENT;
    void* ptrs[] = {m->w, m->wbf, m->grad, m->m1, m->m2, m->loss, m->pairs};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete m;
    return MPM_OK;
}

const char* mpm_mlp_last_error(const mpm_mlp* m) { return m ? m->err.c_str() : "null network"; }

mpm_status mpm_mlp_set_params(mpm_mlp* m, const float* params, size_t count) {
    if (!m || !params || count != (size_t)MlpOff::total) return MPM_ERR_INVALID_ARGUMENT;
    std::vector<__nv_bfloat16> b(count);
    for (size_t i = 0; i < count; ++i) b[i] = __float2bfloat16_rn(params[i]);
    if (cudaMemcpy(m->w, params, sizeof(float) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->wbf, b.data(), sizeof(__nv_bfloat16) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(m->grad, 0, sizeof(float) * count) != cudaSuccess ||
        cudaMemset(m->m1, 0, sizeof(float) * count) != cudaSuccess ||
        cudaMemset(m->m2, 0, sizeof(float) * count) != cudaSuccess) {
        cudaGetLastError();
        m->err = "parameter upload failed";
        return MPM_ERR_CUDA;
    }
    m->step = 0;
    return MPM_OK;
}

mpm_status mpm_mlp_get_params(mpm_mlp* m, float* out, size_t cap) {
    if (!m || !out) return MPM_ERR_INVALID_ARGUMENT;
    if (cap < (size_t)MlpOff::total) return MPM_ERR_CAPACITY;
    if (cudaMemcpy(out, m->w, sizeof(float) * MlpOff::total, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return MPM_ERR_CUDA;
    }
    return MPM_OK;
}

mpm_status mpm_mlp_set_normalization(mpm_mlp* m, const float* in_mean, const float* in_std, const float* out_mean,
                                     const float* out_std) {
    if (!m || !in_mean || !in_std || !out_mean || !out_std) return MPM_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < kMlpIn; ++k) {
        if (!(in_std[k] > 0.f)) return MPM_ERR_INVALID_ARGUMENT;
        m->norm.in_mean[k] = in_mean[k];
        m->norm.in_std[k] = in_std[k];
    }
    for (int k = 0; k < kMlpOut; ++k) {
        if (!(out_std[k] > 0.f)) return MPM_ERR_INVALID_ARGUMENT;
        m->norm.out_mean[k] = out_mean[k];
        m->norm.out_std[k] = out_std[k];
    }
    return MPM_OK;
}

mpm_status mpm_mlp_load_pairs(mpm_mlp* m, const float* pairs, int64_t n) {
    if (!m || n < 0 || (n > 0 && !pairs)) return MPM_ERR_INVALID_ARGUMENT;
    if (m->pairs) cudaFree(m->pairs);
    m->pairs = nullptr;
    m->n_pairs = 0;
    if (n == 0) return MPM_OK;
    if (dalloc(&m->pairs, (size_t)n * 20)) { cudaGetLastError(); return MPM_ERR_OUT_OF_MEMORY; }
    if (cudaMemcpy(m->pairs, pairs, sizeof(float) * 20 * (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        return MPM_ERR_CUDA;
    }
    m->n_pairs = n;
    return MPM_OK;
}

static mpm_status mlp_launch_grad(mpm_mlp* m, const float* dpairs, long long np, const int* didx, int rows,
                                  unsigned seed, float* dloss) {
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpTrainSmem)) !=
            cudaSuccess) {
            cudaGetLastError();
            return MPM_ERR_CUDA;
        }
        attr = true;
    }
    const int blocks = (rows + kMlpTrainRows - 1) / kMlpTrainRows;
    k_mlp_train<<<blocks, 128, sizeof(MlpTrainSmem)>>>(dpairs, np, didx, rows, seed, m->wbf, m->w, m->norm, m->grad,
                                                        dloss);
    return cudaGetLastError() == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
}

mpm_status mpm_mlp_train(mpm_mlp* m, int32_t steps, int32_t batch, float lr, float weight_decay, uint32_t seed,
                         float* loss_out) {
    if (!m || steps < 0 || batch < 1) return MPM_ERR_INVALID_ARGUMENT;
    if (m->n_pairs <= 0) { m->err = "no training pairs loaded"; return MPM_ERR_INVALID_ARGUMENT; }
    if (steps > m->loss_cap) {
        if (m->loss) cudaFree(m->loss);
        m->loss = nullptr;
        if (dalloc(&m->loss, (size_t)steps)) { cudaGetLastError(); return MPM_ERR_OUT_OF_MEMORY; }
        m->loss_cap = steps;
    }
    if (cudaMemset(m->loss, 0, sizeof(float) * steps) != cudaSuccess) return MPM_ERR_CUDA;
    const float b1 = 0.9f, b2 = 0.999f;
    for (int it = 0; it < steps; ++it) {
        // cosine decay to lr / 20
        const float frac = steps > 1 ? float(it) / float(steps - 1) : 0.f;
        const float lr_t = lr * (0.05f + 0.95f * 0.5f * (1.f + std::cos(3.14159265f * frac)));
        mpm_status st = mlp_launch_grad(m, m->pairs, m->n_pairs, nullptr, batch, seed * 2654435761u + (unsigned)it,
                                        m->loss + it);
        if (st != MPM_OK) return st;
        ++m->step;
        const float bc1 = 1.f - std::pow(b1, (float)m->step), bc2 = 1.f - std::pow(b2, (float)m->step);
        k_mlp_adam<<<(MlpOff::total + 255) / 256, 256>>>(m->w, m->wbf, m->grad, m->m1, m->m2, lr_t, b1, b2, 1e-8f,
                                                          weight_decay, bc1, bc2);
        if (cudaGetLastError() != cudaSuccess) return MPM_ERR_CUDA;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) { cudaGetLastError(); return MPM_ERR_CUDA; }
    if (loss_out && steps > 0 &&
        cudaMemcpy(loss_out, m->loss, sizeof(float) * steps, cudaMemcpyDeviceToHost) != cudaSuccess)
        return MPM_ERR_CUDA;
    return MPM_OK;
}

mpm_status mpm_mlp_gradient(mpm_mlp* m, const float* pairs, int64_t n, float* grad_out, float* loss_out) {
    if (!m || !pairs || n < 1 || n > (1 << 24) || !grad_out) return MPM_ERR_INVALID_ARGUMENT;
    float *dp = nullptr, *dl = nullptr;
    int* di = nullptr;
    std::vector<int> idx((size_t)n);
    for (int64_t i = 0; i < n; ++i) idx[i] = (int)i;
    mpm_status st = MPM_OK;
    if (dalloc(&dp, (size_t)n * 20) || dalloc(&dl, 1) || dalloc(&di, (size_t)n)) st = MPM_ERR_OUT_OF_MEMORY;
    if (st == MPM_OK && (cudaMemcpy(dp, pairs, sizeof(float) * 20 * n, cudaMemcpyHostToDevice) != cudaSuccess ||
                         cudaMemcpy(di, idx.data(), sizeof(int) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
                         cudaMemset(dl, 0, sizeof(float)) != cudaSuccess ||
                         cudaMemset(m->grad, 0, sizeof(float) * MlpOff::total) != cudaSuccess))
        st = MPM_ERR_CUDA;
    if (st == MPM_OK) st = mlp_launch_grad(m, dp, n, di, (int)n, 0u, dl);
    if (st == MPM_OK && cudaDeviceSynchronize() != cudaSuccess) st = MPM_ERR_CUDA;
    if (st == MPM_OK && cudaMemcpy(grad_out, m->grad, sizeof(float) * MlpOff::total, cudaMemcpyDeviceToHost) != cudaSuccess)
        st = MPM_ERR_CUDA;
    if (st == MPM_OK && loss_out && cudaMemcpy(loss_out, dl, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        st = MPM_ERR_CUDA;
    cudaMemset(m->grad, 0, sizeof(float) * MlpOff::total);
    if (dp) cudaFree(dp);
    if (dl) cudaFree(dl);
    if (di) cudaFree(di);
    cudaGetLastError();
    return st;
}

mpm_status mpm_mlp_predict(mpm_mlp* m, const float* inputs, int64_t n, int32_t stride, float* out) {
    if (!m || !inputs || !out || n < 1 || stride < 10 || n > (1 << 26)) return MPM_ERR_INVALID_ARGUMENT;
    if (!mlp_device_current(m, "mpm_mlp_predict")) return MPM_ERR_INVALID_ARGUMENT;
    float *di = nullptr, *dout = nullptr;
    mpm_status st = MPM_OK;
    if (dalloc(&di, (size_t)n * stride) || dalloc(&dout, (size_t)n * kMlpOut)) st = MPM_ERR_OUT_OF_MEMORY;
    if (st == MPM_OK && cudaMemcpy(di, inputs, sizeof(float) * n * stride, cudaMemcpyHostToDevice) != cudaSuccess)
        st = MPM_ERR_CUDA;
    if (st == MPM_OK) {
        const long long rows = kMlpWarps * 32;
        if (mlp_kernel_attrs() != cudaSuccess) st = MPM_ERR_CUDA;
        else
            k_mlp_forward<<<(unsigned)((n + rows - 1) / rows), kMlpWarps * 32, sizeof(MlpWarpSmem)>>>(
                di, stride, (int)n, m->wbf, m->w, m->norm, dout);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) st = MPM_ERR_CUDA;
    }
    if (st == MPM_OK && cudaMemcpy(out, dout, sizeof(float) * n * kMlpOut, cudaMemcpyDeviceToHost) != cudaSuccess)
        st = MPM_ERR_CUDA;
    if (di) cudaFree(di);
    if (dout) cudaFree(dout);
    cudaGetLastError();
    return st;
}

mpm_status mpm_set_plasticity(mpm_solver* s, int32_t mode, mpm_mlp* mlp, float tolerance) {
    if (!s) return MPM_ERR_INVALID_ARGUMENT;
    if (mode != MPM_PLASTIC_EXACT && mode != MPM_PLASTIC_MLP) return fail(s, MPM_ERR_INVALID_ARGUMENT, "unknown plasticity mode");
    if (mode == MPM_PLASTIC_MLP) {
        if (!mlp) return fail(s, MPM_ERR_INVALID_ARGUMENT, "MLP plasticity needs a network");
        if (s->dim != 3 || !s->tiled || s->stencil != 4)
            return fail(s, MPM_ERR_UNSUPPORTED, "the learned return map is 3D MLS (cubic stencil) only");
        if (!(tolerance > 0.f)) return fail(s, MPM_ERR_INVALID_ARGUMENT, "tolerance must be > 0");
        MPM_CUDA(s, mlp_kernel_attrs());
        if (!s->mlp_counters) {
            MPM_CUDA(s, dalloc(&s->mlp_counters, 2));
            MPM_CUDA(s, cudaMemset(s->mlp_counters, 0, 2 * sizeof(unsigned long long)));
        }
        s->mlp_tol = tolerance;
    }
    invalidate_graphs(s);
    s->plasticity = mode;
    s->mlp = mode == MPM_PLASTIC_MLP ? mlp : nullptr;
    return MPM_OK;
}

mpm_status mpm_get_mlp_stats(mpm_solver* s, uint64_t* accepted, uint64_t* rejected) {
    if (!s) return MPM_ERR_INVALID_ARGUMENT;
    unsigned long long h[2] = {0, 0};
    if (s->mlp_counters) {
        MPM_CUDA(s, cudaMemcpyAsync(h, s->mlp_counters, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
        MPM_CUDA(s, cudaStreamSynchronize(s->stream));
    }
    if (accepted) *accepted = h[0];
    if (rejected) *rejected = h[1];
    return MPM_OK;
}

mpm_status mpm_pair_log_enable(mpm_solver* s, int64_t capacity) {
    if (!s || capacity < 0) return MPM_ERR_INVALID_ARGUMENT;
    if (s->dim != 3 || !s->tiled) return fail(s, MPM_ERR_UNSUPPORTED, "pair logging is 3D MLS only");
    invalidate_graphs(s);
    if (s->log_data) cudaFree(s->log_data);
    s->log_data = nullptr;
    s->log_cap = 0;
    if (capacity == 0) return MPM_OK;
    if (!s->log_n) MPM_CUDA(s, dalloc(&s->log_n, 1));
    MPM_CUDA(s, dalloc(&s->log_data, (size_t)capacity * 20));
    MPM_CUDA(s, cudaMemset(s->log_n, 0, sizeof(unsigned long long)));
    s->log_cap = capacity;
    return MPM_OK;
}

mpm_status mpm_pair_log_read(mpm_solver* s, float* out, int64_t cap_pairs, int64_t* n_pairs) {
    if (!s || !n_pairs || cap_pairs < 0 || (cap_pairs > 0 && !out)) return MPM_ERR_INVALID_ARGUMENT;
    unsigned long long n = 0;
    if (s->log_n) {
        MPM_CUDA(s, cudaMemcpyAsync(&n, s->log_n, sizeof(n), cudaMemcpyDeviceToHost, s->stream));
        MPM_CUDA(s, cudaStreamSynchronize(s->stream));
    }
    const long long avail = (long long)n < s->log_cap ? (long long)n : s->log_cap;
    const long long take = avail < cap_pairs ? avail : cap_pairs;
    if (take > 0)
        MPM_CUDA(s, cudaMemcpy(out, s->log_data, sizeof(float) * 20 * (size_t)take, cudaMemcpyDeviceToHost));
    if (s->log_n) MPM_CUDA(s, cudaMemset(s->log_n, 0, sizeof(unsigned long long)));
    *n_pairs = take;
    return MPM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Headless frames (Visualize + saveFrame, src/main.cpp:51-205).
namespace {

void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

void normalise3(double* v) {
    const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (l > 0) for (int k = 0; k < 3; ++k) v[k] /= l;
}

// Host copy of render_project (for the line sample counts).
bool host_project(const RenderView& V, const float* p, double& px, double& py) {
    if (V.dim == 2) {
        px = p[0] * V.sx;
        py = V.height - p[1] * V.sy;
        return true;
    }
    double d[3], xv = 0, yv = 0, w = 0;
    for (int k = 0; k < 3; ++k) d[k] = p[k] - V.eye[k];
    for (int k = 0; k < 3; ++k) { xv += V.s[k] * d[k]; yv += V.u[k] * d[k]; w += V.f[k] * d[k]; }
    if (!(w >= V.znear && w <= V.zfar)) return false;
    px = (V.px_scale * xv / w + 1.0) * 0.5 * V.width;
    py = V.height - (V.py_scale * yv / w + 1.0) * 0.5 * V.height;
    return true;
}

}  // namespace

extern "C" {

void mpm_render_params_default(mpm_render_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->width = 1200;   // WINDOW_WIDTH (Parameters.h:64)
    p->height = 600;   // WINDOW_HEIGHT (Parameters.h:65)
    p->point_size = 1.f;           // PARTICLE_SIZE (Parameters.h:73)
    p->camera_angle = 0.f;         // main.cpp:51-53
    p->camera_elevation = 30.f;
    p->camera_distance = 300.f;
    p->fov_degrees = 45.f;         // main.cpp:61
}

mpm_status mpm_render(mpm_solver* s, const mpm_render_params* p, uint8_t* rgb, size_t cap_bytes) {
    if (!s || !p || !rgb) return MPM_ERR_INVALID_ARGUMENT;
    if (p->width < 1 || p->height < 1 || p->width > 16384 || p->height > 16384 || !(p->point_size > 0.f) ||
        !(p->point_size <= 64.f) || !(p->fov_degrees > 0.f && p->fov_degrees < 180.f) || !(p->camera_distance > 0.f))
        return fail(s, MPM_ERR_INVALID_ARGUMENT, "bad render parameters");
    const long long pixels = (long long)p->width * p->height;
    if (cap_bytes < (size_t)pixels * 3) return fail(s, MPM_ERR_CAPACITY, "image buffer smaller than width * height * 3");
    if (pixels > s->render_pixels) {
        if (s->render_fb) cudaFree(s->render_fb);
        if (s->render_rgb) cudaFree(s->render_rgb);
        s->render_fb = nullptr;
        s->render_rgb = nullptr;
        s->render_pixels = 0;
        MPM_CUDA(s, dalloc(&s->render_fb, (size_t)pixels));
        MPM_CUDA(s, dalloc(&s->render_rgb, (size_t)pixels * 3));
        s->render_pixels = pixels;
    }
    RenderView V{};
    V.dim = s->dim;
    V.width = p->width;
    V.height = p->height;
    V.radius = 0.5f * p->point_size;
    const float m = (float)s->params.border_margin, W = (float)s->params.width, H = (float)s->params.height,
                Dp = s->dim == 3 ? (float)s->params.depth : 0.f;
    RenderLines L{};
    if (s->dim == 2) {  // glOrtho(0, WIDTH, 0, HEIGHT) onto the window (main.cpp:260-261)
        V.sx = (float)p->width / W;
        V.sy = (float)p->height / H;
        const float c[4][3] = {{m, m, 0}, {W - m, m, 0}, {W - m, H - m, 0}, {m, H - m, 0}};
        for (int k = 0; k < 4; ++k)
            for (int c3 = 0; c3 < 3; ++c3) { L.a[k][c3] = c[k][c3]; L.b[k][c3] = c[(k + 1) % 4][c3]; }
        L.count = 4;
    } else {  // SetupCamera (main.cpp:56-80)
        const double center[3] = {0.5 * W, 0.5 * H, 0.5 * Dp};
        const double rad = p->camera_angle * M_PI / 180.0, elev = p->camera_elevation * M_PI / 180.0;
        const double eye[3] = {center[0] + p->camera_distance * std::cos(elev) * std::sin(rad),
                               center[1] + p->camera_distance * std::sin(elev),
                               center[2] + p->camera_distance * std::cos(elev) * std::cos(rad)};
        double f[3] = {center[0] - eye[0], center[1] - eye[1], center[2] - eye[2]};
        normalise3(f);
        const double up[3] = {0, 1, 0};
        double sv[3], u[3];
        cross3(f, up, sv);
        normalise3(sv);
        cross3(sv, f, u);
        const double t = std::tan(0.5 * p->fov_degrees * M_PI / 180.0), aspect = (double)p->width / p->height;
        for (int k = 0; k < 3; ++k) {
            V.eye[k] = (float)eye[k];
            V.f[k] = (float)f[k];
            V.s[k] = (float)sv[k];
            V.u[k] = (float)u[k];
        }
        V.px_scale = (float)(1.0 / (aspect * t));
        V.py_scale = (float)(1.0 / t);
        V.znear = 1.f;
        V.zfar = 1000.f;
        // wireframe box (main.cpp:85-111): bottom, top, pillars
        const float x0 = m, y0 = m, z0 = m, x1 = W - m, y1 = H - m, z1 = Dp - m;
        const float e[12][6] = {{x0, y0, z0, x1, y0, z0}, {x1, y0, z0, x1, y0, z1}, {x1, y0, z1, x0, y0, z1},
                                {x0, y0, z1, x0, y0, z0}, {x0, y1, z0, x1, y1, z0}, {x1, y1, z0, x1, y1, z1},
                                {x1, y1, z1, x0, y1, z1}, {x0, y1, z1, x0, y1, z0}, {x0, y0, z0, x0, y1, z0},
                                {x1, y0, z0, x1, y1, z0}, {x1, y0, z1, x1, y1, z1}, {x0, y0, z1, x0, y1, z1}};
        for (int k = 0; k < 12; ++k)
            for (int c3 = 0; c3 < 3; ++c3) { L.a[k][c3] = e[k][c3]; L.b[k][c3] = e[k][3 + c3]; }
        L.count = 12;
    }
    for (int k = 0; k < L.count; ++k) {
        double ax, ay, bx, by;
        if (host_project(V, L.a[k], ax, ay) && host_project(V, L.b[k], bx, by)) {
            const double len = std::sqrt((bx - ax) * (bx - ax) + (by - ay) * (by - ay));
            L.samples[k] = (int)std::min(65536.0, std::ceil(2.0 * len) + 1.0);
        } else {
            L.samples[k] = 4096;
        }
    }
    const int threads = 256;
    const unsigned pblocks = (unsigned)((pixels + threads - 1) / threads);
    k_render_clear<<<pblocks, threads, 0, s->stream>>>(s->render_fb, pixels);
    k_render_lines<<<L.count, threads, 0, s->stream>>>(V, L, s->render_fb);
    if (s->n > 0)
        k_render_points<<<(s->n + threads - 1) / threads, threads, 0, s->stream>>>(V, s->x, s->n, s->render_fb);
    k_render_pack<<<pblocks, threads, 0, s->stream>>>(s->render_fb, pixels, s->render_rgb);
    MPM_CUDA(s, cudaGetLastError());
    MPM_CUDA(s, cudaMemcpyAsync(rgb, s->render_rgb, (size_t)pixels * 3, cudaMemcpyDeviceToHost, s->stream));
    MPM_CUDA(s, cudaStreamSynchronize(s->stream));
    return MPM_OK;
}

}  // extern "C"


// ---------------------------------------------------------------------------
// Inference without allocation: fixed scratch in the device image.
constexpr int kNoallocRows = MPM_MLP_NOALLOC_MAX_ROWS;
// [rows][kMlpIn] staged inputs, then [rows][kMlpOut] outputs. Host code sees
// only a stand-in under this name; kernels get the device address that
// cudaGetSymbolAddress returns.
static __device__ __align__(256) float g_noalloc_scratch[(size_t)kNoallocRows * (kMlpIn + kMlpOut)];
namespace {
constexpr int kNoallocMaxDevices = 64;
// Per device: the scratch address and a non-blocking stream of its own (so a
// call neither waits for nor holds up work on the legacy default stream).
// Set up under the mutex on the first call that succeeds; a failed set-up is
// not remembered, so a later call tries again.
struct NoallocDevice {
    float* scratch = nullptr;
    cudaStream_t stream = nullptr;
    bool ready = false;
};
NoallocDevice g_noalloc[kNoallocMaxDevices];
std::mutex g_noalloc_mutex;

cudaError_t noalloc_setup(int dev) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoallocDevice& d = g_noalloc[dev];
    if (d.ready) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    if (!d.scratch) e = cudaGetSymbolAddress(reinterpret_cast<void**>(&d.scratch), g_noalloc_scratch);
    if (e == cudaSuccess) e = mlp_kernel_attrs();
    if (e == cudaSuccess && !d.stream) e = cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e;
    }
    d.ready = true;
    return cudaSuccess;
}
}  // namespace

extern "C" {

mpm_status mpm_mlp_predict_noalloc(mpm_mlp* m, const float* inputs, int64_t n, int32_t stride, float* out) {
    if (!m || !inputs || !out || n < 1 || stride < kMlpIn) return MPM_ERR_INVALID_ARGUMENT;
    if (n > kNoallocRows) {
        m->err = "mpm_mlp_predict_noalloc: n = " + std::to_string(n) + " exceeds the scratch capacity of " +
                 std::to_string(kNoallocRows) + " rows";
        return MPM_ERR_CAPACITY;
    }
    if (!mlp_device_current(m, "mpm_mlp_predict_noalloc")) return MPM_ERR_INVALID_ARGUMENT;
    const int dev = m->device;
    if (dev < 0 || dev >= kNoallocMaxDevices) {
        m->err = "mpm_mlp_predict_noalloc: device ordinal beyond the supported range";
        return MPM_ERR_UNSUPPORTED;
    }
    cudaError_t e = noalloc_setup(dev);
    if (e != cudaSuccess) {
        m->err = std::string("mpm_mlp_predict_noalloc: scratch set-up failed: ") + cudaGetErrorString(e);
        return MPM_ERR_CUDA;
    }
    const NoallocDevice& d = g_noalloc[dev];
    float* din = d.scratch;
    float* dout = din + (size_t)kNoallocRows * kMlpIn;
    e = cudaMemcpy2DAsync(din, sizeof(float) * kMlpIn, inputs, sizeof(float) * (size_t)stride, sizeof(float) * kMlpIn,
                          (size_t)n, cudaMemcpyHostToDevice, d.stream);
    if (e == cudaSuccess) {
        const int64_t rows = kMlpWarps * 32;
        k_mlp_forward<<<(unsigned)((n + rows - 1) / rows), kMlpWarps * 32, sizeof(MlpWarpSmem), d.stream>>>(
            din, kMlpIn, (int)n, m->wbf, m->w, m->norm, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, dout, sizeof(float) * kMlpOut * (size_t)n, cudaMemcpyDeviceToHost, d.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(d.stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        m->err = std::string("mpm_mlp_predict_noalloc: ") + cudaGetErrorString(e);
        return MPM_ERR_CUDA;
    }
    return MPM_OK;
}

}  // extern "C"
