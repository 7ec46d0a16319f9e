// hhs_api.cu -- C ABI: particle systems, the context, the reference-shaped entry
// points (timesteps / split / kick_slow / kick_sf / drift / update_system) and the
// host-driven HOLD schedule.
#include <atomic>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "hhs_ctx.h"
#include "hhs_kernels.h"

namespace {

constexpr size_t kAlign = 256;
inline size_t align_up(size_t v) { return (v + kAlign - 1) & ~(kAlign - 1); }

SoA soa_of(const hhs_particle_system* s) {
    SoA r;
    r.x = s->x; r.y = s->y; r.z = s->z;
    r.vx = s->vx; r.vy = s->vy; r.vz = s->vz;
    r.m = s->m; r.ts = s->ts; r.id = s->id;
    return r;
}

bool sys_ok(const hhs_particle_system* s) { return s && s->_base && s->n > 0; }

// (de)interleave vec3<double> arrays through the acc region (3n contiguous doubles)
__global__ void k_deinterleave(const double* __restrict__ v3, double* __restrict__ x,
                               double* __restrict__ y, double* __restrict__ z, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = v3[3 * (size_t)i];
        y[i] = v3[3 * (size_t)i + 1];
        z[i] = v3[3 * (size_t)i + 2];
    }
}

__global__ void k_interleave(double* __restrict__ v3, const double* __restrict__ x,
                             const double* __restrict__ y, const double* __restrict__ z,
                             int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        v3[3 * (size_t)i] = x[i];
        v3[3 * (size_t)i + 1] = y[i];
        v3[3 * (size_t)i + 2] = z[i];
    }
}

inline int small_grid(int n) {
    int g = (n + 255) / 256;
    return g < 1 ? 1 : (g > 1184 ? 1184 : g);
}

}  // namespace

static std::atomic<unsigned long long> g_launches{0};
void hhs_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
extern "C" uint64_t hhs_kernel_launch_count(void) { return g_launches.load(); }

// Event profiler of the host-driven schedule: an event pair around each timed launch,
// resolved when the profile is read.
struct Profiler {
    struct Rec {
        int kind;
        cudaEvent_t a, b;
        double pairs;
    };
    bool on = false;
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    hhs_profile acc{};
    cudaEvent_t get() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void begin(Rec& r, int kind, double pairs, cudaStream_t s) {
        r.kind = kind; r.pairs = pairs; r.a = get(); r.b = get();
        cudaEventRecord(r.a, s);
    }
    void end(Rec& r, cudaStream_t s) {
        cudaEventRecord(r.b, s);
        pending.push_back(r);
    }
    void resolve() {
        for (auto& r : pending) {
            float ms = 0.f;
            cudaEventSynchronize(r.b);
            cudaEventElapsedTime(&ms, r.a, r.b);
            acc.launches[r.kind] += 1;
            acc.ms[r.kind] += ms;
            acc.pairs[r.kind] += r.pairs;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        pending.clear();
    }
    ~Profiler() {
        resolve();
        for (auto e : pool) cudaEventDestroy(e);
    }
};

extern "C" const char* hhs_status_string(hhs_status s) {
    switch (s) {
        case HHS_OK: return "HHS_OK";
        case HHS_ERR_INVALID_ARG: return "HHS_ERR_INVALID_ARG";
        case HHS_ERR_CUDA: return "HHS_ERR_CUDA";
        case HHS_ERR_OOM: return "HHS_ERR_OOM";
        case HHS_ERR_TIMEOUT: return "HHS_ERR_TIMEOUT";
        case HHS_ERR_DEVICE_FAULT_FLAG: return "HHS_ERR_DEVICE_FAULT_FLAG";
        case HHS_ERR_DEPTH: return "HHS_ERR_DEPTH";
        case HHS_ERR_CAPACITY: return "HHS_ERR_CAPACITY";
        case HHS_ERR_PEER: return "HHS_ERR_PEER";
    }
    return "HHS_ERR_UNKNOWN";
}

// ------------------------------------------------------------------ particle systems
namespace {
// One device allocation per system: x y z vx vy vz ts m, then ax ay az (3n contiguous
// doubles), id, parent_id, each array 256-byte aligned. A peer mapping of the
// allocation (hhs_ipc_open) is laid out by the same function.
size_t system_bytes(int32_t n) {
    const size_t dbl = align_up(sizeof(double) * (size_t)n);
    const size_t acc3 = align_up(sizeof(double) * 3 * (size_t)n);
    const size_t i32 = align_up(sizeof(int32_t) * (size_t)n);
    return 8 * dbl + acc3 + 2 * i32;
}
void lay_out_system(hhs_particle_system* sys, void* base, int32_t n) {
    const size_t dbl = align_up(sizeof(double) * (size_t)n);
    const size_t acc3 = align_up(sizeof(double) * 3 * (size_t)n);
    const size_t i32 = align_up(sizeof(int32_t) * (size_t)n);
    char* p = static_cast<char*>(base);
    double** f[8] = {&sys->x, &sys->y, &sys->z, &sys->vx, &sys->vy, &sys->vz, &sys->ts, &sys->m};
    for (int k = 0; k < 8; k++) { *f[k] = reinterpret_cast<double*>(p); p += dbl; }
    sys->ax = reinterpret_cast<double*>(p);  // ax, ay, az contiguous: 3n doubles
    sys->ay = sys->ax + n;
    sys->az = sys->ax + 2 * (size_t)n;
    p += acc3;
    sys->id = reinterpret_cast<int32_t*>(p); p += i32;
    sys->parent_id = reinterpret_cast<int32_t*>(p);
    sys->n = n;
    sys->_base = base;
}
}  // namespace

extern "C" hhs_status hhs_particle_system_alloc(hhs_particle_system* sys, int32_t n) {
    if (!sys || n <= 0) return HHS_ERR_INVALID_ARG;
    std::memset(sys, 0, sizeof(*sys));
    const size_t total = system_bytes(n);
    void* base = nullptr;
    cudaError_t e = cudaMalloc(&base, total);
    if (e != cudaSuccess) return hhs_from_cuda(e);
    lay_out_system(sys, base, n);
    e = cudaMemset(base, 0, total);
    if (e != cudaSuccess) { cudaFree(base); std::memset(sys, 0, sizeof(*sys)); return hhs_from_cuda(e); }
    return HHS_OK;
}

extern "C" hhs_status hhs_particle_system_free(hhs_particle_system* sys) {
    if (!sys) return HHS_ERR_INVALID_ARG;
    if (sys->_base) {
        cudaError_t e = cudaFree(sys->_base);
        std::memset(sys, 0, sizeof(*sys));
        if (e != cudaSuccess) return hhs_from_cuda(e);
    }
    return HHS_OK;
}

extern "C" hhs_status hhs_particle_system_upload(hhs_particle_system* sys, int32_t n,
                                                 const double* x, const double* y,
                                                 const double* z, const double* vx,
                                                 const double* vy, const double* vz,
                                                 const double* m, const double* ts,
                                                 const int32_t* id, void* stream) {
    if (!sys_ok(sys) || n < 0) return HHS_ERR_INVALID_ARG;
    if (n > sys->n) return HHS_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t b = sizeof(double) * (size_t)n;
    const double* src[8] = {x, y, z, vx, vy, vz, m, ts};
    double* dst[8] = {sys->x, sys->y, sys->z, sys->vx, sys->vy, sys->vz, sys->m, sys->ts};
    for (int k = 0; k < 8; k++)
        if (src[k]) HHS_CUDA_TRY(cudaMemcpyAsync(dst[k], src[k], b, cudaMemcpyHostToDevice, s));
    if (id) HHS_CUDA_TRY(cudaMemcpyAsync(sys->id, id, sizeof(int32_t) * (size_t)n,
                                         cudaMemcpyHostToDevice, s));
    return HHS_OK;
}

extern "C" hhs_status hhs_particle_system_download(const hhs_particle_system* sys, int32_t n,
                                                   double* x, double* y, double* z,
                                                   double* vx, double* vy, double* vz,
                                                   double* m, double* ts, int32_t* id,
                                                   void* stream) {
    if (!sys_ok(sys) || n < 0) return HHS_ERR_INVALID_ARG;
    if (n > sys->n) return HHS_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t b = sizeof(double) * (size_t)n;
    double* dst[8] = {x, y, z, vx, vy, vz, m, ts};
    const double* src[8] = {sys->x, sys->y, sys->z, sys->vx, sys->vy, sys->vz, sys->m, sys->ts};
    for (int k = 0; k < 8; k++)
        if (dst[k]) HHS_CUDA_TRY(cudaMemcpyAsync(dst[k], src[k], b, cudaMemcpyDeviceToHost, s));
    if (id) HHS_CUDA_TRY(cudaMemcpyAsync(id, sys->id, sizeof(int32_t) * (size_t)n,
                                         cudaMemcpyDeviceToHost, s));
    return HHS_OK;
}

extern "C" hhs_status hhs_particle_system_upload_aos(hhs_particle_system* sys, int32_t n,
                                                     const double* pos3, const double* vel3,
                                                     const double* m, const double* ts,
                                                     const int32_t* id, void* stream) {
    if (!sys_ok(sys) || n < 0) return HHS_ERR_INVALID_ARG;
    if (n > sys->n) return HHS_ERR_CAPACITY;
    if (n == 0) return HHS_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t b3 = sizeof(double) * 3 * (size_t)n;
    if (pos3) {
        HHS_CUDA_TRY(cudaMemcpyAsync(sys->ax, pos3, b3, cudaMemcpyHostToDevice, s));
        k_deinterleave<<<small_grid(n), 256, 0, s>>>(sys->ax, sys->x, sys->y, sys->z, n);
        HHS_LAUNCH_CHECK();
    }
    if (vel3) {
        HHS_CUDA_TRY(cudaMemcpyAsync(sys->ax, vel3, b3, cudaMemcpyHostToDevice, s));
        k_deinterleave<<<small_grid(n), 256, 0, s>>>(sys->ax, sys->vx, sys->vy, sys->vz, n);
        HHS_LAUNCH_CHECK();
    }
    return hhs_particle_system_upload(sys, n, nullptr, nullptr, nullptr, nullptr, nullptr,
                                      nullptr, m, ts, id, stream);
}

extern "C" hhs_status hhs_particle_system_download_aos(const hhs_particle_system* sys,
                                                       int32_t n, double* pos3, double* vel3,
                                                       double* m, double* ts, int32_t* id,
                                                       void* stream) {
    if (!sys_ok(sys) || n < 0) return HHS_ERR_INVALID_ARG;
    if (n > sys->n) return HHS_ERR_CAPACITY;
    if (n == 0) return HHS_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t b3 = sizeof(double) * 3 * (size_t)n;
    if (pos3) {
        k_interleave<<<small_grid(n), 256, 0, s>>>(sys->ax, sys->x, sys->y, sys->z, n);
        HHS_LAUNCH_CHECK();
        HHS_CUDA_TRY(cudaMemcpyAsync(pos3, sys->ax, b3, cudaMemcpyDeviceToHost, s));
    }
    if (vel3) {
        // a second staging round trip: the first copy must finish before reuse
        HHS_CUDA_TRY(cudaStreamSynchronize(s));
        k_interleave<<<small_grid(n), 256, 0, s>>>(sys->ax, sys->vx, sys->vy, sys->vz, n);
        HHS_LAUNCH_CHECK();
        HHS_CUDA_TRY(cudaMemcpyAsync(vel3, sys->ax, b3, cudaMemcpyDeviceToHost, s));
    }
    return hhs_particle_system_download(sys, n, nullptr, nullptr, nullptr, nullptr, nullptr,
                                        nullptr, m, ts, id, stream);
}

// ------------------------------------------------------------------ context
namespace {
struct CtxLayout {
    size_t lists, counts, ws, leaf, err, stats, engine, total;
};
CtxLayout ctx_layout(int n_max, int max_levels) {
    CtxLayout L;
    L.lists = align_up(sizeof(int32_t) * (size_t)n_max * (size_t)max_levels);
    L.counts = align_up(sizeof(hhs_partition) * (size_t)max_levels);
    L.ws = align_up(split_workspace_bytes(n_max));
    L.leaf = align_up(sizeof(double));
    L.err = align_up(sizeof(unsigned));
    L.stats = align_up(sizeof(hhs_stats));
    L.engine = align_up(engine_workspace_bytes(n_max, max_levels));
    L.total = 2 * L.lists + L.counts + L.ws + L.leaf + L.err + L.stats + L.engine;
    return L;
}
}  // namespace

extern "C" size_t hhs_workspace_size(int32_t n_max, int32_t max_levels) {
    if (n_max <= 0 || max_levels <= 0) return 0;
    return ctx_layout(n_max, max_levels).total;
}

extern "C" hhs_status hhs_ctx_create(int32_t n_max, int32_t max_levels, hhs_params params,
                                     hhs_ctx** out) {
    if (!out || n_max <= 0 || max_levels <= 0 || max_levels > 1024) return HHS_ERR_INVALID_ARG;
    if (!(params.eta > 0.0)) return HHS_ERR_INVALID_ARG;
    *out = nullptr;
    hhs_ctx* c = new (std::nothrow) hhs_ctx();
    if (!c) return HHS_ERR_OOM;
    c->n_max = n_max;
    c->max_levels = max_levels;
    c->params = params;
    cudaGetDevice(&c->device);
    const CtxLayout L = ctx_layout(n_max, max_levels);
    cudaError_t e = cudaMalloc(&c->arena, L.total);
    if (e != cudaSuccess) { delete c; return hhs_from_cuda(e); }
    c->arena_bytes = L.total;
    e = cudaMemset(c->arena, 0, L.total);
    if (e != cudaSuccess) { cudaFree(c->arena); delete c; return hhs_from_cuda(e); }
    char* p = static_cast<char*>(c->arena);
    c->fast_lists = reinterpret_cast<int32_t*>(p); p += L.lists;
    c->slow_lists = reinterpret_cast<int32_t*>(p); p += L.lists;
    c->counts = reinterpret_cast<hhs_partition*>(p); p += L.counts;
    c->split_ws = p; p += L.ws;
    c->leaf_time = reinterpret_cast<double*>(p); p += L.leaf;
    c->err = reinterpret_cast<unsigned*>(p); p += L.err;
    c->stats = reinterpret_cast<hhs_stats*>(p); p += L.stats;
    c->engine = p;
    c->engine_bytes = L.engine;
    e = cudaMallocHost(&c->host_counts, sizeof(hhs_partition) * (size_t)max_levels);
    if (e != cudaSuccess) { cudaFree(c->arena); delete c; return hhs_from_cuda(e); }
    hhs_status st = engine_init(c, c->engine);
    if (st != HHS_OK) { cudaFreeHost(c->host_counts); cudaFree(c->arena); delete c; return st; }
    c->prof = new (std::nothrow) Profiler();
    *out = c;
    return HHS_OK;
}

extern "C" hhs_status hhs_ctx_destroy(hhs_ctx* c) {
    if (!c) return HHS_ERR_INVALID_ARG;
    delete static_cast<Profiler*>(c->prof);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    engine_destroy(c);
    cudaError_t e1 = cudaFreeHost(c->host_counts);
    cudaError_t e2 = cudaFree(c->arena);
    delete c;
    if (e1 != cudaSuccess) return hhs_from_cuda(e1);
    return hhs_from_cuda(e2);
}

extern "C" hhs_status hhs_ctx_set_params(hhs_ctx* c, hhs_params params) {
    if (!c || !(params.eta > 0.0)) return HHS_ERR_INVALID_ARG;
    c->params = params;
    return HHS_OK;
}

extern "C" hhs_status hhs_ctx_get_simtime(hhs_ctx* c, double* simtime, void* stream) {
    if (!c || !simtime) return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HHS_CUDA_TRY(cudaMemcpyAsync(simtime, c->leaf_time, sizeof(double), cudaMemcpyDeviceToHost, s));
    HHS_CUDA_TRY(cudaStreamSynchronize(s));
    return HHS_OK;
}

extern "C" hhs_status hhs_ctx_flush_simtime(hhs_ctx* c, void* stream) {
    if (!c) return HHS_ERR_INVALID_ARG;
    HHS_CUDA_TRY(cudaMemsetAsync(c->leaf_time, 0, sizeof(double), static_cast<cudaStream_t>(stream)));
    return HHS_OK;
}

extern "C" hhs_status hhs_ctx_check(hhs_ctx* c, void* stream) {
    if (!c) return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HHS_CUDA_TRY(cudaStreamSynchronize(s));
    unsigned e1 = 0, e2 = 0;
    HHS_CUDA_TRY(cudaMemcpy(&e1, c->err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    HHS_CUDA_TRY(cudaMemcpy(&e2, scan_workspace_error_word(c->split_ws), sizeof(unsigned),
                            cudaMemcpyDeviceToHost));
    const unsigned e = e1 | e2;
    if (e & (HHS_ERRBIT_LOOKBACK_TIMEOUT | HHS_ERRBIT_BARRIER_TIMEOUT)) return HHS_ERR_TIMEOUT;
    if (e & HHS_ERRBIT_DEPTH) return HHS_ERR_DEPTH;
    if (e & HHS_ERRBIT_CAPACITY) return HHS_ERR_CAPACITY;
    if (e) return HHS_ERR_DEVICE_FAULT_FLAG;
    return HHS_OK;
}

extern "C" hhs_status hhs_ctx_clear_errors(hhs_ctx* c, void* stream) {
    if (!c) return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HHS_CUDA_TRY(cudaMemsetAsync(c->err, 0, sizeof(unsigned), s));
    HHS_CUDA_TRY(cudaMemsetAsync(scan_workspace_error_word(c->split_ws), 0, sizeof(unsigned), s));
    return engine_reset_barrier(c, s);
}

extern "C" hhs_status hhs_ctx_set_tuning(hhs_ctx* c, const hhs_tuning* t) {
    if (!c || !t) return HHS_ERR_INVALID_ARG;
    return engine_set_tuning(c, *t);
}

extern "C" hhs_status hhs_ctx_get_tuning(hhs_ctx* c, hhs_tuning* t) {
    if (!c || !t) return HHS_ERR_INVALID_ARG;
    return engine_get_tuning(c, t);
}

extern "C" hhs_status hhs_engine_kick_accelerations(hhs_ctx* c, hhs_particle_system* sys,
                                                    int32_t n, void* stream) {
    if (!c || !sys_ok(sys) || n < 2 || n > sys->n || n > c->n_max) return HHS_ERR_INVALID_ARG;
    return engine_kick_accelerations(c, soa_of(sys), sys->ax, sys->ay, sys->az, n,
                                     static_cast<cudaStream_t>(stream));
}

extern "C" hhs_status hhs_engine_timestep_rates(hhs_ctx* c, hhs_particle_system* sys, int32_t n,
                                                void* stream) {
    if (!c || !sys_ok(sys) || n < 2 || n > sys->n || n > c->n_max) return HHS_ERR_INVALID_ARG;
    return engine_timestep_rates(c, soa_of(sys), n, static_cast<cudaStream_t>(stream));
}

extern "C" hhs_status hhs_ctx_set_trace(hhs_ctx* c, int32_t* d_nodes, int64_t capacity,
                                        uint64_t* d_count) {
    if (!c) return HHS_ERR_INVALID_ARG;
    return engine_set_trace(c, d_nodes, capacity, reinterpret_cast<unsigned long long*>(d_count));
}

extern "C" hhs_status hhs_ctx_get_launch(hhs_ctx* c, int32_t* grid_ctas, int32_t* smem_bytes) {
    if (!c) return HHS_ERR_INVALID_ARG;
    return engine_get_launch(c, grid_ctas, smem_bytes);
}

extern "C" hhs_status hhs_ctx_get_stats(hhs_ctx* c, hhs_stats* out, void* stream) {
    if (!c || !out) return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HHS_CUDA_TRY(cudaMemcpyAsync(out, c->stats, sizeof(hhs_stats), cudaMemcpyDeviceToHost, s));
    HHS_CUDA_TRY(cudaStreamSynchronize(s));
    return HHS_OK;
}

extern "C" hhs_status hhs_ctx_reset_stats(hhs_ctx* c, void* stream) {
    if (!c) return HHS_ERR_INVALID_ARG;
    HHS_CUDA_TRY(cudaMemsetAsync(c->stats, 0, sizeof(hhs_stats), static_cast<cudaStream_t>(stream)));
    return HHS_OK;
}

extern "C" hhs_status hhs_ctx_set_profiling(hhs_ctx* c, int32_t on) {
    if (!c || !c->prof) return HHS_ERR_INVALID_ARG;
    auto* p = static_cast<Profiler*>(c->prof);
    p->resolve();
    p->on = on != 0;
    p->acc = hhs_profile{};
    hhs_profile scratch{};
    return engine_get_profile(c, &scratch, true);
}

extern "C" hhs_status hhs_ctx_get_profile(hhs_ctx* c, hhs_profile* out) {
    if (!c || !c->prof || !out) return HHS_ERR_INVALID_ARG;
    auto* p = static_cast<Profiler*>(c->prof);
    p->resolve();
    *out = p->acc;
    return engine_get_profile(c, out, false);
}

extern "C" hhs_status hhs_ctx_get_level_profile(hhs_ctx* c, double* ms, uint64_t* counts) {
    if (!c) return HHS_ERR_INVALID_ARG;
    return engine_get_level_profile(c, ms, counts);
}

extern "C" hhs_status hhs_measure_fma_peaks(double* fp32_tflops, double* fp64_tflops,
                                            void* stream) {
    if (!fp32_tflops || !fp64_tflops) return HHS_ERR_INVALID_ARG;
    return measure_fma_peaks(fp32_tflops, fp64_tflops, static_cast<cudaStream_t>(stream));
}

extern "C" hhs_status hhs_measure_fma2_peak(double* fp32x2_tflops, void* stream) {
    if (!fp32x2_tflops) return HHS_ERR_INVALID_ARG;
    return measure_fma2_peak(fp32x2_tflops, static_cast<cudaStream_t>(stream));
}

// ------------------------------------------------------------------ reference-shaped ops
extern "C" hhs_status hhs_timesteps(hhs_ctx* c, hhs_particle_system* sys, int32_t n,
                                    hhs_precision prec, void* stream) {
    if (!c || !sys_ok(sys) || n < 0) return HHS_ERR_INVALID_ARG;
    if (n > sys->n) return HHS_ERR_CAPACITY;
    return launch_timesteps(soa_of(sys), nullptr, n, c->params.eta, prec,
                            static_cast<cudaStream_t>(stream));
}

extern "C" hhs_status hhs_split(hhs_ctx* c, const hhs_particle_system* total,
                                hhs_particle_system* slow, hhs_particle_system* fast,
                                int32_t* predicate, int32_t* scanned_predicate, double pivot,
                                int32_t n, hhs_partition* part, void* stream) {
    if (!c || !sys_ok(total) || !sys_ok(slow) || !sys_ok(fast) || !part || n <= 0)
        return HHS_ERR_INVALID_ARG;
    if (n > total->n || n > slow->n || n > fast->n || n > c->n_max) return HHS_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    hhs_status st = launch_split_list(nullptr, n, total->ts, pivot, c->fast(0), c->slow(0),
                                      predicate, scanned_predicate, part, nullptr, 0.0, nullptr,
                                      0, 0, c->split_ws, s);
    if (st != HHS_OK) return st;
    return launch_gather_split(soa_of(total), soa_of(slow), slow->parent_id, soa_of(fast),
                               fast->parent_id, c->slow(0), c->fast(0), part, n, s);
}

extern "C" hhs_status hhs_kick_slow(hhs_particle_system* sys, double dt, double fac, int32_t n,
                                    hhs_precision prec, void* stream) {
    if (!sys_ok(sys) || n < 0) return HHS_ERR_INVALID_ARG;
    if (n > sys->n) return HHS_ERR_CAPACITY;
    const SoA P = soa_of(sys);
    return launch_kick_pair(P, sys->ax, sys->ay, sys->az, P, n, n, fac * dt, prec,
                            static_cast<cudaStream_t>(stream));
}

extern "C" hhs_status hhs_kick_sf(const hhs_particle_system* so_sys,
                                  hhs_particle_system* si_sys, double dt, double fac,
                                  int32_t n_sink, int32_t m_src, hhs_precision prec,
                                  void* stream) {
    if (!sys_ok(so_sys) || !sys_ok(si_sys) || n_sink < 0 || m_src < 0) return HHS_ERR_INVALID_ARG;
    if (n_sink > si_sys->n || m_src > so_sys->n) return HHS_ERR_CAPACITY;
    return launch_kick_pair(soa_of(si_sys), si_sys->ax, si_sys->ay, si_sys->az, soa_of(so_sys),
                            n_sink, m_src, fac * dt, prec, static_cast<cudaStream_t>(stream));
}

extern "C" hhs_status hhs_drift(hhs_particle_system* sys, double dt, double fac, int32_t n,
                                void* stream) {
    if (!sys_ok(sys) || n < 0) return HHS_ERR_INVALID_ARG;
    if (n > sys->n) return HHS_ERR_CAPACITY;
    return launch_drift(soa_of(sys), n, dt * fac, static_cast<cudaStream_t>(stream));
}

extern "C" hhs_status hhs_update_system(hhs_particle_system* prev,
                                        const hhs_particle_system* cur, int32_t n,
                                        void* stream) {
    if (!sys_ok(prev) || !sys_ok(cur) || n < 0) return HHS_ERR_INVALID_ARG;
    if (n > cur->n) return HHS_ERR_CAPACITY;
    return launch_update_system(soa_of(prev), soa_of(cur), cur->parent_id, n,
                                static_cast<cudaStream_t>(stream));
}

// ------------------------------------------------------------------ multi-GPU
// One system on several GPUs: every rank holds a replica; the O(n^2) launches of the
// host-driven schedule are split by sink and their kernels store each result into every
// replica (PeerOut). No counterpart in the reference, which runs on one GPU.
struct hhs_dist {
    int rank = 0, world = 1;
    int n_cap = 0;
    SoA peer[kMaxPeers];  // the other ranks' replicas, in rank order
    double* peer_ax[kMaxPeers];  // their acceleration arrays: pair-rate words of the timestep
    unsigned* rate_words = nullptr;  // this rank's (its system's ax), set per step
    hhs_barrier_fn barrier = nullptr;
    void* user = nullptr;
    long long min_pairs = 0;
    bool engine_below = true;  // subtrees below min_pairs on the engine
    hhs_minmax_fn agree = nullptr;  // min/max of a value over the ranks (configuration check)
    void* agree_user = nullptr;
};

namespace {
// First sink of rank r: the smallest s whose cumulative cost reaches r/world of the
// total, sinks [0, nf) costing ns pair terms each and [nf, nf+ns) costing ns+nf.
int shard_bound(long long nf, long long ns, int r, int world) {
    const long long n = nf + ns;
    if (r <= 0) return 0;
    if (r >= world) return (int)n;
    const __int128 cf = ns, cs = ns + nf;
    const __int128 total = (__int128)nf * cf + (__int128)ns * cs;
    if (total == 0) return (int)((__int128)n * r / world);
    const __int128 target = total * r;  // cost(s) * world >= target
    const __int128 fast_total = (__int128)nf * cf * world;
    __int128 b;
    if (cf > 0 && fast_total >= target) {
        const __int128 q = cf * world;
        b = (target + q - 1) / q;
    } else {
        const __int128 q = cs * world;
        b = nf + (target - fast_total + q - 1) / q;
    }
    return (int)(b < n ? b : n);
}

// One sink-partitioned launch: barrier, this rank's shard (stores into every replica),
// barrier. Every rank takes both barriers even with an empty shard.
template <class Launch>
hhs_status dist_launch(const hhs_dist* d, int n_fast, int n_slow, cudaStream_t s,
                       Launch&& launch) {
    PeerOut po = peer_out_local();
    po.lo = shard_bound(n_fast, n_slow, d->rank, d->world);
    po.hi = shard_bound(n_fast, n_slow, d->rank + 1, d->world);
    po.n_peer = d->world - 1;
    for (int r = 0; r < po.n_peer; r++) {
        po.vx[r] = d->peer[r].vx; po.vy[r] = d->peer[r].vy; po.vz[r] = d->peer[r].vz;
        po.ts[r] = d->peer[r].ts;
        po.rate[r] = reinterpret_cast<unsigned*>(d->peer_ax[r]);
    }
    if (d->barrier(d->user, s) != 0) return HHS_ERR_PEER;
    const hhs_status st = launch(po);
    if (st != HHS_OK) return st;
    if (d->barrier(d->user, s) != 0) return HHS_ERR_PEER;
    return HHS_OK;
}

bool dist_shares(const hhs_dist* d, double pairs) {
    return d && pairs >= (double)d->min_pairs;
}

// Sink-block share [b_lo, b_hi) of this rank for a kick of a split level: the sink shards
// of equal pair cost, rounded to whole blocks of `blk` sinks (the same on every rank).
void kick_blocks(const hhs_dist* d, int nf, int ns, int blk, int* b_lo, int* b_hi) {
    const int nsb = (nf + ns + blk - 1) / blk;
    auto bound = [&](int r) {
        if (r <= 0) return 0;
        if (r >= d->world) return nsb;
        const int b = (shard_bound(nf, ns, r, d->world) + blk / 2) / blk;
        return b < nsb ? b : nsb;
    };
    *b_lo = bound(d->rank);
    *b_hi = bound(d->rank + 1);
}

// ------------------------------------------------------------------ host-driven HOLD
// The schedule of src/hold.cuh:51-181 driven from the host: after each split the
// partition counts are read back (the reference synchronises the device at the same
// point, src/split.cuh:430) to decide the recursion. Level k's subsystem is the fast
// list of level k-1 (the whole system at level 0). With d, the timestep and kick
// launches of at least d->min_pairs pair terms are split across the ranks, and a subtree
// too small for that (no launch in it reaches min_pairs: a kick has at most n(n-1) pair
// terms) runs as one launch of the device-resident engine from its own level,
// identically on every rank.
hhs_status hold_host(hhs_ctx* c, const SoA& P, const int32_t* S, int n, int level, double dt,
                     bool calc, hhs_precision prec, cudaStream_t s, const hhs_dist* d) {
    if (level >= c->max_levels) return HHS_ERR_DEPTH;
    if (d && d->engine_below && c->engine_host && c->engine_bytes &&
        (double)n * (double)(n - 1) < (double)d->min_pairs)
        return engine_hold_step(c, P, n, std::ldexp(dt, level), calc, prec, false, s, level);
    auto* prof = static_cast<Profiler*>(c->prof);
    const bool timed = prof && prof->on;
    Profiler::Rec rec{};
    hhs_status st;
    if (calc) {
        const double pairs = (double)n * (double)(n - 1);
        if (timed) prof->begin(rec, 0, pairs, s);
        if (dist_shares(d, pairs) && c->engine_host && d->rate_words) {
            // the engine's tiled timestep over this rank's share; mixed: the symmetric
            // pair-rate maxima go to every replica's rate words, converted after the barrier
            if (prec != HHS_PREC_FP64)
                HHS_CUDA_TRY(cudaMemsetAsync(d->rate_words, 0, sizeof(unsigned) * (size_t)n, s));
            st = dist_launch(d, 0, n, s, [&](const PeerOut& po) {
                return engine_shard_timesteps(c, P, d->rate_words, S, n, prec, d->rank, d->world,
                                              po, s);
            });
            if (st == HHS_OK && prec != HHS_PREC_FP64)
                st = engine_rates_to_ts(c, P, d->rate_words, S, n, s);
        } else if (dist_shares(d, pairs)) {
            st = dist_launch(d, 0, n, s, [&](const PeerOut& po) {
                return launch_timesteps(P, S, n, c->params.eta, prec, s, po);
            });
        } else {
            st = launch_timesteps(P, S, n, c->params.eta, prec, s);
        }
        if (st != HHS_OK) return st;
        if (timed) prof->end(rec, s);
    }
    int32_t* F = c->fast(level);
    int32_t* L = c->slow(level);
    hhs_partition* cnt = c->counts + level;
    if (timed) prof->begin(rec, 2, 0.0, s);
    st = launch_split_list(S, n, P.ts, dt, F, L, nullptr, nullptr, cnt, c->leaf_time, dt,
                           c->stats, level, calc ? 1 : 0, c->split_ws, s);
    if (st != HHS_OK) return st;
    if (timed) prof->end(rec, s);
    HHS_CUDA_TRY(cudaMemcpyAsync(&c->host_counts[level], cnt, sizeof(hhs_partition),
                                 cudaMemcpyDeviceToHost, s));
    HHS_CUDA_TRY(cudaStreamSynchronize(s));
    const int nf = c->host_counts[level].n_fast, ns = c->host_counts[level].n_slow;
    if (nf < 0 || ns < 0 || nf + ns != n) return HHS_ERR_DEVICE_FAULT_FLAG;
    if (nf > 0) {
        st = hold_host(c, P, F, nf, level + 1, dt / 2, false, prec, s, d);
        if (st != HHS_OK) return st;
    }
    if (ns > 0) {
        st = launch_drift_slow(P, L, cnt, ns, dt * 0.5, s);
        if (st != HHS_OK) return st;
        const double pairs = (double)ns * (ns - 1.0) + 2.0 * (double)ns * (double)nf;
        if (timed) prof->begin(rec, 1, pairs, s);
        const double eps2 = c->params.eps * c->params.eps;
        bool done = false;
        if (dist_shares(d, pairs) && c->engine_host) {
            // the engine's tiled kick over this rank's sink blocks
            int b_lo = 0, b_hi = 0;
            kick_blocks(d, nf, ns, engine_shard_kick_block(prec), &b_lo, &b_hi);
            // mixed precision needs the level's packed-source array (every rank decides
            // alike: the contexts have the same level capacity)
            if (prec == HHS_PREC_FP64 || level < engine_pk_levels(c)) {
                st = dist_launch(d, nf, ns, s, [&](const PeerOut& po) {
                    return engine_shard_kick(c, P, F, L, nf, ns, level, dt, prec, b_lo, b_hi, po, s);
                });
                done = true;
            }
        }
        if (!done) {
            if (dist_shares(d, pairs))
                st = dist_launch(d, nf, ns, s, [&](const PeerOut& po) {
                    return launch_kick_level(P, F, L, cnt, n, dt, eps2, prec, s, po);
                });
            else
                st = launch_kick_level(P, F, L, cnt, n, dt, eps2, prec, s);
        }
        if (st != HHS_OK) return st;
        if (timed) prof->end(rec, s);
        st = launch_drift_slow(P, L, cnt, ns, dt * 0.5, s);
        if (st != HHS_OK) return st;
    }
    if (nf > 0) {
        st = hold_host(c, P, F, nf, level + 1, dt / 2, true, prec, s, d);
        if (st != HHS_OK) return st;
    }
    return HHS_OK;
}
}  // namespace

extern "C" hhs_status hhs_hold_step_host(hhs_ctx* c, hhs_particle_system* sys, int32_t n,
                                         double dt, int32_t calc_timestep, hhs_precision prec,
                                         void* stream) {
    if (!c || !sys_ok(sys) || n <= 0 || !(dt > 0.0)) return HHS_ERR_INVALID_ARG;
    if (n > sys->n || n > c->n_max) return HHS_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    hhs_status st = hold_host(c, soa_of(sys), nullptr, n, 0, dt, calc_timestep != 0, prec, s,
                              nullptr);
    if (st != HHS_OK) return st;
    return hhs_ctx_check(c, stream);
}

extern "C" hhs_status hhs_dist_create(hhs_dist** out, int32_t rank, int32_t world,
                                      const hhs_particle_system* replicas,
                                      hhs_barrier_fn barrier, void* user, int64_t min_pairs) {
    if (!out) return HHS_ERR_INVALID_ARG;
    *out = nullptr;
    if (world < 1 || world > HHS_DIST_MAX_RANKS || world - 1 > kMaxPeers || rank < 0 ||
        rank >= world || !barrier || min_pairs < 0 || (world > 1 && !replicas))
        return HHS_ERR_INVALID_ARG;
    int cap = 0;
    for (int r = 0; r < world; r++) {
        if (r == rank) continue;
        const hhs_particle_system* p = &replicas[r];
        if (!p->vx || !p->vy || !p->vz || !p->ts || !p->ax || p->n <= 0) return HHS_ERR_INVALID_ARG;
        if (cap != 0 && p->n != cap) return HHS_ERR_INVALID_ARG;
        cap = p->n;
    }
    auto* d = new (std::nothrow) hhs_dist;
    if (!d) return HHS_ERR_OOM;
    d->rank = rank;
    d->world = world;
    d->n_cap = cap;
    int k = 0;
    for (int r = 0; r < world; r++)
        if (r != rank) {
            d->peer_ax[k] = replicas[r].ax;
            d->peer[k++] = soa_of(&replicas[r]);
        }
    d->barrier = barrier;
    d->user = user;
    d->min_pairs = min_pairs;
    *out = d;
    return HHS_OK;
}

extern "C" hhs_status hhs_dist_set_subtree_engine(hhs_dist* d, int32_t on) {
    if (!d) return HHS_ERR_INVALID_ARG;
    d->engine_below = on != 0;
    return HHS_OK;
}

extern "C" hhs_status hhs_dist_set_agreement(hhs_dist* d, hhs_minmax_fn fn, void* user) {
    if (!d) return HHS_ERR_INVALID_ARG;
    d->agree = fn;
    d->agree_user = user;
    return HHS_OK;
}

// FNV-1a over the fields that fix the operation order of a step: the precision, the
// engine's launch shape and tuning, the system size, the step and the parameters.
extern "C" hhs_status hhs_dist_config_hash(const hhs_tuning* t, int32_t grid_ctas,
                                           hhs_precision prec, int32_t n, double dt,
                                           hhs_params params, uint64_t* out) {
    if (!t || !out) return HHS_ERR_INVALID_ARG;
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        for (int k = 0; k < 8; k++) {
            h ^= (v >> (8 * k)) & 0xffu;
            h *= 1099511628211ull;
        }
    };
    auto bits = [](double v) {
        uint64_t u;
        std::memcpy(&u, &v, sizeof(u));
        return u;
    };
    mix((uint64_t)prec);
    mix((uint64_t)(uint32_t)grid_ctas);
    mix((uint64_t)(uint32_t)t->small_n);
    mix((uint64_t)(uint32_t)t->units_per_cta);
    mix((uint64_t)(uint32_t)t->ctas_per_sm);
    mix((uint64_t)(uint32_t)t->warp_n);
    mix((uint64_t)(uint32_t)t->cluster_size);
    mix((uint64_t)(uint32_t)t->mid_n);
    mix((uint64_t)(uint32_t)t->packed);
    mix((uint64_t)(uint32_t)t->mid_dist_n);
    mix((uint64_t)(uint32_t)t->overlap);
    mix((uint64_t)(uint32_t)n);
    mix(bits(dt));
    mix(bits(params.eta));
    mix(bits(params.eps));
    *out = h;
    return HHS_OK;
}

extern "C" hhs_status hhs_dist_check(hhs_dist* d, uint64_t config_hash) {
    if (!d) return HHS_ERR_INVALID_ARG;
    if (!d->agree) return HHS_OK;
    uint64_t lo = 0, hi = 0;
    if (d->agree(d->agree_user, config_hash, &lo, &hi) != 0) return HHS_ERR_PEER;
    return lo == hi ? HHS_OK : HHS_ERR_INVALID_ARG;
}

extern "C" hhs_status hhs_dist_destroy(hhs_dist* d) {
    delete d;
    return HHS_OK;
}

extern "C" hhs_status hhs_dist_shard(int32_t n_fast, int32_t n_slow, int32_t rank,
                                     int32_t world, int32_t* lo, int32_t* hi) {
    if (!lo || !hi || n_fast < 0 || n_slow < 0 || world < 1 || rank < 0 || rank >= world ||
        (long long)n_fast + n_slow > 0x7fffffffLL)
        return HHS_ERR_INVALID_ARG;
    *lo = shard_bound(n_fast, n_slow, rank, world);
    *hi = shard_bound(n_fast, n_slow, rank + 1, world);
    return HHS_OK;
}

extern "C" hhs_status hhs_hold_step_dist(hhs_ctx* c, hhs_dist* d, hhs_particle_system* sys,
                                         int32_t n, double dt, int32_t calc_timestep,
                                         hhs_precision prec, void* stream) {
    if (!c || !d || !sys_ok(sys) || n <= 0 || !(dt > 0.0)) return HHS_ERR_INVALID_ARG;
    if (n > sys->n || n > c->n_max || (d->world > 1 && n > d->n_cap)) return HHS_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (d->agree) {
        // every rank must run the same operations in the same order, or replicas drift
        hhs_tuning t{};
        int32_t grid[2] = {0, 0};
        hhs_status st = engine_get_tuning(c, &t);
        if (st == HHS_OK) st = engine_get_launch(c, grid, nullptr);
        uint64_t h = 0;
        if (st == HHS_OK)
            st = hhs_dist_config_hash(&t, grid[prec == HHS_PREC_FP64 ? 0 : 1], prec, n, dt,
                                      c->params, &h);
        if (st == HHS_OK) st = hhs_dist_check(d, h);
        if (st != HHS_OK) return st;
    }
    d->rate_words = reinterpret_cast<unsigned*>(sys->ax);
    hhs_status st = hold_host(c, soa_of(sys), nullptr, n, 0, dt, calc_timestep != 0, prec, s, d);
    d->rate_words = nullptr;
    if (st != HHS_OK) return st;
    return hhs_ctx_check(c, stream);
}

static_assert(sizeof(cudaIpcMemHandle_t) == HHS_IPC_HANDLE_BYTES, "IPC handle size");

extern "C" hhs_status hhs_ipc_handle(const hhs_particle_system* sys, void* handle_out) {
    if (!sys_ok(sys) || !handle_out) return HHS_ERR_INVALID_ARG;
    cudaIpcMemHandle_t h;
    HHS_CUDA_TRY(cudaIpcGetMemHandle(&h, sys->_base));
    std::memcpy(handle_out, &h, sizeof(h));
    return HHS_OK;
}

extern "C" hhs_status hhs_ipc_open(const void* handle, int32_t n, hhs_particle_system* view_out) {
    if (!handle || !view_out || n <= 0) return HHS_ERR_INVALID_ARG;
    std::memset(view_out, 0, sizeof(*view_out));
    cudaIpcMemHandle_t h;
    std::memcpy(&h, handle, sizeof(h));
    void* base = nullptr;
    HHS_CUDA_TRY(cudaIpcOpenMemHandle(&base, h, cudaIpcMemLazyEnablePeerAccess));
    lay_out_system(view_out, base, n);
    return HHS_OK;
}

extern "C" hhs_status hhs_ipc_close(hhs_particle_system* view) {
    if (!view || !view->_base) return HHS_ERR_INVALID_ARG;
    const cudaError_t e = cudaIpcCloseMemHandle(view->_base);
    std::memset(view, 0, sizeof(*view));
    return e == cudaSuccess ? HHS_OK : hhs_from_cuda(e);
}

extern "C" hhs_status hhs_hold_step(hhs_ctx* c, int32_t clevel, hhs_particle_system* sys,
                                    int32_t n, double stime, double etime, double dt,
                                    int32_t calc_timestep, hhs_precision prec, void* stream) {
    (void)clevel; (void)stime; (void)etime;
    if (!c || !sys_ok(sys) || n <= 0 || !(dt > 0.0)) return HHS_ERR_INVALID_ARG;
    if (n > sys->n || n > c->n_max) return HHS_ERR_CAPACITY;
    if (c->engine_bytes == 0 || !c->engine_host)
        return hhs_hold_step_host(c, sys, n, dt, calc_timestep, prec, stream);
    auto* prof = static_cast<Profiler*>(c->prof);
    const bool on = prof && prof->on;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Profiler::Rec rec{};
    if (on) prof->begin(rec, 4, 0.0, s);
    hhs_status st = engine_hold_step(c, soa_of(sys), n, dt, calc_timestep != 0, prec, on, s);
    if (st == HHS_OK && on) prof->end(rec, s);
    return st;
}

// ------------------------------------------------------------------ autotuner
// Times the device-resident step for a grid of (small_n, units_per_cta) candidates on the
// caller's own system: the state is snapshotted once, restored before every trial (one
// untimed warm-up step, then two timed steps) and restored at the end; the fastest
// candidate is kept. Pair throughput depends on how the hierarchy is cut between
// grid-wide phases and single-CTA subtrees, which is a property of the system, so the
// tuning is done on it rather than on a synthetic proxy.
extern "C" hhs_status hhs_ctx_autotune(hhs_ctx* c, hhs_particle_system* sys, int32_t n,
                                       double dt, hhs_precision prec, hhs_tuning* out,
                                       void* stream) {
    if (!c || !sys_ok(sys) || n <= 0 || n > sys->n || n > c->n_max || !(dt > 0.0))
        return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    hhs_particle_system snap;
    hhs_status st = hhs_particle_system_alloc(&snap, n);
    if (st != HHS_OK) return st;
    const size_t b = sizeof(double) * (size_t)n;
    double* src[8] = {sys->x, sys->y, sys->z, sys->vx, sys->vy, sys->vz, sys->ts, sys->m};
    double* dst[8] = {snap.x, snap.y, snap.z, snap.vx, snap.vy, snap.vz, snap.ts, snap.m};
    auto copy_all = [&](bool save) -> hhs_status {
        for (int k = 0; k < 8; k++)
            HHS_CUDA_TRY(cudaMemcpyAsync(save ? dst[k] : src[k], save ? src[k] : dst[k], b,
                                         cudaMemcpyDeviceToDevice, s));
        return HHS_OK;
    };
    hhs_tuning best{}, cur{};
    engine_get_tuning(c, &cur);
    best = cur;
    best.ms_per_step = 1e300;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double leaf = 0.0;
    cudaMemcpy(&leaf, c->leaf_time, sizeof(double), cudaMemcpyDeviceToHost);
    hhs_stats stats_saved{};
    cudaMemcpy(&stats_saved, c->stats, sizeof(hhs_stats), cudaMemcpyDeviceToHost);
    st = copy_all(true);
    // (small_n, mid_n, cluster_size) tiers, then units per CTA and CTAs per SM
    struct Tier { int sn, mid, cs; };
    const Tier tiers[] = {{64, 0, 1},   {128, 0, 1},  {64, 0, 2},   {64, 640, 1},
                          {64, 640, 2}, {64, 256, 2}, {64, 640, 4}, {64, 640, 8},
                          {64, 640, 16}};
    const int upc_cands[] = {8, 16};
    constexpr int kTimed = 3;
    c->tune_table.clear();
    for (int cps = 1; cps <= 2; cps++)
    for (const Tier& tr : tiers) {
        for (int upc : upc_cands) {
            if (st != HHS_OK) break;
            hhs_tuning t{tr.sn, upc, cps, cur.warp_n, tr.cs, tr.mid, cur.packed, cur.mid_dist_n,
                         cur.overlap, 0.0};
            if (engine_set_tuning(c, t) != HHS_OK) continue;  // e.g. no cluster occupancy
            st = copy_all(false);
            if (st == HHS_OK) st = engine_hold_step(c, soa_of(sys), n, dt, true, prec, false, s);
            if (st == HHS_OK) st = copy_all(false);
            if (st != HHS_OK) break;
            cudaEventRecord(e0, s);
            for (int r = 0; r < kTimed && st == HHS_OK; r++)
                st = engine_hold_step(c, soa_of(sys), n, dt, true, prec, false, s);
            cudaEventRecord(e1, s);
            if (st == HHS_OK) st = hhs_ctx_check(c, stream);
            if (st != HHS_OK) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            t.ms_per_step = ms / kTimed;
            c->tune_table.push_back(t);
            if (t.ms_per_step < best.ms_per_step) best = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    hhs_status st2 = copy_all(false);
    cudaMemcpyAsync(c->leaf_time, &leaf, sizeof(double), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(c->stats, &stats_saved, sizeof(hhs_stats), cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    hhs_particle_system_free(&snap);
    if (st == HHS_OK) st = st2;
    if (st != HHS_OK) {
        engine_set_tuning(c, cur);
        return st;
    }
    engine_set_tuning(c, best);
    if (out) *out = best;
    return HHS_OK;
}

extern "C" hhs_status hhs_ctx_autotune_results(hhs_ctx* c, hhs_tuning* out, int32_t capacity,
                                               int32_t* count) {
    if (!c || !count || capacity < 0 || (capacity > 0 && !out)) return HHS_ERR_INVALID_ARG;
    *count = (int32_t)c->tune_table.size();
    for (int32_t k = 0; k < capacity && k < *count; k++) out[k] = c->tune_table[k];
    return HHS_OK;
}

// ------------------------------------------------------------------ graph-captured steps
// `steps` consecutive top-level HOLD steps captured once into a CUDA graph (one node per
// persistent-kernel launch) and replayed on later calls with the same system, size, step,
// precision and tuning. Replays cost one graph launch instead of `steps` kernel launches.
// If the stream cannot be captured, the steps are launched directly.
extern "C" hhs_status hhs_hold_integrate(hhs_ctx* c, hhs_particle_system* sys, int32_t n,
                                         double dt, int32_t steps, hhs_precision prec,
                                         void* stream) {
    if (!c || !sys_ok(sys) || n <= 0 || steps <= 0 || !(dt > 0.0)) return HHS_ERR_INVALID_ARG;
    if (n > sys->n || n > c->n_max) return HHS_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    hhs_tuning t{};
    engine_get_tuning(c, &t);
    unsigned long long dtbits;
    std::memcpy(&dtbits, &dt, sizeof(dtbits));
    const unsigned long long key[6] = {
        reinterpret_cast<uintptr_t>(sys->x), (unsigned long long)n, dtbits,
        ((unsigned long long)steps << 32) | ((unsigned long long)t.mid_dist_n << 8) |
            (unsigned long long)prec,
        ((unsigned long long)t.small_n << 32) | (unsigned)t.mid_n,
        ((unsigned long long)t.units_per_cta << 32) |
            (unsigned)(t.ctas_per_sm | (t.warp_n << 8) | (t.cluster_size << 16) | (t.packed << 24) |
                       (t.overlap << 25))};
    const bool hit = c->graph_exec && std::memcmp(key, c->graph_key, sizeof(key)) == 0;
    if (!hit) {
        if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
        cudaGraph_t g = nullptr;
        bool captured = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        hhs_status st = HHS_OK;
        if (captured) {
            for (int k = 0; k < steps && st == HHS_OK; k++)
                st = engine_hold_step(c, soa_of(sys), n, dt, true, prec, false, s);
            const cudaError_t e = cudaStreamEndCapture(s, &g);
            captured = (st == HHS_OK && e == cudaSuccess && g != nullptr);
            if (captured && cudaGraphInstantiate(&c->graph_exec, g, 0) != cudaSuccess) {
                c->graph_exec = nullptr;
                captured = false;
            }
            if (g) cudaGraphDestroy(g);
        }
        cudaGetLastError();
        if (!captured) {
            for (int k = 0; k < steps; k++) {
                hhs_status st2 = engine_hold_step(c, soa_of(sys), n, dt, true, prec, false, s);
                if (st2 != HHS_OK) return st2;
            }
            return HHS_OK;
        }
        std::memcpy(c->graph_key, key, sizeof(key));
    }
    HHS_CUDA_TRY(cudaGraphLaunch(c->graph_exec, s));
    hhs_count_launch();
    return HHS_OK;
}
