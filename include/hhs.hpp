// hhs.hpp -- the reference's C++ template API (parallel-hhs, src/*.cuh) over the C ABI.
//
// A caller written against parallel-hhs swaps `#include "hold.cuh"` for
// `#include "hhs.hpp"`, links libhhs_b200.so, and keeps its code: the same class and
// function names, template parameters and argument orders as
//   particle_system<T>, nbodysystem_globals<T>, partition, nbody_params<T>, vec3<T>
//     (src/particle_system.cuh:8-132, src/vec.cuh:5-53)
//   hold_step<T,BS>            src/hold.cuh:16-18,51-53
//   timesteps<T,BS>            src/timestep.cuh:7-8
//   split<T,BS,U>              src/split.cuh:573-579
//   kick_slow<T,BS>, kick_sf   src/kick.cuh:6-13
//   drift<T,BS>                src/drift.cuh:7-11
//   update_system<T,BS>        src/update_system.cuh:29-30
// Differences a caller can see: state is FP64 (T must be double); the device side of a
// particle_system is SoA (x, y, z arrays) rather than vec3 arrays, so code that reads
// `gpu_sys->pos` directly must use `gpu_sys->dev` instead; errors throw hhs_error
// instead of calling exit(); the kick is attractive gravity. The template BLOCKSIZE and
// UNROLL arguments are accepted and ignored (the library picks its own launch shapes).
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <stdexcept>
#include <string>

#include "hhs.h"

struct hhs_error : std::runtime_error {
    hhs_status status;
    hhs_error(hhs_status s, const char* what)
        : std::runtime_error(std::string(what) + ": " + hhs_status_string(s)), status(s) {}
};

inline void hhs_check(hhs_status s, const char* what) {
    if (s != HHS_OK) throw hhs_error(s, what);
}

// Precision used by the template wrappers (FP64 reproduces the reference's FP64 path).
inline hhs_precision& hhs_compat_precision() {
    static hhs_precision p = HHS_PREC_FP64;
    return p;
}

template <typename T>
struct vec3 {
    T x, y, z;
    vec3() : x(0), y(0), z(0) {}
    vec3(const T& a, const T& b, const T& c) : x(a), y(b), z(c) {}
    vec3 operator+(const vec3& v) const { return vec3(v.x + x, v.y + y, v.z + z); }
    vec3 operator-(const vec3& v) const { return vec3(x - v.x, y - v.y, z - v.z); }
    T operator*(const vec3& v) const { return v.x * x + v.y * y + v.z * z; }
    vec3 operator*(const T& v) const { return vec3(x * v, y * v, z * v); }
    vec3 operator-() const { return vec3(-x, -y, -z); }
    T norm2() const { return x * x + y * y + z * z; }
    T norm() const { return std::sqrt(norm2()); }
};
static_assert(sizeof(vec3<double>) == 3 * sizeof(double), "vec3<double> must be packed");

struct partition {
    int N_slow;
    int N_fast;
};
static_assert(sizeof(partition) == sizeof(hhs_partition), "partition layout");

template <typename T>
struct nbody_params {
    T eta;
    T eps;
};

template <typename T>
class particle_system {
    static_assert(sizeof(T) == sizeof(double), "the B200 library keeps FP64 state: use double");

   public:
    // host ('c') store: AoS arrays as in the reference
    vec3<T>* pos = nullptr;
    vec3<T>* vel = nullptr;
    vec3<T>* acc = nullptr;
    T* timestep = nullptr;
    T* m = nullptr;
    int N;
    int* id = nullptr;
    int* parent_id = nullptr;
    char store;
    // device ('g') store: SoA arrays owned by the library
    hhs_particle_system dev{};

    particle_system(int N_init, char s) : N(N_init), store(s) {}

    void gpu_alloc() {
        if (store == 'c') throw hhs_error(HHS_ERR_INVALID_ARG, "gpu_alloc on a CPU store");
        hhs_check(hhs_particle_system_alloc(&dev, N), "gpu_alloc");
    }
    void gpu_free() {
        if (store == 'c') throw hhs_error(HHS_ERR_INVALID_ARG, "gpu_free on a CPU store");
        hhs_check(hhs_particle_system_free(&dev), "gpu_free");
    }
    void cpu_alloc() {
        if (store == 'g') throw hhs_error(HHS_ERR_INVALID_ARG, "cpu_alloc on a GPU store");
        pos = new vec3<T>[N];
        vel = new vec3<T>[N];
        acc = new vec3<T>[N];
        timestep = new T[N];
        m = new T[N];
        id = new int[N];
        parent_id = new int[N];
    }
    void cpu_free() {
        if (store == 'g') throw hhs_error(HHS_ERR_INVALID_ARG, "cpu_free on a GPU store");
        delete[] pos; delete[] vel; delete[] acc; delete[] timestep;
        delete[] m; delete[] id; delete[] parent_id;
        pos = vel = acc = nullptr; timestep = m = nullptr; id = parent_id = nullptr;
    }
    // this (GPU store) <- host_system (CPU store)
    void host_to_gpu(particle_system* host_system) {
        if (store == 'c') throw hhs_error(HHS_ERR_INVALID_ARG, "host_to_gpu on a CPU store");
        hhs_check(hhs_particle_system_upload_aos(
                      &dev, N, reinterpret_cast<const double*>(host_system->pos),
                      reinterpret_cast<const double*>(host_system->vel), host_system->m,
                      host_system->timestep, host_system->id, nullptr),
                  "host_to_gpu");
        hhs_check(cudaStreamSynchronize(nullptr) == cudaSuccess ? HHS_OK : HHS_ERR_CUDA,
                  "host_to_gpu");
    }
    // this (CPU store) <- gpu_system (GPU store)
    void gpu_to_host(particle_system* gpu_system) {
        if (store == 'g') throw hhs_error(HHS_ERR_INVALID_ARG, "gpu_to_host on a GPU store");
        hhs_check(hhs_particle_system_download_aos(&gpu_system->dev, N,
                                                   reinterpret_cast<double*>(pos),
                                                   reinterpret_cast<double*>(vel), m, timestep,
                                                   id, nullptr),
                  "gpu_to_host");
        hhs_check(cudaStreamSynchronize(nullptr) == cudaSuccess ? HHS_OK : HHS_ERR_CUDA,
                  "gpu_to_host");
    }
};

// The library context takes the place of the reference's globals (predicate buffers,
// parameters, simtime) and of the per-call level buffers.
template <typename T>
class nbodysystem_globals {
   public:
    int* predicate = nullptr;
    int* scanned_predicate = nullptr;
    T simtime;
    int N_total;
    nbody_params<T> params_host;
    nbody_params<T>* params = &params_host;
    hhs_ctx* ctx = nullptr;

    nbodysystem_globals(int N_init, T eta, T eps, int max_levels = 64)
        : simtime(0), N_total(N_init), params_host{eta, eps} {
        hhs_check(hhs_ctx_create(N_init, max_levels, hhs_params{(double)eta, (double)eps}, &ctx),
                  "nbodysystem_globals");
        if (cudaMalloc(&predicate, sizeof(int) * N_init) != cudaSuccess ||
            cudaMalloc(&scanned_predicate, sizeof(int) * N_init) != cudaSuccess)
            throw hhs_error(HHS_ERR_OOM, "nbodysystem_globals");
    }
    ~nbodysystem_globals() {
        cudaFree(predicate);
        cudaFree(scanned_predicate);
        hhs_ctx_destroy(ctx);
    }
    void flush_simtime() {
        simtime = 0;
        hhs_check(hhs_ctx_flush_simtime(ctx, nullptr), "flush_simtime");
    }
    void print_simtime() { std::printf("simtime: %g\n", (double)simtime); }
};

namespace hhs_detail {
// A context for the entry points whose reference signature carries no globals (split).
inline hhs_ctx* default_ctx(int n) {
    static hhs_ctx* c = nullptr;
    static int cap = 0;
    if (!c || n > cap) {
        if (c) hhs_ctx_destroy(c);
        cap = n;
        hhs_check(hhs_ctx_create(n, 4, hhs_params{0.03, 0.0}, &c), "split context");
    }
    return c;
}
}  // namespace hhs_detail

template <typename T, int BLOCKSIZE>
void hold_step(int clevel, nbodysystem_globals<T>* globals, particle_system<T>* sys,
               const int N_total, T stime, T etime, T dt, bool calc_timestep) {
    hhs_check(hhs_hold_step(globals->ctx, clevel, &sys->dev, N_total, stime, etime, dt,
                            calc_timestep ? 1 : 0, hhs_compat_precision(), nullptr),
              "hold_step");
    hhs_check(hhs_ctx_check(globals->ctx, nullptr), "hold_step");
    double t = 0;
    hhs_check(hhs_ctx_get_simtime(globals->ctx, &t, nullptr), "hold_step");
    globals->simtime = (T)t;
}

template <typename T, int BLOCKSIZE>
void timesteps(particle_system<T>* sys, nbodysystem_globals<T>* globals, const int N) {
    hhs_check(hhs_timesteps(globals->ctx, &sys->dev, N, hhs_compat_precision(), nullptr),
              "timesteps");
}

template <typename T, int BLOCKSIZE, int UNROLL>
void split(particle_system<T>* total, particle_system<T>* slow, particle_system<T>* fast,
           int* predicate, int* scanned_predicate, const T pivot, const int N, partition* part) {
    hhs_check(hhs_split(hhs_detail::default_ctx(N), &total->dev, &slow->dev, &fast->dev,
                        predicate, scanned_predicate, (double)pivot, N,
                        reinterpret_cast<hhs_partition*>(part), nullptr),
              "split");
    hhs_check(cudaDeviceSynchronize() == cudaSuccess ? HHS_OK : HHS_ERR_CUDA, "split");
}

template <typename T, int BLOCKSIZE>
void kick_slow(particle_system<T>* sys, T dt, T fac, const int N) {
    hhs_check(hhs_kick_slow(&sys->dev, dt, fac, N, hhs_compat_precision(), nullptr), "kick_slow");
}

template <typename T, int BLOCKSIZE>
void kick_sf(particle_system<T>* so_sys, particle_system<T>* si_sys, T dt, T fac, const int N,
             const int M) {
    hhs_check(hhs_kick_sf(&so_sys->dev, &si_sys->dev, dt, fac, N, M, hhs_compat_precision(),
                          nullptr),
              "kick_sf");
}

template <typename T, int BLOCKSIZE>
void drift(particle_system<T>* sys, const T dt, const T fac, const int N) {
    hhs_check(hhs_drift(&sys->dev, dt, fac, N, nullptr), "drift");
}

template <typename T, int BLOCKSIZE>
void update_system(particle_system<T>* prev_level_sys, particle_system<T>* cur_level_sys,
                   int N) {
    if (N == 0) return;
    hhs_check(hhs_update_system(&prev_level_sys->dev, &cur_level_sys->dev, N, nullptr),
              "update_system");
}
