// test_compat.cpp -- a reference-style caller compiled against include/hhs.hpp.
//
// It is written the way the reference's own programs use its headers (particle_system
// with CPU and GPU stores, host_to_gpu / gpu_to_host, hold_step<T,BS>, split<T,BS,U>
// with a managed partition, the PASS/FAIL printing of tests/harness.h), so it shows
// that such code builds and runs unchanged on this library. It prints one JSON line
// that the pytest wrapper checks against the C ABI driven from Python.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hhs.hpp"

#define TEST_ASSERT(name, cond) \
    std::printf("%s %s\n", (cond) ? "[PASS]" : "[FAIL]", name)

static unsigned long long fnv(const void* p, size_t n, unsigned long long h) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ull; }
    return h;
}

int main(int argc, char** argv) {
    const int N = argc > 1 ? std::atoi(argv[1]) : 1024;
    const int steps = argc > 2 ? std::atoi(argv[2]) : 2;
    const double dt = 1.0 / 64, eta = 0.03;

    std::vector<double> x(N), y(N), z(N), vx(N), vy(N), vz(N), m(N);
    if (hhs_ic_plummer(N, 99, HHS_MASS_EQUAL, x.data(), y.data(), z.data(), vx.data(),
                       vy.data(), vz.data(), m.data()) != HHS_OK)
        return 2;

    particle_system<double> host(N, 'c'), gpu(N, 'g');
    host.cpu_alloc();
    for (int i = 0; i < N; i++) {
        host.pos[i] = vec3<double>(x[i], y[i], z[i]);
        host.vel[i] = vec3<double>(vx[i], vy[i], vz[i]);
        host.m[i] = m[i];
        host.timestep[i] = 0.0;
        host.id[i] = i;
    }
    gpu.gpu_alloc();
    gpu.host_to_gpu(&host);

    nbodysystem_globals<double> globals(N, eta, 0.0);
    double t = 0;
    for (int s = 0; s < steps; s++) {
        hold_step<double, 256>(0, &globals, &gpu, N, t, t + dt, dt, true);
        t += dt;
    }
    host.gpu_to_host(&gpu);
    TEST_ASSERT("simtime advanced", globals.simtime > 0.0);

    // split of the final timesteps, as the reference's split tests do (counts and sides)
    particle_system<double> slow(N, 'g'), fast(N, 'g');
    slow.gpu_alloc();
    fast.gpu_alloc();
    partition* part = nullptr;
    cudaMallocManaged(&part, sizeof(partition));
    const double pivot = dt / 8;
    split<double, 256, 4>(&gpu, &slow, &fast, globals.predicate, globals.scanned_predicate,
                          pivot, N, part);
    TEST_ASSERT("Total size check (slow + fast == total)", part->N_slow + part->N_fast == N);
    int below = 0;
    for (int i = 0; i < N; i++) below += host.timestep[i] <= pivot;
    TEST_ASSERT("fast count", part->N_fast == (below == 1 ? 0 : below));

    unsigned long long h = 1469598103934665603ull;
    h = fnv(host.pos, sizeof(vec3<double>) * N, h);
    h = fnv(host.vel, sizeof(vec3<double>) * N, h);
    h = fnv(host.timestep, sizeof(double) * N, h);
    std::printf("{\"n\": %d, \"steps\": %d, \"simtime\": %.17g, \"n_fast\": %d, "
                "\"n_slow\": %d, \"fnv\": \"%016llx\", \"x0\": %.17g}\n",
                N, steps, (double)globals.simtime, part->N_fast, part->N_slow, h, host.pos[0].x);
    cudaFree(part);
    slow.gpu_free();
    fast.gpu_free();
    gpu.gpu_free();
    host.cpu_free();
    return 0;
}
