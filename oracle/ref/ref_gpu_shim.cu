// ref_gpu_shim.cu -- C entry points around the reference's own GPU code, compiled from
// the reference tree as it lies (src/hold.cuh and the headers it includes).
// TEST INFRASTRUCTURE ONLY: it pins the oracle and the CUDA path against the reference
// on a GPU; the product never loads it.
//
// Exposed: the exclusive scan of split<T,BS,4> (src/split.cuh:585-599), the timestep
// kernel (src/timestep.cuh:65-99), kick_slow / kick_sf (src/kick.cuh:158-181) and drift
// (src/drift.cuh:30-43). Not exposed: _set_predicate (its __syncthreads sits inside a
// divergent branch, src/split.cuh:311,332) and hold_step (allocates per call and never
// frees, src/hold.cuh:56). Arrays are the reference's AoS vec3<double> layout.
#include "hold.cuh"

static particle_system<double> view(int n, double* pos3, double* vel3, double* acc3, double* m) {
    particle_system<double> s(n, 'g');
    s.pos = reinterpret_cast<vec3<double>*>(pos3);
    s.vel = reinterpret_cast<vec3<double>*>(vel3);
    s.acc = reinterpret_cast<vec3<double>*>(acc3);
    s.m = m;
    return s;
}

extern "C" int ref_scan_predicate(int* d_pred, int* d_scan, int n, int blocksize) {
    const int unroll = 4;  // UNROLL_FAC, src/hold.cuh:14
    if (n > unroll * blocksize) scan_predicate_large<4>(d_pred, d_scan, n, blocksize);
    else scan_predicate_small<4>(d_pred, d_scan, n);
    return (int)cudaDeviceSynchronize();
}

// N % 256 == 0 keeps the timestep kernel's tail tile (src/timestep.cuh:70) out of play.
extern "C" int ref_timesteps(double* pos3, double* vel3, double* m, double* ts, double eta, int n) {
    nbody_params<double>* params = nullptr;
    cudaMalloc(&params, sizeof(nbody_params<double>));
    nbody_params<double> h{eta, 0.0};
    cudaMemcpy(params, &h, sizeof(h), cudaMemcpyHostToDevice);
    dim3 block(256), grid((256 + n - 1) / 256);
    _timesteps<double, 256><<<grid, block>>>(reinterpret_cast<vec3<double>*>(pos3),
                                             reinterpret_cast<vec3<double>*>(vel3), m, ts,
                                             params, n);
    int e = (int)cudaDeviceSynchronize();
    cudaFree(params);
    return e;
}

extern "C" int ref_kick_slow(double* pos3, double* vel3, double* acc3, double* m, double dt,
                             double fac, int n) {
    particle_system<double> s = view(n, pos3, vel3, acc3, m);
    kick_slow<double, 256>(&s, dt, fac, n);
    return (int)cudaDeviceSynchronize();
}

extern "C" int ref_kick_sf(double* so_pos3, double* so_m, double* si_pos3, double* si_vel3,
                           double* si_acc3, double dt, double fac, int n_sink, int m_src) {
    particle_system<double> so = view(m_src, so_pos3, nullptr, nullptr, so_m);
    particle_system<double> si = view(n_sink, si_pos3, si_vel3, si_acc3, nullptr);
    kick_sf<double, 256>(&so, &si, dt, fac, n_sink, m_src);
    return (int)cudaDeviceSynchronize();
}

extern "C" int ref_drift(double* pos3, double* vel3, double dt, double fac, int n) {
    particle_system<double> s = view(n, pos3, vel3, nullptr, nullptr);
    drift<double, 256>(&s, dt, fac, n);
    return (int)cudaDeviceSynchronize();
}
