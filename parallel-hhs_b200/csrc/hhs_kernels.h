// hhs_kernels.h -- host-side launchers shared between the library's .cu files.
#pragma once
#include <cuda_runtime.h>

#include "hhs_internal.h"

struct SoA;

// ---- scan / split (hhs_scan.cu)
size_t scan_workspace_bytes(long long n, int tile);
size_t split_workspace_bytes(int n);
unsigned* scan_workspace_error_word(void* ws);
hhs_status launch_split_list(const int32_t* list_in, int n, const double* ts, double pivot,
                             int32_t* fast_out, int32_t* slow_out, int32_t* pred_out,
                             int32_t* scan_out, hhs_partition* counts, double* leaf_time,
                             double dt, hhs_stats* stats, int level, int calc_ts, void* ws,
                             cudaStream_t stream);

// ---- pair kernels, drift, gathers (hhs_pairs.cu)
// Sink-partitioned launch of a pair kernel (the multi-GPU HOLD step): only sinks
// [lo, hi) of the launch's sink index space are computed, and every result is stored
// both in the local arrays and in each peer replica's arrays (P2P stores over NVLink,
// or plain stores when the replicas share a device). hi < 0 selects every sink and
// n_peer = 0 writes the local arrays only: the single-GPU launch.
constexpr int kMaxPeers = 7;  // an 8-GPU NVSwitch node
struct PeerOut {
    int lo, hi, n_peer;
    double* vx[kMaxPeers];
    double* vy[kMaxPeers];
    double* vz[kMaxPeers];
    double* ts[kMaxPeers];
    unsigned* rate[kMaxPeers];  // peers' pair-rate words (their ax arrays, reinterpreted)
};
inline PeerOut peer_out_local() {
    PeerOut p{};
    p.lo = 0; p.hi = -1; p.n_peer = 0;
    return p;
}
// Timesteps of the subsystem given by list (identity when nullptr), min over j != i.
hhs_status launch_timesteps(const SoA& P, const int32_t* list, int n, double eta,
                            hhs_precision prec, cudaStream_t stream,
                            const PeerOut& po = peer_out_local());
// One HOLD kick of a split level: slow sinks get slow then fast sources, fast sinks get
// slow sources; v += a*dt. Counts are read from the device (n_max bounds the grid). The
// sink index space is the fast list, then the slow list.
hhs_status launch_kick_level(const SoA& P, const int32_t* fast_list,
                             const int32_t* slow_list, const hhs_partition* counts,
                             int n_max, double dt, double eps2, hhs_precision prec,
                             cudaStream_t stream, const PeerOut& po = peer_out_local());
// Standalone kick: sinks = sink[0..n_sink), sources = src[0..n_src); acc written.
hhs_status launch_kick_pair(const SoA& sink, double* ax, double* ay, double* az,
                            const SoA& src, int n_sink, int n_src, double dtfac,
                            hhs_precision prec, cudaStream_t stream);
// pos += vel*h for the slow part of a split level (count read from the device).
hhs_status launch_drift_slow(const SoA& P, const int32_t* slow_list,
                             const hhs_partition* counts, int n_max, double h,
                             cudaStream_t stream);
hhs_status launch_drift(const SoA& P, int n, double h, cudaStream_t stream);
hhs_status launch_update_system(const SoA& prev, const SoA& cur, const int32_t* parent_id,
                                int n, cudaStream_t stream);
hhs_status launch_gather_split(const SoA& total, const SoA& slow, int32_t* slow_parent,
                               const SoA& fast, int32_t* fast_parent,
                               const int32_t* slow_list, const int32_t* fast_list,
                               const hhs_partition* counts, int n_max, cudaStream_t stream);

// ---- diagnostics (hhs_diag.cu)
hhs_status measure_fma_peaks(double* fp32_tflops, double* fp64_tflops, cudaStream_t stream);
hhs_status measure_fma2_peak(double* tflops, cudaStream_t stream);
