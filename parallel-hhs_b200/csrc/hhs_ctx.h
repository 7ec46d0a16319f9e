// hhs_ctx.h -- the library context (definition shared by the host translation units).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "hhs_common.cuh"

// nbodysystem_globals<T> (src/particle_system.cuh:65-104) plus a preallocated
// per-level arena replacing the per-call nbodysystem_buffers<T> of src/hold.cuh:56.
// Level k holds the split of the level-k subsystem into a fast and a slow index list
// (global particle indices, stable order); the level-(k+1) subsystem is the fast
// list of level k, so no particle data is copied between levels.
struct hhs_ctx {
    int n_max = 0;
    int max_levels = 0;
    hhs_params params{0.03, 0.0};
    int device = 0;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    int32_t* fast_lists = nullptr;  // [max_levels][n_max]
    int32_t* slow_lists = nullptr;  // [max_levels][n_max]
    hhs_partition* counts = nullptr;  // [max_levels] device
    void* split_ws = nullptr;         // self-resetting scan workspace
    double* leaf_time = nullptr;      // device: sum of leaf dt (globals->simtime)
    unsigned* err = nullptr;          // device error word (HHS_ERRBIT_*)
    hhs_partition* host_counts = nullptr;  // pinned mirror for the host-driven schedule
    hhs_stats* stats = nullptr;            // device work counters
    void* prof = nullptr;                  // host-side event profiler (hhs_api.cu)
    // device-resident engine state (hhs_engine.cu)
    void* engine = nullptr;
    size_t engine_bytes = 0;
    void* engine_host = nullptr;
    // CUDA graph of a captured multi-step integration (hhs_hold_integrate)
    cudaGraphExec_t graph_exec = nullptr;
    unsigned long long graph_key[6] = {0, 0, 0, 0, 0, 0};
    // candidates timed by the last hhs_ctx_autotune (ms_per_step filled)
    std::vector<hhs_tuning> tune_table;

    int32_t* fast(int level) const { return fast_lists + (size_t)level * n_max; }
    int32_t* slow(int level) const { return slow_lists + (size_t)level * n_max; }
};

// Engine entry points (hhs_engine.cu)
size_t engine_workspace_bytes(int n_max, int max_levels);
hhs_status engine_init(hhs_ctx* c, void* base);
void engine_destroy(hhs_ctx* c);
hhs_status engine_set_tuning(hhs_ctx* c, const hhs_tuning& t);
hhs_status engine_get_tuning(hhs_ctx* c, hhs_tuning* t);
hhs_status engine_get_launch(hhs_ctx* c, int32_t* grid, int32_t* smem_bytes);
hhs_status engine_get_profile(hhs_ctx* c, hhs_profile* out, bool reset);
hhs_status engine_get_level_profile(hhs_ctx* c, double* ms, uint64_t* counts);
hhs_status engine_reset_barrier(hhs_ctx* c, cudaStream_t stream);
hhs_status engine_set_trace(hhs_ctx* c, int32_t* nodes, int64_t capacity,
                            unsigned long long* count);
hhs_status engine_kick_accelerations(hhs_ctx* c, const SoA& P, double* ax, double* ay,
                                     double* az, int n, cudaStream_t stream);
hhs_status engine_timestep_rates(hhs_ctx* c, const SoA& P, int n, cudaStream_t stream);
// Sharded phases of the multi-GPU step (one rank's share; results into every replica).
// Mixed timesteps leave pair-rate maxima in rate_words (local) and the peers' words;
// engine_rates_to_ts turns them into timesteps on every rank after the barrier.
struct PeerOut;
hhs_status engine_shard_timesteps(hhs_ctx* c, const SoA& P, unsigned* rate_words,
                                  const int32_t* S, int n, hhs_precision prec, int rank,
                                  int world, const PeerOut& po, cudaStream_t s);
hhs_status engine_rates_to_ts(hhs_ctx* c, const SoA& P, unsigned* rate_words, const int32_t* S,
                              int n, cudaStream_t s);
// levels with packed kick sources (the mixed sharded kick runs below this level)
int engine_pk_levels(hhs_ctx* c);
// sinks per block of the sharded kick (rank shares are whole blocks)
int engine_shard_kick_block(hhs_precision prec);
// Kick of a split level (positions already drifted), sink blocks [b_lo, b_hi); mixed
// precision returns HHS_ERR_CAPACITY for levels without packed sources (no work done).
hhs_status engine_shard_kick(hhs_ctx* c, const SoA& P, const int32_t* F, const int32_t* L,
                             int nf, int ns, int level, double dt, hhs_precision prec, int b_lo,
                             int b_hi, const PeerOut& po, cudaStream_t s);
// top_level > 0: the launch walks the subtree of the level-top_level node, whose members
// are the fast list of level top_level - 1 (written by the host-driven schedule); dt is
// the top-level step and the node's own step is dt / 2^top_level.
hhs_status engine_hold_step(hhs_ctx* c, const SoA& P, int n, double dt, bool calc_ts,
                            hhs_precision prec, bool profile, cudaStream_t stream,
                            int top_level = 0);
