/*
 * hhs.h -- C ABI of the B200-native HOLD (Hierarchical Hamiltonian Splitting) step.
 *
 * Drop-in boundary for the header-only C++ templates of parallel-hhs
 * (paths relative to that project's root). Every function returns an hhs_status,
 * never calls exit(), and runs stream-ordered on the caller's cudaStream_t
 * (passed as void*; NULL = legacy default stream). No function allocates device
 * memory while a step runs: particle systems and contexts are allocated up front.
 *
 * Floating point: FP64 state (positions, velocities, masses, timesteps).
 * HHS_PREC_FP64 evaluates every pair term in FP64 with the reference's operation
 * order and no fused multiply-add, so it reproduces the CPU FP64 restatement bit
 * for bit. HHS_PREC_MIXED evaluates pair terms in FP32 from FP64 relative
 * coordinates and accumulates with compensated FP32 sums applied in FP64.
 */
#ifndef HHS_H
#define HHS_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces gpuErrchk -> exit(code) (src/utils.cuh:4-12) and the exit(1) store checks
 * (src/particle_system.cuh:138-141,164-167,181-184,198-201,214-217,232-235). */
typedef enum {
    HHS_OK = 0,
    HHS_ERR_INVALID_ARG = 1,
    HHS_ERR_CUDA = 2,
    HHS_ERR_OOM = 3,
    HHS_ERR_TIMEOUT = 4,             /* a bounded device wait gave up */
    HHS_ERR_DEVICE_FAULT_FLAG = 5,   /* a device-side check recorded an error word */
    HHS_ERR_DEPTH = 6,               /* hierarchy deeper than the context's level capacity */
    HHS_ERR_CAPACITY = 7,            /* n larger than the object was created for */
    HHS_ERR_PEER = 8                 /* a peer rank failed or missed a barrier (multi-GPU) */
} hhs_status;

typedef enum { HHS_PREC_FP64 = 0, HHS_PREC_MIXED = 1 } hhs_precision;

typedef enum {
    HHS_MASS_EQUAL = 0,
    HHS_MASS_SALPETER = 1,       /* dN/dm ~ m^-2.35 on [0.1, 100] */
    HHS_MASS_TWO_COMPONENT = 2   /* 90% m = 1, 10% m = 10 */
} hhs_mass_spectrum;

/* {N_slow, N_fast} -- struct partition, src/particle_system.cuh:8-11 */
typedef struct {
    int32_t n_slow;
    int32_t n_fast;
} hhs_partition;

/* nbody_params<T>, src/particle_system.cuh:13-17. The reference stores eps but never
 * applies it (TODOs at src/hold.cuh:136,141,157); here every kick of the HOLD step
 * (hhs_hold_step, hhs_hold_step_host, hhs_hold_batched) uses d^2 + eps^2, and eps = 0
 * reproduces the unsoftened reference bit for bit. */
typedef struct {
    double eta;
    double eps;
} hhs_params;

/* particle_system<T>, src/particle_system.cuh:20-54, as true SoA FP64 device arrays.
 * The caller owns the struct; hhs_particle_system_alloc fills the pointers from one
 * device allocation (256-byte aligned arrays). */
typedef struct {
    int32_t n;                /* capacity */
    double *x, *y, *z;        /* pos */
    double *vx, *vy, *vz;     /* vel */
    double *ax, *ay, *az;     /* acc (written by the standalone kicks) */
    double *ts;               /* timestep */
    double *m;
    int32_t *id, *parent_id;
    void* _base;              /* owning allocation */
} hhs_particle_system;

/* gpu_alloc / gpu_free: src/particle_system.cuh:135-177 */
hhs_status hhs_particle_system_alloc(hhs_particle_system* sys, int32_t n);
hhs_status hhs_particle_system_free(hhs_particle_system* sys);

/* host_to_gpu / gpu_to_host: src/particle_system.cuh:212-247. Host arrays are SoA;
 * any pointer may be NULL to skip that field. Copies are async on `stream`
 * (pinned host memory makes them truly asynchronous). */
hhs_status hhs_particle_system_upload(hhs_particle_system* sys, int32_t n,
                                      const double* x, const double* y, const double* z,
                                      const double* vx, const double* vy, const double* vz,
                                      const double* m, const double* ts, const int32_t* id,
                                      void* stream);
hhs_status hhs_particle_system_download(const hhs_particle_system* sys, int32_t n,
                                        double* x, double* y, double* z,
                                        double* vx, double* vy, double* vz,
                                        double* m, double* ts, int32_t* id, void* stream);
/* Interleaved (vec3<double>, AoS) host layout of the reference: pos/vel as 3n doubles. */
hhs_status hhs_particle_system_upload_aos(hhs_particle_system* sys, int32_t n,
                                          const double* pos3, const double* vel3,
                                          const double* m, const double* ts,
                                          const int32_t* id, void* stream);
hhs_status hhs_particle_system_download_aos(const hhs_particle_system* sys, int32_t n,
                                            double* pos3, double* vel3, double* m,
                                            double* ts, int32_t* id, void* stream);

/* Library context: nbodysystem_globals<T> (src/particle_system.cuh:65-104) plus the
 * per-level arena that replaces the per-call nbodysystem_buffers<T> allocations of
 * src/hold.cuh:56 (and the per-call scan cudaMalloc of src/split.cuh:512-514).
 * One context per stream; distinct contexts are independent. */
typedef struct hhs_ctx hhs_ctx;

size_t hhs_workspace_size(int32_t n_max, int32_t max_levels);
hhs_status hhs_ctx_create(int32_t n_max, int32_t max_levels, hhs_params params,
                          hhs_ctx** out);
hhs_status hhs_ctx_destroy(hhs_ctx* ctx);
hhs_status hhs_ctx_set_params(hhs_ctx* ctx, hhs_params params);
/* globals->simtime (sum of leaf dt, src/hold.cuh:106-114) -- synchronises the stream */
hhs_status hhs_ctx_get_simtime(hhs_ctx* ctx, double* simtime, void* stream);
hhs_status hhs_ctx_flush_simtime(hhs_ctx* ctx, void* stream);
/* Synchronises the stream and converts the device error words (bounded waits that
 * gave up, depth or capacity overflow) into a status. */
hhs_status hhs_ctx_check(hhs_ctx* ctx, void* stream);
hhs_status hhs_ctx_clear_errors(hhs_ctx* ctx, void* stream);
/* Device-schedule tuning. small_n: nodes with at most small_n particles are solved, with
 * their whole subtree, by a single CTA of the persistent HOLD kernel (0 = never).
 * units_per_cta: target number of (sink block, source chunk) work units per CTA when a
 * node's pair work is cut into source chunks (1..64). ctas_per_sm: 1 or 2 (fewer CTAs make
 * the grid barrier cheaper, more CTAs hide latency better). */
typedef struct {
    int32_t small_n;
    int32_t units_per_cta;
    int32_t ctas_per_sm;     /* CTAs of the persistent kernel per SM (1 or 2) */
    int32_t warp_n;          /* nodes with at most warp_n (<= 32) particles run on one warp */
    int32_t cluster_size;    /* launch the persistent kernel in thread-block clusters (1,2,4,8,
                                or 16 where the device allows clusters beyond 8) */
    int32_t mid_n;           /* nodes with n <= mid_n (at most 640) run, with their whole subtree,
                                from shared memory on the first cluster (on CTA 0 when
                                cluster_size is 1); 0 = never */
    int32_t packed;          /* mixed kick: two sinks per thread in packed FP32x2 arithmetic */
    int32_t mid_dist_n;      /* in such a subtree, nodes with more than mid_dist_n particles spread
                                their pair work over the cluster's CTAs */
    int32_t overlap;         /* mixed: while such a subtree's first pass runs on the first
                                cluster, the other CTAs compute its parent's kick terms between
                                slow particles (1, the default) or wait (0) */
    double ms_per_step;      /* filled by hhs_ctx_autotune: time of the chosen setting */
} hhs_tuning;
hhs_status hhs_ctx_set_tuning(hhs_ctx* ctx, const hhs_tuning* t);
hhs_status hhs_ctx_get_tuning(hhs_ctx* ctx, hhs_tuning* t);
/* Launch shape of the persistent HOLD kernel under the current tuning: grid_ctas[0] for
 * HHS_PREC_FP64 and grid_ctas[1] for HHS_PREC_MIXED (CTAs of 256 threads), and its
 * dynamic shared memory per CTA. Either pointer may be NULL. */
hhs_status hhs_ctx_get_launch(hhs_ctx* ctx, int32_t* grid_ctas, int32_t* smem_bytes);
/* Autotuner: times hold_step on the caller's system for a grid of tuning candidates,
 * restoring the particle state before every trial and at the end, and keeps the fastest.
 * Allocates a snapshot of the system (call it outside any timed or captured region). */
hhs_status hhs_ctx_autotune(hhs_ctx* ctx, hhs_particle_system* sys, int32_t n, double dt,
                            hhs_precision prec, hhs_tuning* out, void* stream);
/* The candidates the last hhs_ctx_autotune timed, in trial order, each with its
 * ms_per_step (the mean of three steps after one warm-up step): *count receives their
 * number, out the first `capacity` of them. Host-only. */
hhs_status hhs_ctx_autotune_results(hhs_ctx* ctx, hhs_tuning* out, int32_t capacity,
                                    int32_t* count);

/* timesteps<T,BS>(sys, globals, N): src/timestep.cuh:103-118 (kernel :65-99) */
hhs_status hhs_timesteps(hhs_ctx* ctx, hhs_particle_system* sys, int32_t n,
                         hhs_precision prec, void* stream);

/* split<T,BS,U>(total, slow, fast, pred, scan, pivot, N, part): src/split.cuh:573-610.
 * Predicate ts <= pivot, exact exclusive scan, stable scatter of pos, vel, m, ts, id
 * with parent_id = source index, N_fast == 1 folded into slow (lone particle last).
 * `part` is a device (or managed) pointer written on the stream; `predicate` and
 * `scanned_predicate` are optional device int32[n] outputs (NULL = not written). */
hhs_status hhs_split(hhs_ctx* ctx, const hhs_particle_system* total,
                     hhs_particle_system* slow, hhs_particle_system* fast,
                     int32_t* predicate, int32_t* scanned_predicate, double pivot,
                     int32_t n, hhs_partition* part, void* stream);

/* kick_slow<T,BS>(sys, dt, fac, N): src/kick.cuh:158-168. acc = sum over the set;
 * vel += acc * (fac*dt). Attractive gravity, as the reference's CPU force test has it
 * (tests/test_nbforce.cu:14-18); the reference GPU kernel adds the opposite sign
 * (src/kick.cuh:23,28). */
hhs_status hhs_kick_slow(hhs_particle_system* sys, double dt, double fac, int32_t n,
                         hhs_precision prec, void* stream);
/* kick_sf<T,BS>(so_sys, si_sys, dt, fac, N_sink, M_src): src/kick.cuh:170-181 */
hhs_status hhs_kick_sf(const hhs_particle_system* so_sys, hhs_particle_system* si_sys,
                       double dt, double fac, int32_t n_sink, int32_t m_src,
                       hhs_precision prec, void* stream);
/* drift<T,BS>(sys, dt, fac, N): src/drift.cuh:30-43 */
hhs_status hhs_drift(hhs_particle_system* sys, double dt, double fac, int32_t n,
                     void* stream);
/* update_system<T,BS>(prev, cur, N): src/update_system.cuh:29-43 */
hhs_status hhs_update_system(hhs_particle_system* prev, const hhs_particle_system* cur,
                             int32_t n, void* stream);

/* hold_step<T,BS>(clevel, globals, sys, N, stime, etime, dt, calc_timestep):
 * src/hold.cuh:51-181. The whole recursive step on the first n particles of sys as one
 * persistent cooperative kernel, stream-ordered and asynchronous: partition counts stay
 * on the device and no host synchronisation happens inside the step (errors surface
 * through hhs_ctx_check). clevel, stime and etime are accepted for the reference's
 * signature; the top level is always 0. */
hhs_status hhs_hold_step(hhs_ctx* ctx, int32_t clevel, hhs_particle_system* sys,
                         int32_t n, double stime, double etime, double dt,
                         int32_t calc_timestep, hhs_precision prec, void* stream);

/* `steps` consecutive top-level steps (calc_timestep = 1 each), captured once into a CUDA
 * graph and replayed on later calls with the same system, n, dt, steps, precision and
 * tuning (one graph launch per call). Falls back to direct launches when the stream
 * cannot be captured. Not for use inside another stream capture. */
hhs_status hhs_hold_integrate(hhs_ctx* ctx, hhs_particle_system* sys, int32_t n, double dt,
                              int32_t steps, hhs_precision prec, void* stream);

/* The same step driven from the host: the partition counts are read back after every
 * split (the reference synchronises at the same point, src/split.cuh:430) and the
 * recursion runs on the CPU. Synchronous; the plain baseline schedule. */
hhs_status hhs_hold_step_host(hhs_ctx* ctx, hhs_particle_system* sys, int32_t n, double dt,
                              int32_t calc_timestep, hhs_precision prec, void* stream);

/* ---- one system on several GPUs (sink-partitioned kick) --------------------------- */
/* Every rank (one per GPU) holds a full replica of the system and runs the host-driven
 * schedule of hhs_hold_step_host on it. Each timestep and kick launch of at least
 * min_pairs pair terms is split by sink across the ranks: a rank computes its shard of
 * the sinks and its kernel stores every result both locally and straight into each
 * peer replica (P2P stores over NVLink), so the launch is the all-gather. A barrier
 * before the launch (no peer still reads the old values) and one after it (every
 * store has landed) bracket each shared launch. Everything else (splits, drifts, small
 * levels) runs replicated and bit-identically on every rank, so all replicas stay
 * equal, and equal to hhs_hold_step_host on one GPU: per sink, a shard computes the
 * same operations in the same order as the whole launch.
 *
 * The barrier is the host's: hhs_barrier_fn(user, stream) must return 0 once the work
 * enqueued on `stream` by every rank before the call is complete before any rank's
 * later work starts (an NCCL all-reduce of one value on the stream, or a stream
 * synchronise followed by a host barrier), or non-zero if a peer failed or did not
 * arrive in time, which ends the step with HHS_ERR_PEER. Every rank takes the same
 * barrier steps in the same order. */
typedef int32_t (*hhs_barrier_fn)(void* user, void* stream);
typedef struct hhs_dist hhs_dist;
#define HHS_DIST_MAX_RANKS 8
/* replicas[world]: each rank's system, as this process addresses it (a peer's arrays
 * opened with hhs_ipc_open, or the systems themselves when the ranks share a process);
 * replicas[rank] is not used. All replicas have the same capacity. */
hhs_status hhs_dist_create(hhs_dist** out, int32_t rank, int32_t world,
                           const hhs_particle_system* replicas, hhs_barrier_fn barrier,
                           void* user, int64_t min_pairs);
hhs_status hhs_dist_destroy(hhs_dist* d);
/* Sink range [lo, hi) of `rank` for a launch whose first n_fast sinks cost n_slow pair
 * terms each and whose other n_slow sinks cost n_slow + n_fast each (one kick of a split
 * level; a timestep launch over n particles is n_fast = 0, n_slow = n): ranks get
 * contiguous ranges of equal cost to within one sink. Host-only arithmetic. */
hhs_status hhs_dist_shard(int32_t n_fast, int32_t n_slow, int32_t rank, int32_t world,
                          int32_t* lo, int32_t* hi);
/* Subtrees in which no launch reaches min_pairs pair terms run, by default, as one
 * launch of the device-resident engine (the kernel of hhs_hold_step) from their own
 * level, identically on every rank. on = 0 keeps them on the host-driven schedule. With
 * the engine, the FP64 replicas still equal hhs_hold_step_host bit for bit; the mixed
 * ones equal a one-rank run with the same min_pairs. */
hhs_status hhs_dist_set_subtree_engine(hhs_dist* d, int32_t on);
/* Configuration agreement. The order of the mixed-precision sums (and so the bits of
 * every replica) depends on the engine's launch shape and tuning, which each rank sets
 * on its own context. fn(user, value, out_min, out_max) returns in *out_min / *out_max
 * the minimum and maximum of `value` over all ranks (for example two all-reduces on the
 * ranks' communicator) and 0, or non-zero if a peer failed. With it set, every
 * hhs_hold_step_dist first compares a hash of this rank's configuration
 * (hhs_dist_config_hash) across the ranks and returns HHS_ERR_INVALID_ARG on every rank
 * when they differ, before any kernel runs; HHS_ERR_PEER if fn fails. Host-only. */
typedef int32_t (*hhs_minmax_fn)(void* user, uint64_t value, uint64_t* out_min,
                                 uint64_t* out_max);
hhs_status hhs_dist_set_agreement(hhs_dist* d, hhs_minmax_fn fn, void* user);
/* The hash compared by the agreement check: precision, launch shape (grid CTAs of the
 * persistent kernel for that precision), tuning, n, dt, eta and eps. Host-only. */
hhs_status hhs_dist_config_hash(const hhs_tuning* t, int32_t grid_ctas, hhs_precision prec,
                                int32_t n, double dt, hhs_params params, uint64_t* out);
/* Runs the agreement check on a given hash: HHS_OK when every rank passed the same
 * value (or no agreement function is set), HHS_ERR_INVALID_ARG when they differ,
 * HHS_ERR_PEER if the function failed. Every rank must call it. Host-only. */
hhs_status hhs_dist_check(hhs_dist* d, uint64_t config_hash);
/* One top-level step (hold_step, src/hold.cuh:51-181) of the rank's replica sys. */
hhs_status hhs_hold_step_dist(hhs_ctx* ctx, hhs_dist* d, hhs_particle_system* sys, int32_t n,
                              double dt, int32_t calc_timestep, hhs_precision prec,
                              void* stream);
/* Peer mappings of a system's device allocation (CUDA IPC): the handle is 64 bytes;
 * hhs_ipc_open maps another process's system of capacity n into this one (peer access
 * enabled) and fills a view whose arrays address it; close a view with hhs_ipc_close,
 * never hhs_particle_system_free. */
#define HHS_IPC_HANDLE_BYTES 64
hhs_status hhs_ipc_handle(const hhs_particle_system* sys, void* handle_out);
hhs_status hhs_ipc_open(const void* handle, int32_t n, hhs_particle_system* view_out);
hhs_status hhs_ipc_close(hhs_particle_system* view);

/* Exact exclusive prefix sum of int32 values (the contract of
 * scan_predicate_small/large, src/split.cuh:438-565): one decoupled-lookback pass below
 * 2^22 values, two passes over chunks (chunk sums, then chunk scans) up to 2^25, and from
 * 2^25 values (16-byte aligned input and output) one streamed pass: a cooperative launch
 * of resident CTAs that bulk-copy chunks into shared memory and exchange chunk
 * aggregates two rounds ahead (unaligned pointers keep the two-pass form).
 * d_workspace: hhs_scan_workspace_size(n) bytes of device memory (need not be zeroed;
 * the call clears what it uses). */
size_t hhs_scan_workspace_size(int64_t n);
hhs_status hhs_scan_exclusive_i32(const int32_t* d_in, int32_t* d_out, int64_t n,
                                  void* d_workspace, size_t workspace_bytes, void* stream);
/* Allocation-free exclusive scan. No counterpart in the reference: it is an addition for
 * callers that must not allocate device memory -- an application that has handed the
 * device to its own memory pool, or a step loop that must run under a fixed device-memory
 * budget -- and so cannot provide the workspace hhs_scan_exclusive_i32 needs. The same
 * kernels (the single pass below 2^22 values, the two-pass form up to 2^25, the streamed
 * pass above) run with their workspace in a fixed 128.3 KiB array inside the library's own
 * device memory, present on every device that loads the library until the process
 * exits. Limit: n <= HHS_SCAN_NOALLOC_MAX_N (2^26 values); larger n returns
 * HHS_ERR_CAPACITY. The call allocates nothing; it clears the part of the array it uses
 * with cudaMemsetAsync before the launch. Every call shares the one array, so calls
 * that overlap on the GPU (different streams, or several host threads at once) race:
 * serialise them. The first call on each device looks up the array's device address;
 * make that first call before any stream capture. */
#define HHS_SCAN_NOALLOC_MAX_N (1LL << 26)
hhs_status hhs_scan_exclusive_i32_noalloc(const int32_t* d_in, int32_t* d_out, int64_t n,
                                          void* stream);
/* Status of the last hhs_scan_exclusive_i32_noalloc on the current device (its bounded
 * look-back waits record a timeout in the array instead of hanging): synchronises the
 * stream; HHS_ERR_TIMEOUT if a wait gave up, in which case the output is not valid.
 * The array's device address is looked up once per device and kept for the life of the
 * process; it does not survive cudaDeviceReset (the library's module is reloaded), so
 * do not call these functions after a device reset. */
hhs_status hhs_scan_noalloc_status(void* stream);
/* Bounded-wait self-test on the same static array: the scan with its first tile left
 * out, every look-back giving up after max_polls (1..2^22) polls. Synchronises the
 * stream; returns HHS_ERR_TIMEOUT when the waits ran out as designed. 8192 <= n <= 2^26. */
hhs_status hhs_scan_noalloc_selftest_stalled_predecessor(const int32_t* d_in, int32_t* d_out,
                                                         int64_t n, uint32_t max_polls,
                                                         void* stream);

/* Stream compaction (the split of a flag array, src/split.cuh:573-610 on int32 data):
 * d_idx[k] = index of the k-th nonzero flag, *d_count = number of nonzero flags, and
 * d_scan (optional, NULL = not written) = exclusive scan of (flag != 0). One pass below
 * 2^22 flags; from there on chunk sums then chunk scans (from 2^24 flags in one
 * cooperative launch, in waves of 2^24 flags). Workspace as for hhs_scan_exclusive_i32. */
hhs_status hhs_compact_flags_i32(const int32_t* d_flags, int32_t* d_scan, int32_t* d_idx,
                                 int32_t* d_count, int64_t n, void* d_workspace,
                                 size_t workspace_bytes, void* stream);
/* Synchronises the stream; HHS_ERR_TIMEOUT if a look-back wait of the last scan on this
 * workspace gave up. */
hhs_status hhs_scan_workspace_status(const void* d_workspace, void* stream);
/* The split in the (unstable) particle order of the HHS CPU integrators: the permutation
 * left by cpu_split's in-place two-pointer partition (src/cpu_scan.h:20-50) of d_ts
 * against pivot. d_order[0..n_fast) = fast (ts <= pivot), d_order[n_fast..n) = slow;
 * *d_counts on the device. No N_fast == 1 fold (cpu_split has none). Workspace: 256-byte
 * aligned, hhs_split_cpu_order_workspace_size(n) bytes. */
size_t hhs_split_cpu_order_workspace_size(int64_t n);
hhs_status hhs_split_cpu_order(const double* d_ts, int32_t n, double pivot, int32_t* d_order,
                               hhs_partition* d_counts, void* d_workspace,
                               size_t workspace_bytes, void* stream);
/* Failure-detection self-test of the bounded look-back wait (no counterpart in the
 * reference, whose waits are unbounded): runs the scan with its first tile left out, so
 * every look-back waits for a predecessor that never publishes; each wait gives up after
 * max_polls (1..2^22) polls, records the timeout in the workspace and returns. Synchronises
 * the stream; returns HHS_ERR_TIMEOUT when the waits ran out as designed. n >= 8192. */
hhs_status hhs_scan_selftest_stalled_predecessor(const int32_t* d_in, int32_t* d_out, int64_t n,
                                                 void* d_workspace, size_t workspace_bytes,
                                                 uint32_t max_polls, void* stream);
/* Failure-detection self-test of the bounded grid barrier of the wave-form scan (the
 * one-launch form that stream compaction uses from 2^24 values): runs it with every
 * barrier waiting for one CTA more than the launch has; each wait gives up after
 * timeout_us (1..10^7) microseconds, records the timeout in the workspace and returns.
 * d_out is left unspecified. Synchronises the stream; returns HHS_ERR_TIMEOUT when the
 * waits ran out as designed. n >= 2^22. */
hhs_status hhs_scan_selftest_wave_barrier(const int32_t* d_in, int32_t* d_out, int64_t n,
                                          void* d_workspace, size_t workspace_bytes,
                                          uint32_t timeout_us, void* stream);

/* ---- diagnostics ---------------------------------------------------------------- */
/* Work recorded by the HOLD schedule since the last reset (device counters). */
typedef struct {
    uint64_t nodes;          /* hold_step calls (split nodes) */
    int32_t max_level;
    int32_t _pad;
    double kick_pairs;       /* sum over nodes of N_s(N_s-1) + 2 N_s N_f */
    double ts_pairs;         /* sum over timestep evaluations of N(N-1) */
} hhs_stats;
hhs_status hhs_ctx_get_stats(hhs_ctx* ctx, hhs_stats* out, void* stream);
hhs_status hhs_ctx_reset_stats(hhs_ctx* ctx, void* stream);

/* Per-kernel timing of the pair kernels (CUDA events on the launching stream) while
 * profiling is on; kinds: 0 timesteps, 1 kick, 2 split, 3 drift, 4 whole-step engine. */
typedef struct {
    uint64_t launches[8];
    double ms[8];
    double pairs[8];
} hhs_profile;
hhs_status hhs_ctx_set_profiling(hhs_ctx* ctx, int32_t on);
hhs_status hhs_ctx_get_profile(hhs_ctx* ctx, hhs_profile* out);
/* The device schedule's phase times per kind and level since profiling was switched on:
 * ms[kind*64 + level] milliseconds and counts[kind*64 + level] phases (either may be NULL). */
hhs_status hhs_ctx_get_level_profile(hhs_ctx* ctx, double* ms, uint64_t* counts);

/* Node trace of the device-resident step (hhs_hold_step): while set, every node of the
 * recursion -- each call of the reference's hold_step, src/hold.cuh:51-181 -- appends
 * {level, n, n_fast, calc_timestep} (4 int32) to d_nodes in call order, and *d_count
 * (device uint64, zeroed by the caller) counts the nodes, also past capacity. n_fast is
 * the count after the N_fast == 1 fold. d_nodes is 16-byte aligned device memory; NULL
 * (with d_count NULL) switches the trace off. The same record as the CPU restatement's
 * trace, so a hierarchy can be compared node by node. */
hhs_status hhs_ctx_set_trace(hhs_ctx* ctx, int32_t* d_nodes, int64_t capacity,
                             uint64_t* d_count);

/* Accelerations computed by the mixed-precision kick phase of hhs_hold_step -- the same
 * packed tiles, work units, FP32 pair arithmetic, column sums and compensated sums --
 * for the first n >= 2 particles taken as one split node whose fast set is every third
 * particle (index % 3 == 0) and whose slow set is the rest, positions as they are:
 * fast particles get the pull of the slow set, slow particles that of all others, as
 * in the kick of src/hold.cuh:135-143. Written to sys->ax, ay, az. A diagnostic for
 * checking that arithmetic against an FP64 direct sum; it uses the context's level
 * lists and kick scratch, so do not run it concurrently with a step on the context. */
hhs_status hhs_engine_kick_accelerations(hhs_ctx* ctx, hhs_particle_system* sys, int32_t n,
                                         void* stream);

/* Timesteps computed by the mixed-precision timestep phase of hhs_hold_step -- the same
 * packed members, bulk-copied column tiles, symmetric FP32 pair rates (one evaluation per
 * unordered pair) and row/column maxima -- for the first n >= 2 particles taken as one
 * node (every other particle of the n is a source), converted to timesteps as the split
 * does (1 / max rate, capped at 1e30) and written to sys->ts. The counterpart of
 * _timesteps / timesteps (src/timestep.cuh:65-118) in mixed precision; a diagnostic for
 * checking that arithmetic against the FP64 expression. It uses the context's packed
 * member arrays and rate words, so do not run it concurrently with a step on the
 * context. */
hhs_status hhs_engine_timestep_rates(hhs_ctx* ctx, hhs_particle_system* sys, int32_t n,
                                     void* stream);

/* Kernel launches issued by this library since it was loaded (all contexts). */
uint64_t hhs_kernel_launch_count(void);

/* Measured arithmetic peaks of the current device: a register-resident chain of FP32
 * (and FP64) fused multiply-adds on every SM, timed with CUDA events. TFLOP/s. */
hhs_status hhs_measure_fma_peaks(double* fp32_tflops, double* fp64_tflops, void* stream);
/* The same chain with packed FP32 pairs (sm_100 fma.rn.f32x2). TFLOP/s. */
hhs_status hhs_measure_fma2_peak(double* fp32x2_tflops, void* stream);

/* ---- batched systems ------------------------------------------------------------ */
/* Many independent systems packed back to back in one particle system: system k holds
 * particles [offsets[k], offsets[k+1]) (host array, offsets[0] = 0). hhs_hold_batched
 * advances every system by one top-level HOLD step in ONE launch: hardware thread-block
 * clusters take the large systems (largest first, one cluster per system, cluster
 * barriers between phases), then single CTAs take the rest, each split being a
 * per-system (segmented) scan and compaction. Per-system leaf times are kept. */
typedef struct hhs_batch hhs_batch;
hhs_status hhs_batch_create(int32_t n_sys, const int32_t* offsets, int32_t max_levels,
                            hhs_params params, hhs_batch** out);
hhs_status hhs_batch_destroy(hhs_batch* b);
/* big_n: systems with more particles run on a thread-block cluster; small_n: inside a
 * system, nodes with at most small_n particles run on one CTA; units_per_cta as above. */
hhs_status hhs_batch_set_tuning(hhs_batch* b, int32_t big_n, int32_t small_n,
                                int32_t units_per_cta);
/* Subtrees of at most mid_n (<= 640) particles run from shared memory: on the system's
 * cluster for large systems (nodes above mid_dist_n spread over its CTAs), on one CTA for
 * the others (default 640 and 96; mid_n = 0 turns it off). */
hhs_status hhs_batch_set_mid(hhs_batch* b, int32_t mid_n, int32_t mid_dist_n);
/* Tuning of the batched launch, as hhs_batch_set_tuning / hhs_batch_set_mid set it. */
typedef struct {
    int32_t big_n, small_n, units_per_cta, mid_n, mid_dist_n;
    double ms_per_step;      /* filled by hhs_batch_autotune */
} hhs_batch_tuning;
/* Batched autotuner: times hhs_hold_batched on the caller's systems for a grid of
 * (big_n, units_per_cta, mid_dist_n) candidates -- the state, per-system leaf times and
 * work counters restored before every trial and at the end -- and keeps the fastest.
 * out (optional) receives it; table (optional, capacity entries) every candidate timed,
 * *count (optional) their number. Allocates a snapshot of the state: call it outside
 * any timed or captured region. */
hhs_status hhs_batch_autotune(hhs_batch* b, hhs_particle_system* sys, double dt,
                              hhs_precision prec, hhs_batch_tuning* out,
                              hhs_batch_tuning* table, int32_t capacity, int32_t* count,
                              void* stream);
hhs_status hhs_hold_batched(hhs_batch* b, hhs_particle_system* sys, double dt,
                            int32_t calc_timestep, hhs_precision prec, void* stream);
hhs_status hhs_batch_get_simtime(hhs_batch* b, double* per_system, void* stream);
hhs_status hhs_batch_get_stats(hhs_batch* b, hhs_stats* out, void* stream);
hhs_status hhs_batch_reset_stats(hhs_batch* b, void* stream);
hhs_status hhs_batch_check(hhs_batch* b, void* stream);

/* Multi-GPU sharding of a batch (host only, no device work): assigns each of the n_sys
 * independent systems (sizes[k] particles) to one of n_ranks ranks so that the per-rank
 * sums of sizes[k]^2 (the O(N^2) pair work) are balanced: longest-processing-time greedy,
 * systems taken by decreasing size (ties by index), each to the least-loaded rank (ties by
 * rank). Deterministic, so every rank computes the same rank_of[n_sys] without an
 * exchange. load (optional, n_ranks entries) receives each rank's sum of sizes^2. */
hhs_status hhs_batch_partition(int32_t n_sys, const int32_t* sizes, int32_t n_ranks,
                               int32_t* rank_of, double* load);

/* ---- driver: hold(), energy diagnostic, snapshots ------------------------------ */
/* FP64 total energy of the first n particles (kinetic and potential, compensated sums,
 * pair potential with softening length eps). Uses the system's acceleration arrays as
 * scratch; synchronises the stream. */
hhs_status hhs_energy(hhs_particle_system* sys, int32_t n, double eps, double* kinetic,
                      double* potential, void* stream);
/* Binary snapshot (checkpoint): an 80-byte header ("HHSSNAP1", n, time, eta, eps, dt,
 * step) followed by the FP64 SoA arrays x y z vx vy vz m ts and the int32 ids. */
hhs_status hhs_snapshot_write(const hhs_particle_system* sys, int32_t n, double time,
                              const hhs_params* params, double dt, int32_t step,
                              const char* path, void* stream);
hhs_status hhs_snapshot_read(hhs_particle_system* sys, const char* path, int32_t* n_out,
                             double* time, int32_t* step, void* stream);
/* Energy log filled by hhs_hold: one (time, energy) entry per diagnostic. */
typedef struct {
    double* time;
    double* energy;
    int32_t capacity;
    int32_t n_entries;
} hhs_run_log;
/* hold(...) of the reference (declared at src/hold.cuh:20-23, sketched at :26-35, never
 * defined): integrate from stime to etime in top-level steps of dt. Every
 * snapshot_every steps and at the end the energy is logged and, with a non-empty
 * prefix, "<prefix>_<step>.hhs" is written. Segments run as graph-captured steps. */
hhs_status hhs_hold(hhs_ctx* ctx, hhs_particle_system* sys, int32_t n, double stime,
                    double etime, double dt, hhs_precision prec, int32_t snapshot_every,
                    const char* snapshot_prefix, hhs_run_log* log, void* stream);

/* Host-side utilities (no GPU): seeded Plummer initial conditions in Henon units,
 * and FP64 energies with compensated sums. */
hhs_status hhs_ic_plummer(int32_t n, uint64_t seed, int32_t mass_spectrum, double* x,
                          double* y, double* z, double* vx, double* vy, double* vz,
                          double* m);
double hhs_host_potential_energy(int32_t n, const double* x, const double* y,
                                 const double* z, const double* m);
double hhs_host_kinetic_energy(int32_t n, const double* vx, const double* vy,
                               const double* vz, const double* m);

/* Human-readable name of a status code. */
const char* hhs_status_string(hhs_status s);

#ifdef __cplusplus
}
#endif
#endif /* HHS_H */
