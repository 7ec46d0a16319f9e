/*
 * hhs_oracle.h -- CPU FP64 restatement of the HOLD step of parallel-hhs.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker against which the CUDA path is
 * compared. Only the test suite, the smoke check and the CPU-baseline leg of the
 * benchmark may load it; the product library never links or calls it.
 *
 * Every function restates one piece of the reference (paths relative to the
 * parallel-hhs project root):
 *   oracle_timesteps      src/timestep.cuh:10-99  (pair timestep, min over j != i;
 *                         the tail-tile read of uninitialised shared memory at
 *                         src/timestep.cuh:70,84-88 is NOT reproduced: the min runs
 *                         over every j != i)
 *   oracle_scan_exclusive src/split.cuh:131-302,372-394,438-565 (exact exclusive
 *                         prefix sum of the 0/1 predicate)
 *   oracle_split          src/split.cuh:107-117,304-370,573-610 (predicate ts <= pivot,
 *                         stable scatter, N_fast==1 fold with the lone fast particle
 *                         placed last in the slow set -- the intended semantics of
 *                         src/split.cuh:321-324,361-368)
 *   oracle_kick           src/kick.cuh:15-55,59-155 (direct sum, d2==0 skipped;
 *                         ATTRACTIVE sign as in tests/test_nbforce.cu:14-18)
 *   oracle_drift          src/drift.cuh:16-28
 *   oracle_hold_step      src/hold.cuh:51-181 (recursive schedule, per-level copies,
 *                         update_system of src/update_system.cuh:10-25)
 *
 * All arithmetic is IEEE binary64 with no fused multiply-add (the file is compiled
 * with -ffp-contract=off) and the operation order of the reference expressions.
 */
#ifndef HHS_ORACLE_H
#define HHS_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* one node of the recorded HOLD call tree (call order) */
typedef struct {
    int32_t level;
    int32_t n;        /* particles in this (sub)system */
    int32_t n_fast;   /* after the N_fast==1 fold */
    int32_t calc_ts;  /* 1 if timesteps were recomputed at this node */
} oracle_node;

typedef struct {
    oracle_node* nodes;   /* caller buffer, may be NULL */
    int64_t capacity;     /* entries available in nodes */
    int64_t count;        /* nodes visited (may exceed capacity) */
    int32_t max_level;
    double  leaf_time;    /* sum of dt over leaves (reference globals->simtime) */
    double  kick_pairs;   /* N_s(N_s-1)+2 N_s N_f summed over nodes */
    double  ts_pairs;     /* N(N-1) summed over nodes with calc_ts */
} oracle_trace;

void oracle_timesteps(int n, const double* x, const double* y, const double* z,
                      const double* vx, const double* vy, const double* vz,
                      const double* m, double eta, double* ts);

void oracle_scan_exclusive_i32(int64_t n, const int32_t* in, int32_t* out);

/* Writes the permutation of parent indices: order[0..n_fast) = fast set,
 * order[n_fast..n) = slow set, and returns n_fast (after the fold). */
int oracle_split(int n, const double* ts, double pivot, int32_t* order);

/* cpu_split (src/cpu_scan.h:20-50) on indices: the unstable in-place partition of the
 * HHS CPU integrators. order receives fast then slow indices; returns n_fast. */
int oracle_split_cpu_order(int n, const double* ts, double pivot, int32_t* order);

/* sinks: positions (read) and velocities (updated by acc*dtfac); sources: positions
 * and masses. acc (3 arrays, may be NULL) receives this call's acceleration. */
void oracle_kick(int n_sink, const double* sx, const double* sy, const double* sz,
                 double* svx, double* svy, double* svz,
                 double* ax, double* ay, double* az,
                 int n_src, const double* px, const double* py, const double* pz,
                 const double* pm, double dtfac);

/* oracle_kick with a softening length: d2 = dx.dx + eps2 (eps2 = eps^2). */
void oracle_kick_soft(int n_sink, const double* sx, const double* sy, const double* sz,
                      double* svx, double* svy, double* svz,
                      double* ax, double* ay, double* az,
                      int n_src, const double* px, const double* py, const double* pz,
                      const double* pm, double dtfac, double eps2);

void oracle_drift(int n, double* x, double* y, double* z,
                  const double* vx, const double* vy, const double* vz, double dtfac);

/* One recursive HOLD step on the whole system, in place. id is carried along. */
void oracle_hold_step(int n, double* x, double* y, double* z,
                      double* vx, double* vy, double* vz, double* m, double* ts,
                      int32_t* id, double dt, int calc_ts, double eta,
                      oracle_trace* trace);

/* oracle_hold_step with every kick softened by eps2 = eps^2. */
void oracle_hold_step_soft(int n, double* x, double* y, double* z,
                           double* vx, double* vy, double* vz, double* m, double* ts,
                           int32_t* id, double dt, int calc_ts, double eta, double eps2,
                           oracle_trace* trace);

/* Total energy with Neumaier-compensated sums: out[0]=kinetic, out[1]=potential. */
void oracle_energy(int n, const double* x, const double* y, const double* z,
                   const double* vx, const double* vy, const double* vz,
                   const double* m, double* out);

/* Seeded Plummer sphere in Henon units (mass_spectrum 0 equal, 1 Salpeter on [0.1,100],
 * 2 two-component 90/10): the inputs of the benchmark's CPU-baseline leg, identical bit
 * for bit to the product generator's for the same seed. Returns 0, or 1 on bad
 * arguments. */
int oracle_plummer(int n, uint64_t seed, int mass_spectrum, double* x, double* y, double* z,
                   double* vx, double* vy, double* vz, double* m);

/* Single-threaded variants for the timed CPU baseline are the same functions with
 * OMP_NUM_THREADS=1; oracle_threads reports the OpenMP thread count in use. */
int oracle_threads(void);

#ifdef __cplusplus
}
#endif
#endif
