// hhs_engine.cu -- device-resident HOLD schedule.
//
// The reference walks the recursion of src/hold.cuh:51-181 on the host, with a
// device synchronisation and a host read of N_fast after every split
// (src/split.cuh:430, src/hold.cuh:106-173) and 10-15 launches per node. Here the
// whole top-level step is ONE persistent cooperative kernel: every CTA walks the
// same recursion (explicit per-level state kept in registers; decisions are read
// from device counts after grid barriers, so control flow is uniform), big nodes run
// as grid-wide phases separated by bounded grid barriers, and small nodes (n at or
// below a threshold) are solved with their whole subtree by one CTA while the others
// wait at the next barrier.
//
// Phases of a big node at level k (S = fast list of level k-1, or all particles):
//   [calc]  TS-units   : (sink block, source chunk) units, partial min/max per chunk
//           TS-reduce  : per-sink reduction -> timestep, predicate, per-tile counts
//   [!calc] COUNT      : predicate ts <= dt, per-tile counts
//           SCATTER    : tile prefix, stable scatter into F_k / L_k, N_fast == 1 fold,
//                        counts, leaf time (globals->simtime), work counters
//   child (F_k, dt/2, calc = false)
//           KICK-units : (sink block, source chunk) units; slow sources drifted by dt/2
//                        on the fly (the first drift of src/hold.cuh:123-124)
//           KICK-reduce: per-sink sum of partial accelerations, v += a*dt, and for
//                        slow sinks both half drifts (src/hold.cuh:124,159)
//   child (F_k, dt/2, calc = true)
// Index lists replace the per-level copies and update_system of the reference
// (src/split.cuh:341-356, src/update_system.cuh:14-23): particle data stays in the
// caller's SoA arrays and every level works on global indices.
#include <cooperative_groups.h>
#include <type_traits>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <new>
#include <numeric>
#include <vector>

#include "hhs_ctx.h"
#include "hhs_kernels.h"
#include "hhs_pairmath.cuh"
#include "hhs_scan.cuh"
#include "hhs_tma.cuh"

using namespace hhs;

namespace {

constexpr int kEB = 256;          // engine block size (one sink per thread per unit)
constexpr int kKB = 2 * kEB;      // sinks per block of the mixed grid kick (two per thread)
constexpr int kTS = 1024;         // source records per shared-memory tile of that kick
constexpr int kTX = 256;          // slow records per tile of the symmetric grid kick
constexpr int kTW = 256;          // widest column tile of the packed grid timestep
constexpr int kMaxFsb = 64;       // fast super-blocks of that kick (column-partial slots)
constexpr int kMaxChunks = 32;    // source chunks per node (partial-sum slots)
constexpr int kMaxLevels = 64;    // per-level state is kept in 64-bit masks
constexpr unsigned long long kBarrierTimeoutNs = 60ull * 1000000000ull;

enum ProfKind {
    kProfTs = 0, kProfKick = 1, kProfSplit = 2, kProfUpdate = 3, kProfSubtree = 5, kProfCluster = 6
};

struct EngineState {
    unsigned bar_count;   // grid-barrier arrivals of this launch (cleared before each launch)
    unsigned bar_gen;
    unsigned pad[2];
    unsigned kick_ctr[2][kMaxLevels];  // dynamic work counters of each level's kick units
    unsigned long long prof_ns[8];
    unsigned long long prof_cnt[8];
    double prof_pairs[8];
    unsigned long long lvl_ns[8][kMaxLevels];   // per phase kind and level
    unsigned long long lvl_cnt[8][kMaxLevels];
};

struct EParams {
    SoA P;
    int n_top, n_max, max_levels, small_n, calc_top, profile, units_per_cta, warp_n, mid_n;
    int mid_dist_n;  // cluster subtree solver: nodes above this size are spread over the cluster
    int packed;  // mixed kick: two sinks per thread in packed FP32x2 arithmetic
    int top_level;  // level of the node the launch starts from (0: the whole system)
    double dt_top, eta, eta_s2, eps2;
    float inv_eta_s2, inv_eta, eps2f;
    int32_t* fast_lists;
    int32_t* slow_lists;
    hhs_partition* counts;
    double* leaf_time;
    hhs_stats* stats;
    double* ts_part;   // [kMaxChunks][n_max] (float view for mixed)
    double* k_part;    // [kMaxChunks*3][n_max] (mixed) or [6][n_max] (FP64)
    double* c_part;    // [kMaxFsb*3][n_max]: column sums of the symmetric kick (slow sinks)
    int* tile_counts;  // [n_max/kEB + 1]
    unsigned long long* tile_status;  // [n_max/kEB + 2] look-back words, cleared per launch
    unsigned* rate_acc;  // [n_max] max pair rate per list position (FP32 bits), kept at 0
    EngineState* st;
    unsigned* err;
    // packed kick sources of each grid level (mixed precision): slow particle q of the
    // level's slow list, drifted by half the level's step, as double-single position
    // in pairs: entry e of a level holds records 2e and 2e + 1 as four float4
    // (x hi, y hi), (z hi, mass), (x lo, y lo), (z lo, 0), written by the split, read by
    // bulk copies and unpacked into f32x2 operands
    float4* pk;             // [pk_levels][pk_stride][4]
    long long pk_stride;    // pair entries per level
    int pk_levels;
    // the members of the current grid node packed for the mixed timestep, in list order,
    // in pairs: five arrays of tq_stride float4, member 2p + h at component h (and 2 + h)
    // of entry p: (x hi, y hi), (z hi, mass), (x lo, y lo), (z lo, vx), (vy, vz)
    float4* tq;
    long long tq_stride;
    int prec_mixed;  // this launch runs the mixed-precision kernels
    int overlap;     // slow-only kick units beside a subtree's first pass (tuning)
    int4* trace;                        // node record {level, n, n_fast, calc} in call order
    unsigned long long* trace_count;    // nodes recorded (may exceed trace_cap)
    long long trace_cap;
};

// Cluster subtree solver state (one replica per CTA of the cluster): a subsystem of at
// most kMid particles with its whole subtree lives in shared memory.
constexpr int kMid = 640;
constexpr int kMidW = kMid / 32;
struct __align__(16) MidState {
    double x[kMid], y[kMid], z[kMid], vx[kMid], vy[kMid], vz[kMid], m[kMid], ts[kMid];
    float4 A[kMid], B[kMid], V[kMid];     // mixed: position hi + mass, position lo, velocity
    int g[kMid];                          // global index of each slot
    unsigned fmask[kMaxLevels][kMidW];    // fast set (slot bitmask) chosen at each depth
    int lone[kMaxLevels];                 // slot folded into the slow set, or -1
    int nmem[kMaxLevels];                 // member count of the node at each depth
    short mem[kMid];                      // member slots of the current node, increasing
    unsigned rmax[kMid];                  // mixed: maximum pair rate of each slot (FP32 bits)
    short kl[kMid];                       // kick order: slow slots (lone last), then fast
    union {
        double pmin[8][32];               // partial timesteps (FP64)
        float pmax[8][32];                // partial pair rates (mixed)
        float part[8][3][32];             // partial accelerations (mixed)
    } red;
    unsigned allw[kMidW];                 // members of the subtree's root (every slot)
    short wslot[32];                      // warp solver: slot of each lane's particle
    unsigned wf[kMaxLevels];              // warp solver: fast-lane mask per depth
    int wl[kMaxLevels];                   // warp solver: lane folded into the slow set, or -1
    int wbase[kMidW], wbase2[kMidW];
    int wcnt[kEB / 32];
    int total, total2;
};

// fast sets of at least kX2Min sinks take two sinks per thread in the cross units; slow
// sets of at least kSymMin evaluate each slow-slow pair once for both particles (below
// that, the units would be too few and the column sums of one-row passes cost more than
// the halved pair count saves)
constexpr int kX2Min = 8192;
constexpr int kSymMin = 12288;
static_assert(kSymMin > kMaxChunks * kEB, "symmetric slow chunks are whole two-row passes");

struct KickPlan {
    int R;               // fast sinks per thread in the cross units (1 or 2)
    int ncs, Cs;         // slow chunks: ncs chunks of Cs slow particles (the partial-sum slots)
    int nsub, FB, nfsb;  // fast sub-blocks of R*kEB sinks; FB of them per super-block
    int nsb;             // blocks of kEB slow sinks
    int sym, Rs, noff;   // symmetric slow-slow units: Rs sinks per thread, noff chunk pairs
    int nx, nsl;         // cross units (nfsb x ncs) and slow units
};

struct __align__(16) Smem {
    float colred[kEB / 32][64];
    unsigned long long prof_ns[8][kMaxLevels];  // phase times of this launch (CTA 0)
    unsigned prof_cnt[8][kMaxLevels];
    double prof_pairs[8];
    unsigned wfast[kMaxLevels];   // warp solver: fast-lane mask per depth
    int wlone[kMaxLevels];        // warp solver: lane folded into the slow set, or -1
    int warp_tot[kEB / 32];
    int red[kEB / 32];
    int ok;
    int bcast;
    unsigned bar_k;               // grid barriers passed by this CTA in this launch
    unsigned epoch;               // look-back epoch of the current split
    unsigned kphase;              // parity of the next phase of kbar
    unsigned tphase;              // parities of the next phases of tbar[0], tbar[1]
    __align__(8) uint64_t kbar;   // completion barrier of the kick's source-tile copies
    __align__(8) uint64_t tbar[2];  // completion barriers of the timestep's column tiles
    KickPlan kp;                  // unit layout of the running kick (read from shared memory
                                  // after every unit, so it holds no registers meanwhile)
    // last, so that the persistent kernel's dynamic allocation can extend it to a MidState
    union {
        struct { float4 A[kEB], B[kEB], V[kEB]; } tsm;         // mixed timestep tiles
        struct { double x[kEB], y[kEB], z[kEB], vx[kEB], vy[kEB], vz[kEB], m[kEB]; } tsd;
        struct { float4 A[kEB], B[kEB]; } km;                   // mixed kick tiles
        struct { float4 A[kTS], B[kTS]; } kt;                   // grid kick source tile
        struct {                                                  // symmetric kick
            float4 T[2][kTX / 2][4];                              // source pairs
            float colw[kEB / 32][kTX][3];
        } kc;
        struct {                                                  // packed timestep tiles
            float4 Q[2][5][kTW / 2];                              // column pairs
            float colred[2][kEB / 32][kTW];
        } ts2;
        struct { float4 P0[kEB], P1[kEB], P2[kEB]; float2 M[kEB]; } kx;  // packed kick tiles
        struct { double x[kEB], y[kEB], z[kEB], m[kEB]; } kd;   // FP64 kick tiles
        struct {                                                  // tiny-subtree state
            double x[32], y[32], z[32], vx[32], vy[32], vz[32], m[32], ts[32];
            float4 A[32], B[32], V[32];
            double pmin[kEB / 32][32];
            float pmax[kEB / 32][32];
            float part[kEB / 32][3][32];
            int g[32];
        } tiny;
    } u;
};

// dynamic shared memory of the persistent kernel: Smem with its last member grown to
// hold a MidState
constexpr size_t kEngineSmem =
    offsetof(Smem, u) + (sizeof(MidState) > sizeof(Smem::u) ? sizeof(MidState) : sizeof(Smem::u));

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// One node of the recursion, recorded in call order (the order of the reference's
// hold_step calls) when the caller asked for a trace.
__device__ __forceinline__ void trace_node(const EParams& E, int level, int n, int nf, bool calc) {
    if (!E.trace) return;
    const unsigned long long k = atomicAdd(E.trace_count, 1ull);
    if ((long long)k < E.trace_cap) E.trace[k] = make_int4(level, n, nf, calc ? 1 : 0);
}

// E.dt_top * 2^-lvl, exact (the same double as ldexp(E.dt_top, -lvl) for the levels
// kept, which stay far from the subnormal range)
__device__ __forceinline__ double dt_at(const EParams& E, int lvl) {
    return __dmul_rn(E.dt_top, __longlong_as_double((long long)(1023 - lvl) << 52));
}

__device__ __forceinline__ int ld_volatile_i32(const int32_t* p) {
    return *reinterpret_cast<const volatile int32_t*>(p);
}

// ---------------------------------------------------------------- grid barrier
// Counting barrier over all CTAs of the cooperative grid: the arrival counter is cleared
// before each launch, the k-th barrier of the launch is passed when it reaches k times the
// grid size. Arrivals are fire-and-forget release reductions (no CTA waits for its own
// atomic to return); waiters poll with acquire loads, give up after kBarrierTimeoutNs (or
// as soon as another CTA recorded an error) and report failure instead of hanging.
__device__ bool grid_barrier(const EParams& E, Smem& sm) {
    __syncthreads();
    if (threadIdx.x == 0) {
        // The CTA barrier above orders every thread's writes before this thread's
        // release; the acquire loads of the waiters make them visible, so no separate
        // fences are needed.
        int ok = 1;
        EngineState* st = E.st;
        const unsigned target = (++sm.bar_k) * gridDim.x;
        red_add_release_u32(&st->bar_count, 1u);
        unsigned polls = 0;
        unsigned long long t0 = 0;
        while (ld_acquire_u32(&st->bar_count) < target) {
            if (++polls < 256) continue;  // tight polling first
            if (t0 == 0) t0 = gtimer();
            if (*reinterpret_cast<volatile unsigned*>(E.err) != 0u) { ok = 0; break; }
            __nanosleep(32);
            if (gtimer() - t0 > kBarrierTimeoutNs) {
                atomicOr(E.err, HHS_ERRBIT_BARRIER_TIMEOUT);
                ok = 0;
                break;
            }
        }
        sm.ok = ok;
    }
    __syncthreads();
    return sm.ok != 0;
}

// Workers: the whole cooperative grid (one worker per CTA), a hardware thread-block
// cluster (one worker per CTA of the cluster; batched systems), or one CTA alone.
enum { kModeBlock = 0, kModeGrid = 1, kModeCluster = 2 };
struct Workers {
    int id, count, mode;
};

__device__ __forceinline__ bool phase_barrier(const EParams& E, Smem& sm, const Workers& W) {
    if (W.mode == kModeGrid) return grid_barrier(E, sm);
    if (W.mode == kModeCluster) {
        cooperative_groups::this_cluster().sync();
        return true;
    }
    __syncthreads();
    return true;
}

// Phase timing by CTA 0 of the grid: the time from the previous mark to the release of
// the barrier that ends the phase (the phase's makespan over all CTAs), per kind and
// level, accumulated in shared memory and added to the context's counters at the end of
// the launch.
__device__ __forceinline__ void prof_mark(const EParams& E, const Workers& W,
                                          unsigned long long& t_last, int kind, double pairs,
                                          Smem& sm, int level = 0) {
    if (!E.profile || W.mode != kModeGrid || threadIdx.x != 0 || W.id != 0) return;
    const unsigned long long t = gtimer();
    if (kind >= 0) {
        const int l = level < kMaxLevels ? level : kMaxLevels - 1;
        sm.prof_ns[kind][l] += t - t_last;
        sm.prof_cnt[kind][l] += 1;
        sm.prof_pairs[kind] += pairs;
    }
    t_last = t;
}

__device__ void prof_begin(const EParams& E, Smem& sm) {
    if (!E.profile || blockIdx.x != 0) return;
    for (int i = threadIdx.x; i < 8 * kMaxLevels; i += blockDim.x) {
        (&sm.prof_ns[0][0])[i] = 0ull;
        (&sm.prof_cnt[0][0])[i] = 0u;
    }
    if (threadIdx.x < 8) sm.prof_pairs[threadIdx.x] = 0.0;
    __syncthreads();
}

__device__ void prof_end(const EParams& E, Smem& sm) {
    if (!E.profile || blockIdx.x != 0) return;
    __syncthreads();
    EngineState* st = E.st;
    for (int i = threadIdx.x; i < 8 * kMaxLevels; i += blockDim.x) {
        const int k = i / kMaxLevels, l = i % kMaxLevels;
        const unsigned long long ns = sm.prof_ns[k][l];
        const unsigned c = sm.prof_cnt[k][l];
        if (c) {
            st->lvl_ns[k][l] += ns;
            st->lvl_cnt[k][l] += c;
        }
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        unsigned long long ns = 0, c = 0;
        for (int l = 0; l < kMaxLevels; l++) {
            ns += sm.prof_ns[threadIdx.x][l];
            c += sm.prof_cnt[threadIdx.x][l];
        }
        st->prof_ns[threadIdx.x] += ns;
        st->prof_cnt[threadIdx.x] += c;
        st->prof_pairs[threadIdx.x] += sm.prof_pairs[threadIdx.x];
    }
}

// number of source chunks for a node of n sinks
__device__ __forceinline__ int chunks_for(int n, const Workers& W, bool split_ok, int upc,
                                          int block = kEB) {
    if (W.mode == kModeBlock || !split_ok) return 1;
    const int nsb = (n + block - 1) / block;
    int c = (upc * W.count + nsb - 1) / nsb;
    c = c < 1 ? 1 : (c > kMaxChunks ? kMaxChunks : c);
    const int maxc = (n + 63) / 64;  // at least 64 sources per chunk
    return c < maxc ? c : (maxc < 1 ? 1 : maxc);
}

__device__ __forceinline__ int list_at(const int32_t* S, int i) { return S ? S[i] : i; }

// ---------------------------------------------------------------- block scan helpers
// exclusive prefix of a 0/1 flag over the CTA (one flag per thread) and the CTA total
__device__ __forceinline__ int block_excl_flag(int flag, Smem& sm, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned b = __ballot_sync(HHS_FULL_MASK, flag);
    const int within = __popc(b & ((1u << lane) - 1u));
    __syncthreads();
    if (lane == 0) sm.warp_tot[warp] = __popc(b);
    __syncthreads();
    int before = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kEB / 32; w++) {
        const int t = sm.warp_tot[w];
        before += (w < warp) ? t : 0;
        tot += t;
    }
    total = tot;
    return before + within;
}

__device__ __forceinline__ int block_sum(int v, Smem& sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sm.red[warp] = v;
    __syncthreads();
    int t = 0;
#pragma unroll
    for (int w = 0; w < kEB / 32; w++) t += sm.red[w];
    return t;
}

// ---------------------------------------------------------------- timestep units
template <int PREC>
__device__ void ts_unit(const EParams& E, const int32_t* S, int n, int ib, int j0, int j1,
                        double* out64, float* out32, Smem& sm) {
    const int i = ib * kEB + threadIdx.x;
    const bool act = i < n;
    const int gi = act ? list_at(S, i) : 0;
    const SoA& P = E.P;
    if (PREC == HHS_PREC_FP64) {
        double xi = 0, yi = 0, zi = 0, vxi = 0, vyi = 0, vzi = 0, mi = 0;
        if (act) {
            xi = P.x[gi]; yi = P.y[gi]; zi = P.z[gi];
            vxi = P.vx[gi]; vyi = P.vy[gi]; vzi = P.vz[gi]; mi = P.m[gi];
        }
        double minval = 1.e30;
        for (int t0 = j0; t0 < j1; t0 += kEB) {
            const int tl = min(kEB, j1 - t0);
            __syncthreads();
            if ((int)threadIdx.x < tl) {
                const int gj = list_at(S, t0 + threadIdx.x);
                sm.u.tsd.x[threadIdx.x] = P.x[gj]; sm.u.tsd.y[threadIdx.x] = P.y[gj];
                sm.u.tsd.z[threadIdx.x] = P.z[gj]; sm.u.tsd.vx[threadIdx.x] = P.vx[gj];
                sm.u.tsd.vy[threadIdx.x] = P.vy[gj]; sm.u.tsd.vz[threadIdx.x] = P.vz[gj];
                sm.u.tsd.m[threadIdx.x] = P.m[gj];
            }
            __syncthreads();
            if (act) {
                for (int jl = 0; jl < tl; jl++) {
                    if (t0 + jl == i) continue;
                    ts_pair_fp64(f64_sub(xi, sm.u.tsd.x[jl]), f64_sub(yi, sm.u.tsd.y[jl]),
                                 f64_sub(zi, sm.u.tsd.z[jl]), f64_sub(vxi, sm.u.tsd.vx[jl]),
                                 f64_sub(vyi, sm.u.tsd.vy[jl]), f64_sub(vzi, sm.u.tsd.vz[jl]),
                                 mi, sm.u.tsd.m[jl], E.eta, E.eta_s2, minval);
                }
            }
        }
        if (act) out64[i] = minval;
    } else {
        DS xi{0, 0}, yi{0, 0}, zi{0, 0};
        float vxi = 0, vyi = 0, vzi = 0, mi = 0;
        if (act) {
            xi = ds_split(P.x[gi]); yi = ds_split(P.y[gi]); zi = ds_split(P.z[gi]);
            vxi = (float)P.vx[gi]; vyi = (float)P.vy[gi]; vzi = (float)P.vz[gi];
            mi = (float)P.m[gi];
        }
        float maxrate = 0.0f;
        for (int t0 = j0; t0 < j1; t0 += kEB) {
            const int tl = min(kEB, j1 - t0);
            __syncthreads();
            if ((int)threadIdx.x < tl) {
                const int gj = list_at(S, t0 + threadIdx.x);
                const DS a = ds_split(P.x[gj]), b = ds_split(P.y[gj]), c = ds_split(P.z[gj]);
                sm.u.tsm.A[threadIdx.x] = make_float4(a.hi, b.hi, c.hi, (float)P.m[gj]);
                sm.u.tsm.B[threadIdx.x] = make_float4(a.lo, b.lo, c.lo, 0.0f);
                sm.u.tsm.V[threadIdx.x] =
                    make_float4((float)P.vx[gj], (float)P.vy[gj], (float)P.vz[gj], 0.0f);
            }
            __syncthreads();
            if (act) {
                for (int jl = 0; jl < tl; jl++) {
                    if (t0 + jl == i) continue;
                    const float4 A = sm.u.tsm.A[jl], B = sm.u.tsm.B[jl], V = sm.u.tsm.V[jl];
                    const float r = ts_pair_rate_mixed(
                        ds_diff(xi.hi, xi.lo, A.x, B.x), ds_diff(yi.hi, yi.lo, A.y, B.y),
                        ds_diff(zi.hi, zi.lo, A.z, B.z), vxi - V.x, vyi - V.y, vzi - V.z,
                        mi + A.w, E.inv_eta_s2, E.inv_eta);
                    maxrate = fmaxf(maxrate, r);
                }
            }
        }
        if (act) out32[i] = maxrate;
    }
}


// ---------------------------------------------------------------- symmetric timestep
// The pair timestep is exactly symmetric under i <-> j (dr, dv negate exactly, squares,
// products of two negated values and the mass sum are unchanged), so each unordered pair
// is evaluated once, in the unit (row block of kEB list positions, column block of kCB)
// that holds it with i < j. Rows keep their running max rate in a register; the column
// maxima of a warp's 32 rows come from one warp max-reduction (redux.sync) per column.
// Both are merged into rate_acc with an integer atomicMax on the FP32 bit pattern (rates
// are >= 0, so integer order is float order). Max is exact and
// order-independent: the result equals the all-pairs evaluation bit for bit.
constexpr int kCB = 32;
constexpr int kTsRows = 1;                // rows per thread in the symmetric timestep
constexpr int kTsBlock = kTsRows * kEB;   // rows per unit

// Units [u0, u1) of the upper triangle of (256-row block, kCB-column block) tiles, in
// row-major order: a contiguous range per CTA, so consecutive units mostly share their row
// block, whose particles stay in registers (and whose row maximum is merged once).
// Every max also goes to the peer replicas' rate words when po is given (the sharded
// timestep of the multi-GPU step).
__device__ __forceinline__ void rate_max(const EParams& E, const PeerOut* po, int i, float v) {
    atomicMax(&E.rate_acc[i], __float_as_uint(v));
    if (po)
        for (int r = 0; r < po->n_peer; r++) atomicMax(&po->rate[r][i], __float_as_uint(v));
}

__device__ void ts_sym_range(const EParams& E, const int32_t* S, int n, int u0, int u1,
                             Smem& sm, const PeerOut* po = nullptr) {
    const SoA& P = E.P;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int R = kTsRows;
    constexpr int kRowStep = kTsBlock / kCB;
    const int nrb = (n + kTsBlock - 1) / kTsBlock, ncb = (n + kCB - 1) / kCB;
    int rb = 0, off = u0;  // unit u0 = (rb, rb * kRowStep + off)
    while (rb < nrb && off >= ncb - rb * kRowStep) {
        off -= ncb - rb * kRowStep;
        rb++;
    }
    int cur = -1;
    int i[R];
    bool act[R];
    DS xi[R], yi[R], zi[R];
    float vxi[R], vyi[R], vzi[R], mi[R], rowmax[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        i[r] = 0; act[r] = false; rowmax[r] = 0.0f;
        xi[r] = yi[r] = zi[r] = DS{0.f, 0.f};
        vxi[r] = vyi[r] = vzi[r] = mi[r] = 0.0f;
    }
    // the next unit's columns are loaded into registers while this unit computes
    double px = 0, py = 0, pz = 0, pvx = 0, pvy = 0, pvz = 0, pm = 0;
    bool have = false;
    for (int u = u0; u < u1 && rb < nrb; u++) {
        if (rb != cur) {
#pragma unroll
            for (int r = 0; r < R; r++) {
                if (act[r] && rowmax[r] > 0.0f) rate_max(E, po, i[r], rowmax[r]);
                rowmax[r] = 0.0f;
                i[r] = rb * kTsBlock + r * kEB + (int)threadIdx.x;
                act[r] = i[r] < n;
                if (act[r]) {
                    const int gi = list_at(S, i[r]);
                    xi[r] = ds_split(P.x[gi]); yi[r] = ds_split(P.y[gi]); zi[r] = ds_split(P.z[gi]);
                    vxi[r] = (float)P.vx[gi]; vyi[r] = (float)P.vy[gi]; vzi[r] = (float)P.vz[gi];
                    mi[r] = (float)P.m[gi];
                }
            }
            cur = rb;
        }
        const int c0 = (rb * kRowStep + off) * kCB;
        const int ncol = min(kCB, n - c0);
        if (!have && (int)threadIdx.x < ncol) {
            const int gj = list_at(S, c0 + threadIdx.x);
            px = P.x[gj]; py = P.y[gj]; pz = P.z[gj];
            pvx = P.vx[gj]; pvy = P.vy[gj]; pvz = P.vz[gj]; pm = P.m[gj];
        }
        __syncthreads();
        if ((int)threadIdx.x < ncol) {
            const DS a = ds_split(px), b = ds_split(py), c = ds_split(pz);
            sm.u.tsm.A[threadIdx.x] = make_float4(a.hi, b.hi, c.hi, (float)pm);
            sm.u.tsm.B[threadIdx.x] = make_float4(a.lo, b.lo, c.lo, 0.0f);
            sm.u.tsm.V[threadIdx.x] = make_float4((float)pvx, (float)pvy, (float)pvz, 0.0f);
        }
        __syncthreads();
        {
            int rb2 = rb, off2 = off + 1;
            if (off2 >= ncb - rb * kRowStep) { off2 = 0; rb2++; }
            have = false;
            if (u + 1 < u1 && rb2 < nrb) {
                have = true;
                const int c0n = (rb2 * kRowStep + off2) * kCB;
                if ((int)threadIdx.x < min(kCB, n - c0n)) {
                    const int gj = list_at(S, c0n + threadIdx.x);
                    px = P.x[gj]; py = P.y[gj]; pz = P.z[gj];
                    pvx = P.vx[gj]; pvy = P.vy[gj]; pvz = P.vz[gj]; pm = P.m[gj];
                }
            }
        }
        // column maxima over the warp's rows: one warp max-reduction per column on the
        // rates' bit patterns (rates are >= 0 or +inf, so integer order is float order);
        // lane c keeps column c's maximum
        unsigned colmax = 0u;
#pragma unroll 8
        for (int jl = 0; jl < kCB; jl++) {
            const float4 A = sm.u.tsm.A[jl], B = sm.u.tsm.B[jl], V = sm.u.tsm.V[jl];
            float cmax = 0.0f;
#pragma unroll
            for (int r = 0; r < R; r++) {
                const float rate = ts_pair_rate_mixed(
                    ds_diff(xi[r].hi, xi[r].lo, A.x, B.x), ds_diff(yi[r].hi, yi[r].lo, A.y, B.y),
                    ds_diff(zi[r].hi, zi[r].lo, A.z, B.z), vxi[r] - V.x, vyi[r] - V.y,
                    vzi[r] - V.z, mi[r] + A.w, E.inv_eta_s2, E.inv_eta);
                const bool ok = act[r] && (jl < ncol) && (c0 + jl > i[r]);
                const float rr = ok ? rate : 0.0f;
                rowmax[r] = fmaxf(rowmax[r], rr);
                cmax = fmaxf(cmax, rr);
            }
            const unsigned cm = __reduce_max_sync(HHS_FULL_MASK, __float_as_uint(cmax));
            colmax = lane == jl ? cm : colmax;
        }
        sm.colred[warp][lane] = __uint_as_float(colmax);
        __syncthreads();
        if ((int)threadIdx.x < ncol) {
            float cm = 0.0f;
#pragma unroll
            for (int w = 0; w < kEB / 32; w++) cm = fmaxf(cm, sm.colred[w][threadIdx.x]);
            if (cm > 0.0f) rate_max(E, po, c0 + (int)threadIdx.x, cm);
        }
        if (++off >= ncb - rb * kRowStep) {
            off = 0;
            rb++;
        }
    }
#pragma unroll
    for (int r = 0; r < R; r++)
        if (act[r] && rowmax[r] > 0.0f) rate_max(E, po, i[r], rowmax[r]);
}

// Units of the upper triangle of (kTsBlock-row block, kCB-column block) tiles of a node
__host__ __device__ __forceinline__ long long ts_sym_units(int n) {
    constexpr int kRowStep = kTsBlock / kCB;
    const long long nrb = (n + kTsBlock - 1) / kTsBlock, ncb = (n + kCB - 1) / kCB;
    long long units = 0;
    for (long long r = 0; r < nrb; r++) units += ncb - r * kRowStep > 0 ? ncb - r * kRowStep : 0;
    return units;
}


// ---------------------------------------------------------------- packed grid timestep
// The same symmetric evaluation on the whole grid from the node's packed members (list
// order, written by the kick-reduce phase that last changed them, or by pack_ts): units
// are (kEB-row block, CW-column block) tiles of the upper triangle, CW chosen per node
// (the widest of 256/128/64/32 that still gives every CTA two units). A CTA takes a
// contiguous range of units in row-major order; each unit's columns arrive by bulk copy
// into one of two shared buffers while the previous unit computes.
__device__ __forceinline__ long long ts_tile_units(int n, int cw) {
    const long long nrb = (n + kEB - 1) / kEB, ncb = (n + cw - 1) / cw, step = kEB / cw;
    long long units = 0;
    for (long long r = 0; r < nrb; r++) units += ncb - r * step > 0 ? ncb - r * step : 0;
    return units;
}

__device__ __forceinline__ int ts_tile_width(int n, int workers) {
    int cw = kTW;
    while (cw > 32 && ts_tile_units(n, cw) < 2LL * workers) cw >>= 1;
    return cw;
}

// Member i of the packed timestep arrays: pair entry i / 2, component i % 2 (and 2 + i % 2)
// of each of the five arrays.
__device__ __forceinline__ void tq_put(const EParams& E, int i, double x, double y, double z,
                                       double m, double vx, double vy, double vz) {
    const DS X = ds_split(x), Y = ds_split(y), Z = ds_split(z);
    float* q = reinterpret_cast<float*>(E.tq) + 4 * (size_t)(i >> 1) + (i & 1);
    const size_t a = 4 * (size_t)E.tq_stride;  // floats per array
    q[0] = X.hi;
    q[2] = Y.hi;
    q[a] = Z.hi;
    q[a + 2] = (float)m;
    q[2 * a] = X.lo;
    q[2 * a + 2] = Y.lo;
    q[3 * a] = Z.lo;
    q[3 * a + 2] = (float)vx;
    q[4 * a] = (float)vy;
    q[4 * a + 2] = (float)vz;
}

// Member i as a sink of the packed timestep: negated, each value in both lanes.
__device__ __forceinline__ TsSink2 tq_sink(const EParams& E, int i) {
    const float* q = reinterpret_cast<const float*>(E.tq) + 4 * (size_t)(i >> 1) + (i & 1);
    const size_t a = 4 * (size_t)E.tq_stride;
    return TsSink2{f2dup(-q[0]), f2dup(-q[2]), f2dup(-q[a]), f2dup(-q[2 * a]),
                   f2dup(-q[2 * a + 2]), f2dup(-q[3 * a]), f2dup(-q[3 * a + 2]),
                   f2dup(-q[4 * a]), f2dup(-q[4 * a + 2]), f2dup(q[a + 2])};
}

// The node's members (list S, n of them) into the packed timestep arrays.
__device__ void pack_ts(const EParams& E, const int32_t* S, int n, const Workers& W) {
    const SoA& P = E.P;
    for (int i = W.id * kEB + (int)threadIdx.x; i < n; i += W.count * kEB) {
        const int g = list_at(S, i);
        tq_put(E, i, P.x[g], P.y[g], P.z[g], P.m[g], P.vx[g], P.vy[g], P.vz[g]);
    }
}

// unit u of the triangle -> (row block, column block)
__device__ __forceinline__ void ts_tile_of(long long u, int nrb, int ncb, int step, int& rb,
                                           int& cb) {
    rb = 0;
    while (rb < nrb && u >= ncb - (long long)rb * step) {
        u -= ncb - (long long)rb * step;
        rb++;
    }
    cb = rb * step + (int)u;
}

// columns [c0, c0 + ncol), c0 even: their (ncol + 1) / 2 pair entries of the five arrays
__device__ __forceinline__ void ts_tile_stage(const EParams& E, int buf, int c0, int ncol,
                                              Smem& sm) {
    const unsigned bytes = (unsigned)((ncol + 1) >> 1) * (unsigned)sizeof(float4);
    mbar_arrive_expect_tx(&sm.tbar[buf], 5u * bytes);
#pragma unroll
    for (int k = 0; k < 5; k++)
        bulk_load(sm.u.ts2.Q[buf][k], E.tq + (size_t)k * E.tq_stride + (c0 >> 1), bytes,
                  &sm.tbar[buf]);
}

__device__ void ts_sym_tiles(const EParams& E, int n, int cw, long long u0, long long u1,
                             Smem& sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int step = kEB / cw;
    const int nrb = (n + kEB - 1) / kEB, ncb = (n + cw - 1) / cw;
    if (u0 >= u1) return;
    int rb = 0, cb = 0;
    ts_tile_of(u0, nrb, ncb, step, rb, cb);
    // prologue: the first two units' columns
    if (threadIdx.x == 0) {
        int r2 = rb, c2 = cb;
        for (int k = 0; k < 2 && u0 + k < u1; k++) {
            const int c0 = c2 * cw;
            ts_tile_stage(E, k, c0, min(cw, n - c0), sm);
            if (++c2 >= ncb) { r2++; c2 = r2 * step; }
        }
    }
    int cur = -1, i = 0;
    bool act = false;
    TsSink2 si{};
    float rowmax = 0.0f;
    unsigned phase = sm.tphase;
    int nrb_n = rb, ncb_n = cb;  // the unit two ahead, for the refill
    for (int k = 0; k < 2; k++)
        if (++ncb_n >= ncb) { nrb_n++; ncb_n = nrb_n * step; }
    for (long long u = u0; u < u1; u++) {
        const int buf = (int)((u - u0) & 1);
        if (rb != cur) {
            if (act && rowmax > 0.0f) rate_max(E, nullptr, i, rowmax);
            cur = rb;
            rowmax = 0.0f;
            i = rb * kEB + threadIdx.x;
            act = i < n;
            if (act) si = tq_sink(E, i);
        }
        const int c0 = cb * cw;
        const int ncol = min(cw, n - c0);
        if (!mbar_wait(&sm.tbar[buf], (phase >> buf) & 1u, E.err))
            (void)mbar_wait(&sm.tbar[buf], (phase >> buf) & 1u, nullptr);
        phase ^= 1u << buf;
        const float4* Q0 = sm.u.ts2.Q[buf][0];
        const float4* Q1 = sm.u.ts2.Q[buf][1];
        const float4* Q2 = sm.u.ts2.Q[buf][2];
        const float4* Q3 = sm.u.ts2.Q[buf][3];
        const float4* Q4 = sm.u.ts2.Q[buf][4];
        // pairs need a mask only in the tiles that cross the diagonal (j > i), hold rows
        // past the end or end in half a column pair
        const int diag_end = (rb + 1) * kEB;  // columns from here see every row as j > i
        const int mask = c0 < diag_end ? 2 : ((diag_end > n || (ncol & 1)) ? 1 : 0);
        auto cols = [&](auto MASK) {
            constexpr int M = decltype(MASK)::value;
            for (int g = 0; g < ncol; g += 32) {
                const int np = (min(32, ncol - g) + 1) >> 1;  // column pairs of this group
                unsigned colmax = 0u;
#pragma unroll 4
                for (int q = 0; q < np; q++) {
                    const int e = (g >> 1) + q;  // pair entry: columns c0 + 2e, c0 + 2e + 1
                    const float4 a0 = Q0[e], a1 = Q1[e], a2 = Q2[e], a3 = Q3[e], a4 = Q4[e];
                    const float2 rate = ts_pair_rate_mixed2(
                        make_float2(a0.x, a0.y), make_float2(a0.z, a0.w), make_float2(a1.x, a1.y),
                        make_float2(a2.x, a2.y), make_float2(a2.z, a2.w), make_float2(a3.x, a3.y),
                        make_float2(a3.z, a3.w), make_float2(a4.x, a4.y), make_float2(a4.z, a4.w),
                        make_float2(a1.z, a1.w), si, E.inv_eta_s2, E.inv_eta);
                    float r0 = rate.x, r1 = rate.y;
                    if (M != 0) {
                        const int c = c0 + 2 * e;
                        const bool ok0 = act && c < n && (M == 1 || c > i);
                        const bool ok1 = act && c + 1 < n && (M == 1 || c + 1 > i);
                        r0 = ok0 ? r0 : 0.0f;
                        r1 = ok1 ? r1 : 0.0f;
                    }
                    rowmax = fmaxf(rowmax, fmaxf(r0, r1));
                    const unsigned m0 = __reduce_max_sync(HHS_FULL_MASK, __float_as_uint(r0));
                    const unsigned m1 = __reduce_max_sync(HHS_FULL_MASK, __float_as_uint(r1));
                    colmax = lane == 2 * q ? m0 : colmax;
                    colmax = lane == 2 * q + 1 ? m1 : colmax;
                }
                sm.u.ts2.colred[buf][warp][g + lane] = __uint_as_float(colmax);
            }
        };
        if (mask == 0) cols(std::integral_constant<int, 0>{});
        else if (mask == 1) cols(std::integral_constant<int, 1>{});
        else cols(std::integral_constant<int, 2>{});
        __syncthreads();  // this buffer's columns are read, colred[buf] is complete
        if ((int)threadIdx.x < ncol) {
            float cm = 0.0f;
#pragma unroll
            for (int w = 0; w < kEB / 32; w++) cm = fmaxf(cm, sm.u.ts2.colred[buf][w][threadIdx.x]);
            if (cm > 0.0f) rate_max(E, nullptr, c0 + (int)threadIdx.x, cm);
        }
        if (threadIdx.x == 0 && u + 2 < u1) {
            const int cn = ncb_n * cw;
            ts_tile_stage(E, buf, cn, min(cw, n - cn), sm);
        }
        if (++ncb_n >= ncb) { nrb_n++; ncb_n = nrb_n * step; }
        if (++cb >= ncb) { rb++; cb = rb * step; }
    }
    if (act && rowmax > 0.0f) rate_max(E, nullptr, i, rowmax);
    __syncthreads();  // colred and the buffers are free; every wait of this range is done
    if (threadIdx.x == 0) sm.tphase = phase;
    __syncthreads();
}

// ---------------------------------------------------------------- kick units
// Sinks s in [0, nf + ns): s < nf -> F[s] (fast), else L[s - nf] (slow). Sources j in
// [0, ns + nf): j < ns -> L[j] (drifted by h on the fly), else F[j - ns]. Fast sinks
// see slow sources only.
template <int PREC>
__device__ void kick_unit(const EParams& E, const int32_t* F, const int32_t* L, int nf, int ns,
                          double h, int ib, int jc, int j0, int j1, Smem& sm) {
    const int n = nf + ns;
    const int s = ib * kEB + threadIdx.x;
    const bool act = s < n;
    const bool slow = s >= nf;
    const int g = act ? (slow ? L[s - nf] : F[s]) : 0;
    const int jend = slow ? j1 : min(j1, ns);
    const SoA& P = E.P;
    const int n_max = E.n_max;
    if (PREC == HHS_PREC_FP64) {
        double xi = 0, yi = 0, zi = 0;
        if (act) {
            xi = P.x[g]; yi = P.y[g]; zi = P.z[g];
            if (slow) {
                xi = f64_add(xi, f64_mul(P.vx[g], h));
                yi = f64_add(yi, f64_mul(P.vy[g], h));
                zi = f64_add(zi, f64_mul(P.vz[g], h));
            }
        }
        double aL[3] = {0, 0, 0}, aF[3] = {0, 0, 0};
        for (int t0 = j0; t0 < j1; t0 += kEB) {
            const int tl = min(kEB, j1 - t0);
            __syncthreads();
            if ((int)threadIdx.x < tl) {
                const int j = t0 + threadIdx.x;
                const bool js = j < ns;
                const int gj = js ? L[j] : F[j - ns];
                double x = P.x[gj], y = P.y[gj], z = P.z[gj];
                if (js) {
                    x = f64_add(x, f64_mul(P.vx[gj], h));
                    y = f64_add(y, f64_mul(P.vy[gj], h));
                    z = f64_add(z, f64_mul(P.vz[gj], h));
                }
                sm.u.kd.x[threadIdx.x] = x; sm.u.kd.y[threadIdx.x] = y;
                sm.u.kd.z[threadIdx.x] = z; sm.u.kd.m[threadIdx.x] = P.m[gj];
            }
            __syncthreads();
            if (act) {
                const int je = min(tl, jend - t0);
                for (int jl = 0; jl < je; jl++) {
                    double* a = (t0 + jl < ns) ? aL : aF;
                    kick_pair_fp64(f64_sub(sm.u.kd.x[jl], xi), f64_sub(sm.u.kd.y[jl], yi),
                                   f64_sub(sm.u.kd.z[jl], zi), sm.u.kd.m[jl], a[0], a[1], a[2],
                                   E.eps2);
                }
            }
        }
        if (act) {
            double* part = E.k_part;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                part[(size_t)k * n_max + s] = aL[k];
                part[(size_t)(3 + k) * n_max + s] = aF[k];
            }
        }
    } else {
        DS xi{0, 0}, yi{0, 0}, zi{0, 0};
        if (act) {
            double x = P.x[g], y = P.y[g], z = P.z[g];
            if (slow) { x = fma(P.vx[g], h, x); y = fma(P.vy[g], h, y); z = fma(P.vz[g], h, z); }
            xi = ds_split(x); yi = ds_split(y); zi = ds_split(z);
        }
        float acc[3] = {0, 0, 0}, cmp[3] = {0, 0, 0};
        for (int t0 = j0; t0 < j1; t0 += kEB) {
            const int tl = min(kEB, j1 - t0);
            __syncthreads();
            if ((int)threadIdx.x < tl) {
                const int j = t0 + threadIdx.x;
                const bool js = j < ns;
                const int gj = js ? L[j] : F[j - ns];
                double x = P.x[gj], y = P.y[gj], z = P.z[gj];
                if (js) { x = fma(P.vx[gj], h, x); y = fma(P.vy[gj], h, y); z = fma(P.vz[gj], h, z); }
                const DS a = ds_split(x), b = ds_split(y), c = ds_split(z);
                sm.u.km.A[threadIdx.x] = make_float4(a.hi, b.hi, c.hi, (float)P.m[gj]);
                sm.u.km.B[threadIdx.x] = make_float4(a.lo, b.lo, c.lo, 0.0f);
            }
            __syncthreads();
            if (act) {
                const int je = min(tl, jend - t0);
                // blocked compensated summation: 32-pair FP32 blocks, Kahan across blocks
                // (full blocks unrolled so that consecutive pairs overlap); 1/r^3 from
                // rsqrtf with one Newton correction
                auto pair = [&](int jl, float& bx, float& by, float& bz) {
                    const float4 A = sm.u.km.A[jl], B = sm.u.km.B[jl];
                    const float dx = ds_diff(A.x, B.x, xi.hi, xi.lo);
                    const float dy = ds_diff(A.y, B.y, yi.hi, yi.lo);
                    const float dz = ds_diff(A.z, B.z, zi.hi, zi.lo);
                    const float d2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, E.eps2f)));
                    const float mr3 = mr3_nr(A.w, d2);
                    bx = fmaf(dx, mr3, bx);
                    by = fmaf(dy, mr3, by);
                    bz = fmaf(dz, mr3, bz);
                };
                int jb = 0;
                for (; jb + 32 <= je; jb += 32) {
                    float bx = 0.0f, by = 0.0f, bz = 0.0f;
#pragma unroll 8
                    for (int jl = jb; jl < jb + 32; jl++) pair(jl, bx, by, bz);
                    kahan_add(acc[0], cmp[0], bx);
                    kahan_add(acc[1], cmp[1], by);
                    kahan_add(acc[2], cmp[2], bz);
                }
                if (jb < je) {
                    float bx = 0.0f, by = 0.0f, bz = 0.0f;
                    for (int jl = jb; jl < je; jl++) pair(jl, bx, by, bz);
                    kahan_add(acc[0], cmp[0], bx);
                    kahan_add(acc[1], cmp[1], by);
                    kahan_add(acc[2], cmp[2], bz);
                }
            }
        }
        if (act) {
            double* part = E.k_part;
#pragma unroll
            for (int k = 0; k < 3; k++)
                part[(size_t)(jc * 3 + k) * n_max + s] = (double)acc[k] - (double)cmp[k];
        }
    }
}


// ---------------------------------------------------------------- grid kick (mixed)
// The kick of a large node on the whole grid, mixed precision. Sources are staged in
// shared memory tiles of up to kTS records: the slow ones (the majority of every node's
// sources) arrive by bulk copy from the level's packed array, which the split wrote
// once (position drifted by half the step, split to double-single, mass), and the fast
// ones are gathered and split by the CTA. Work units are (block of 512 sinks, source
// chunk) in chunk-major order, a contiguous range per CTA, so a CTA keeps its chunk
// resident across consecutive units and stages it once. Each thread carries two sinks,
// which share every shared-memory read. Pair terms are FP32: 1/d^3 from rsqrtf with one
// Newton correction applied to its cube (y^3 (5/2 - 3/2 d2 y^2), the first-order Newton
// step for d2^-3/2), summed per sink in 32-pair FP32 blocks that are added into Kahan-
// compensated sums; the per-chunk sums go to k_part for the reduce phase as before.
// Self pairs contribute exactly 0 (zero separation times a finite 1/d^3: d2 is floored
// at 1e-20, which no separation in the state arrays ever reaches).
struct SinkDS {
    float nxh, nyh, nzh, nxl, nyl, nzl;  // negated double-single position
};

// The packed kick sources of a level, and record q of them.
__device__ __forceinline__ float4* pk_level(const EParams& E, int lvl) {
    return E.pk + (size_t)lvl * (size_t)E.pk_stride * 4;
}
__device__ __forceinline__ void pk_put(float4* L, int q, const DS& x, const DS& y, const DS& z,
                                       float m) {
    float* p = reinterpret_cast<float*>(L + 4 * (size_t)(q >> 1)) + (q & 1);
    p[0] = x.hi;
    p[2] = y.hi;
    p[4] = z.hi;
    p[6] = m;
    p[8] = x.lo;
    p[10] = y.lo;
    p[12] = z.lo;
    p[14] = 0.0f;
}
// record q as (hi x, y, z, m) and (lo x, y, z, 0)
__device__ __forceinline__ void pk_get(const float4* L, int q, float4& a, float4& b) {
    const float* p = reinterpret_cast<const float*>(L + 4 * (size_t)(q >> 1)) + (q & 1);
    a = make_float4(p[0], p[2], p[4], p[6]);
    b = make_float4(p[8], p[10], p[12], 0.0f);
}

__device__ __forceinline__ void kick_pair_nr(const float4 A, const float4 B, const SinkDS& q,
                                             float eps2, float& bx, float& by, float& bz) {
    const float dx = __fadd_rn(__fadd_rn(A.x, q.nxh), __fadd_rn(B.x, q.nxl));
    const float dy = __fadd_rn(__fadd_rn(A.y, q.nyh), __fadd_rn(B.y, q.nyl));
    const float dz = __fadd_rn(__fadd_rn(A.z, q.nzh), __fadd_rn(B.z, q.nzl));
    const float d2 = fmaxf(fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2))), 1e-20f);
    const float y = rsqrtf(d2);
    const float y2 = __fmul_rn(y, y);
    const float c = fmaf(-1.5f, __fmul_rn(d2, y2), 2.5f);
    const float mr3 = __fmul_rn(__fmul_rn(A.w, __fmul_rn(y2, y)), c);
    bx = fmaf(dx, mr3, bx);
    by = fmaf(dy, mr3, by);
    bz = fmaf(dz, mr3, bz);
}

// Sources [lo, hi) of the shared tile on one sink (32-pair blocks, Kahan across blocks).
__device__ __forceinline__ void kick_span1(const Smem& sm, int lo, int hi, const SinkDS& q,
                                           float eps2, float (&acc)[3], float (&cmp)[3]) {
    int jb = lo;
    for (; jb < hi; jb += 32) {
        const int je = min(hi, jb + 32);
        float b[3] = {0.f, 0.f, 0.f};
#pragma unroll 4
        for (int j = jb; j < je; j++) kick_pair_nr(sm.u.kt.A[j], sm.u.kt.B[j], q, eps2, b[0], b[1], b[2]);
#pragma unroll
        for (int c = 0; c < 3; c++) kahan_add(acc[c], cmp[c], b[c]);
    }
}

// Sources [lo, hi) of the shared tile on two sinks at once (each record read once).
__device__ __forceinline__ void kick_span2(const Smem& sm, int lo, int hi, const SinkDS& q0,
                                           const SinkDS& q1, float eps2, float (&acc)[2][3],
                                           float (&cmp)[2][3]) {
    int jb = lo;
    for (; jb + 32 <= hi; jb += 32) {
        float b0[3] = {0.f, 0.f, 0.f}, b1[3] = {0.f, 0.f, 0.f};
#pragma unroll 4
        for (int j = jb; j < jb + 32; j++) {
            const float4 A = sm.u.kt.A[j], B = sm.u.kt.B[j];
            kick_pair_nr(A, B, q0, eps2, b0[0], b0[1], b0[2]);
            kick_pair_nr(A, B, q1, eps2, b1[0], b1[1], b1[2]);
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            kahan_add(acc[0][c], cmp[0][c], b0[c]);
            kahan_add(acc[1][c], cmp[1][c], b1[c]);
        }
    }
    if (jb < hi) {
        float b0[3] = {0.f, 0.f, 0.f}, b1[3] = {0.f, 0.f, 0.f};
        for (int j = jb; j < hi; j++) {
            const float4 A = sm.u.kt.A[j], B = sm.u.kt.B[j];
            kick_pair_nr(A, B, q0, eps2, b0[0], b0[1], b0[2]);
            kick_pair_nr(A, B, q1, eps2, b1[0], b1[1], b1[2]);
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            kahan_add(acc[0][c], cmp[0][c], b0[c]);
            kahan_add(acc[1][c], cmp[1][c], b1[c]);
        }
    }
}

// Stages source records [a, b) of the node into sm.u.kt: slow records [a, min(b, ns))
// from the level's packed pairs, fast ones gathered from the state arrays.
__device__ void kick_stage_tile(const EParams& E, const int32_t* F, const float4* PK, int a,
                                int b, int ns, Smem& sm) {
    __syncthreads();  // every thread is done reading the previous tile
    const int sb = min(b, ns);
    for (int j = a + (int)threadIdx.x; j < sb; j += kEB)
        pk_get(PK, j, sm.u.kt.A[j - a], sm.u.kt.B[j - a]);
    const SoA& P = E.P;
    for (int j = max(a, ns) + (int)threadIdx.x; j < b; j += kEB) {
        const int g = F[j - ns];
        const DS x = ds_split(P.x[g]), y = ds_split(P.y[g]), z = ds_split(P.z[g]);
        sm.u.kt.A[j - a] = make_float4(x.hi, y.hi, z.hi, (float)P.m[g]);
        sm.u.kt.B[j - a] = make_float4(x.lo, y.lo, z.lo, 0.0f);
    }
    __syncthreads();
}

// Work units (sink block ib, source chunk jc) of a node, as up to three rectangles
// {chunks [jc0, jc1) x blocks [ib0, ib1)}, enumerated chunk-major.
struct UnitGroups {
    int n;
    int jc0[3], jc1[3], ib0[3], ib1[3];
    __device__ long long count(int k) const {
        const int a = jc1[k] - jc0[k], b = ib1[k] - ib0[k];
        return (a > 0 && b > 0) ? (long long)a * b : 0;
    }
    __device__ void add(int j0, int j1, int i0, int i1) {
        jc0[n] = j0; jc1[n] = j1; ib0[n] = i0; ib1[n] = i1; n++;
    }
};

// Which units of a node's kick: every one, only those independent of the fast set
// (blocks of slow sinks x chunks of slow sources; they can run while the fast set is
// still being advanced), or the others.
enum { kUnitsAll = 0, kUnitsSlowOnly = 1, kUnitsRest = 2 };

__device__ UnitGroups kick_unit_groups(int nf, int ns, int nch, int C, int part, int ib_lo,
                                       int ib_hi) {
    const int ntot = nf + ns;
    const int nsb = (ntot + kKB - 1) / kKB;
    const int nfb = nf / kKB;                        // blocks of fast sinks only
    const int ibs = (nf + kKB - 1) / kKB;            // first block of slow sinks only
    const int ncs = min(nch, (ns + C - 1) / C);      // chunks holding slow sources
    const int ncss = min(nch, ns / C);               // chunks of slow sources only
    UnitGroups g;
    g.n = 0;
    if (part == kUnitsAll) {
        g.add(0, ncs, 0, nsb);
        g.add(ncs, nch, nfb, nsb);
    } else if (part == kUnitsSlowOnly) {
        g.add(0, ncss, ibs, nsb);
    } else {
        g.add(0, ncss, 0, ibs);
        g.add(ncss, ncs, 0, nsb);
        g.add(ncs, nch, nfb, nsb);
    }
    for (int k = 0; k < g.n; k++) {
        g.ib0[k] = max(g.ib0[k], ib_lo);
        g.ib1[k] = min(g.ib1[k], ib_hi);
    }
    return g;
}

// Sink blocks [ib_lo, ib_hi) of the node (all of them by default; a rank's share in the
// sharded kick of the multi-GPU step); `part` selects the units (kUnits*).
__device__ void kick_units_grid(const EParams& E, const int32_t* F, int nf, int ns, int lvl,
                                int nch, int C, const Workers& W, Smem& sm, int ib_lo = 0,
                                int ib_hi = -1, int part = kUnitsAll) {
    const int ntot = nf + ns;
    const SoA& P = E.P;
    const float4* PK = pk_level(E, lvl);
    if (ib_hi < 0) ib_hi = (ntot + kKB - 1) / kKB;
    if (ib_hi <= ib_lo || W.count <= 0) return;
    const UnitGroups grp = kick_unit_groups(nf, ns, nch, C, part, ib_lo, ib_hi);
    long long units = 0;
    for (int k = 0; k < grp.n; k++) units += grp.count(k);
    const long long u0 = units * W.id / W.count, u1 = units * (W.id + 1) / W.count;
    const float eps2 = E.eps2f;
    int res_a = -1, res_b = -1;  // source records resident in sm.u.kt
    for (long long u = u0; u < u1; u++) {
        int jc = 0, ib = 0;
        long long v = u;
        for (int k = 0; k < grp.n; k++) {
            const long long c = grp.count(k);
            if (v < c) {
                const int nb = grp.ib1[k] - grp.ib0[k];
                jc = grp.jc0[k] + (int)(v / nb);
                ib = grp.ib0[k] + (int)(v % nb);
                break;
            }
            v -= c;
        }
        const int j0 = jc * C, j1 = min(ntot, j0 + C);
        int sk[2], jend[2];
        SinkDS q[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            sk[k] = ib * kKB + k * kEB + (int)threadIdx.x;
            const bool act = sk[k] < ntot;
            const bool slow = sk[k] >= nf;
            q[k] = SinkDS{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (act) {
                if (slow) {
                    float4 a, b;
                    pk_get(PK, sk[k] - nf, a, b);
                    q[k] = SinkDS{-a.x, -a.y, -a.z, -b.x, -b.y, -b.z};
                } else {
                    const int g = F[sk[k]];
                    const DS x = ds_split(P.x[g]), y = ds_split(P.y[g]), z = ds_split(P.z[g]);
                    q[k] = SinkDS{-x.hi, -y.hi, -z.hi, -x.lo, -y.lo, -z.lo};
                }
            }
            jend[k] = act ? (slow ? j1 : min(j1, ns)) : j0;
        }
        float acc[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        float cmp[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        for (int a = j0; a < j1; a += kTS) {
            const int b = min(j1, a + kTS);
            if (a != res_a || b != res_b) {
                kick_stage_tile(E, F, PK, a, b, ns, sm);
                res_a = a;
                res_b = b;
            }
            const int e0 = max(0, min(b, jend[0]) - a), e1 = max(0, min(b, jend[1]) - a);
            const int m = min(e0, e1);
            kick_span2(sm, 0, m, q[0], q[1], eps2, acc, cmp);
            if (e0 > m) kick_span1(sm, m, e0, q[0], eps2, acc[0], cmp[0]);
            if (e1 > m) kick_span1(sm, m, e1, q[1], eps2, acc[1], cmp[1]);
        }
        double* part = E.k_part;
#pragma unroll
        for (int k = 0; k < 2; k++)
            if (sk[k] < ntot)
#pragma unroll
                for (int c = 0; c < 3; c++)
                    part[(size_t)(jc * 3 + c) * E.n_max + sk[k]] =
                        (double)acc[k][c] - (double)cmp[k][c];
    }
}

// ---------------------------------------------------------------- symmetric grid kick
// The kick of a large grid node in mixed precision, with each (fast, slow) pair
// evaluated once. The pair vector w = (x_j - x_i) / |x_j - x_i|^3 (fast i, slow j, slow
// position drifted by half the step) gives the fast sink m_j w and the slow sink -m_i w
// (Newton's third law); the reference evaluates the two kicks of the pair separately
// (src/kick.cuh:111-155 and :59-106). Work units, taken dynamically from a counter:
//  - cross units (fast super-block, slow chunk): rows are the super-block's fast sinks,
//    kEB at a time, one per thread; columns are the chunk's slow particles, bulk-copied
//    into shared memory in tiles of kTX. Rows sum their pair terms in 32-pair FP32 blocks
//    into Kahan-compensated sums (one partial per chunk); each column's terms are summed
//    over the warp by a transposed butterfly, over the CTA's warps in order and over the
//    super-block's rows in order, into one FP64 partial per (super-block, slow sink);
//  - slow units (block of kEB slow sinks, slow chunk): the slow-slow pairs, per sink.
// The reduce phase adds, per sink, its chunk partials in order and (slow sinks) its
// super-block partials in order: every sum has a fixed order, so a step is deterministic.
// Unit layout of the mixed grid kick of a node with nf fast and ns slow particles.
// Cross units (fast super-block, slow chunk) evaluate each fast-slow pair once for both
// particles. Slow units are either (sym) the chunk pairs a < b, each evaluating the pairs
// of chunk a x chunk b once for both particles, followed by one unit per block of kEB
// slow sinks against its own chunk; or (small slow sets, where those units would be too
// coarse to spread over the grid) blocks of kEB slow sinks x chunks, one direction only.
// Either way every slow particle receives exactly one partial per chunk slot.
__device__ __forceinline__ KickPlan kick_plan(int nf, int ns, int workers) {
    KickPlan p;
    p.R = nf >= kX2Min ? 2 : 1;
    p.nsub = (nf + p.R * kEB - 1) / (p.R * kEB);
    const int f = p.nsub < kMaxFsb ? p.nsub : kMaxFsb;
    p.FB = f > 0 ? (p.nsub + f - 1) / f : 1;
    p.nfsb = (p.nsub + p.FB - 1) / p.FB;
    p.nsb = (ns + kEB - 1) / kEB;
    p.sym = ns >= kSymMin;
    if (p.sym) {
        // chunks of whole two-row passes, at most kMaxChunks of them
        p.Rs = 2;
        const int rb = p.Rs * kEB, span = kMaxChunks * rb;
        p.Cs = rb * ((ns + span - 1) / span);
        p.ncs = (ns + p.Cs - 1) / p.Cs;
        p.noff = p.ncs * (p.ncs - 1) / 2;
        p.nsl = p.noff + p.nsb;
    } else {
        const int per = p.nfsb + p.nsb;  // units per chunk
        int c = (3 * workers + per - 1) / per;  // about three units per CTA
        const int cmax = min(kMaxChunks, (ns + 31) / 32);  // at least 32 slow particles a chunk
        c = c < 1 ? 1 : (c > cmax ? cmax : c);
        p.Cs = ((ns + c - 1) / c + 1) & ~1;  // even: chunks start on whole source pairs
        p.ncs = (ns + p.Cs - 1) / p.Cs;
        p.Rs = 1;
        p.noff = 0;
        p.nsl = p.nsb * p.ncs;
    }
    p.nx = p.nfsb * p.ncs;
    return p;
}

// chunk pair (a, b), a < b, of symmetric slow unit v (row-major over the upper triangle)
__device__ __forceinline__ void sym_pair_of(int v, int G, int& a, int& b) {
    a = 0;
    while (v >= G - 1 - a) {
        v -= G - 1 - a;
        a++;
    }
    b = a + 1 + v;
}

// Column sums over the warp of eight columns (three components each): lane l ends with
// the sums of column ((l >> 2) & 7) in r (every lane of a group of four holds them).
__device__ __forceinline__ void warp_colsum8(const float (&v)[8][3], float (&r)[3], int lane) {
    float a[4][3], b[2][3];
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
#pragma unroll
    for (int c = 0; c < 4; c++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float keep = b4 ? v[c + 4][k] : v[c][k], send = b4 ? v[c][k] : v[c + 4][k];
            a[c][k] = keep + __shfl_xor_sync(HHS_FULL_MASK, send, 16);
        }
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float keep = b3 ? a[c + 2][k] : a[c][k], send = b3 ? a[c][k] : a[c + 2][k];
            b[c][k] = keep + __shfl_xor_sync(HHS_FULL_MASK, send, 8);
        }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float keep = b2 ? b[1][k] : b[0][k], send = b2 ? b[0][k] : b[1][k];
        float t = keep + __shfl_xor_sync(HHS_FULL_MASK, send, 4);
        t += __shfl_xor_sync(HHS_FULL_MASK, t, 2);
        t += __shfl_xor_sync(HHS_FULL_MASK, t, 1);
        r[k] = t;
    }
}

// Two shared buffers of slow records: the tile a unit computes on, and the first tile of
// the next unit, copied in while this one computes. State is uniform across the CTA.
struct TileCache {
    int a[2], b[2];      // records [a, b) of the level's packed array held (or on their way)
    bool pending[2];     // a copy into the buffer was issued and not yet waited for
    unsigned phase;      // parities of the buffers' barriers (sm.tbar)
};

// thread 0: copy records [a, b) (a even: whole pair entries) into buffer c
__device__ __forceinline__ void tc_issue(const float4* PK, int a, int b, int c, Smem& sm) {
    const unsigned bytes = (unsigned)((b - a + 1) >> 1) * (unsigned)(4 * sizeof(float4));
    mbar_arrive_expect_tx(&sm.tbar[c], bytes);
    bulk_load(sm.u.kc.T[c], PK + 4 * (size_t)(a >> 1), bytes, &sm.tbar[c]);
}

// Makes records [a, b) available in buffer c (every thread calls it): copies them unless
// they are held or on their way, waits for an outstanding copy, and zeroes the records
// after b up to the next multiple of eight (massless at the origin: their pair terms
// vanish).
__device__ void tc_use(const EParams& E, const float4* PK, int a, int b, int c, TileCache& tc,
                       Smem& sm) {
    if (tc.a[c] != a || tc.b[c] != b) {
        __syncthreads();  // every thread is done with the buffer's previous records
        if (threadIdx.x == 0) tc_issue(PK, a, b, c, sm);
        tc.a[c] = a;
        tc.b[c] = b;
        tc.pending[c] = true;
    }
    if (tc.pending[c]) {
        if (!mbar_wait(&sm.tbar[c], (tc.phase >> c) & 1u, E.err))
            (void)mbar_wait(&sm.tbar[c], (tc.phase >> c) & 1u, nullptr);
        tc.phase ^= 1u << c;
        tc.pending[c] = false;
        const int len = b - a, len8 = (len + 7) & ~7;
        if ((int)threadIdx.x < len8 - len) {
            const int r = len + (int)threadIdx.x;
            float* q = reinterpret_cast<float*>(sm.u.kc.T[c][r >> 1]) + (r & 1);
#pragma unroll
            for (int k = 0; k < 8; k++) q[2 * k] = 0.0f;
        }
        __syncthreads();
    }
}

// A sink against a pair entry of sources in f32x2 arithmetic (the sink negated, each
// value in both lanes); each lane runs the scalar pair operations in their order.
struct SinkDS2 {
    float2 nxh, nyh, nzh, nxl, nyl, nzl;
};
__device__ __forceinline__ SinkDS2 sink2(const SinkDS& q) {
    return SinkDS2{f2dup(q.nxh), f2dup(q.nyh), f2dup(q.nzh),
                   f2dup(q.nxl), f2dup(q.nyl), f2dup(q.nzl)};
}

// offsets d = source - sink of the entry's two sources, and d2 = |d|^2 + eps^2 (floored)
__device__ __forceinline__ void pair_d2(const float4& Q0, const float4& Q1, const float4& Q2,
                                        const float4& Q3, const SinkDS2& q, float eps2,
                                        float2& dx, float2& dy, float2& dz, float2& d2) {
    dx = __fadd2_rn(__fadd2_rn(make_float2(Q0.x, Q0.y), q.nxh),
                    __fadd2_rn(make_float2(Q2.x, Q2.y), q.nxl));
    dy = __fadd2_rn(__fadd2_rn(make_float2(Q0.z, Q0.w), q.nyh),
                    __fadd2_rn(make_float2(Q2.z, Q2.w), q.nyl));
    dz = __fadd2_rn(__fadd2_rn(make_float2(Q1.x, Q1.y), q.nzh),
                    __fadd2_rn(make_float2(Q3.x, Q3.y), q.nzl));
    const float2 t = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, f2dup(eps2))));
    d2 = make_float2(fmaxf(t.x, 1e-20f), fmaxf(t.y, 1e-20f));
}

// 1/|d|^3 with one Newton correction, per lane
__device__ __forceinline__ float2 r3_nr2(float2 d2) {
    const float2 y = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
    const float2 y2 = __fmul2_rn(y, y);
    const float2 c = __ffma2_rn(f2dup(-1.5f), __fmul2_rn(d2, y2), f2dup(2.5f));
    return __fmul2_rn(__fmul2_rn(y2, y), c);
}

// Pair terms of rows [r0, r1) (sinks: the fast list, or the level's packed slow records)
// against the packed slow records [j0, j1) (columns), each pair evaluated once for both
// particles. R sinks per thread, so one column butterfly serves R rows. Row partials (the
// rows' accelerations from these columns) go to rout[k * nmx + row]; column partials (the
// columns' accelerations from these rows) to cout[k * nmx + j], summed over the row passes
// in order (the first pass stores).
template <int R>
__device__ void kick_pair_block(const EParams& E, const int32_t* F, bool rows_fast, int r0,
                                int r1, int j0, int j1, int lvl, double* rout, double* cout,
                                Smem& sm, TileCache& tc, int cb) {
    const SoA& P = E.P;
    const size_t nmx = E.n_max;
    const float4* PK = pk_level(E, lvl);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float eps2 = E.eps2f;
    for (int rp = r0; rp < r1; rp += R * kEB) {
        int s[R];
        SinkDS2 q[R];
        float nmi[R];  // -m_i: the column terms
#pragma unroll
        for (int r = 0; r < R; r++) {
            s[r] = rp + r * kEB + (int)threadIdx.x;
            SinkDS q1{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            nmi[r] = 0.0f;
            if (s[r] < r1) {
                if (rows_fast) {
                    const int g = F[s[r]];
                    const DS x = ds_split(P.x[g]), y = ds_split(P.y[g]), z = ds_split(P.z[g]);
                    q1 = SinkDS{-x.hi, -y.hi, -z.hi, -x.lo, -y.lo, -z.lo};
                    nmi[r] = -(float)P.m[g];
                } else {
                    float4 a, b;
                    pk_get(PK, s[r], a, b);
                    q1 = SinkDS{-a.x, -a.y, -a.z, -b.x, -b.y, -b.z};
                    nmi[r] = -a.w;
                }
            }
            q[r] = sink2(q1);
        }
        float acc[R][3], cmp[R][3];
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
            for (int k = 0; k < 3; k++) acc[r][k] = cmp[r][k] = 0.0f;
        for (int a = j0; a < j1; a += kTX) {
            const int b = min(j1, a + kTX), len = b - a;
            tc_use(E, PK, a, b, cb, tc, sm);
            const float4(*T)[4] = sm.u.kc.T[cb];
            // rows' sums of the even and odd columns in the two lanes
            float2 bl[R][3];
#pragma unroll
            for (int r = 0; r < R; r++) bl[r][0] = bl[r][1] = bl[r][2] = make_float2(0.f, 0.f);
            int nb = 0;
            for (int g8 = 0; g8 < len; g8 += 8) {
                float2 v2[4][3];  // column terms of the four entries (eight columns)
#pragma unroll
                for (int c2 = 0; c2 < 4; c2++) {
                    const int e = (g8 >> 1) + c2;
                    const float4 Q0 = T[e][0], Q1 = T[e][1], Q2 = T[e][2], Q3 = T[e][3];
                    const float2 m = make_float2(Q1.z, Q1.w);
#pragma unroll
                    for (int r = 0; r < R; r++) {
                        float2 dx, dy, dz, d2;
                        pair_d2(Q0, Q1, Q2, Q3, q[r], eps2, dx, dy, dz, d2);
                        const float2 r3 = r3_nr2(d2);
                        const float2 wx = __fmul2_rn(dx, r3), wy = __fmul2_rn(dy, r3),
                                     wz = __fmul2_rn(dz, r3);
                        bl[r][0] = __ffma2_rn(wx, m, bl[r][0]);
                        bl[r][1] = __ffma2_rn(wy, m, bl[r][1]);
                        bl[r][2] = __ffma2_rn(wz, m, bl[r][2]);
                        const float2 nm = f2dup(nmi[r]);
                        if (r == 0) {
                            v2[c2][0] = __fmul2_rn(wx, nm);
                            v2[c2][1] = __fmul2_rn(wy, nm);
                            v2[c2][2] = __fmul2_rn(wz, nm);
                        } else {
                            v2[c2][0] = __ffma2_rn(wx, nm, v2[c2][0]);
                            v2[c2][1] = __ffma2_rn(wy, nm, v2[c2][1]);
                            v2[c2][2] = __ffma2_rn(wz, nm, v2[c2][2]);
                        }
                    }
                }
                float v[8][3];
#pragma unroll
                for (int c2 = 0; c2 < 4; c2++)
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        v[2 * c2][k] = v2[c2][k].x;
                        v[2 * c2 + 1][k] = v2[c2][k].y;
                    }
                float rs[3];
                warp_colsum8(v, rs, lane);
                const int col = ((lane >> 2) & 7);
                if ((lane & 3) == 0 && g8 + col < len) {
                    sm.u.kc.colw[warp][g8 + col][0] = rs[0];
                    sm.u.kc.colw[warp][g8 + col][1] = rs[1];
                    sm.u.kc.colw[warp][g8 + col][2] = rs[2];
                }
                if (++nb == 4) {  // 32 pairs a row: into the compensated sums
#pragma unroll
                    for (int r = 0; r < R; r++)
#pragma unroll
                        for (int k = 0; k < 3; k++) {
                            kahan_add(acc[r][k], cmp[r][k], bl[r][k].x + bl[r][k].y);
                            bl[r][k] = make_float2(0.f, 0.f);
                        }
                    nb = 0;
                }
            }
            if (nb) {
#pragma unroll
                for (int r = 0; r < R; r++)
#pragma unroll
                    for (int k = 0; k < 3; k++)
                        kahan_add(acc[r][k], cmp[r][k], bl[r][k].x + bl[r][k].y);
            }
            __syncthreads();
            // the tile's column sums: the CTA's warps in order, then the row passes in order
            for (int t = threadIdx.x; t < 3 * len; t += kEB) {
                const int jl = t / 3, k = t - 3 * jl;
                double sum = 0.0;
#pragma unroll
                for (int w = 0; w < kEB / 32; w++) sum += (double)sm.u.kc.colw[w][jl][k];
                double* o = cout + (size_t)k * nmx + a + jl;
                *o = rp == r0 ? sum : *o + sum;
            }
            __syncthreads();  // colw is rewritten by the next pass
        }
#pragma unroll
        for (int r = 0; r < R; r++)
            if (s[r] < r1)
#pragma unroll
                for (int k = 0; k < 3; k++)
                    rout[(size_t)k * nmx + s[r]] = (double)acc[r][k] - (double)cmp[r][k];
    }
}

// One-directional slow unit: the block sb of kEB slow sinks against slow chunk jc, in
// f32x2 arithmetic over the chunk's source pairs (the even and odd sources' sums in the
// two lanes, 32 sources a block into the compensated sums).
__device__ void kick_slow_unit(const EParams& E, int nf, int lvl, const KickPlan& p, int sb,
                               int jc, int ns, Smem& sm, TileCache& tc, int cb) {
    const size_t nmx = E.n_max;
    const float4* PK = pk_level(E, lvl);
    const int j0 = jc * p.Cs, j1 = min(ns, j0 + p.Cs);
    const int qs = sb * kEB + (int)threadIdx.x;  // slow sink position
    const bool act = qs < ns;
    SinkDS q1{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (act) {
        float4 a, b;
        pk_get(PK, qs, a, b);
        q1 = SinkDS{-a.x, -a.y, -a.z, -b.x, -b.y, -b.z};
    }
    const SinkDS2 q = sink2(q1);
    const float eps2 = E.eps2f;
    float acc[3] = {0.f, 0.f, 0.f}, cmp[3] = {0.f, 0.f, 0.f};
    for (int a = j0; a < j1; a += kTX) {
        const int b = min(j1, a + kTX), len = b - a;
        tc_use(E, PK, a, b, cb, tc, sm);
        const float4(*T)[4] = sm.u.kc.T[cb];
        for (int jb = 0; jb < len; jb += 32) {
            const int ne = (min(len, jb + 32) - jb + 1) >> 1;  // entries of this block
            float2 bl[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll 4
            for (int i = 0; i < ne; i++) {
                const int e = (jb >> 1) + i;
                const float4 Q0 = T[e][0], Q1 = T[e][1], Q2 = T[e][2], Q3 = T[e][3];
                float2 dx, dy, dz, d2;
                pair_d2(Q0, Q1, Q2, Q3, q, eps2, dx, dy, dz, d2);
                const float2 mr3 = __fmul2_rn(make_float2(Q1.z, Q1.w), r3_nr2(d2));
                bl[0] = __ffma2_rn(dx, mr3, bl[0]);
                bl[1] = __ffma2_rn(dy, mr3, bl[1]);
                bl[2] = __ffma2_rn(dz, mr3, bl[2]);
            }
#pragma unroll
            for (int k = 0; k < 3; k++) kahan_add(acc[k], cmp[k], bl[k].x + bl[k].y);
        }
    }
    if (act)
#pragma unroll
        for (int k = 0; k < 3; k++)
            E.k_part[(size_t)(jc * 3 + k) * nmx + nf + qs] = (double)acc[k] - (double)cmp[k];
}

// Units of one kind set, taken from the level's counter `set` until none is left:
// kinds 0 = cross units then slow units, 1 = slow units only, 2 = cross units only.
// While a unit computes, thread 0 already takes the next unit and starts the copy of its
// first tile into the other buffer.
__device__ __forceinline__ int unit_chunk(const KickPlan& p, int nx, int u) {
    if (u < nx) return u / p.nfsb;
    const int v = u - nx;
    if (!p.sym) return v / p.nsb;
    if (v >= p.noff) return (v - p.noff) * kEB / p.Cs;  // a block of slow sinks: its own chunk
    int a, b;
    sym_pair_of(v, p.ncs, a, b);
    return b;
}

__device__ __forceinline__ void unit_first_tile(const KickPlan& p, int nx, int u, int& a, int& b) {
    a = unit_chunk(p, nx, u) * p.Cs;
    b = a + min(p.Cs, kTX);
}

__device__ void kick_sym_units(const EParams& E, const int32_t* F, int nf, int ns, int lvl,
                               const KickPlan& plan, int set, int kinds, Smem& sm) {
    const int nx = kinds == 1 ? 0 : plan.nx;
    const int total = nx + (kinds == 2 ? 0 : plan.nsl);
    if (threadIdx.x == 0) sm.kp = plan;  // read back after each barrier below
    const KickPlan& p = sm.kp;
    const float4* PK = pk_level(E, lvl);
    unsigned* ctr = &E.st->kick_ctr[set][lvl];
    TileCache tc;
    tc.a[0] = tc.a[1] = tc.b[0] = tc.b[1] = -1;
    tc.pending[0] = tc.pending[1] = false;
    tc.phase = sm.tphase;
    __syncthreads();  // every thread has read sm.tphase and the previous phase's sm.bcast
    if (threadIdx.x == 0) sm.bcast = (int)atomicAdd(ctr, 1u);
    __syncthreads();
    int u = sm.bcast, c = 0;
    auto clip = [&](int& a, int& b) { b = min(b, ns); };
    if (u < total) {
        int a, b;
        unit_first_tile(p, nx, u, a, b);
        clip(a, b);
        if (threadIdx.x == 0) tc_issue(PK, a, b, c, sm);
        tc.a[c] = a; tc.b[c] = b; tc.pending[c] = true;
    }
    while (u < total) {
        __syncthreads();  // every thread has read sm.bcast
        if (threadIdx.x == 0) {
            const int un = (int)atomicAdd(ctr, 1u);
            sm.bcast = un;
            if (un < total) {
                int a, b;
                unit_first_tile(p, nx, un, a, b);
                clip(a, b);
                if (tc.a[c ^ 1] != a || tc.b[c ^ 1] != b) tc_issue(PK, a, b, c ^ 1, sm);
            }
        }
        // one call site per kind of block keeps the inlined pair loops to three copies
        {
            const size_t nmx = E.n_max;
            int kind = 0, r0 = 0, r1 = 0, j0 = 0, j1 = 0, sb = 0, jc = 0;
            double *rout = nullptr, *cout = nullptr;
            const int v = u - nx;
            if (u < nx) {  // cross unit: fast super-block fsb x slow chunk jc
                const int fsb = u % p.nfsb, rb = p.R * kEB;
                jc = u / p.nfsb;
                kind = p.R == 2 ? 2 : 1;
                r0 = fsb * p.FB * rb;
                r1 = min(nf, r0 + p.FB * rb);
                rout = E.k_part + (size_t)jc * 3 * nmx;
                cout = E.c_part + (size_t)fsb * 3 * nmx + nf;
            } else if (p.sym && v < p.noff) {  // slow chunk a x slow chunk b > a
                int a, b;
                sym_pair_of(v, p.ncs, a, b);
                kind = 3;
                r0 = a * p.Cs;
                r1 = min(ns, r0 + p.Cs);
                jc = b;
                rout = E.k_part + (size_t)b * 3 * nmx + nf;
                cout = E.k_part + (size_t)a * 3 * nmx + nf;
            } else if (p.sym) {  // a block of slow sinks against its own chunk
                sb = v - p.noff;
                jc = sb * kEB / p.Cs;
            } else {
                sb = v % p.nsb;
                jc = v / p.nsb;
            }
            j0 = jc * p.Cs;
            j1 = min(ns, j0 + p.Cs);
            if (kind >= 2)
                kick_pair_block<2>(E, F, kind == 2, r0, r1, j0, j1, lvl, rout, cout, sm, tc, c);
            else if (kind == 1)
                kick_pair_block<1>(E, F, true, r0, r1, j0, j1, lvl, rout, cout, sm, tc, c);
            else
                kick_slow_unit(E, nf, lvl, p, sb, jc, ns, sm, tc, c);
        }
        __syncthreads();  // the unit is done; sm.bcast holds the next one
        const int un = sm.bcast;
        if (un < total) {
            int a, b;
            unit_first_tile(p, nx, un, a, b);
            clip(a, b);
            if (tc.a[c ^ 1] != a || tc.b[c ^ 1] != b) {
                tc.a[c ^ 1] = a; tc.b[c ^ 1] = b; tc.pending[c ^ 1] = true;
            }
        }
        u = un;
        c ^= 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) sm.tphase = tc.phase;
    __syncthreads();
}

// ---------------------------------------------------------------- packed kick units
// The mixed kick with two sinks per thread (s and s + kEB) evaluated together in packed
// FP32 pairs (fma/add/mul.rn.f32x2 of sm_100): one instruction advances both sinks'
// pair terms, so the per-pair instruction count halves. Sources are staged once per
// tile with each coordinate duplicated, so a 128-bit shared load fills two packed
// operands. Self pairs (d2 == 0) contribute exactly 0 through a 1e-20 floor on d2
// (finite rsqrt, zero numerator); for d2 >= 1e-20 the floor never changes d2.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// lim0: sources at or beyond lim0 do not act on the first sink (a fast sink sharing the
// thread with a slow one sees slow sources only)
__device__ __forceinline__ void kick_x2_pairs(const Smem& sm, int jbeg, int jend, float2 nxh,
                                              float2 nyh, float2 nzh, float2 nxl, float2 nyl,
                                              float2 nzl, int lim0, float2 eps2, float2& ax,
                                              float2& ay, float2& az) {
    const float2 half = f2(-0.5f, -0.5f), three_half = f2(1.5f, 1.5f);
#pragma unroll 4
    for (int jl = jbeg; jl < jend; jl++) {
        const float4 P0 = sm.u.kx.P0[jl], P1 = sm.u.kx.P1[jl], P2 = sm.u.kx.P2[jl];
        float2 M = sm.u.kx.M[jl];
        if (jl >= lim0) M.x = 0.0f;
        const float2 dx = __fadd2_rn(__fadd2_rn(f2(P0.x, P0.y), nxh), __fadd2_rn(f2(P1.z, P1.w), nxl));
        const float2 dy = __fadd2_rn(__fadd2_rn(f2(P0.z, P0.w), nyh), __fadd2_rn(f2(P2.x, P2.y), nyl));
        const float2 dz = __fadd2_rn(__fadd2_rn(f2(P1.x, P1.y), nzh), __fadd2_rn(f2(P2.z, P2.w), nzl));
        float2 d2 = __ffma2_rn(dz, dz, eps2);
        d2 = __ffma2_rn(dy, dy, d2);
        d2 = __ffma2_rn(dx, dx, d2);
        d2.x = fmaxf(d2.x, 1e-20f);
        d2.y = fmaxf(d2.y, 1e-20f);
        const float2 y = f2(rsqrtf(d2.x), rsqrtf(d2.y));
        const float2 ri = __fmul2_rn(y, __ffma2_rn(__fmul2_rn(d2, half), __fmul2_rn(y, y), three_half));
        const float2 ri2 = __fmul2_rn(ri, ri);
        const float2 mr3 = __fmul2_rn(__fmul2_rn(M, ri2), ri);
        ax = __ffma2_rn(dx, mr3, ax);
        ay = __ffma2_rn(dy, mr3, ay);
        az = __ffma2_rn(dz, mr3, az);
    }
}

__device__ void kick_unit_x2(const EParams& E, const int32_t* F, const int32_t* L, int nf,
                             int ns, double h, int ib, int jc, int j0, int j1, Smem& sm) {
    const int n = nf + ns;
    const SoA& P = E.P;
    const int n_max = E.n_max;
    int s[2];
    s[0] = ib * (2 * kEB) + threadIdx.x;
    s[1] = s[0] + kEB;
    DS sx[2], sy[2], sz[2];
    int jend[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const bool act = s[q] < n;
        const bool slow = s[q] >= nf;
        jend[q] = act ? (slow ? j1 : min(j1, ns)) : j0;
        double x = 0, y = 0, z = 0;
        if (act) {
            const int g = slow ? L[s[q] - nf] : F[s[q]];
            x = P.x[g]; y = P.y[g]; z = P.z[g];
            if (slow) { x = fma(P.vx[g], h, x); y = fma(P.vy[g], h, y); z = fma(P.vz[g], h, z); }
        }
        sx[q] = ds_split(x); sy[q] = ds_split(y); sz[q] = ds_split(z);
    }
    const float2 nxh = f2(-sx[0].hi, -sx[1].hi), nyh = f2(-sy[0].hi, -sy[1].hi),
                 nzh = f2(-sz[0].hi, -sz[1].hi), nxl = f2(-sx[0].lo, -sx[1].lo),
                 nyl = f2(-sy[0].lo, -sy[1].lo), nzl = f2(-sz[0].lo, -sz[1].lo);
    float acc[2][3] = {{0, 0, 0}, {0, 0, 0}}, cmp[2][3] = {{0, 0, 0}, {0, 0, 0}};
    for (int t0 = j0; t0 < j1; t0 += kEB) {
        const int tl = min(kEB, j1 - t0);
        __syncthreads();
        if ((int)threadIdx.x < tl) {
            const int j = t0 + threadIdx.x;
            const bool js = j < ns;
            const int gj = js ? L[j] : F[j - ns];
            double x = P.x[gj], y = P.y[gj], z = P.z[gj];
            if (js) { x = fma(P.vx[gj], h, x); y = fma(P.vy[gj], h, y); z = fma(P.vz[gj], h, z); }
            const DS a = ds_split(x), b = ds_split(y), c = ds_split(z);
            sm.u.kx.P0[threadIdx.x] = make_float4(a.hi, a.hi, b.hi, b.hi);
            sm.u.kx.P1[threadIdx.x] = make_float4(c.hi, c.hi, a.lo, a.lo);
            sm.u.kx.P2[threadIdx.x] = make_float4(b.lo, b.lo, c.lo, c.lo);
            const float m = (float)P.m[gj];
            sm.u.kx.M[threadIdx.x] = make_float2(m, m);
        }
        __syncthreads();
        // fast sinks come first in a block, so when the two sinks' source limits differ
        // the first sink is the fast one (smaller limit); an inactive second sink's
        // results are never written
        const int e0 = min(tl, jend[0] - t0), e1 = min(tl, jend[1] - t0);
        const int emax = max(e0, e1);
        for (int jb = 0; jb < emax; jb += 32) {
            float2 bx = f2(0.f, 0.f), by = f2(0.f, 0.f), bz = f2(0.f, 0.f);
            kick_x2_pairs(sm, jb, min(jb + 32, emax), nxh, nyh, nzh, nxl, nyl, nzl, e0,
                          make_float2(E.eps2f, E.eps2f), bx, by, bz);
            kahan_add(acc[0][0], cmp[0][0], bx.x);
            kahan_add(acc[0][1], cmp[0][1], by.x);
            kahan_add(acc[0][2], cmp[0][2], bz.x);
            kahan_add(acc[1][0], cmp[1][0], bx.y);
            kahan_add(acc[1][1], cmp[1][1], by.y);
            kahan_add(acc[1][2], cmp[1][2], bz.y);
        }
    }
    double* part = E.k_part;
#pragma unroll
    for (int q = 0; q < 2; q++)
        if (s[q] < n)
#pragma unroll
            for (int k = 0; k < 3; k++)
                part[(size_t)(jc * 3 + k) * n_max + s[q]] = (double)acc[q][k] - (double)cmp[q][k];
}

// ---------------------------------------------------------------- node phases
// Per-sink reduction of the timestep partials (calc) or plain predicate (no calc),
// writing per-tile predicate counts.
template <int PREC>
__device__ void count_phase(const EParams& E, const int32_t* S, int n, double dt, bool calc,
                            int nch, const Workers& W, Smem& sm) {
    const int ntiles = (n + kEB - 1) / kEB;
    for (int t = W.id; t < ntiles; t += W.count) {
        const int i = t * kEB + threadIdx.x;
        int flag = 0;
        if (i < n) {
            const int gi = list_at(S, i);
            double ts;
            if (calc) {
                if (PREC == HHS_PREC_FP64) {
                    double mv = 1.e30;
                    for (int c = 0; c < nch; c++) {
                        const double v = E.ts_part[(size_t)c * E.n_max + i];
                        if (v < mv) mv = v;
                    }
                    ts = mv;
                } else {
                    const float mr = __uint_as_float(E.rate_acc[i]);
                    E.rate_acc[i] = 0u;
                    const double tv = 1.0 / (double)mr;
                    ts = tv < 1.e30 ? tv : 1.e30;
                }
                E.P.ts[gi] = ts;
            } else {
                ts = E.P.ts[gi];
            }
            flag = ts <= dt;
        }
        const int c = block_sum(flag, sm);
        if (threadIdx.x == 0) E.tile_counts[t] = c;
    }
}

// Stable scatter into F_k / L_k with the N_fast == 1 fold (src/split.cuh:304-370).
__device__ void scatter_phase(const EParams& E, const int32_t* S, int n, double dt, int level,
                              bool calc, const Workers& W, Smem& sm) {
    const int ntiles = (n + kEB - 1) / kEB;
    int32_t* F = E.fast_lists + (size_t)level * E.n_max;
    int32_t* L = E.slow_lists + (size_t)level * E.n_max;
    // grand total (every worker computes it; identical everywhere)
    int part = 0;
    for (int t = threadIdx.x; t < ntiles; t += kEB) part += E.tile_counts[t];
    const int nf_raw = block_sum(part, sm);
    const bool fold = nf_raw == 1;
    for (int t = W.id; t < ntiles; t += W.count) {
        int pre = 0;
        for (int u = threadIdx.x; u < t; u += kEB) pre += E.tile_counts[u];
        const int prefix = block_sum(pre, sm);
        const int i = t * kEB + threadIdx.x;
        int flag = 0, gi = 0;
        if (i < n) {
            gi = list_at(S, i);
            flag = E.P.ts[gi] <= dt;
        }
        int tot;
        const int ex = block_excl_flag(flag, sm, tot);
        if (i < n) {
            const int p = prefix + ex;
            if (flag) {
                if (fold) L[n - 1] = gi;
                else F[p] = gi;
            } else {
                L[i - p] = gi;
            }
        }
    }
    if (W.id == 0 && threadIdx.x == 0) {
        const int nf = fold ? 0 : nf_raw;
        E.counts[level].n_fast = nf;
        E.counts[level].n_slow = n - nf;
        trace_node(E, level, n, nf, calc);
        if (nf == 0) *E.leaf_time += dt;
        const double ns = (double)(n - nf), nfd = (double)nf;
        atomicAdd(reinterpret_cast<unsigned long long*>(&E.stats->nodes), 1ull);
        atomicMax(&E.stats->max_level, level);
        atomicAdd(&E.stats->kick_pairs, ns * (ns - 1.0) + 2.0 * ns * nfd);
        if (calc) atomicAdd(&E.stats->ts_pairs, (double)n * (double)(n - 1));
    }
}

// Predicate and stable scatter in one pass (grid mode): each 256-particle tile publishes
// its fast count and finds its prefix by a decoupled look-back over the tiles before it
// (hhs_scan.cuh), so no grid barrier separates counting from scattering. Tiles are taken
// in increasing order by every CTA of the co-resident grid, so every look-back ends. The
// N_fast == 1 fold costs nothing: the first fast particle is also written to L[n-1],
// which is the lone particle's place after the fold and an unused slot otherwise (every
// slow particle lands below n-1 once one fast particle exists). The tile that ends the
// list writes the counts and the work counters.
template <int PREC>
__device__ void split_phase(const EParams& E, const int32_t* S, int n, double dt, int level,
                            bool calc, int nch, const Workers& W, Smem& sm) {
    const int ntiles = (n + kEB - 1) / kEB;
    int32_t* F = E.fast_lists + (size_t)level * E.n_max;
    int32_t* L = E.slow_lists + (size_t)level * E.n_max;
    if (threadIdx.x == 0) sm.epoch = (sm.bar_k + 1u) & 0x3fffffffu;
    __syncthreads();
    const unsigned epoch = sm.epoch;
    for (int t = W.id; t < ntiles; t += W.count) {
        const int i = t * kEB + threadIdx.x;
        int flag = 0, gi = 0;
        if (i < n) {
            gi = list_at(S, i);
            double ts;
            if (calc) {
                if (PREC == HHS_PREC_FP64) {
                    double mv = 1.e30;
                    for (int c = 0; c < nch; c++) {
                        const double v = E.ts_part[(size_t)c * E.n_max + i];
                        if (v < mv) mv = v;
                    }
                    ts = mv;
                } else {
                    const float mr = __uint_as_float(E.rate_acc[i]);
                    E.rate_acc[i] = 0u;
                    const double tv = 1.0 / (double)mr;
                    ts = tv < 1.e30 ? tv : 1.e30;
                }
                E.P.ts[gi] = ts;
            } else {
                ts = E.P.ts[gi];
            }
            flag = ts <= dt;
        }
        int tot;
        const int ex = block_excl_flag(flag, sm, tot);
        if (threadIdx.x < 32) {
            const unsigned pre = scan_lookback_w<1>(E.tile_status, t, (unsigned)tot, epoch, E.err,
                                                    HHS_SPIN_LIMIT);
            if (threadIdx.x == 0) sm.bcast = (int)pre;
        }
        __syncthreads();
        const int prefix = sm.bcast;
        if (i < n) {
            const int p = prefix + ex;
            int q = -1;  // slow-list position (the first fast particle: the fold's slot)
            if (flag) {
                F[p] = gi;
                if (p == 0) {
                    L[n - 1] = gi;
                    q = n - 1;
                }
            } else {
                L[i - p] = gi;
                q = i - p;
            }
            if (PREC != HHS_PREC_FP64 && q >= 0 && E.pk && level < E.pk_levels) {
                // packed kick source: the slow particle at its drifted kick position
                const double h = dt * 0.5;
                const DS x = ds_split(fma(E.P.vx[gi], h, E.P.x[gi]));
                const DS y = ds_split(fma(E.P.vy[gi], h, E.P.y[gi]));
                const DS z = ds_split(fma(E.P.vz[gi], h, E.P.z[gi]));
                pk_put(pk_level(E, level), q, x, y, z, (float)E.P.m[gi]);
            }
        }
        if (t == ntiles - 1 && threadIdx.x == 0) {
            const int nf_raw = prefix + tot;
            const int nf = nf_raw == 1 ? 0 : nf_raw;
            E.counts[level].n_fast = nf;
            E.counts[level].n_slow = n - nf;
            if (E.st && level < kMaxLevels) {  // the level's kick takes its units afresh
                E.st->kick_ctr[0][level] = 0u;
                E.st->kick_ctr[1][level] = 0u;
            }
            trace_node(E, level, n, nf, calc);
            if (nf == 0) *E.leaf_time += dt;
            const double ns = (double)(n - nf), nfd = (double)nf;
            atomicAdd(reinterpret_cast<unsigned long long*>(&E.stats->nodes), 1ull);
            atomicMax(&E.stats->max_level, level);
            atomicAdd(&E.stats->kick_pairs, ns * (ns - 1.0) + 2.0 * ns * nfd);
            if (calc) atomicAdd(&E.stats->ts_pairs, (double)n * (double)(n - 1));
        }
        __syncthreads();
    }
}

// Sum of the per-chunk partial accelerations, v += a*dt, and for slow sinks both half
// drifts. Mixed: one thread per (sink, component) adds its chunks with eight independent
// loads in flight, so the reduction of a node spreads over the whole grid; FP64: one
// thread per sink (slow then fast sources, the reference's order).
// nfsb >= 0: the symmetric kick's partials (nch = its chunk count: fast sinks add their
// nch chunk partials, slow sinks those and then their nfsb super-block partials).
template <int PREC>
__device__ void kick_reduce_phase(const EParams& E, const int32_t* F, const int32_t* L, int nf,
                                  int ns, double dt, int nch, int C, const Workers& W,
                                  Smem& sm, int nfsb = -1) {
    const int n = nf + ns;
    const double h = dt * 0.5;
    const SoA& P = E.P;
    if (PREC == HHS_PREC_FP64) {
        const int ntiles = (n + kEB - 1) / kEB;
        for (int t = W.id; t < ntiles; t += W.count) {
            const int s = t * kEB + threadIdx.x;
            if (s >= n) continue;
            const bool slow = s >= nf;
            const int g = slow ? L[s - nf] : F[s];
            const double v0[3] = {P.vx[g], P.vy[g], P.vz[g]};
            double v1[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                double v = f64_add(v0[k], f64_mul(E.k_part[(size_t)k * E.n_max + s], dt));
                if (slow && nf > 0)
                    v = f64_add(v, f64_mul(E.k_part[(size_t)(3 + k) * E.n_max + s], dt));
                v1[k] = v;
            }
            P.vx[g] = v1[0]; P.vy[g] = v1[1]; P.vz[g] = v1[2];
            if (slow) {
                P.x[g] = f64_add(f64_add(P.x[g], f64_mul(v0[0], h)), f64_mul(v1[0], h));
                P.y[g] = f64_add(f64_add(P.y[g], f64_mul(v0[1], h)), f64_mul(v1[1], h));
                P.z[g] = f64_add(f64_add(P.z[g], f64_mul(v0[2], h)), f64_mul(v1[2], h));
            }
        }
        return;
    }
    constexpr int kPer = kEB / 3;  // sinks per CTA iteration (3 components each)
    const int ntiles = (n + kPer - 1) / kPer;
    const int lastf = nfsb >= 0 ? nch : min(nch, (ns + C - 1) / C);  // chunks for fast sinks
    double* red = reinterpret_cast<double*>(&sm.u);
    for (int t = W.id; t < ntiles; t += W.count) {
        const int q = (int)threadIdx.x / 3, k = (int)threadIdx.x % 3;
        const int s = t * kPer + q;
        double a = 0.0;
        if (q < kPer && s < n) {
            const int last = s >= nf ? nch : lastf;
            const double* part = E.k_part + (size_t)k * E.n_max + s;
            const size_t stride = (size_t)3 * E.n_max;
            int c = 0;
            for (; c + 8 <= last; c += 8) {
                double v[8];
#pragma unroll
                for (int u = 0; u < 8; u++) v[u] = part[(size_t)(c + u) * stride];
#pragma unroll
                for (int u = 0; u < 8; u++) a += v[u];
            }
            for (; c < last; c++) a += part[(size_t)c * stride];
            if (nfsb > 0 && s >= nf) {
                const double* cpart = E.c_part + (size_t)k * E.n_max + s;
                for (int f = 0; f < nfsb; f++) a += cpart[(size_t)f * stride];
            }
        }
        __syncthreads();
        red[threadIdx.x] = a;
        __syncthreads();
        if ((int)threadIdx.x < kPer) {
            const int s2 = t * kPer + (int)threadIdx.x;
            if (s2 < n) {
                const bool slow = s2 >= nf;
                const int g = slow ? L[s2 - nf] : F[s2];
                const double v0[3] = {P.vx[g], P.vy[g], P.vz[g]};
                double v1[3];
#pragma unroll
                for (int c = 0; c < 3; c++) v1[c] = fma(red[3 * threadIdx.x + c], dt, v0[c]);
                P.vx[g] = v1[0]; P.vy[g] = v1[1]; P.vz[g] = v1[2];
                if (!slow && E.tq && W.mode == kModeGrid) {
                    // the fast set's next pass recomputes its timesteps from these records
                    tq_put(E, s2, P.x[g], P.y[g], P.z[g], P.m[g], v1[0], v1[1], v1[2]);
                }
                if (slow) {
                    P.x[g] = fma(v1[0], h, fma(v0[0], h, P.x[g]));
                    P.y[g] = fma(v1[1], h, fma(v0[1], h, P.y[g]));
                    P.z[g] = fma(v1[2], h, fma(v0[2], h, P.z[g]));
                }
            }
        }
    }
}


// ---------------------------------------------------------------- tiny subtree solver
// A subsystem of at most 32 particles, with its whole subtree, on one CTA: the state
// lives in shared memory (FP64), each level's subset is a 32-bit slot mask, the split is
// a ballot (stable order = slot order; the N_fast == 1 fold keeps the lone slot and
// visits it last among the slow sources). Pair work is spread over the CTA's 8 warps:
// lane = sink slot, warp = source group (slots w, w+8, w+16, w+24), partial results
// reduced by warp 0. The FP64 kick sums stay sequential per sink (warp 0) so the FP64
// form keeps the reference's summation order and stays bit-exact. No list, count or
// partial-sum traffic to global memory; the state is written back once.
template <int PREC>
__device__ void tiny_hold(const EParams& E, const int32_t* S, int n, int level0, bool calc0,
                          Smem& sm) {
    auto& T = sm.u.tiny;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const SoA& P = E.P;
    if (warp == 0) {
        const bool act = lane < n;
        const int g = act ? list_at(S, lane) : 0;
        T.g[lane] = g;
        T.x[lane] = act ? P.x[g] : 0.0; T.y[lane] = act ? P.y[g] : 0.0;
        T.z[lane] = act ? P.z[g] : 0.0; T.vx[lane] = act ? P.vx[g] : 0.0;
        T.vy[lane] = act ? P.vy[g] : 0.0; T.vz[lane] = act ? P.vz[g] : 0.0;
        T.m[lane] = act ? P.m[g] : 0.0; T.ts[lane] = act ? P.ts[g] : 1.e30;
    }
    __syncthreads();
    const unsigned top_mask = n >= 32 ? 0xffffffffu : ((1u << n) - 1u);
    unsigned long long after1 = 0, after2 = 0, calcm = calc0 ? 1ull : 0ull;
    int d = 0;
    while (d >= 0) {
        const int lvl = level0 + d;
        const unsigned long long bit = 1ull << d;
        const unsigned mask = d == 0 ? top_mask : sm.wfast[d - 1];
        const bool in = (mask >> lane) & 1u;
        const double dt = dt_at(E, lvl);
        if (!(after1 & bit)) {
            if (lvl >= E.max_levels || lvl >= kMaxLevels - 1) {
                if (threadIdx.x == 0) atomicOr(E.err, HHS_ERRBIT_DEPTH);
                break;
            }
            const int cnt = __popc(mask);
            if (calcm & bit) {
                if (PREC == HHS_PREC_FP64) {
                    double mv = 1.e30;
                    if (in) {
#pragma unroll 1
                        for (int j = warp; j < 32; j += kEB / 32) {
                            if (!((mask >> j) & 1u) || j == lane) continue;
                            ts_pair_fp64(f64_sub(T.x[lane], T.x[j]), f64_sub(T.y[lane], T.y[j]),
                                         f64_sub(T.z[lane], T.z[j]), f64_sub(T.vx[lane], T.vx[j]),
                                         f64_sub(T.vy[lane], T.vy[j]), f64_sub(T.vz[lane], T.vz[j]),
                                         T.m[lane], T.m[j], E.eta, E.eta_s2, mv);
                        }
                    }
                    T.pmin[warp][lane] = mv;
                    __syncthreads();
                    if (warp == 0 && in) {
                        double m = 1.e30;
#pragma unroll
                        for (int w = 0; w < kEB / 32; w++) m = T.pmin[w][lane] < m ? T.pmin[w][lane] : m;
                        T.ts[lane] = m;
                    }
                } else {
                    if (warp == 0) {
                        const DS a = ds_split(T.x[lane]), b = ds_split(T.y[lane]),
                                 c = ds_split(T.z[lane]);
                        T.A[lane] = make_float4(a.hi, b.hi, c.hi, (float)T.m[lane]);
                        T.B[lane] = make_float4(a.lo, b.lo, c.lo, 0.0f);
                        T.V[lane] = make_float4((float)T.vx[lane], (float)T.vy[lane],
                                                (float)T.vz[lane], 0.0f);
                    }
                    __syncthreads();
                    float mr = 0.0f;
                    if (in) {
                        const float4 Ai = T.A[lane], Bi = T.B[lane], Vi = T.V[lane];
#pragma unroll 1
                        for (int j = warp; j < 32; j += kEB / 32) {
                            if (!((mask >> j) & 1u) || j == lane) continue;
                            const float4 A = T.A[j], B = T.B[j], V = T.V[j];
                            mr = fmaxf(mr, ts_pair_rate_mixed(
                                               ds_diff(Ai.x, Bi.x, A.x, B.x), ds_diff(Ai.y, Bi.y, A.y, B.y),
                                               ds_diff(Ai.z, Bi.z, A.z, B.z), Vi.x - V.x, Vi.y - V.y,
                                               Vi.z - V.z, Ai.w + A.w, E.inv_eta_s2, E.inv_eta));
                        }
                    }
                    T.pmax[warp][lane] = mr;
                    __syncthreads();
                    if (warp == 0 && in) {
                        float m = 0.0f;
#pragma unroll
                        for (int w = 0; w < kEB / 32; w++) m = fmaxf(m, T.pmax[w][lane]);
                        const double tv = 1.0 / (double)m;
                        T.ts[lane] = tv < 1.e30 ? tv : 1.e30;
                    }
                }
                __syncthreads();
            }
            if (warp == 0) {
                unsigned F = __ballot_sync(HHS_FULL_MASK, in && T.ts[lane] <= dt);
                int lone = -1;
                if (__popc(F) == 1) { lone = __ffs(F) - 1; F = 0u; }
                if (lane == 0) {
                    sm.wfast[d] = F;
                    sm.wlone[d] = lone;
                    const int nf = __popc(F);
                    trace_node(E, lvl, cnt, nf, (calcm & bit) != 0);
                    const double ns = (double)(cnt - nf), nfd = (double)nf;
                    if (nf == 0) *E.leaf_time += dt;
                    atomicAdd(reinterpret_cast<unsigned long long*>(&E.stats->nodes), 1ull);
                    atomicMax(&E.stats->max_level, lvl);
                    atomicAdd(&E.stats->kick_pairs, ns * (ns - 1.0) + 2.0 * ns * nfd);
                    if (calcm & bit) atomicAdd(&E.stats->ts_pairs, (double)cnt * (double)(cnt - 1));
                }
            }
            __syncthreads();
            after1 |= bit;
            if (sm.wfast[d]) {
                d++;
                const unsigned long long cb = 1ull << d;
                calcm &= ~cb; after1 &= ~cb; after2 &= ~cb;
                continue;
            }
        }
        if (!(after2 & bit)) {
            const unsigned F = sm.wfast[d];
            const int lone = sm.wlone[d];
            const unsigned L = mask & ~F;
            const bool is_slow = (L >> lane) & 1u, is_fast = (F >> lane) & 1u;
            const double h = dt * 0.5;
            if (L) {
                if (warp == 0) {
                    // first half drift of the slow slots (src/hold.cuh:123-124)
                    if (is_slow) {
                        if (PREC == HHS_PREC_FP64) {
                            T.x[lane] = f64_add(T.x[lane], f64_mul(T.vx[lane], h));
                            T.y[lane] = f64_add(T.y[lane], f64_mul(T.vy[lane], h));
                            T.z[lane] = f64_add(T.z[lane], f64_mul(T.vz[lane], h));
                        } else {
                            T.x[lane] = fma(T.vx[lane], h, T.x[lane]);
                            T.y[lane] = fma(T.vy[lane], h, T.y[lane]);
                            T.z[lane] = fma(T.vz[lane], h, T.z[lane]);
                        }
                    }
                    if (PREC != HHS_PREC_FP64) {
                        __syncwarp();
                        const DS a = ds_split(T.x[lane]), b = ds_split(T.y[lane]),
                                 c = ds_split(T.z[lane]);
                        T.A[lane] = make_float4(a.hi, b.hi, c.hi, (float)T.m[lane]);
                        T.B[lane] = make_float4(a.lo, b.lo, c.lo, 0.0f);
                    }
                }
                __syncthreads();
                if (PREC == HHS_PREC_FP64) {
                    if (warp == 0 && (is_slow || is_fast)) {
                        const double xi = T.x[lane], yi = T.y[lane], zi = T.z[lane];
                        const unsigned Lord = lone >= 0 ? (L & ~(1u << lone)) : L;
                        double aL[3] = {0, 0, 0}, aF[3] = {0, 0, 0};
#pragma unroll 1
                        for (unsigned mm = Lord; mm; mm &= mm - 1u) {
                            const int j = __ffs(mm) - 1;
                            kick_pair_fp64(f64_sub(T.x[j], xi), f64_sub(T.y[j], yi),
                                           f64_sub(T.z[j], zi), T.m[j], aL[0], aL[1], aL[2],
                                           E.eps2);
                        }
                        if (lone >= 0)
                            kick_pair_fp64(f64_sub(T.x[lone], xi), f64_sub(T.y[lone], yi),
                                           f64_sub(T.z[lone], zi), T.m[lone], aL[0], aL[1], aL[2],
                                           E.eps2);
                        if (is_slow) {
#pragma unroll 1
                            for (unsigned mm = F; mm; mm &= mm - 1u) {
                                const int j = __ffs(mm) - 1;
                                kick_pair_fp64(f64_sub(T.x[j], xi), f64_sub(T.y[j], yi),
                                               f64_sub(T.z[j], zi), T.m[j], aF[0], aF[1], aF[2],
                                               E.eps2);
                            }
                        }
                        double vx = f64_add(T.vx[lane], f64_mul(aL[0], dt));
                        double vy = f64_add(T.vy[lane], f64_mul(aL[1], dt));
                        double vz = f64_add(T.vz[lane], f64_mul(aL[2], dt));
                        if (is_slow && F) {
                            vx = f64_add(vx, f64_mul(aF[0], dt));
                            vy = f64_add(vy, f64_mul(aF[1], dt));
                            vz = f64_add(vz, f64_mul(aF[2], dt));
                        }
                        __syncwarp(__activemask());
                        T.vx[lane] = vx; T.vy[lane] = vy; T.vz[lane] = vz;
                        if (is_slow) {
                            T.x[lane] = f64_add(xi, f64_mul(vx, h));
                            T.y[lane] = f64_add(yi, f64_mul(vy, h));
                            T.z[lane] = f64_add(zi, f64_mul(vz, h));
                        }
                    }
                } else {
                    float a[3] = {0, 0, 0};
                    const unsigned srcs = is_slow ? (L | F) : (is_fast ? L : 0u);
                    if (srcs) {
                        const float4 Ai = T.A[lane], Bi = T.B[lane];
#pragma unroll 1
                        for (int j = warp; j < 32; j += kEB / 32) {
                            if (!((srcs >> j) & 1u)) continue;
                            const float4 A = T.A[j], B = T.B[j];
                            const float dx = ds_diff(A.x, B.x, Ai.x, Bi.x);
                            const float dy = ds_diff(A.y, B.y, Ai.y, Bi.y);
                            const float dz = ds_diff(A.z, B.z, Ai.z, Bi.z);
                            const float d2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, E.eps2f)));
                            const float mr3 = mr3_nr(A.w, d2);
                            a[0] = fmaf(dx, mr3, a[0]);
                            a[1] = fmaf(dy, mr3, a[1]);
                            a[2] = fmaf(dz, mr3, a[2]);
                        }
                    }
                    T.part[warp][0][lane] = a[0];
                    T.part[warp][1][lane] = a[1];
                    T.part[warp][2][lane] = a[2];
                    __syncthreads();
                    if (warp == 0 && (is_slow || is_fast)) {
                        double acc[3] = {0, 0, 0};
#pragma unroll
                        for (int w = 0; w < kEB / 32; w++)
#pragma unroll
                            for (int k = 0; k < 3; k++) acc[k] += (double)T.part[w][k][lane];
                        const double vx = fma(acc[0], dt, T.vx[lane]);
                        const double vy = fma(acc[1], dt, T.vy[lane]);
                        const double vz = fma(acc[2], dt, T.vz[lane]);
                        T.vx[lane] = vx; T.vy[lane] = vy; T.vz[lane] = vz;
                        if (is_slow) {
                            T.x[lane] = fma(vx, h, T.x[lane]);
                            T.y[lane] = fma(vy, h, T.y[lane]);
                            T.z[lane] = fma(vz, h, T.z[lane]);
                        }
                    }
                }
                __syncthreads();
            }
            after2 |= bit;
            if (F) {
                d++;
                const unsigned long long cb = 1ull << d;
                calcm = (calcm & ~cb) | cb;
                after1 &= ~cb; after2 &= ~cb;
                continue;
            }
        }
        calcm &= ~bit; after1 &= ~bit; after2 &= ~bit;
        d--;
    }
    __syncthreads();
    if ((int)threadIdx.x < n) {
        const int g = T.g[threadIdx.x];
        P.x[g] = T.x[threadIdx.x]; P.y[g] = T.y[threadIdx.x]; P.z[g] = T.z[threadIdx.x];
        P.vx[g] = T.vx[threadIdx.x]; P.vy[g] = T.vy[threadIdx.x]; P.vz[g] = T.vz[threadIdx.x];
        P.ts[g] = T.ts[threadIdx.x];
    }
    __syncthreads();
}

// ---------------------------------------------------------------- cluster subtree solver
// A subsystem of at most kMid particles, with its whole subtree, on one thread-block
// cluster (or one CTA). Every CTA of the cluster holds a replica of the subsystem in
// shared memory and walks the same recursion; the members of each level are slot
// bitmasks (stable order = slot order, the N_fast == 1 fold visits the lone slot last
// among the slow ones). Splits and drifts are computed redundantly in every CTA (the
// same arithmetic in the same order keeps the replicas identical). The pair work of a
// node with more than `dist_n` members is divided among the cluster's CTAs: each CTA
// computes its share of the sinks and stores the results (timesteps or velocities)
// into every replica through distributed shared memory, between two cluster barriers
// (the first one makes sure no CTA is still reading what the stores overwrite). Nodes
// of up to 32 members run with their subtree on one warp of every CTA (warp_subtree);
// the others are computed whole by every CTA with CTA barriers only. Global memory is
// read once at entry and written once at exit.
namespace mid {

// slots of the set bits of words[0..nw) in increasing order -> out; returns the count
__device__ __forceinline__ int compact(const unsigned* words, int nw, short* out,
                                       MidState& M) {
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid < 32) {
        const int c = lane < nw ? __popc(words[lane]) : 0;
        const int inc = warp_incl_scan(c, lane);
        if (lane < nw) M.wbase[lane] = inc - c;
        if (lane == 31) M.total = inc;
    }
    __syncthreads();
    for (int s = tid; s < nw * 32; s += kEB) {
        const unsigned w = words[s >> 5];
        const int b = s & 31;
        if ((w >> b) & 1u) out[M.wbase[s >> 5] + __popc(w & ((1u << b) - 1u))] = (short)s;
    }
    const int total = M.total;
    __syncthreads();
    return total;
}

// kick order of a node in one pass: the slow members (stable; the lone slot, if any,
// last) then the fast ones. Returns the number of slow slots; *nf_out the fast count.
__device__ __forceinline__ int kick_order(const unsigned* memw, const unsigned* fastw, int lone,
                                          int nw, short* out, MidState& M, int* nf_out) {
    const int tid = threadIdx.x, lane = tid & 31;
    const unsigned lone_word = lone >= 0 ? (unsigned)(lone >> 5) : 0xffffffffu;
    const unsigned lone_keep = lone >= 0 ? ~(1u << (lone & 31)) : ~0u;
    if (tid < 32) {
        unsigned sw = 0u, fw = 0u;
        if (lane < nw) {
            fw = fastw[lane];
            sw = memw[lane] & ~fw;
            if ((unsigned)lane == lone_word) sw &= lone_keep;
        }
        const int cs_ = __popc(sw), cf = __popc(fw);
        const int is = warp_incl_scan(cs_, lane), iff = warp_incl_scan(cf, lane);
        if (lane < nw) {
            M.wbase[lane] = is - cs_;
            M.wbase2[lane] = iff - cf;
        }
        if (lane == 31) {
            M.total = is + (lone >= 0 ? 1 : 0);
            M.total2 = iff;
        }
    }
    __syncthreads();
    const int ns = M.total, nf = M.total2;
    for (int s = tid; s < nw * 32; s += kEB) {
        const int w = s >> 5, b = s & 31;
        const unsigned fw = fastw[w];
        unsigned sw = memw[w] & ~fw;
        if ((unsigned)w == lone_word) sw &= lone_keep;
        const unsigned below = (1u << b) - 1u;
        if ((sw >> b) & 1u) out[M.wbase[w] + __popc(sw & below)] = (short)s;
        else if ((fw >> b) & 1u) out[ns + M.wbase2[w] + __popc(fw & below)] = (short)s;
    }
    if (tid == 0 && lone >= 0) out[ns - 1] = (short)lone;
    __syncthreads();
    *nf_out = nf;
    return ns;
}

// mixed-precision views of slot k (double-single position, FP32 velocity)
__device__ __forceinline__ void refresh_pos(MidState& M, int k) {
    const DS a = ds_split(M.x[k]), b = ds_split(M.y[k]), c = ds_split(M.z[k]);
    M.A[k] = make_float4(a.hi, b.hi, c.hi, (float)M.m[k]);
    M.B[k] = make_float4(a.lo, b.lo, c.lo, 0.0f);
}
__device__ __forceinline__ void refresh_vel(MidState& M, int k) {
    M.V[k] = make_float4((float)M.vx[k], (float)M.vy[k], (float)M.vz[k], 0.0f);
}

// a result for slot p: into this replica only, or into every replica of the cluster
template <class T>
__device__ __forceinline__ void put(T* p, T v, bool dist, int cs) {
    if (!dist) {
        *p = v;
        return;
    }
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    for (int r = 0; r < cs; r++) *cl.map_shared_rank(p, (unsigned)r) = v;
}

// atomic maximum of a slot's rate word in this replica only, or in every replica
__device__ __forceinline__ void put_max(unsigned* p, unsigned v, bool dist, int cs) {
    if (!dist) {
        atomicMax(p, v);
        return;
    }
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    for (int r = 0; r < cs; r++) atomicMax(cl.map_shared_rank(p, (unsigned)r), v);
}

// Mixed timesteps of the node's members (M.mem[0..nm)), each unordered pair evaluated
// once (the pair rate is exactly symmetric): 32 x 32 tiles of the upper triangle over
// the warps of the CTA, or of the whole cluster when dist; row maxima in registers,
// column maxima by one warp max-reduction per column; both merged into every replica's
// per-slot maxima, then every CTA turns them into timesteps. The result equals the
// maximum over all ordered pairs bit for bit.
__device__ void mid_timesteps_sym(const EParams& E, MidState& M, int nm, bool dist, int cs,
                                  int rank) {
    namespace cg = cooperative_groups;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k = tid; k < nm; k += kEB) M.rmax[M.mem[k]] = 0u;
    if (dist) cg::this_cluster().sync();
    else __syncthreads();
    const int nb = (nm + 31) >> 5;
    const int tiles = nb * (nb + 1) / 2;
    const int gw = (dist ? rank : 0) * (kEB / 32) + warp;
    const int nwarps = (dist ? cs : 1) * (kEB / 32);
    for (int t = gw; t < tiles; t += nwarps) {
        int rb = 0, rem = t;
        while (rem >= nb - rb) {
            rem -= nb - rb;
            rb++;
        }
        const int cb = rb + rem;
        const int p = rb * 32 + lane;
        const bool act = p < nm;
        const int i = act ? M.mem[p] : 0;
        const float4 Ai = M.A[i], Bi = M.B[i], Vi = M.V[i];
        float rowmax = 0.0f;
        unsigned colmax = 0u;
        const int ncol = min(32, nm - cb * 32);
#pragma unroll 4
        for (int c = 0; c < ncol; c++) {
            const int q = cb * 32 + c;
            const int j = M.mem[q];
            const float4 A = M.A[j], B = M.B[j], V = M.V[j];
            const float r = ts_pair_rate_mixed(ds_diff(Ai.x, Bi.x, A.x, B.x),
                                               ds_diff(Ai.y, Bi.y, A.y, B.y),
                                               ds_diff(Ai.z, Bi.z, A.z, B.z), Vi.x - V.x,
                                               Vi.y - V.y, Vi.z - V.z, Ai.w + A.w,
                                               E.inv_eta_s2, E.inv_eta);
            const float rr = (act && q > p) ? r : 0.0f;
            rowmax = fmaxf(rowmax, rr);
            const unsigned cm = __reduce_max_sync(HHS_FULL_MASK, __float_as_uint(rr));
            colmax = lane == c ? cm : colmax;
        }
        if (act && rowmax > 0.0f) put_max(&M.rmax[i], __float_as_uint(rowmax), dist, cs);
        if (lane < ncol && colmax > 0u) put_max(&M.rmax[M.mem[cb * 32 + lane]], colmax, dist, cs);
    }
    if (dist) cg::this_cluster().sync();
    else __syncthreads();
    for (int k = tid; k < nm; k += kEB) {
        const int slot = M.mem[k];
        const double tv = 1.0 / (double)__uint_as_float(M.rmax[slot]);
        M.ts[slot] = tv < 1.e30 ? tv : 1.e30;
    }
    __syncthreads();
}

// the CTA's share [s0, s1) of n sinks and the (sink group, source part) work layout
struct Share {
    int s0, s1, ng, wpg;
};
__device__ __forceinline__ Share share_of(int n, bool dist, int cs, int rank) {
    Share sh;
    const int parts = dist ? cs : 1;
    const int r = dist ? rank : 0;
    const int q = (n + parts - 1) / parts;
    sh.s0 = min(n, r * q);
    sh.s1 = min(n, sh.s0 + q);
    sh.ng = (sh.s1 - sh.s0 + 31) / 32;
    sh.wpg = sh.ng >= kEB / 32 ? 1 : (sh.ng > 0 ? (kEB / 32) / sh.ng : 1);
    return sh;
}

// max pair rate of sink i over the sources list[q], q = q0, q0 + step, ... < qn (the sink
// itself excluded); four independent pairs per iteration
__device__ __forceinline__ float rate_over(const EParams& E, const MidState& M, const short* list,
                                           int q0, int qn, int step, int i) {
    const float4 Ai = M.A[i], Bi = M.B[i], Vi = M.V[i];
    float mr = 0.0f;
    int q = q0;
    auto one = [&](int j) {
        const float4 A = M.A[j], B = M.B[j], V = M.V[j];
        const float r = ts_pair_rate_mixed(ds_diff(Ai.x, Bi.x, A.x, B.x), ds_diff(Ai.y, Bi.y, A.y, B.y),
                                           ds_diff(Ai.z, Bi.z, A.z, B.z), Vi.x - V.x, Vi.y - V.y,
                                           Vi.z - V.z, Ai.w + A.w, E.inv_eta_s2, E.inv_eta);
        return j == i ? 0.0f : r;
    };
#pragma unroll 1
    for (; q + 3 * step < qn; q += 4 * step) {
        const int j0 = list[q], j1 = list[q + step], j2 = list[q + 2 * step], j3 = list[q + 3 * step];
        const float r0 = one(j0), r1 = one(j1), r2 = one(j2), r3 = one(j3);
        mr = fmaxf(mr, fmaxf(fmaxf(r0, r1), fmaxf(r2, r3)));
    }
#pragma unroll 1
    for (; q < qn; q += step) mr = fmaxf(mr, one(list[q]));
    return mr;
}

// mixed acceleration of sink i from the sources list[q], q = q0, q0 + step, ... < qn
__device__ __forceinline__ void acc_over(const EParams& E, const MidState& M, const short* list,
                                         int q0, int qn, int step, int i, float (&a)[3]) {
    const float4 Ai = M.A[i], Bi = M.B[i];
    auto one = [&](int j) {
        const float4 A = M.A[j], B = M.B[j];
        const float dx = ds_diff(A.x, B.x, Ai.x, Bi.x);
        const float dy = ds_diff(A.y, B.y, Ai.y, Bi.y);
        const float dz = ds_diff(A.z, B.z, Ai.z, Bi.z);
        const float d2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, E.eps2f)));
        const float mr3 = mr3_nr(A.w, d2);
        a[0] = fmaf(dx, mr3, a[0]);
        a[1] = fmaf(dy, mr3, a[1]);
        a[2] = fmaf(dz, mr3, a[2]);
    };
    int q = q0;
#pragma unroll 1
    for (; q + 3 * step < qn; q += 4 * step) {
        const int j0 = list[q], j1 = list[q + step], j2 = list[q + 2 * step], j3 = list[q + 3 * step];
        one(j0); one(j1); one(j2); one(j3);
    }
#pragma unroll 1
    for (; q < qn; q += step) one(list[q]);
}

}  // namespace mid

// Fine-grained timing inside the cluster subtree solver (profiling only; CTA 0, thread 0):
// kind 7 of the level table, slots 56 load, 57 timesteps, 58 split, 59 kick, 60 warp
// subtrees (of which 62 their timesteps, 63 their kicks and drifts), 61 write-back.
__device__ __forceinline__ void mid_mark(const EParams& E, Smem& sm, unsigned long long& t,
                                         int slot) {
    if (!E.profile || blockIdx.x != 0 || threadIdx.x != 0) return;
    const unsigned long long now = gtimer();
    if (slot >= 0) {
        sm.prof_ns[7][slot] += now - t;
        sm.prof_cnt[7][slot] += 1;
    }
    t = now;
}

// Warp solver for a node of at most 32 members with its whole subtree (every node below
// it is smaller): warp 0 of the CTA, one member per lane, warp barriers only. Lanes are
// members in increasing slot order (the stable order); the state stays in the MidState
// arrays, read and written by slot. Work counters go to lane 0's accumulators.
template <int PREC>
__device__ void warp_subtree(const EParams& E, MidState& M, const unsigned* memw, int nw,
                             int cnt, int level0, bool calc0, unsigned long long& nodes,
                             int& maxl, double& kpairs, double& tpairs, double& leaf,
                             bool& ok, bool rec, Smem& sm) {
    const int lane = threadIdx.x & 31;
    unsigned long long tw = 0;
    // lane l takes the l-th member
    {
        // member slot w * 32 + l (bit l of word w) is the k-th member, k = the members in
        // the words before w plus the set bits below l
        const int c = lane < nw ? __popc(memw[lane]) : 0;
        const int base = warp_incl_scan(c, lane) - c;
        for (int w = 0; w < nw; w++) {
            const unsigned mw = memw[w];
            if (!mw) continue;
            const int bw = __shfl_sync(HHS_FULL_MASK, base, w);
            if ((mw >> lane) & 1u)
                M.wslot[bw + __popc(mw & ((1u << lane) - 1u))] = (short)(w * 32 + lane);
        }
        __syncwarp();
    }
    const int me = lane < cnt ? M.wslot[lane] : 0;
    const unsigned top = cnt >= 32 ? 0xffffffffu : ((1u << cnt) - 1u);
    unsigned long long after1 = 0, after2 = 0, calcm = calc0 ? 1ull : 0ull;
    int dd = 0;
    while (dd >= 0) {
        const int lvl = level0 + dd;
        const unsigned long long bit = 1ull << dd;
        const double dt = dt_at(E, lvl);
        const unsigned mk = dd == 0 ? top : M.wf[dd - 1];
        const bool in = (mk >> lane) & 1u;
        if (!(after1 & bit)) {
            if (lvl >= E.max_levels || lvl >= kMaxLevels - 1) {
                if (lane == 0) atomicOr(E.err, HHS_ERRBIT_DEPTH);
                ok = false;
                return;
            }
            const int n_here = __popc(mk);
            if (calcm & bit) {
                mid_mark(E, sm, tw, -1);
                if (in) {
                    const unsigned srcs = mk & ~(1u << lane);
                    if (PREC == HHS_PREC_FP64) {
                        const double xi = M.x[me], yi = M.y[me], zi = M.z[me];
                        const double vxi = M.vx[me], vyi = M.vy[me], vzi = M.vz[me], mi = M.m[me];
                        double mv = 1.e30;
#pragma unroll 1
                        for (unsigned m = srcs; m; m &= m - 1u) {
                            const int j = M.wslot[__ffs(m) - 1];
                            ts_pair_fp64(f64_sub(xi, M.x[j]), f64_sub(yi, M.y[j]),
                                         f64_sub(zi, M.z[j]), f64_sub(vxi, M.vx[j]),
                                         f64_sub(vyi, M.vy[j]), f64_sub(vzi, M.vz[j]), mi, M.m[j],
                                         E.eta, E.eta_s2, mv);
                        }
                        M.ts[me] = mv;
                    } else {
                        const float4 Ai = M.A[me], Bi = M.B[me], Vi = M.V[me];
                        auto rate = [&](int j) {
                            const float4 A = M.A[j], B = M.B[j], V = M.V[j];
                            return ts_pair_rate_mixed(
                                ds_diff(Ai.x, Bi.x, A.x, B.x), ds_diff(Ai.y, Bi.y, A.y, B.y),
                                ds_diff(Ai.z, Bi.z, A.z, B.z), Vi.x - V.x, Vi.y - V.y, Vi.z - V.z,
                                Ai.w + A.w, E.inv_eta_s2, E.inv_eta);
                        };
                        float mr = 0.0f;
                        unsigned m = srcs;
#pragma unroll 1
                        while (__popc(m) >= 4) {  // four independent pairs per iteration
                            const int l0 = __ffs(m) - 1;
                            m &= m - 1u;
                            const int l1 = __ffs(m) - 1;
                            m &= m - 1u;
                            const int l2 = __ffs(m) - 1;
                            m &= m - 1u;
                            const int l3 = __ffs(m) - 1;
                            m &= m - 1u;
                            const float r0 = rate(M.wslot[l0]), r1 = rate(M.wslot[l1]);
                            const float r2 = rate(M.wslot[l2]), r3 = rate(M.wslot[l3]);
                            mr = fmaxf(mr, fmaxf(fmaxf(r0, r1), fmaxf(r2, r3)));
                        }
#pragma unroll 1
                        for (; m; m &= m - 1u) mr = fmaxf(mr, rate(M.wslot[__ffs(m) - 1]));
                        const double tv = 1.0 / (double)mr;
                        M.ts[me] = tv < 1.e30 ? tv : 1.e30;
                    }
                }
                __syncwarp();
                if (lane == 0) tpairs += (double)n_here * (double)(n_here - 1);
                mid_mark(E, sm, tw, 62);
            }
            unsigned F = __ballot_sync(HHS_FULL_MASK, in && M.ts[me] <= dt);
            int lone = -1;
            if (__popc(F) == 1) {
                lone = __ffs(F) - 1;
                F = 0u;
            }
            if (lane == 0) {
                M.wf[dd] = F;
                M.wl[dd] = lone;
                const int nf = __popc(F);
                if (rec) trace_node(E, lvl, n_here, nf, (calcm & bit) != 0);
                const double ns = (double)(n_here - nf), nfd = (double)nf;
                nodes++;
                maxl = max(maxl, lvl);
                kpairs += ns * (ns - 1.0) + 2.0 * ns * nfd;
                if (nf == 0) leaf += dt;
            }
            __syncwarp();
            after1 |= bit;
            if (F) {
                dd++;
                const unsigned long long cb = 1ull << dd;
                calcm &= ~cb; after1 &= ~cb; after2 &= ~cb;
                continue;
            }
        }
        if (!(after2 & bit)) {
            const unsigned F = M.wf[dd];
            const int lone = M.wl[dd];
            const unsigned L = mk & ~F;
            const bool is_slow = (L >> lane) & 1u, is_fast = (F >> lane) & 1u;
            const double h = dt * 0.5;
            if (L) {
                mid_mark(E, sm, tw, -1);
                // first half drift of the slow lanes (src/hold.cuh:123-124)
                if (is_slow) {
                    if (PREC == HHS_PREC_FP64) {
                        M.x[me] = f64_add(M.x[me], f64_mul(M.vx[me], h));
                        M.y[me] = f64_add(M.y[me], f64_mul(M.vy[me], h));
                        M.z[me] = f64_add(M.z[me], f64_mul(M.vz[me], h));
                    } else {
                        M.x[me] = fma(M.vx[me], h, M.x[me]);
                        M.y[me] = fma(M.vy[me], h, M.y[me]);
                        M.z[me] = fma(M.vz[me], h, M.z[me]);
                        mid::refresh_pos(M, me);
                    }
                }
                __syncwarp();
                double vx = 0.0, vy = 0.0, vz = 0.0;
                if (is_slow || is_fast) {
                    if (PREC == HHS_PREC_FP64) {
                        const double xi = M.x[me], yi = M.y[me], zi = M.z[me];
                        const unsigned Lord = lone >= 0 ? (L & ~(1u << lone)) : L;
                        double aL[3] = {0, 0, 0}, aF[3] = {0, 0, 0};
#pragma unroll 1
                        for (unsigned m = Lord; m; m &= m - 1u) {
                            const int j = M.wslot[__ffs(m) - 1];
                            kick_pair_fp64(f64_sub(M.x[j], xi), f64_sub(M.y[j], yi),
                                           f64_sub(M.z[j], zi), M.m[j], aL[0], aL[1], aL[2],
                                           E.eps2);
                        }
                        if (lone >= 0) {
                            const int j = M.wslot[lone];
                            kick_pair_fp64(f64_sub(M.x[j], xi), f64_sub(M.y[j], yi),
                                           f64_sub(M.z[j], zi), M.m[j], aL[0], aL[1], aL[2],
                                           E.eps2);
                        }
                        if (is_slow) {
#pragma unroll 1
                            for (unsigned m = F; m; m &= m - 1u) {
                                const int j = M.wslot[__ffs(m) - 1];
                                kick_pair_fp64(f64_sub(M.x[j], xi), f64_sub(M.y[j], yi),
                                               f64_sub(M.z[j], zi), M.m[j], aF[0], aF[1], aF[2],
                                               E.eps2);
                            }
                        }
                        vx = f64_add(M.vx[me], f64_mul(aL[0], dt));
                        vy = f64_add(M.vy[me], f64_mul(aL[1], dt));
                        vz = f64_add(M.vz[me], f64_mul(aL[2], dt));
                        if (is_slow && F) {
                            vx = f64_add(vx, f64_mul(aF[0], dt));
                            vy = f64_add(vy, f64_mul(aF[1], dt));
                            vz = f64_add(vz, f64_mul(aF[2], dt));
                        }
                    } else {
                        const float4 Ai = M.A[me], Bi = M.B[me];
                        float a[3] = {0, 0, 0};
                        auto acc = [&](int j) {
                            const float4 A = M.A[j], B = M.B[j];
                            const float dx = ds_diff(A.x, B.x, Ai.x, Bi.x);
                            const float dy = ds_diff(A.y, B.y, Ai.y, Bi.y);
                            const float dz = ds_diff(A.z, B.z, Ai.z, Bi.z);
                            const float d2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, E.eps2f)));
                            const float mr3 = mr3_nr(A.w, d2);
                            a[0] = fmaf(dx, mr3, a[0]);
                            a[1] = fmaf(dy, mr3, a[1]);
                            a[2] = fmaf(dz, mr3, a[2]);
                        };
                        unsigned m = is_slow ? (L | F) : L;
#pragma unroll 1
                        while (__popc(m) >= 4) {
                            const int l0 = __ffs(m) - 1;
                            m &= m - 1u;
                            const int l1 = __ffs(m) - 1;
                            m &= m - 1u;
                            const int l2 = __ffs(m) - 1;
                            m &= m - 1u;
                            const int l3 = __ffs(m) - 1;
                            m &= m - 1u;
                            acc(M.wslot[l0]);
                            acc(M.wslot[l1]);
                            acc(M.wslot[l2]);
                            acc(M.wslot[l3]);
                        }
#pragma unroll 1
                        for (; m; m &= m - 1u) acc(M.wslot[__ffs(m) - 1]);
                        vx = fma((double)a[0], dt, M.vx[me]);
                        vy = fma((double)a[1], dt, M.vy[me]);
                        vz = fma((double)a[2], dt, M.vz[me]);
                    }
                }
                __syncwarp();  // every lane's reads of the positions precede the drifts
                if (is_slow || is_fast) {
                    M.vx[me] = vx; M.vy[me] = vy; M.vz[me] = vz;
                    if (PREC != HHS_PREC_FP64) mid::refresh_vel(M, me);
                }
                if (is_slow) {
                    // second half drift (src/hold.cuh:158-159)
                    if (PREC == HHS_PREC_FP64) {
                        M.x[me] = f64_add(M.x[me], f64_mul(vx, h));
                        M.y[me] = f64_add(M.y[me], f64_mul(vy, h));
                        M.z[me] = f64_add(M.z[me], f64_mul(vz, h));
                    } else {
                        M.x[me] = fma(vx, h, M.x[me]);
                        M.y[me] = fma(vy, h, M.y[me]);
                        M.z[me] = fma(vz, h, M.z[me]);
                        mid::refresh_pos(M, me);
                    }
                }
                __syncwarp();
                mid_mark(E, sm, tw, 63);
            }
            after2 |= bit;
            if (F) {
                dd++;
                const unsigned long long cb = 1ull << dd;
                calcm = (calcm & ~cb) | cb;
                after1 &= ~cb; after2 &= ~cb;
                continue;
            }
        }
        calcm &= ~bit; after1 &= ~bit; after2 &= ~bit;
        dd--;
    }
}

// cs, rank: the hardware cluster that runs the subtree (every CTA of it calls mid_hold),
// or cs = 1 for one CTA alone whatever cluster it belongs to.
template <int PREC>
__device__ void mid_hold(const EParams& E, const int32_t* S, int n, int level0, bool calc0,
                         int dist_n, int cs, int rank, Smem& sm) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    MidState& M = *reinterpret_cast<MidState*>(&sm.u);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const SoA& P = E.P;
    const int nw = (n + 31) >> 5;
    unsigned long long tm = 0;
    mid_mark(E, sm, tm, -1);
    for (int k = tid; k < n; k += kEB) {
        const int g = list_at(S, k);
        M.g[k] = g;
        M.x[k] = P.x[g]; M.y[k] = P.y[g]; M.z[k] = P.z[g];
        M.vx[k] = P.vx[g]; M.vy[k] = P.vy[g]; M.vz[k] = P.vz[g];
        M.m[k] = P.m[g]; M.ts[k] = P.ts[g];
        if (PREC != HHS_PREC_FP64) { mid::refresh_pos(M, k); mid::refresh_vel(M, k); }
    }
    if (tid < kMidW)
        M.allw[tid] = tid < nw ? (tid == nw - 1 && (n & 31) ? (1u << (n & 31)) - 1u : ~0u) : 0u;
    if (tid == 0) M.nmem[0] = n;
    __syncthreads();
    mid_mark(E, sm, tm, 56);
    // work counters of this subtree (thread 0; added to the context once, by CTA 0)
    unsigned long long nodes = 0;
    int maxl = 0;
    double kpairs = 0.0, tpairs = 0.0, leaf = 0.0;
    unsigned long long after1 = 0, after2 = 0, calcm = calc0 ? 1ull : 0ull;
    int d = 0;
    bool ok = true;
    while (d >= 0) {
        const int lvl = level0 + d;
        const unsigned long long bit = 1ull << d;
        const double dt = dt_at(E, lvl);
        const unsigned* memw = d == 0 ? M.allw : M.fmask[d - 1];
        if (!(after1 & bit)) {
            if (lvl >= E.max_levels || lvl >= kMaxLevels - 1) {
                if (tid == 0) atomicOr(E.err, HHS_ERRBIT_DEPTH);
                ok = false;
                break;
            }
            if (M.nmem[d] <= 32) {
                // at most 32 members: the whole subtree on warp 0 of every CTA
                mid_mark(E, sm, tm, -1);
                if (warp == 0)
                    warp_subtree<PREC>(E, M, memw, nw, M.nmem[d], lvl, (calcm & bit) != 0,
                                       nodes, maxl, kpairs, tpairs, leaf, ok, rank == 0, sm);
                __syncthreads();
                mid_mark(E, sm, tm, 60);
                calcm &= ~bit; after1 &= ~bit; after2 &= ~bit;
                d--;
                continue;
            }
            mid_mark(E, sm, tm, -1);
            if (calcm & bit) {
                // ---- timesteps of the members (min over all other members)
                const int nm = mid::compact(memw, nw, M.mem, M);
                const bool dist = cs > 1 && nm > dist_n;
                if (PREC != HHS_PREC_FP64) {
                    mid::mid_timesteps_sym(E, M, nm, dist, cs, rank);
                    if (tid == 0) tpairs += (double)nm * (double)(nm - 1);
                } else {
                if (dist) cl.sync();
                const mid::Share sh = mid::share_of(nm, dist, cs, rank);
                const int items = sh.ng * sh.wpg;
                for (int it = warp; it < items; it += kEB / 32) {
                    const int grp = it / sh.wpg, part = it % sh.wpg;
                    const int p = sh.s0 + grp * 32 + lane;
                    const bool act = p < sh.s1;
                    const int i = act ? M.mem[p] : 0;
                    if (PREC == HHS_PREC_FP64) {
                        double mv = 1.e30;
                        if (act) {
                            const double xi = M.x[i], yi = M.y[i], zi = M.z[i];
                            const double vxi = M.vx[i], vyi = M.vy[i], vzi = M.vz[i], mi = M.m[i];
#pragma unroll 1
                            for (int q = part; q < nm; q += sh.wpg) {
                                const int j = M.mem[q];
                                if (j == i) continue;
                                ts_pair_fp64(f64_sub(xi, M.x[j]), f64_sub(yi, M.y[j]),
                                             f64_sub(zi, M.z[j]), f64_sub(vxi, M.vx[j]),
                                             f64_sub(vyi, M.vy[j]), f64_sub(vzi, M.vz[j]), mi,
                                             M.m[j], E.eta, E.eta_s2, mv);
                            }
                        }
                        if (sh.wpg > 1) M.red.pmin[it][lane] = mv;
                        else if (act) mid::put(&M.ts[i], mv, dist, cs);
                    } else {
                        const float mr = act ? mid::rate_over(E, M, M.mem, part, nm, sh.wpg, i) : 0.0f;
                        if (sh.wpg > 1) {
                            M.red.pmax[it][lane] = mr;
                        } else if (act) {
                            const double tv = 1.0 / (double)mr;
                            mid::put(&M.ts[i], tv < 1.e30 ? tv : 1.e30, dist, cs);
                        }
                    }
                }
                if (sh.wpg > 1) {
                    __syncthreads();
                    const int t = tid;
                    if (t < sh.s1 - sh.s0) {
                        const int grp = t >> 5, l = t & 31;
                        const int i = M.mem[sh.s0 + t];
                        if (PREC == HHS_PREC_FP64) {
                            double mv = 1.e30;
                            for (int q = 0; q < sh.wpg; q++) {
                                const double v = M.red.pmin[grp * sh.wpg + q][l];
                                mv = v < mv ? v : mv;
                            }
                            mid::put(&M.ts[i], mv, dist, cs);
                        } else {
                            float mr = 0.0f;
                            for (int q = 0; q < sh.wpg; q++) mr = fmaxf(mr, M.red.pmax[grp * sh.wpg + q][l]);
                            const double tv = 1.0 / (double)mr;
                            mid::put(&M.ts[i], tv < 1.e30 ? tv : 1.e30, dist, cs);
                        }
                    }
                }
                if (dist) cl.sync();
                else __syncthreads();
                if (tid == 0) tpairs += (double)nm * (double)(nm - 1);
                }
            }
            mid_mark(E, sm, tm, 57);
            // ---- split: fast = members with ts <= dt, N_fast == 1 folded into the slow set
            int cnt = 0, mcnt = 0;
            for (int w = warp; w < nw; w += kEB / 32) {
                const unsigned mw = memw[w];
                const bool in = (mw >> lane) & 1u;
                const unsigned f = __ballot_sync(HHS_FULL_MASK, in && M.ts[w * 32 + lane] <= dt);
                if (lane == 0) M.fmask[d][w] = f;
                cnt += __popc(f);
                mcnt += __popc(mw);
            }
            if (tid >= nw && tid < kMidW) M.fmask[d][tid] = 0u;
            if (lane == 0) M.wcnt[warp] = cnt | (mcnt << 16);
            __syncthreads();
            int nf = 0, nm = 0;
#pragma unroll
            for (int w = 0; w < kEB / 32; w++) {
                nf += M.wcnt[w] & 0xffff;
                nm += M.wcnt[w] >> 16;
            }
            int lone = -1;
            if (nf == 1) {
                for (int w = 0; w < nw; w++)
                    if (M.fmask[d][w]) lone = w * 32 + __ffs(M.fmask[d][w]) - 1;
                nf = 0;
            }
            if (tid == 0) {
                M.lone[d] = lone;
                if (nf > 0) M.nmem[d + 1] = nf;
                if (rank == 0) trace_node(E, lvl, nm, nf, (calcm & bit) != 0);
                const double ns = (double)(nm - nf), nfd = (double)nf;
                nodes++;
                maxl = max(maxl, lvl);
                kpairs += ns * (ns - 1.0) + 2.0 * nfd * ns;
                if (nf == 0) leaf += dt;
            }
            __syncthreads();  // everyone has read fmask[d] before the fold clears it
            if (lone >= 0 && tid == 0) M.fmask[d][lone >> 5] = 0u;
            mid_mark(E, sm, tm, 58);
            after1 |= bit;
            if (nf > 0) {
                d++;
                const unsigned long long cb = 1ull << d;
                calcm &= ~cb; after1 &= ~cb; after2 &= ~cb;
                continue;
            }
            __syncthreads();
        }
        if (!(after2 & bit)) {
            mid_mark(E, sm, tm, -1);
            // ---- kick order: slow slots (stable, lone last), then fast slots
            int nf = 0;
            const int ns = mid::kick_order(memw, M.fmask[d], M.lone[d], nw, M.kl, M, &nf);
            const int nk = ns + nf;
            const double h = dt * 0.5;
            if (ns > 0) {
                // first half drift of the slow slots (src/hold.cuh:123-124), every replica
                for (int p = tid; p < ns; p += kEB) {
                    const int k = M.kl[p];
                    if (PREC == HHS_PREC_FP64) {
                        M.x[k] = f64_add(M.x[k], f64_mul(M.vx[k], h));
                        M.y[k] = f64_add(M.y[k], f64_mul(M.vy[k], h));
                        M.z[k] = f64_add(M.z[k], f64_mul(M.vz[k], h));
                    } else {
                        M.x[k] = fma(M.vx[k], h, M.x[k]);
                        M.y[k] = fma(M.vy[k], h, M.y[k]);
                        M.z[k] = fma(M.vz[k], h, M.z[k]);
                        mid::refresh_pos(M, k);
                    }
                }
                // ---- kicks (src/hold.cuh:138-143): slow sinks from slow + fast sources,
                // fast sinks from slow sources
                const bool dist = cs > 1 && nk > dist_n;
                if (dist) cl.sync();
                else __syncthreads();
                const mid::Share sh = mid::share_of(nk, dist, cs, rank);
                if (PREC == HHS_PREC_FP64) {
                    // one thread per sink, sources in the reference's order
                    for (int p = sh.s0 + tid; p < sh.s1; p += kEB) {
                        const int i = M.kl[p];
                        const bool slow = p < ns;
                        const double xi = M.x[i], yi = M.y[i], zi = M.z[i];
                        double aL[3] = {0, 0, 0}, aF[3] = {0, 0, 0};
#pragma unroll 1
                        for (int q = 0; q < ns; q++) {
                            const int j = M.kl[q];
                            kick_pair_fp64(f64_sub(M.x[j], xi), f64_sub(M.y[j], yi),
                                           f64_sub(M.z[j], zi), M.m[j], aL[0], aL[1], aL[2],
                                           E.eps2);
                        }
                        if (slow) {
#pragma unroll 1
                            for (int q = ns; q < nk; q++) {
                                const int j = M.kl[q];
                                kick_pair_fp64(f64_sub(M.x[j], xi), f64_sub(M.y[j], yi),
                                               f64_sub(M.z[j], zi), M.m[j], aF[0], aF[1],
                                               aF[2], E.eps2);
                            }
                        }
                        double vx = f64_add(M.vx[i], f64_mul(aL[0], dt));
                        double vy = f64_add(M.vy[i], f64_mul(aL[1], dt));
                        double vz = f64_add(M.vz[i], f64_mul(aL[2], dt));
                        if (slow && nf > 0) {
                            vx = f64_add(vx, f64_mul(aF[0], dt));
                            vy = f64_add(vy, f64_mul(aF[1], dt));
                            vz = f64_add(vz, f64_mul(aF[2], dt));
                        }
                        mid::put(&M.vx[i], vx, dist, cs);
                        mid::put(&M.vy[i], vy, dist, cs);
                        mid::put(&M.vz[i], vz, dist, cs);
                    }
                } else {
                    const int items = sh.ng * sh.wpg;
                    for (int it = warp; it < items; it += kEB / 32) {
                        const int grp = it / sh.wpg, part = it % sh.wpg;
                        const int p = sh.s0 + grp * 32 + lane;
                        const bool act = p < sh.s1;
                        const int i = act ? M.kl[p] : 0;
                        float a[3] = {0, 0, 0};
                        if (act) mid::acc_over(E, M, M.kl, part, p < ns ? nk : ns, sh.wpg, i, a);
                        if (sh.wpg > 1) {
                            M.red.part[it][0][lane] = a[0];
                            M.red.part[it][1][lane] = a[1];
                            M.red.part[it][2][lane] = a[2];
                        } else if (act) {
                            mid::put(&M.vx[i], fma((double)a[0], dt, M.vx[i]), dist, cs);
                            mid::put(&M.vy[i], fma((double)a[1], dt, M.vy[i]), dist, cs);
                            mid::put(&M.vz[i], fma((double)a[2], dt, M.vz[i]), dist, cs);
                        }
                    }
                    if (sh.wpg > 1) {
                        __syncthreads();
                        const int t = tid;
                        if (t < sh.s1 - sh.s0) {
                            const int grp = t >> 5, l = t & 31;
                            const int i = M.kl[sh.s0 + t];
                            double acc[3] = {0, 0, 0};
                            for (int q = 0; q < sh.wpg; q++)
#pragma unroll
                                for (int c = 0; c < 3; c++)
                                    acc[c] += (double)M.red.part[grp * sh.wpg + q][c][l];
                            mid::put(&M.vx[i], fma(acc[0], dt, M.vx[i]), dist, cs);
                            mid::put(&M.vy[i], fma(acc[1], dt, M.vy[i]), dist, cs);
                            mid::put(&M.vz[i], fma(acc[2], dt, M.vz[i]), dist, cs);
                        }
                    }
                }
                if (dist) cl.sync();
                else __syncthreads();
                // second half drift of the slow slots (src/hold.cuh:158-159), every replica
                for (int p = tid; p < nk; p += kEB) {
                    const int k = M.kl[p];
                    if (p < ns) {
                        if (PREC == HHS_PREC_FP64) {
                            M.x[k] = f64_add(M.x[k], f64_mul(M.vx[k], h));
                            M.y[k] = f64_add(M.y[k], f64_mul(M.vy[k], h));
                            M.z[k] = f64_add(M.z[k], f64_mul(M.vz[k], h));
                        } else {
                            M.x[k] = fma(M.vx[k], h, M.x[k]);
                            M.y[k] = fma(M.vy[k], h, M.y[k]);
                            M.z[k] = fma(M.vz[k], h, M.z[k]);
                            mid::refresh_pos(M, k);
                        }
                    }
                    if (PREC != HHS_PREC_FP64) mid::refresh_vel(M, k);
                }
                __syncthreads();
            }
            mid_mark(E, sm, tm, 59);
            after2 |= bit;
            if (nf > 0) {
                d++;
                const unsigned long long cb = 1ull << d;
                calcm = (calcm & ~cb) | cb;
                after1 &= ~cb; after2 &= ~cb;
                continue;
            }
        }
        calcm &= ~bit; after1 &= ~bit; after2 &= ~bit;
        d--;
    }
    mid_mark(E, sm, tm, -1);
    // write back this CTA's share of the slots; work counters once per subtree
    for (int k = rank + cs * tid; k < n; k += cs * kEB) {
        const int g = M.g[k];
        P.x[g] = M.x[k]; P.y[g] = M.y[k]; P.z[g] = M.z[k];
        P.vx[g] = M.vx[k]; P.vy[g] = M.vy[k]; P.vz[g] = M.vz[k];
        P.ts[g] = M.ts[k];
    }
    if (ok && rank == 0 && tid == 0 && nodes) {
        *E.leaf_time += leaf;
        atomicAdd(reinterpret_cast<unsigned long long*>(&E.stats->nodes), nodes);
        atomicMax(&E.stats->max_level, maxl);
        atomicAdd(&E.stats->kick_pairs, kpairs);
        atomicAdd(&E.stats->ts_pairs, tpairs);
    }
    if (cs > 1) cl.sync();
    else __syncthreads();
    mid_mark(E, sm, tm, 61);
}

// True when the kick of level lvl (a grid node with a fast set of at most mid_n) runs its
// slow-only units beside the fast set's first pass on the first cluster: mixed precision,
// packed sources at that level, and CTAs outside the first cluster.
__device__ __forceinline__ bool kick_overlaps(const EParams& E, int lvl, const Workers& W) {
    namespace cg = cooperative_groups;
    return W.mode == kModeGrid && E.overlap && E.pk && lvl < E.pk_levels && !E.packed &&
           E.prec_mixed && (int)cg::this_cluster().num_blocks() < W.count &&
           ld_volatile_i32(&E.counts[lvl].n_slow) > 0;
}

// ---------------------------------------------------------------- the recursion
// Walks the HOLD recursion from `top` (whose subsystem is already defined by the
// counts/lists above it). Grid and cluster modes delegate nodes with n <= small_n,
// with their whole subtree, to worker 0 alone.
template <int PREC, int MODE>
__device__ bool run_hold(const EParams& E, int top, bool top_calc, const Workers& W, Smem& sm,
                         unsigned long long& t_last) {
    unsigned long long after1 = 0, after2 = 0, calcm = 0;  // per-level state bits
    if (top_calc) calcm |= 1ull << top;
    int lvl = top;
    while (lvl >= top) {
        const unsigned long long bit = 1ull << lvl;
        const int n = (lvl == 0) ? E.n_top : ld_volatile_i32(&E.counts[lvl - 1].n_fast);
        const int32_t* S = (lvl == 0) ? nullptr : E.fast_lists + (size_t)(lvl - 1) * E.n_max;
        const double dt = dt_at(E, lvl);
        const bool calc = (calcm & bit) != 0;
        int32_t* F = E.fast_lists + (size_t)lvl * E.n_max;
        int32_t* L = E.slow_lists + (size_t)lvl * E.n_max;
        if (!(after1 & bit)) {
            if (lvl >= E.max_levels || lvl >= kMaxLevels - 1) {
                if (threadIdx.x == 0) atomicOr(E.err, HHS_ERRBIT_DEPTH);
                return false;
            }
            if (n <= E.mid_n && n <= kMid) {
                // the whole subtree from shared memory: on the grid's first cluster (or
                // CTA 0), on this hardware cluster, or on this CTA alone
                if constexpr (MODE == kModeGrid) {
                    namespace cg = cooperative_groups;
                    const int cs = (int)cg::this_cluster().num_blocks();
                    if ((int)blockIdx.x < cs) {
                        mid_hold<PREC>(E, S, n, lvl, calc, E.mid_dist_n, cs,
                                       (int)cg::this_cluster().block_rank(), sm);
                    } else if (!calc && lvl > top && kick_overlaps(E, lvl - 1, W)) {
                        // meanwhile the other CTAs run the parent's kick units that do not
                        // involve the fast set (this node), which mid_hold is advancing
                        const int pl = lvl - 1;
                        const int pnf = n, pns = ld_volatile_i32(&E.counts[pl].n_slow);
                        const KickPlan kp = kick_plan(pnf, pns, W.count);
                        kick_sym_units(E, E.fast_lists + (size_t)pl * E.n_max, pnf, pns, pl, kp, 1,
                                       1, sm);
                    }
                } else {
                    mid_hold<PREC>(E, S, n, lvl, calc, E.mid_dist_n, W.count, W.id, sm);
                }
                if (!phase_barrier(E, sm, W)) return false;
                prof_mark(E, W, t_last, kProfCluster, 0.0, sm, lvl);
                calcm &= ~bit; after1 &= ~bit; after2 &= ~bit;
                lvl--;
                continue;
            }
            if (n <= E.warp_n) {
                if (W.id == 0) tiny_hold<PREC>(E, S, n, lvl, calc, sm);
                if (!phase_barrier(E, sm, W)) return false;
                prof_mark(E, W, t_last, kProfSubtree, 0.0, sm, lvl);
                calcm &= ~bit; after1 &= ~bit; after2 &= ~bit;
                lvl--;
                continue;
            }
            if (MODE != kModeBlock && n <= E.small_n) {
                if (W.id == 0) {
                    const Workers one{0, 1, kModeBlock};
                    unsigned long long t_sub = 0;
                    run_hold<PREC, kModeBlock>(E, lvl, calc, one, sm, t_sub);
                }
                if (!phase_barrier(E, sm, W)) return false;
                prof_mark(E, W, t_last, kProfSubtree, 0.0, sm, lvl);
                calcm &= ~bit; after1 &= ~bit; after2 &= ~bit;
                lvl--;
                continue;
            }
            int nch = 1;
            if (calc) {
                if (PREC == HHS_PREC_FP64) {
                    nch = chunks_for(n, W, true, E.units_per_cta);
                    const int C = (n + nch - 1) / nch;
                    const int nsb = (n + kEB - 1) / kEB;
                    for (int u = W.id; u < nsb * nch; u += W.count) {
                        const int ib = u / nch, jc = u % nch;
                        const int j0 = jc * C, j1 = min(n, j0 + C);
                        ts_unit<PREC>(E, S, n, ib, j0, j1, E.ts_part + (size_t)jc * E.n_max,
                                      nullptr, sm);
                    }
                } else if (MODE == kModeGrid && E.tq) {
                    // packed members: written by the parent's kick-reduce phase when it
                    // ran (the second pass of a fast set), else packed here
                    if (lvl == top || ld_volatile_i32(&E.counts[lvl - 1].n_slow) == 0) {
                        pack_ts(E, S, n, W);
                        if (!phase_barrier(E, sm, W)) return false;
                    }
                    const int cw = ts_tile_width(n, W.count);
                    const long long units = ts_tile_units(n, cw);
                    ts_sym_tiles(E, n, cw, units * W.id / W.count, units * (W.id + 1) / W.count,
                                 sm);
                } else {
                    // only units with a pair j > i: row block rb takes column blocks
                    // cb >= rb * kEB / kCB; each worker takes a contiguous range of that
                    // triangle in row-major order
                    const long long units = ts_sym_units(n);
                    const int u0 = (int)(units * W.id / W.count);
                    const int u1 = (int)(units * (W.id + 1) / W.count);
                    ts_sym_range(E, S, n, u0, u1, sm);
                }
                if (!phase_barrier(E, sm, W)) return false;
                prof_mark(E, W, t_last, kProfTs, (double)n * (double)(n - 1), sm, lvl);
            }
            if constexpr (MODE == kModeGrid) {
                split_phase<PREC>(E, S, n, dt, lvl, calc, nch, W, sm);
            } else {
                count_phase<PREC>(E, S, n, dt, calc, nch, W, sm);
                if (!phase_barrier(E, sm, W)) return false;
                scatter_phase(E, S, n, dt, lvl, calc, W, sm);
            }
            if (!phase_barrier(E, sm, W)) return false;
            prof_mark(E, W, t_last, kProfSplit, 0.0, sm, lvl);
            after1 |= bit;
            const int nf = ld_volatile_i32(&E.counts[lvl].n_fast);
            if (nf > 0) {
                lvl++;
                const unsigned long long cb = 1ull << lvl;
                calcm &= ~cb; after1 &= ~cb; after2 &= ~cb;
                continue;
            }
        }
        if (!(after2 & bit)) {
            const int nf = ld_volatile_i32(&E.counts[lvl].n_fast);
            const int ns = ld_volatile_i32(&E.counts[lvl].n_slow);
            if (ns > 0) {
                const int ntot = nf + ns;
                const bool grid_tma = MODE == kModeGrid && PREC != HHS_PREC_FP64 && !E.packed &&
                                      E.pk && lvl < E.pk_levels;
                const bool x2 = PREC != HHS_PREC_FP64 && E.packed;
                const int blk = (x2 || grid_tma) ? 2 * kEB : kEB;
                const int nch = chunks_for(ntot, W, PREC != HHS_PREC_FP64, E.units_per_cta, blk);
                const int C = (ntot + nch - 1) / nch;
                const int nsb = (ntot + blk - 1) / blk;
                const double h = dt * 0.5;
                // blocks of fast sinks only need the slow-source chunks: the work units
                // are the first nfb blocks x jcs chunks, then the other blocks x nch
                const int nfb = nf / blk;
                const int jcs = min(nch, (ns + C - 1) / C);
                const int uf = nfb * jcs;
                const int units = grid_tma ? 0 : uf + (nsb - nfb) * nch;
                KickPlan kp{};
                if (grid_tma) {
                    // the slow units already ran beside the fast set's first pass when that
                    // pass was a subtree on the first cluster
                    const bool overlapped = nf > 0 && nf <= E.mid_n && nf <= kMid &&
                                            kick_overlaps(E, lvl, W);
                    kp = kick_plan(nf, ns, W.count);
                    kick_sym_units(E, F, nf, ns, lvl, kp, 0, overlapped ? 2 : 0, sm);
                }
                for (int u = W.id; u < units; u += W.count) {
                    int ib, jc;
                    if (u < uf) {
                        ib = u / jcs;
                        jc = u % jcs;
                    } else {
                        ib = nfb + (u - uf) / nch;
                        jc = (u - uf) % nch;
                    }
                    const int j0 = jc * C, j1 = min(ntot, j0 + C);
                    if (x2) kick_unit_x2(E, F, L, nf, ns, h, ib, jc, j0, j1, sm);
                    else kick_unit<PREC>(E, F, L, nf, ns, h, ib, jc, j0, j1, sm);
                }
                if (!phase_barrier(E, sm, W)) return false;
                const double ns_d = ns, nf_d = nf;
                prof_mark(E, W, t_last, kProfKick, ns_d * (ns_d - 1.0) + 2.0 * ns_d * nf_d, sm, lvl);
                if (grid_tma) kick_reduce_phase<PREC>(E, F, L, nf, ns, dt, kp.ncs, 0, W, sm, kp.nfsb);
                else kick_reduce_phase<PREC>(E, F, L, nf, ns, dt, nch, C, W, sm);
                if (!phase_barrier(E, sm, W)) return false;
                prof_mark(E, W, t_last, kProfUpdate, 0.0, sm, lvl);
            }
            after2 |= bit;
            if (nf > 0) {
                lvl++;
                const unsigned long long cb = 1ull << lvl;
                calcm = (calcm & ~cb) | cb;
                after1 &= ~cb; after2 &= ~cb;
                continue;
            }
        }
        calcm &= ~bit; after1 &= ~bit; after2 &= ~bit;
        lvl--;
    }
    return true;
}

template <int PREC>
__global__ void __launch_bounds__(kEB, 2) k_engine(EParams E) {
    extern __shared__ __align__(16) unsigned char engine_smem[];
    Smem& sm = *reinterpret_cast<Smem*>(engine_smem);
    const Workers W{(int)blockIdx.x, (int)gridDim.x, kModeGrid};
    if (threadIdx.x == 0) {
        sm.bar_k = 0u;  // thread 0 alone uses it
        sm.kphase = 0u;
        sm.tphase = 0u;
        mbar_init(&sm.kbar, 1u);
        mbar_init(&sm.tbar[0], 1u);
        mbar_init(&sm.tbar[1], 1u);
        fence_barrier_init();
    }
    __syncthreads();
    unsigned long long t_last = 0;
    prof_begin(E, sm);
    prof_mark(E, W, t_last, -1, 0.0, sm);
    run_hold<PREC, kModeGrid>(E, E.top_level, E.calc_top != 0, W, sm, t_last);
    prof_end(E, sm);
}

// Probe of the mixed grid kick: the system as one split node whose fast set is every
// third particle (index % 3 == 0) and whose slow set is the rest, with no drift. The
// level's slow records are packed, the symmetric kick runs its units, and the reduce
// phase's sums give each particle's acceleration (fast: from the slow set; slow: from
// all others), written to E.ts_part / rate_acc / tile_counts reinterpreted as FP64
// ax / ay / az (see engine_kick_accelerations).
__global__ void __launch_bounds__(kEB, 2) k_engine_accel(EParams E) {
    extern __shared__ __align__(16) unsigned char engine_smem[];
    Smem& sm = *reinterpret_cast<Smem*>(engine_smem);
    const Workers W{(int)blockIdx.x, (int)gridDim.x, kModeGrid};
    if (threadIdx.x == 0) {
        sm.bar_k = 0u;
        sm.kphase = 0u;
        sm.tphase = 0u;
        mbar_init(&sm.kbar, 1u);
        mbar_init(&sm.tbar[0], 1u);
        mbar_init(&sm.tbar[1], 1u);
        fence_barrier_init();
    }
    __syncthreads();
    const int n = E.n_top;
    const int nf = (n + 2) / 3, ns = n - nf;
    int32_t* F = E.fast_lists;
    int32_t* L = E.slow_lists;
    for (int i = W.id * kEB + (int)threadIdx.x; i < n; i += W.count * kEB) {
        if (i % 3 == 0) {
            F[i / 3] = i;
        } else {
            const int q = (i / 3) * 2 + (i % 3) - 1;
            L[q] = i;
            const DS x = ds_split(E.P.x[i]), y = ds_split(E.P.y[i]), z = ds_split(E.P.z[i]);
            pk_put(E.pk, q, x, y, z, (float)E.P.m[i]);
        }
    }
    if (W.id == 0 && threadIdx.x == 0) E.st->kick_ctr[0][0] = 0u;
    if (!grid_barrier(E, sm)) return;
    const KickPlan kp = kick_plan(nf, ns, W.count);
    kick_sym_units(E, F, nf, ns, 0, kp, 0, 0, sm);
    if (!grid_barrier(E, sm)) return;
    double* out[3] = {E.ts_part, reinterpret_cast<double*>(E.rate_acc),
                      reinterpret_cast<double*>(E.tile_counts)};
    for (int s = W.id * kEB + (int)threadIdx.x; s < n; s += W.count * kEB)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double a = 0.0;
            for (int c = 0; c < kp.ncs; c++) a += E.k_part[(size_t)(c * 3 + k) * E.n_max + s];
            if (s >= nf)
                for (int f = 0; f < kp.nfsb; f++)
                    a += E.c_part[(size_t)(f * 3 + k) * E.n_max + s];
            out[k][s >= nf ? L[s - nf] : F[s]] = a;
        }
}

// Probe of the mixed grid timestep: the first n particles as one node whose timesteps
// are computed by the packed symmetric tile phase of k_engine (members packed, column
// tiles bulk-copied, one rate per unordered pair, row and column maxima), then converted
// to timesteps as the split phase does, into P.ts (see engine_timestep_rates).
__global__ void __launch_bounds__(kEB, 2) k_engine_ts(EParams E) {
    extern __shared__ __align__(16) unsigned char engine_smem[];
    Smem& sm = *reinterpret_cast<Smem*>(engine_smem);
    const Workers W{(int)blockIdx.x, (int)gridDim.x, kModeGrid};
    if (threadIdx.x == 0) {
        sm.bar_k = 0u;
        sm.kphase = 0u;
        sm.tphase = 0u;
        mbar_init(&sm.kbar, 1u);
        mbar_init(&sm.tbar[0], 1u);
        mbar_init(&sm.tbar[1], 1u);
        fence_barrier_init();
    }
    __syncthreads();
    const int n = E.n_top;
    pack_ts(E, nullptr, n, W);
    if (!grid_barrier(E, sm)) return;
    const int cw = ts_tile_width(n, W.count);
    const long long units = ts_tile_units(n, cw);
    ts_sym_tiles(E, n, cw, units * W.id / W.count, units * (W.id + 1) / W.count, sm);
    if (!grid_barrier(E, sm)) return;
    for (int i = W.id * kEB + (int)threadIdx.x; i < n; i += W.count * kEB) {
        const float mr = __uint_as_float(E.rate_acc[i]);
        E.rate_acc[i] = 0u;
        const double tv = 1.0 / (double)mr;
        E.P.ts[i] = tv < 1.e30 ? tv : 1.e30;
    }
}

// ---------------------------------------------------------------- sharded phases
// The engine's tiled timestep and kick phases over one rank's share of a level, for the
// multi-GPU step (hhs_hold_step_dist): ordinary launches whose CTAs split the rank's
// share; every result also goes into each peer replica (atomic maxima of pair rates,
// stored velocities and timesteps over NVLink). No kernel waits on another rank: the
// host's barrier brackets each launch.
__device__ __forceinline__ void kick_smem_init(Smem& sm) {
    if (threadIdx.x == 0) {
        sm.kphase = 0u;
        mbar_init(&sm.kbar, 1u);
        fence_barrier_init();
    }
    __syncthreads();
}

// Mixed timestep: units [u_lo, u_hi) of the level's symmetric triangle, row and column
// maxima into the local rate words (E.rate_acc) and each peer's.
__global__ void __launch_bounds__(kEB, 2)
    k_shard_ts_mixed(EParams E, const int32_t* S, int n, long long u_lo, long long u_hi,
                     PeerOut po) {
    extern __shared__ __align__(16) unsigned char engine_smem[];
    Smem& sm = *reinterpret_cast<Smem*>(engine_smem);
    const long long span = u_hi - u_lo;
    const int u0 = (int)(u_lo + span * blockIdx.x / gridDim.x);
    const int u1 = (int)(u_lo + span * (blockIdx.x + 1) / gridDim.x);
    ts_sym_range(E, S, n, u0, u1, sm, &po);
    if (po.n_peer > 0) __threadfence_system();
}

// Rate words -> timesteps of the level's members (every rank, after the barrier), the
// conversion of the engine's split phase.
__global__ void k_rates_to_ts(EParams E, const int32_t* S, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float mr = __uint_as_float(E.rate_acc[i]);
        const double tv = 1.0 / (double)mr;
        E.P.ts[list_at(S, i)] = tv < 1.e30 ? tv : 1.e30;
    }
}

// FP64 timestep: sink blocks [ib_lo, ib_hi) x nch source chunks, partial minima per chunk
// in ts_part; then the minimum of each sink of [s_lo, s_hi) to every replica.
__global__ void __launch_bounds__(kEB, 2)
    k_shard_ts_fp64(EParams E, const int32_t* S, int n, int ib_lo, int ib_hi, int nch) {
    extern __shared__ __align__(16) unsigned char engine_smem[];
    Smem& sm = *reinterpret_cast<Smem*>(engine_smem);
    const int C = (n + nch - 1) / nch;
    const int units = (ib_hi - ib_lo) * nch;
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        const int ib = ib_lo + u / nch, jc = u % nch;
        const int j0 = jc * C, j1 = min(n, j0 + C);
        ts_unit<HHS_PREC_FP64>(E, S, n, ib, j0, j1, E.ts_part + (size_t)jc * E.n_max, nullptr, sm);
    }
}

__global__ void k_shard_ts_fp64_reduce(EParams E, const int32_t* S, int s_lo, int s_hi, int nch,
                                       PeerOut po) {
    for (int i = s_lo + blockIdx.x * blockDim.x + threadIdx.x; i < s_hi;
         i += gridDim.x * blockDim.x) {
        double mv = 1.e30;
        for (int c = 0; c < nch; c++) {
            const double v = E.ts_part[(size_t)c * E.n_max + i];
            if (v < mv) mv = v;
        }
        const int g = list_at(S, i);
        E.P.ts[g] = mv;
        for (int r = 0; r < po.n_peer; r++) po.ts[r][g] = mv;
    }
    if (po.n_peer > 0) __threadfence_system();
}

// Slow sources of a level at their current (already drifted) positions, packed for the
// mixed kick's bulk copies (every rank).
__global__ void k_pack_slow(EParams E, const int32_t* L, int ns, int lvl) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ns; q += gridDim.x * blockDim.x) {
        const int g = L[q];
        const DS x = ds_split(E.P.x[g]), y = ds_split(E.P.y[g]), z = ds_split(E.P.z[g]);
        pk_put(pk_level(E, lvl), q, x, y, z, (float)E.P.m[g]);
    }
}

// Mixed kick units of sink blocks [ib_lo, ib_hi) (kKB sinks each), partials in k_part.
__global__ void __launch_bounds__(kEB, 2)
    k_shard_kick_mixed(EParams E, const int32_t* F, int nf, int ns, int lvl, int nch, int C,
                       int ib_lo, int ib_hi) {
    extern __shared__ __align__(16) unsigned char engine_smem[];
    Smem& sm = *reinterpret_cast<Smem*>(engine_smem);
    kick_smem_init(sm);
    const Workers W{(int)blockIdx.x, (int)gridDim.x, kModeGrid};
    kick_units_grid(E, F, nf, ns, lvl, nch, C, W, sm, ib_lo, ib_hi);
}

// FP64 kick units of sink blocks [ib_lo, ib_hi) (kEB sinks each), one chunk: slow then
// fast sources in list order, the reference's order.
__global__ void __launch_bounds__(kEB, 2)
    k_shard_kick_fp64(EParams E, const int32_t* F, const int32_t* L, int nf, int ns, int ib_lo,
                      int ib_hi) {
    extern __shared__ __align__(16) unsigned char engine_smem[];
    Smem& sm = *reinterpret_cast<Smem*>(engine_smem);
    for (int ib = ib_lo + (int)blockIdx.x; ib < ib_hi; ib += gridDim.x)
        kick_unit<HHS_PREC_FP64>(E, F, L, nf, ns, 0.0, ib, 0, 0, nf + ns, sm);
}

// v += a*dt for sinks [s_lo, s_hi) from the per-chunk partials (the kick-reduce phase's
// sums, without its drifts), stored locally and into every peer replica.
template <int PREC>
__global__ void k_shard_kick_reduce(EParams E, const int32_t* F, const int32_t* L, int nf,
                                    int ns, double dt, int nch, int C, int s_lo, int s_hi,
                                    PeerOut po) {
    const SoA& P = E.P;
    const int lastf = min(nch, (ns + C - 1) / C);
    for (int s = s_lo + blockIdx.x * blockDim.x + threadIdx.x; s < s_hi;
         s += gridDim.x * blockDim.x) {
        const bool slow = s >= nf;
        const int g = slow ? L[s - nf] : F[s];
        const double v0[3] = {P.vx[g], P.vy[g], P.vz[g]};
        double v1[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            if (PREC == HHS_PREC_FP64) {
                double v = f64_add(v0[k], f64_mul(E.k_part[(size_t)k * E.n_max + s], dt));
                if (slow && nf > 0)
                    v = f64_add(v, f64_mul(E.k_part[(size_t)(3 + k) * E.n_max + s], dt));
                v1[k] = v;
            } else {
                const int last = slow ? nch : lastf;
                double a = 0.0;
                for (int c = 0; c < last; c++) a += E.k_part[(size_t)(c * 3 + k) * E.n_max + s];
                v1[k] = fma(a, dt, v0[k]);
            }
        }
        P.vx[g] = v1[0]; P.vy[g] = v1[1]; P.vz[g] = v1[2];
        for (int r = 0; r < po.n_peer; r++) {
            po.vx[r][g] = v1[0]; po.vy[r][g] = v1[1]; po.vz[r][g] = v1[2];
        }
    }
    if (po.n_peer > 0) __threadfence_system();
}

// ---------------------------------------------------------------- batched systems
// Many independent systems packed back to back: the hardware clusters of the launch
// first take the large systems from a queue ordered by decreasing size (each cluster
// runs one system at a time with cluster barriers between phases), then every CTA takes
// the remaining small systems one by one and solves each alone. Each worker group owns
// a scratch slot (level lists, counts, partial sums) for the system it is running.
struct Slot {
    int32_t* fast_lists;
    int32_t* slow_lists;
    hhs_partition* counts;
    double* ts_part;
    double* k_part;
    int* tile_counts;
    unsigned* rate_acc;
};

struct BParams {
    EParams E;               // common fields; per-system fields are filled in per system
    const int32_t* offsets;  // [n_sys + 1]
    const int32_t* order;    // systems by decreasing size
    int n_sys, n_big;
    unsigned* queues;        // [0] big-system queue, [1] small-system queue, [2 + c] broadcast
    char* cluster_slots;
    char* cta_slots;
    size_t cluster_slot_bytes, cta_slot_bytes;
    size_t off_lists, off_counts, off_ts, off_k, off_tiles, off_rate;
    double* leaf_times;      // [n_sys]
};

__device__ __forceinline__ EParams system_params(const BParams& B, int sys, const char* slot) {
    EParams E = B.E;
    const int o = B.offsets[sys];
    E.P.x += o; E.P.y += o; E.P.z += o;
    E.P.vx += o; E.P.vy += o; E.P.vz += o;
    E.P.m += o; E.P.ts += o; E.P.id += o;
    E.n_top = B.offsets[sys + 1] - o;
    char* p = const_cast<char*>(slot);
    const size_t lists = (size_t)E.max_levels * E.n_max;
    E.fast_lists = reinterpret_cast<int32_t*>(p + B.off_lists);
    E.slow_lists = E.fast_lists + lists;
    E.counts = reinterpret_cast<hhs_partition*>(p + B.off_counts);
    E.ts_part = reinterpret_cast<double*>(p + B.off_ts);
    E.k_part = reinterpret_cast<double*>(p + B.off_k);
    E.tile_counts = reinterpret_cast<int*>(p + B.off_tiles);
    E.rate_acc = reinterpret_cast<unsigned*>(p + B.off_rate);
    E.leaf_time = B.leaf_times + sys;
    return E;
}

template <int PREC>
__global__ void __launch_bounds__(kEB, 2) k_batched(BParams B) {
    extern __shared__ __align__(16) unsigned char batched_smem[];
    Smem& sm = *reinterpret_cast<Smem*>(batched_smem);
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int cs = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int cid = (int)(blockIdx.x / cs);
    unsigned long long t = 0;
    // large systems: one hardware cluster per system
    while (true) {
        if (rank == 0 && threadIdx.x == 0)
            *reinterpret_cast<volatile unsigned*>(&B.queues[2 + cid]) = atomicAdd(&B.queues[0], 1u);
        cluster.sync();
        const int idx = (int)*reinterpret_cast<volatile unsigned*>(&B.queues[2 + cid]);
        cluster.sync();
        if (idx >= B.n_big) break;
        const int sys = B.order[idx];
        const EParams E = system_params(B, sys, B.cluster_slots + (size_t)cid * B.cluster_slot_bytes);
        const Workers W{rank, cs, kModeCluster};
        run_hold<PREC, kModeCluster>(E, 0, E.calc_top != 0, W, sm, t);
    }
    // small systems: one CTA per system
    while (true) {
        if (threadIdx.x == 0) sm.bcast = (int)atomicAdd(&B.queues[1], 1u);
        __syncthreads();
        const int idx = sm.bcast;
        __syncthreads();
        if (idx >= B.n_sys - B.n_big) break;
        const int sys = B.order[B.n_big + idx];
        const EParams E = system_params(B, sys, B.cta_slots + (size_t)blockIdx.x * B.cta_slot_bytes);
        const Workers W{0, 1, kModeBlock};
        run_hold<PREC, kModeBlock>(E, 0, E.calc_top != 0, W, sm, t);
    }
}

struct EngineHost {
    int grid[2] = {0, 0};
    int sms = 0, occ[2] = {0, 0};
    int ctas_per_sm = 2;
    int small_n = 64;
    int units_per_cta = 16;
    int warp_n = 32;
    int cluster_size = 4;
    int mid_n = 640;
    int mid_dist_n = 96;
    int packed = 0;
    int overlap = 1;
    EngineState* st = nullptr;
    double* ts_part = nullptr;
    double* k_part = nullptr;
    int* tile_counts = nullptr;
    unsigned* rate_acc = nullptr;
    unsigned long long* tile_status = nullptr;
    int n_max = 0;
    float4* pk = nullptr;
    long long pk_stride = 0;
    int pk_levels = 0;
    double* c_part = nullptr;
    float4* tq = nullptr;
    long long tq_stride = 0;
    int32_t* trace = nullptr;                 // caller's node-record buffer (4 int32 each)
    unsigned long long* trace_count = nullptr;
    long long trace_cap = 0;
};

constexpr size_t kAl = 256;
inline size_t al(size_t v) { return (v + kAl - 1) & ~(kAl - 1); }

}  // namespace

// levels with packed kick sources (deeper levels, if they run grid phases at all, gather)
constexpr int kPkLevels = 24;
inline int pk_levels_for(int max_levels) { return max_levels < kPkLevels ? max_levels : kPkLevels; }

size_t engine_workspace_bytes(int n_max, int max_levels) {
    const size_t n = (size_t)n_max;
    return al(sizeof(EngineState)) + al(sizeof(double) * kMaxChunks * n) +
           al(sizeof(double) * kMaxChunks * 3 * n) + al(sizeof(int) * (n / kEB + 2)) +
           al(sizeof(unsigned) * n) + al(sizeof(unsigned long long) * (n / kEB + 2)) +
           al(sizeof(float4) * 4 * (n / 2 + 1) * (size_t)pk_levels_for(max_levels)) +
           al(sizeof(double) * kMaxFsb * 3 * n) + al(sizeof(float4) * 5 * (n / 2 + 1));
}

hhs_status engine_init(hhs_ctx* c, void* base) {
    auto* eh = new (std::nothrow) EngineHost();
    if (!eh) return HHS_ERR_OOM;
    char* p = static_cast<char*>(base);
    const size_t n = (size_t)c->n_max;
    eh->st = reinterpret_cast<EngineState*>(p); p += al(sizeof(EngineState));
    eh->ts_part = reinterpret_cast<double*>(p); p += al(sizeof(double) * kMaxChunks * n);
    eh->k_part = reinterpret_cast<double*>(p); p += al(sizeof(double) * kMaxChunks * 3 * n);
    eh->tile_counts = reinterpret_cast<int*>(p); p += al(sizeof(int) * (n / kEB + 2));
    eh->rate_acc = reinterpret_cast<unsigned*>(p); p += al(sizeof(unsigned) * n);
    eh->tile_status = reinterpret_cast<unsigned long long*>(p);
    p += al(sizeof(unsigned long long) * (n / kEB + 2));
    eh->pk_levels = pk_levels_for(c->max_levels);
    eh->pk_stride = (long long)(n / 2 + 1);
    eh->pk = reinterpret_cast<float4*>(p);
    p += al(sizeof(float4) * 4 * (size_t)eh->pk_stride * (size_t)eh->pk_levels);
    eh->c_part = reinterpret_cast<double*>(p); p += al(sizeof(double) * kMaxFsb * 3 * n);
    eh->tq = reinterpret_cast<float4*>(p);
    eh->tq_stride = (long long)(n / 2 + 1);
    eh->n_max = c->n_max;
    int dev = 0, sms = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) { delete eh; return HHS_ERR_CUDA; }
    int b0 = 0, b1 = 0;
    HHS_CUDA_TRY(cudaFuncSetAttribute(k_engine<HHS_PREC_FP64>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEngineSmem));
    HHS_CUDA_TRY(cudaFuncSetAttribute(k_engine<HHS_PREC_MIXED>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEngineSmem));
    HHS_CUDA_TRY(cudaFuncSetAttribute(k_engine_accel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kEngineSmem));
    HHS_CUDA_TRY(cudaFuncSetAttribute(k_engine_ts, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kEngineSmem));
    // clusters of 16 CTAs (beyond the portable 8) for the subtree solver, where allowed
    if (cudaFuncSetAttribute(k_engine<HHS_PREC_FP64>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_engine<HHS_PREC_MIXED>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_engine_accel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_engine_ts, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess)
        (void)cudaGetLastError();  // cluster size 16 then fails its occupancy check
    HHS_CUDA_TRY(cudaFuncSetAttribute(k_shard_ts_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kEngineSmem));
    HHS_CUDA_TRY(cudaFuncSetAttribute(k_shard_ts_fp64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kEngineSmem));
    HHS_CUDA_TRY(cudaFuncSetAttribute(k_shard_kick_mixed,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEngineSmem));
    HHS_CUDA_TRY(cudaFuncSetAttribute(k_shard_kick_fp64,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEngineSmem));
    HHS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_engine<HHS_PREC_FP64>, kEB,
                                                               kEngineSmem));
    HHS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_engine<HHS_PREC_MIXED>, kEB,
                                                               kEngineSmem));
    eh->sms = sms;
    eh->occ[0] = b0;
    eh->occ[1] = b1;
    eh->grid[0] = sms * (b0 < 2 ? b0 : 2);
    eh->grid[1] = sms * (b1 < 2 ? b1 : 2);
    if (eh->grid[0] <= 0 || eh->grid[1] <= 0) { delete eh; return HHS_ERR_CUDA; }
    c->engine_host = eh;
    // size the grid for the default tuning (thread-block clusters included); without
    // cluster occupancy fall back to plain CTAs
    hhs_tuning t{};
    engine_get_tuning(c, &t);
    if (engine_set_tuning(c, t) != HHS_OK) {
        t.cluster_size = 1;
        if (engine_set_tuning(c, t) != HHS_OK) { engine_destroy(c); return HHS_ERR_CUDA; }
    }
    return HHS_OK;
}

void engine_destroy(hhs_ctx* c) {
    delete static_cast<EngineHost*>(c->engine_host);
    c->engine_host = nullptr;
}

hhs_status engine_set_tuning(hhs_ctx* c, const hhs_tuning& t) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh || t.small_n < 0 || t.units_per_cta < 1 || t.units_per_cta > 64 ||
        t.ctas_per_sm < 1 || t.ctas_per_sm > 2 || t.warp_n < 0 || t.warp_n > 32 ||
        !(t.cluster_size == 1 || t.cluster_size == 2 || t.cluster_size == 4 ||
          t.cluster_size == 8 || t.cluster_size == 16) || t.mid_n < 0 || t.mid_dist_n < 0)
        return HHS_ERR_INVALID_ARG;
    eh->warp_n = t.warp_n;
    eh->cluster_size = t.cluster_size;
    eh->mid_n = t.mid_n;
    eh->mid_dist_n = t.mid_dist_n;
    eh->packed = t.packed != 0;
    eh->overlap = t.overlap != 0;
    eh->small_n = t.small_n;
    eh->units_per_cta = t.units_per_cta;
    eh->ctas_per_sm = t.ctas_per_sm;
    for (int k = 0; k < 2; k++) {
        int g = eh->sms * (eh->occ[k] < t.ctas_per_sm ? eh->occ[k] : t.ctas_per_sm);
        if (t.cluster_size > 1) {
            int nc = 0;
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(t.cluster_size, 1, 1);
            cfg.blockDim = dim3(kEB, 1, 1);
            cfg.dynamicSmemBytes = kEngineSmem;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = t.cluster_size;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            const cudaError_t e =
                k == 0 ? cudaOccupancyMaxActiveClusters(&nc, (void*)k_engine<HHS_PREC_FP64>, &cfg)
                       : cudaOccupancyMaxActiveClusters(&nc, (void*)k_engine<HHS_PREC_MIXED>, &cfg);
            if (e != cudaSuccess || nc <= 0) return HHS_ERR_CUDA;
            const int gc = nc * t.cluster_size;
            g = (g < gc ? g : gc) / t.cluster_size * t.cluster_size;
        }
        eh->grid[k] = g;
    }
    return HHS_OK;
}

hhs_status engine_get_launch(hhs_ctx* c, int32_t* grid, int32_t* smem_bytes) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh) return HHS_ERR_INVALID_ARG;
    if (grid) { grid[0] = eh->grid[0]; grid[1] = eh->grid[1]; }
    if (smem_bytes) *smem_bytes = (int32_t)kEngineSmem;
    return HHS_OK;
}

hhs_status engine_get_tuning(hhs_ctx* c, hhs_tuning* t) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh || !t) return HHS_ERR_INVALID_ARG;
    t->small_n = eh->small_n;
    t->units_per_cta = eh->units_per_cta;
    t->ctas_per_sm = eh->ctas_per_sm;
    t->warp_n = eh->warp_n;
    t->cluster_size = eh->cluster_size;
    t->mid_n = eh->mid_n;
    t->mid_dist_n = eh->mid_dist_n;
    t->packed = eh->packed;
    t->overlap = eh->overlap;
    return HHS_OK;
}

hhs_status engine_get_level_profile(hhs_ctx* c, double* ms, uint64_t* counts) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh) return HHS_ERR_INVALID_ARG;
    EngineState h;
    HHS_CUDA_TRY(cudaMemcpy(&h, eh->st, sizeof(h), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 8; k++)
        for (int l = 0; l < kMaxLevels; l++) {
            if (ms) ms[k * kMaxLevels + l] = (double)h.lvl_ns[k][l] * 1e-6;
            if (counts) counts[k * kMaxLevels + l] = h.lvl_cnt[k][l];
        }
    return HHS_OK;
}

hhs_status engine_get_profile(hhs_ctx* c, hhs_profile* out, bool reset) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh) return HHS_ERR_INVALID_ARG;
    EngineState h;
    HHS_CUDA_TRY(cudaMemcpy(&h, eh->st, sizeof(h), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 8; k++) {
        out->launches[k] += h.prof_cnt[k];
        out->ms[k] += (double)h.prof_ns[k] * 1e-6;
        out->pairs[k] += h.prof_pairs[k];
    }
    if (reset) {
        HHS_CUDA_TRY(cudaMemset(reinterpret_cast<char*>(eh->st) + offsetof(EngineState, prof_ns),
                                0, sizeof(EngineState) - offsetof(EngineState, prof_ns)));
    }
    return HHS_OK;
}

hhs_status engine_set_trace(hhs_ctx* c, int32_t* nodes, int64_t capacity,
                            unsigned long long* count) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh) return HHS_ERR_INVALID_ARG;
    if ((nodes == nullptr) != (count == nullptr) || capacity < 0 ||
        (nodes && (reinterpret_cast<uintptr_t>(nodes) & 15u)))
        return HHS_ERR_INVALID_ARG;
    eh->trace = nodes;
    eh->trace_count = count;
    eh->trace_cap = nodes ? capacity : 0;
    return HHS_OK;
}

hhs_status engine_reset_barrier(hhs_ctx* c, cudaStream_t stream) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh) return HHS_ERR_INVALID_ARG;
    HHS_CUDA_TRY(cudaMemsetAsync(eh->st, 0, 2 * sizeof(unsigned), stream));
    HHS_CUDA_TRY(cudaMemsetAsync(eh->rate_acc, 0, sizeof(unsigned) * (size_t)eh->n_max, stream));
    return HHS_OK;
}

namespace {
EParams engine_params(hhs_ctx* c, EngineHost* eh, const SoA& P, int n, double dt, bool calc_ts,
                      bool profile, int top_level) {
    EParams E;
    E.P = P;
    E.top_level = top_level;
    E.n_top = n;
    E.n_max = c->n_max;
    E.max_levels = c->max_levels < kMaxLevels - 1 ? c->max_levels : kMaxLevels - 1;
    E.small_n = eh->small_n;
    E.units_per_cta = eh->units_per_cta;
    E.warp_n = eh->warp_n;
    E.mid_n = eh->mid_n;
    E.mid_dist_n = eh->mid_dist_n;
    E.packed = eh->packed;
    E.calc_top = calc_ts ? 1 : 0;
    E.profile = profile ? 1 : 0;
    E.dt_top = dt;
    E.eta = c->params.eta;
    E.eps2 = c->params.eps * c->params.eps;
    E.eps2f = (float)E.eps2;
    E.eta_s2 = c->params.eta / 1.41421356237309504880;
    E.inv_eta_s2 = (float)(1.0 / E.eta_s2);
    E.inv_eta = (float)(1.0 / E.eta);
    E.fast_lists = c->fast_lists;
    E.slow_lists = c->slow_lists;
    E.counts = c->counts;
    E.leaf_time = c->leaf_time;
    E.stats = c->stats;
    E.ts_part = eh->ts_part;
    E.k_part = eh->k_part;
    E.c_part = eh->c_part;
    E.tq = eh->tq;
    E.tq_stride = eh->tq_stride;
    E.tile_counts = eh->tile_counts;
    E.tile_status = eh->tile_status;
    E.rate_acc = eh->rate_acc;
    E.st = eh->st;
    E.err = c->err;
    E.pk = eh->pk;
    E.pk_stride = eh->pk_stride;
    E.pk_levels = eh->pk_levels;
    E.prec_mixed = 0;
    E.overlap = eh->overlap;
    E.trace = reinterpret_cast<int4*>(eh->trace);
    E.trace_count = eh->trace_count;
    E.trace_cap = eh->trace_cap;
    return E;
}

// Cooperative launch of a persistent engine kernel in the context's launch shape.
template <class K>
cudaError_t engine_launch(EngineHost* eh, int pi, K kernel, const EParams& E, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(eh->grid[pi], 1, 1);
    cfg.blockDim = dim3(kEB, 1, 1);
    cfg.dynamicSmemBytes = kEngineSmem;
    cfg.stream = stream;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (eh->cluster_size > 1) {
        at[1].id = cudaLaunchAttributeClusterDimension;
        at[1].val.clusterDim.x = eh->cluster_size;
        at[1].val.clusterDim.y = 1;
        at[1].val.clusterDim.z = 1;
        cfg.numAttrs = 2;
    }
    // the grid barrier counts this launch's arrivals from zero; look-back words of earlier
    // launches must not look ready
    cudaError_t e = cudaMemsetAsync(&eh->st->bar_count, 0, sizeof(unsigned), stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(eh->tile_status, 0,
                            sizeof(unsigned long long) * (size_t)(eh->n_max / kEB + 2), stream);
    if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, kernel, E);
    return e;
}
}  // namespace

hhs_status engine_hold_step(hhs_ctx* c, const SoA& P, int n, double dt, bool calc_ts,
                            hhs_precision prec, bool profile, cudaStream_t stream,
                            int top_level) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh) return HHS_ERR_INVALID_ARG;
    if (top_level < 0 || top_level >= c->max_levels) return HHS_ERR_INVALID_ARG;
    EParams E = engine_params(c, eh, P, n, dt, calc_ts, profile, top_level);
    const int pi = prec == HHS_PREC_FP64 ? 0 : 1;
    E.prec_mixed = pi;
    const cudaError_t e = pi == 0 ? engine_launch(eh, 0, k_engine<HHS_PREC_FP64>, E, stream)
                                  : engine_launch(eh, 1, k_engine<HHS_PREC_MIXED>, E, stream);
    hhs_count_launch();
    if (e != cudaSuccess) return hhs_from_cuda(e);
    return HHS_OK;
}

// Accelerations of all n particles from one another with the engine's mixed grid kick
// (the arithmetic of the kick phase of hhs_hold_step), into P's acceleration arrays.
hhs_status engine_kick_accelerations(hhs_ctx* c, const SoA& P, double* ax, double* ay,
                                     double* az, int n, cudaStream_t stream) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh || n < 2 || n > c->n_max || !ax || !ay || !az || eh->pk_levels < 1)
        return HHS_ERR_INVALID_ARG;
    EParams E = engine_params(c, eh, P, n, 1.0, false, false, 0);
    E.ts_part = ax;  // outputs (the probe needs no timestep partials)
    E.rate_acc = reinterpret_cast<unsigned*>(ay);
    E.tile_counts = reinterpret_cast<int*>(az);
    const cudaError_t e = engine_launch(eh, 1, k_engine_accel, E, stream);
    hhs_count_launch();
    if (e != cudaSuccess) return hhs_from_cuda(e);
    return HHS_OK;
}

hhs_status engine_timestep_rates(hhs_ctx* c, const SoA& P, int n, cudaStream_t stream) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh || n < 2 || n > c->n_max) return HHS_ERR_INVALID_ARG;
    EParams E = engine_params(c, eh, P, n, 1.0, true, false, 0);
    if (!E.tq) return HHS_ERR_INVALID_ARG;
    const cudaError_t e = engine_launch(eh, 1, k_engine_ts, E, stream);
    hhs_count_launch();
    if (e != cudaSuccess) return hhs_from_cuda(e);
    return HHS_OK;
}

// ------------------------------------------------------------------ sharded phases (host)
namespace {
// source chunks of the grid kick for a node of n sinks, as chunks_for computes them on
// the device for a grid of `workers` CTAs (so every rank cuts the node the same way)
int chunks_host(int n, int workers, int upc, int block) {
    const int nsb = (n + block - 1) / block;
    int c = (upc * workers + nsb - 1) / nsb;
    c = c < 1 ? 1 : (c > kMaxChunks ? kMaxChunks : c);
    const int maxc = (n + 63) / 64;
    return c < maxc ? c : (maxc < 1 ? 1 : maxc);
}
}  // namespace

hhs_status engine_shard_timesteps(hhs_ctx* c, const SoA& P, unsigned* rate_words,
                                  const int32_t* S, int n, hhs_precision prec, int rank,
                                  int world, const PeerOut& po, cudaStream_t s) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh || n < 1 || world < 1 || rank < 0 || rank >= world) return HHS_ERR_INVALID_ARG;
    EParams E = engine_params(c, eh, P, n, 1.0, true, false, 0);
    const int pi = prec == HHS_PREC_FP64 ? 0 : 1;
    const int grid = eh->grid[pi];
    if (pi == 1) {
        E.rate_acc = rate_words;
        const long long units = ts_sym_units(n);
        const long long u_lo = units * rank / world, u_hi = units * (rank + 1) / world;
        k_shard_ts_mixed<<<grid, kEB, kEngineSmem, s>>>(E, S, n, u_lo, u_hi, po);
        HHS_LAUNCH_CHECK();
        return HHS_OK;
    }
    const int nsb = (n + kEB - 1) / kEB;
    const int b_lo = (int)((long long)nsb * rank / world), b_hi = (int)((long long)nsb * (rank + 1) / world);
    const int nch = chunks_host(n, grid, eh->units_per_cta, kEB);
    if (b_hi > b_lo) {
        k_shard_ts_fp64<<<grid, kEB, kEngineSmem, s>>>(E, S, n, b_lo, b_hi, nch);
        HHS_LAUNCH_CHECK();
        const int s_lo = b_lo * kEB, s_hi = b_hi * kEB < n ? b_hi * kEB : n;
        k_shard_ts_fp64_reduce<<<(s_hi - s_lo + kEB - 1) / kEB, kEB, 0, s>>>(E, S, s_lo, s_hi, nch, po);
        HHS_LAUNCH_CHECK();
    }
    return HHS_OK;
}

hhs_status engine_rates_to_ts(hhs_ctx* c, const SoA& P, unsigned* rate_words, const int32_t* S,
                              int n, cudaStream_t s) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh || n < 1) return HHS_ERR_INVALID_ARG;
    EParams E = engine_params(c, eh, P, n, 1.0, true, false, 0);
    E.rate_acc = rate_words;
    k_rates_to_ts<<<(n + kEB - 1) / kEB, kEB, 0, s>>>(E, S, n);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

int engine_shard_kick_block(hhs_precision prec) { return prec == HHS_PREC_FP64 ? kEB : kKB; }

int engine_pk_levels(hhs_ctx* c) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    return eh ? eh->pk_levels : 0;
}

hhs_status engine_shard_kick(hhs_ctx* c, const SoA& P, const int32_t* F, const int32_t* L,
                             int nf, int ns, int level, double dt, hhs_precision prec, int b_lo,
                             int b_hi, const PeerOut& po, cudaStream_t s) {
    auto* eh = static_cast<EngineHost*>(c->engine_host);
    if (!eh || ns < 1 || nf < 0) return HHS_ERR_INVALID_ARG;
    const int pi = prec == HHS_PREC_FP64 ? 0 : 1;
    if (pi == 1 && level >= eh->pk_levels) return HHS_ERR_CAPACITY;  // caller falls back
    const int ntot = nf + ns;
    EParams E = engine_params(c, eh, P, ntot, dt, false, false, level);
    const int grid = eh->grid[pi];
    if (pi == 1) {
        k_pack_slow<<<(ns + kEB - 1) / kEB, kEB, 0, s>>>(E, L, ns, level);
        HHS_LAUNCH_CHECK();
    }
    if (b_hi <= b_lo) return HHS_OK;
    const int blk = engine_shard_kick_block(prec);
    const int nch = pi == 1 ? chunks_host(ntot, eh->grid[1], eh->units_per_cta, kKB) : 1;
    const int C = (ntot + nch - 1) / nch;
    if (pi == 1)
        k_shard_kick_mixed<<<grid, kEB, kEngineSmem, s>>>(E, F, nf, ns, level, nch, C, b_lo, b_hi);
    else
        k_shard_kick_fp64<<<grid, kEB, kEngineSmem, s>>>(E, F, L, nf, ns, b_lo, b_hi);
    HHS_LAUNCH_CHECK();
    const int s_lo = b_lo * blk, s_hi = b_hi * blk < ntot ? b_hi * blk : ntot;
    const int g2 = (s_hi - s_lo + kEB - 1) / kEB;
    if (pi == 1)
        k_shard_kick_reduce<HHS_PREC_MIXED><<<g2, kEB, 0, s>>>(E, F, L, nf, ns, dt, nch, C, s_lo,
                                                               s_hi, po);
    else
        k_shard_kick_reduce<HHS_PREC_FP64><<<g2, kEB, 0, s>>>(E, F, L, nf, ns, dt, nch, C, s_lo,
                                                              s_hi, po);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

// ------------------------------------------------------------------ batched host side
struct hhs_batch {
    int n_sys = 0, n_total = 0, n_max_sys = 0, max_levels = 0;
    hhs_params params{0.03, 0.0};
    int big_n = 1024, cluster_size = 8, small_n = 64, units_per_cta = 8, warp_n = 32, packed = 0;
    int mid_n = kMid, mid_dist_n = 96;
    int n_big = 0, n_clusters[2] = {0, 0};
    void* arena = nullptr;
    int32_t* d_offsets = nullptr;
    int32_t* d_order = nullptr;
    unsigned* d_queues = nullptr;
    double* d_leaf = nullptr;
    hhs_stats* d_stats = nullptr;
    unsigned* d_err = nullptr;
    char* cluster_slots = nullptr;
    char* cta_slots = nullptr;
    size_t cluster_slot_bytes = 0, cta_slot_bytes = 0;
    size_t off_lists = 0, off_counts = 0, off_ts = 0, off_k = 0, off_tiles = 0, off_rate = 0;
    int max_clusters = 0, max_ctas = 0;
    std::vector<int> sizes, order;
};

namespace {
template <int PREC>
cudaError_t batched_occupancy(int cs, int* clusters) {
    cudaError_t e = cudaFuncSetAttribute(k_batched<PREC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kEngineSmem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs, 1, 1);
    cfg.blockDim = dim3(kEB, 1, 1);
    cfg.dynamicSmemBytes = kEngineSmem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(clusters, (void*)k_batched<PREC>, &cfg);
}

size_t slot_layout(int n, int levels, int chunks, size_t* off) {
    size_t p = 0;
    off[0] = p; p += al(sizeof(int32_t) * 2 * (size_t)levels * n);          // lists
    off[1] = p; p += al(sizeof(hhs_partition) * (size_t)levels);            // counts
    off[2] = p; p += al(sizeof(double) * (size_t)chunks * n);               // ts partials
    off[3] = p; p += al(sizeof(double) * (size_t)(chunks * 3 > 6 ? chunks * 3 : 6) * n);
    off[4] = p; p += al(sizeof(int) * (size_t)(n / kEB + 2));               // tile counts
    off[5] = p; p += al(sizeof(unsigned) * (size_t)n);                      // rate_acc
    return p;
}
}  // namespace

extern "C" hhs_status hhs_batch_create(int32_t n_sys, const int32_t* offsets, int32_t max_levels,
                                       hhs_params params, hhs_batch** out) {
    if (!out || n_sys <= 0 || !offsets || max_levels <= 0 || !(params.eta > 0.0))
        return HHS_ERR_INVALID_ARG;
    *out = nullptr;
    auto* b = new (std::nothrow) hhs_batch();
    if (!b) return HHS_ERR_OOM;
    b->n_sys = n_sys;
    b->max_levels = max_levels < kMaxLevels - 1 ? max_levels : kMaxLevels - 1;
    b->params = params;
    b->sizes.resize(n_sys);
    if (offsets[0] != 0) { delete b; return HHS_ERR_INVALID_ARG; }
    for (int k = 0; k < n_sys; k++) {
        const int sz = offsets[k + 1] - offsets[k];
        if (sz <= 0) { delete b; return HHS_ERR_INVALID_ARG; }
        b->sizes[k] = sz;
        b->n_max_sys = sz > b->n_max_sys ? sz : b->n_max_sys;
    }
    b->n_total = offsets[n_sys];
    b->order.resize(n_sys);
    std::iota(b->order.begin(), b->order.end(), 0);
    std::stable_sort(b->order.begin(), b->order.end(),
                     [&](int a, int c) { return b->sizes[a] > b->sizes[c]; });
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int c0 = 0, c1 = 0;
    if (batched_occupancy<HHS_PREC_FP64>(b->cluster_size, &c0) != cudaSuccess ||
        batched_occupancy<HHS_PREC_MIXED>(b->cluster_size, &c1) != cudaSuccess || c0 <= 0 ||
        c1 <= 0) {
        delete b;
        return HHS_ERR_CUDA;
    }
    b->n_clusters[0] = c0;
    b->n_clusters[1] = c1;
    b->max_clusters = c0 > c1 ? c0 : c1;
    b->max_ctas = b->max_clusters * b->cluster_size;
    size_t offc[6], offs[6];
    b->cluster_slot_bytes = slot_layout(b->n_max_sys, b->max_levels, kMaxChunks, offc);
    b->cta_slot_bytes = slot_layout(b->n_max_sys, b->max_levels, 1, offs);
    // both slot kinds use the same offsets up to their own sizes: lists and counts first
    b->off_lists = offc[0]; b->off_counts = offc[1];
    // offsets beyond counts differ; keep the larger (cluster) layout for both
    b->cta_slot_bytes = b->cluster_slot_bytes;
    b->off_ts = offc[2]; b->off_k = offc[3]; b->off_tiles = offc[4]; b->off_rate = offc[5];
    (void)offs;
    const size_t head = al(sizeof(int32_t) * (n_sys + 1)) + al(sizeof(int32_t) * n_sys) +
                        al(sizeof(unsigned) * (2 + b->max_clusters)) + al(sizeof(double) * n_sys) +
                        al(sizeof(hhs_stats)) + al(sizeof(unsigned));
    const size_t total = head + b->cluster_slot_bytes * (size_t)b->max_clusters +
                         b->cta_slot_bytes * (size_t)b->max_ctas;
    cudaError_t e = cudaMalloc(&b->arena, total);
    if (e != cudaSuccess) { delete b; return hhs_from_cuda(e); }
    e = cudaMemset(b->arena, 0, total);
    char* p = static_cast<char*>(b->arena);
    b->d_offsets = reinterpret_cast<int32_t*>(p); p += al(sizeof(int32_t) * (n_sys + 1));
    b->d_order = reinterpret_cast<int32_t*>(p); p += al(sizeof(int32_t) * n_sys);
    b->d_queues = reinterpret_cast<unsigned*>(p); p += al(sizeof(unsigned) * (2 + b->max_clusters));
    b->d_leaf = reinterpret_cast<double*>(p); p += al(sizeof(double) * n_sys);
    b->d_stats = reinterpret_cast<hhs_stats*>(p); p += al(sizeof(hhs_stats));
    b->d_err = reinterpret_cast<unsigned*>(p); p += al(sizeof(unsigned));
    b->cluster_slots = p; p += b->cluster_slot_bytes * (size_t)b->max_clusters;
    b->cta_slots = p;
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_offsets, offsets, sizeof(int32_t) * (n_sys + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_order, b->order.data(), sizeof(int32_t) * n_sys, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { cudaFree(b->arena); delete b; return hhs_from_cuda(e); }
    for (int k = 0; k < n_sys; k++)
        if (b->sizes[b->order[k]] > b->big_n) b->n_big = k + 1;
    *out = b;
    return HHS_OK;
}

extern "C" hhs_status hhs_batch_destroy(hhs_batch* b) {
    if (!b) return HHS_ERR_INVALID_ARG;
    cudaError_t e = cudaFree(b->arena);
    delete b;
    return hhs_from_cuda(e);
}

extern "C" hhs_status hhs_batch_set_tuning(hhs_batch* b, int32_t big_n, int32_t small_n,
                                           int32_t units_per_cta) {
    if (!b || big_n < 0 || small_n < 0 || units_per_cta < 1 || units_per_cta > 64)
        return HHS_ERR_INVALID_ARG;
    b->big_n = big_n;
    b->small_n = small_n;
    b->units_per_cta = units_per_cta;
    b->n_big = 0;
    for (int k = 0; k < b->n_sys; k++)
        if (b->sizes[b->order[k]] > b->big_n) b->n_big = k + 1;
    return HHS_OK;
}

extern "C" hhs_status hhs_batch_set_mid(hhs_batch* b, int32_t mid_n, int32_t mid_dist_n) {
    if (!b || mid_n < 0 || mid_dist_n < 0) return HHS_ERR_INVALID_ARG;
    b->mid_n = mid_n;
    b->mid_dist_n = mid_dist_n;
    return HHS_OK;
}

extern "C" hhs_status hhs_hold_batched(hhs_batch* b, hhs_particle_system* sys, double dt,
                                       int32_t calc_timestep, hhs_precision prec, void* stream) {
    if (!b || !sys || !sys->_base || !(dt > 0.0)) return HHS_ERR_INVALID_ARG;
    if (b->n_total > sys->n) return HHS_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int pi = prec == HHS_PREC_FP64 ? 0 : 1;
    const int nclu = b->n_clusters[pi];
    HHS_CUDA_TRY(cudaMemsetAsync(b->d_queues, 0, sizeof(unsigned) * (2 + nclu), s));
    BParams B;
    EParams& E = B.E;
    E.P.x = sys->x; E.P.y = sys->y; E.P.z = sys->z;
    E.P.vx = sys->vx; E.P.vy = sys->vy; E.P.vz = sys->vz;
    E.P.m = sys->m; E.P.ts = sys->ts; E.P.id = sys->id;
    E.n_top = 0;
    E.n_max = b->n_max_sys;
    E.max_levels = b->max_levels;
    E.small_n = b->small_n;
    E.calc_top = calc_timestep ? 1 : 0;
    E.profile = 0;
    E.units_per_cta = b->units_per_cta;
    E.warp_n = b->warp_n;
    E.mid_n = b->mid_n;
    E.mid_dist_n = b->mid_dist_n;
    E.packed = b->packed;
    E.top_level = 0;
    E.dt_top = dt;
    E.eta = b->params.eta;
    E.eps2 = b->params.eps * b->params.eps;
    E.eps2f = (float)E.eps2;
    E.eta_s2 = b->params.eta / 1.41421356237309504880;
    E.inv_eta_s2 = (float)(1.0 / E.eta_s2);
    E.inv_eta = (float)(1.0 / E.eta);
    E.fast_lists = E.slow_lists = nullptr;
    E.counts = nullptr;
    E.leaf_time = nullptr;
    E.stats = b->d_stats;
    E.ts_part = E.k_part = E.c_part = nullptr;
    E.tq = nullptr;
    E.tq_stride = 0;
    E.tile_counts = nullptr;
    E.tile_status = nullptr;
    E.rate_acc = nullptr;
    E.st = nullptr;
    E.err = b->d_err;
    E.pk = nullptr;
    E.pk_stride = 0;
    E.pk_levels = 0;
    E.prec_mixed = pi;
    E.overlap = 0;
    E.trace = nullptr;
    E.trace_count = nullptr;
    E.trace_cap = 0;
    B.offsets = b->d_offsets;
    B.order = b->d_order;
    B.n_sys = b->n_sys;
    B.n_big = b->n_big;
    B.queues = b->d_queues;
    B.cluster_slots = b->cluster_slots;
    B.cta_slots = b->cta_slots;
    B.cluster_slot_bytes = b->cluster_slot_bytes;
    B.cta_slot_bytes = b->cta_slot_bytes;
    B.off_lists = b->off_lists; B.off_counts = b->off_counts; B.off_ts = b->off_ts;
    B.off_k = b->off_k; B.off_tiles = b->off_tiles; B.off_rate = b->off_rate;
    B.leaf_times = b->d_leaf;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nclu * b->cluster_size, 1, 1);
    cfg.blockDim = dim3(kEB, 1, 1);
    cfg.dynamicSmemBytes = kEngineSmem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = b->cluster_size;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaError_t e = pi == 0 ? cudaLaunchKernelEx(&cfg, k_batched<HHS_PREC_FP64>, B)
                            : cudaLaunchKernelEx(&cfg, k_batched<HHS_PREC_MIXED>, B);
    hhs_count_launch();
    return hhs_from_cuda(e);
}

// Batched autotuner: times hhs_hold_batched on the caller's systems for a grid of
// (big_n, units_per_cta, mid_dist_n) candidates, restoring the particle state, the
// per-system leaf times and the work counters before every trial and at the end, and
// keeps the fastest. Allocates a snapshot of the state (outside any timed region).
extern "C" hhs_status hhs_batch_autotune(hhs_batch* b, hhs_particle_system* sys, double dt,
                                         hhs_precision prec, hhs_batch_tuning* out,
                                         hhs_batch_tuning* table, int32_t capacity,
                                         int32_t* count, void* stream) {
    if (!b || !sys || !sys->_base || !(dt > 0.0) || capacity < 0 || (capacity > 0 && !table))
        return HHS_ERR_INVALID_ARG;
    if (b->n_total > sys->n) return HHS_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = b->n_total;
    hhs_particle_system snap;
    hhs_status st = hhs_particle_system_alloc(&snap, n);
    if (st != HHS_OK) return st;
    double* leaf = nullptr;
    if (cudaMalloc(&leaf, sizeof(double) * (size_t)b->n_sys) != cudaSuccess) {
        hhs_particle_system_free(&snap);
        return HHS_ERR_OOM;
    }
    const size_t bytes = sizeof(double) * (size_t)n;
    double* src[7] = {sys->x, sys->y, sys->z, sys->vx, sys->vy, sys->vz, sys->ts};
    double* dst[7] = {snap.x, snap.y, snap.z, snap.vx, snap.vy, snap.vz, snap.ts};
    auto copy_all = [&](bool save) -> hhs_status {
        for (int k = 0; k < 7; k++)
            HHS_CUDA_TRY(cudaMemcpyAsync(save ? dst[k] : src[k], save ? src[k] : dst[k], bytes,
                                         cudaMemcpyDeviceToDevice, s));
        HHS_CUDA_TRY(cudaMemcpyAsync(save ? leaf : b->d_leaf, save ? b->d_leaf : leaf,
                                     sizeof(double) * (size_t)b->n_sys, cudaMemcpyDeviceToDevice, s));
        return HHS_OK;
    };
    hhs_stats stats_saved{};
    cudaMemcpyAsync(&stats_saved, b->d_stats, sizeof(hhs_stats), cudaMemcpyDeviceToHost, s);
    const hhs_batch_tuning cur{b->big_n, b->small_n, b->units_per_cta, b->mid_n, b->mid_dist_n, 0.0};
    hhs_batch_tuning best = cur;
    best.ms_per_step = 1e300;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    st = copy_all(true);
    const int big_c[] = {512, 1024, 2048};
    const int upc_c[] = {8, 16};
    const int dist_c[] = {64, 96};
    constexpr int kTimed = 3;
    int k = 0;
    for (int big : big_c)
        for (int upc : upc_c)
            for (int dn : dist_c) {
                if (st != HHS_OK) break;
                hhs_batch_tuning t{big, cur.small_n, upc, cur.mid_n, dn, 0.0};
                if ((st = hhs_batch_set_tuning(b, t.big_n, t.small_n, t.units_per_cta)) != HHS_OK) break;
                if ((st = hhs_batch_set_mid(b, t.mid_n, t.mid_dist_n)) != HHS_OK) break;
                st = copy_all(false);
                if (st == HHS_OK) st = hhs_hold_batched(b, sys, dt, 1, prec, stream);
                if (st == HHS_OK) st = copy_all(false);
                if (st != HHS_OK) break;
                cudaEventRecord(e0, s);
                for (int r = 0; r < kTimed && st == HHS_OK; r++)
                    st = hhs_hold_batched(b, sys, dt, 1, prec, stream);
                cudaEventRecord(e1, s);
                if (st == HHS_OK) st = hhs_batch_check(b, stream);
                if (st != HHS_OK) break;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                t.ms_per_step = ms / kTimed;
                if (k < capacity) table[k] = t;
                k++;
                if (t.ms_per_step < best.ms_per_step) best = t;
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const hhs_status st2 = copy_all(false);
    cudaMemcpyAsync(b->d_stats, &stats_saved, sizeof(hhs_stats), cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    cudaFree(leaf);
    hhs_particle_system_free(&snap);
    if (count) *count = k;
    const hhs_batch_tuning pick = (st == HHS_OK && st2 == HHS_OK) ? best : cur;
    hhs_batch_set_tuning(b, pick.big_n, pick.small_n, pick.units_per_cta);
    hhs_batch_set_mid(b, pick.mid_n, pick.mid_dist_n);
    if (st == HHS_OK) st = st2;
    if (st == HHS_OK && out) *out = best;
    return st;
}

extern "C" hhs_status hhs_batch_get_simtime(hhs_batch* b, double* out, void* stream) {
    if (!b || !out) return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HHS_CUDA_TRY(cudaMemcpyAsync(out, b->d_leaf, sizeof(double) * b->n_sys, cudaMemcpyDeviceToHost, s));
    HHS_CUDA_TRY(cudaStreamSynchronize(s));
    return HHS_OK;
}

extern "C" hhs_status hhs_batch_get_stats(hhs_batch* b, hhs_stats* out, void* stream) {
    if (!b || !out) return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HHS_CUDA_TRY(cudaMemcpyAsync(out, b->d_stats, sizeof(hhs_stats), cudaMemcpyDeviceToHost, s));
    HHS_CUDA_TRY(cudaStreamSynchronize(s));
    return HHS_OK;
}

extern "C" hhs_status hhs_batch_reset_stats(hhs_batch* b, void* stream) {
    if (!b) return HHS_ERR_INVALID_ARG;
    HHS_CUDA_TRY(cudaMemsetAsync(b->d_stats, 0, sizeof(hhs_stats), static_cast<cudaStream_t>(stream)));
    return HHS_OK;
}

extern "C" hhs_status hhs_batch_check(hhs_batch* b, void* stream) {
    if (!b) return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HHS_CUDA_TRY(cudaStreamSynchronize(s));
    unsigned e = 0;
    HHS_CUDA_TRY(cudaMemcpy(&e, b->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (e & (HHS_ERRBIT_LOOKBACK_TIMEOUT | HHS_ERRBIT_BARRIER_TIMEOUT)) return HHS_ERR_TIMEOUT;
    if (e & HHS_ERRBIT_DEPTH) return HHS_ERR_DEPTH;
    if (e) return HHS_ERR_DEVICE_FAULT_FLAG;
    return HHS_OK;
}
