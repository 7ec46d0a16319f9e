// hhs_pairs.cu -- one-thread-per-sink pair kernels (timestep, kick), drift, gathers.
//
// These are the plain kernels of the library: the reference's one-thread-per-sink
// structure with source tiles staged through shared memory (src/timestep.cuh:65-99,
// src/kick.cuh:59-155), but on SoA FP64 arrays addressed through index lists, with
// the tail tile loaded correctly (the reference returns before the cooperative load,
// src/timestep.cuh:70) and every launch sized from device-resident counts.
#include "hhs_common.cuh"
#include "hhs_kernels.h"
#include "hhs_pairmath.cuh"

using namespace hhs;

namespace {

constexpr int kTsBlock = 128;
constexpr int kKickBlock = 128;
constexpr double kHuge = 1.e30;  // src/timestep.cuh:4

__device__ __forceinline__ int list_at(const int32_t* list, int i) { return list ? list[i] : i; }

// The stores of a sink-partitioned launch into the peer replicas, then a system-scope
// fence so that the barrier which follows the launch orders them for every peer.
__device__ __forceinline__ void peer_store_ts(const PeerOut& po, int g, double t) {
    if (po.n_peer == 0) return;
    for (int r = 0; r < po.n_peer; r++) po.ts[r][g] = t;
    __threadfence_system();
}
__device__ __forceinline__ void peer_store_v(const PeerOut& po, int g, double vx, double vy,
                                             double vz) {
    if (po.n_peer == 0) return;
    for (int r = 0; r < po.n_peer; r++) {
        po.vx[r][g] = vx; po.vy[r][g] = vy; po.vz[r][g] = vz;
    }
    __threadfence_system();
}

// ---------------------------------------------------------------- timesteps, FP64
__global__ void __launch_bounds__(kTsBlock)
    k_timesteps_fp64(SoA P, const int32_t* __restrict__ list, int n, double eta,
                     double eta_s2, PeerOut po) {
    __shared__ double sx[kTsBlock], sy[kTsBlock], sz[kTsBlock];
    __shared__ double svx[kTsBlock], svy[kTsBlock], svz[kTsBlock], sm[kTsBlock];
    const int i = po.lo + blockIdx.x * kTsBlock + threadIdx.x;
    const bool active = i < (po.hi < 0 ? n : po.hi);
    const int gi = active ? list_at(list, i) : 0;
    double xi = 0, yi = 0, zi = 0, vxi = 0, vyi = 0, vzi = 0, mi = 0;
    if (active) {
        xi = P.x[gi]; yi = P.y[gi]; zi = P.z[gi];
        vxi = P.vx[gi]; vyi = P.vy[gi]; vzi = P.vz[gi];
        mi = P.m[gi];
    }
    double minval = kHuge;
    for (int jt = 0; jt < n; jt += kTsBlock) {
        const int j = jt + threadIdx.x;
        if (j < n) {
            const int gj = list_at(list, j);
            sx[threadIdx.x] = P.x[gj]; sy[threadIdx.x] = P.y[gj]; sz[threadIdx.x] = P.z[gj];
            svx[threadIdx.x] = P.vx[gj]; svy[threadIdx.x] = P.vy[gj];
            svz[threadIdx.x] = P.vz[gj]; sm[threadIdx.x] = P.m[gj];
        }
        __syncthreads();
        if (active) {
            const int jn = min(kTsBlock, n - jt);
            for (int jl = 0; jl < jn; jl++) {
                if (jt + jl == i) continue;
                ts_pair_fp64(f64_sub(xi, sx[jl]), f64_sub(yi, sy[jl]), f64_sub(zi, sz[jl]),
                             f64_sub(vxi, svx[jl]), f64_sub(vyi, svy[jl]), f64_sub(vzi, svz[jl]), mi,
                             sm[jl], eta, eta_s2, minval);
            }
        }
        __syncthreads();
    }
    if (active) {
        P.ts[gi] = minval;
        peer_store_ts(po, gi, minval);
    }
}

// ---------------------------------------------------------------- timesteps, mixed
__global__ void __launch_bounds__(kTsBlock)
    k_timesteps_mixed(SoA P, const int32_t* __restrict__ list, int n, float inv_eta_s2,
                      float inv_eta, PeerOut po) {
    __shared__ float4 sA[kTsBlock];  // xh, yh, zh, m
    __shared__ float4 sB[kTsBlock];  // xl, yl, zl, -
    __shared__ float4 sV[kTsBlock];  // vx, vy, vz, -
    const int i = po.lo + blockIdx.x * kTsBlock + threadIdx.x;
    const bool active = i < (po.hi < 0 ? n : po.hi);
    const int gi = active ? list_at(list, i) : 0;
    DS xi{0, 0}, yi{0, 0}, zi{0, 0};
    float vxi = 0, vyi = 0, vzi = 0, mi = 0;
    if (active) {
        xi = ds_split(P.x[gi]); yi = ds_split(P.y[gi]); zi = ds_split(P.z[gi]);
        vxi = (float)P.vx[gi]; vyi = (float)P.vy[gi]; vzi = (float)P.vz[gi];
        mi = (float)P.m[gi];
    }
    float maxrate = 0.0f;
    for (int jt = 0; jt < n; jt += kTsBlock) {
        const int j = jt + threadIdx.x;
        if (j < n) {
            const int gj = list_at(list, j);
            const DS a = ds_split(P.x[gj]), b = ds_split(P.y[gj]), c = ds_split(P.z[gj]);
            sA[threadIdx.x] = make_float4(a.hi, b.hi, c.hi, (float)P.m[gj]);
            sB[threadIdx.x] = make_float4(a.lo, b.lo, c.lo, 0.0f);
            sV[threadIdx.x] =
                make_float4((float)P.vx[gj], (float)P.vy[gj], (float)P.vz[gj], 0.0f);
        }
        __syncthreads();
        if (active) {
            const int jn = min(kTsBlock, n - jt);
            for (int jl = 0; jl < jn; jl++) {
                if (jt + jl == i) continue;
                const float4 A = sA[jl], B = sB[jl], V = sV[jl];
                const float rate = ts_pair_rate_mixed(
                    ds_diff(xi.hi, xi.lo, A.x, B.x), ds_diff(yi.hi, yi.lo, A.y, B.y),
                    ds_diff(zi.hi, zi.lo, A.z, B.z), vxi - V.x, vyi - V.y, vzi - V.z, mi + A.w,
                    inv_eta_s2, inv_eta);
                maxrate = fmaxf(maxrate, rate);
            }
        }
        __syncthreads();
    }
    if (active) {
        double t = 1.0 / (double)maxrate;
        t = (t < kHuge) ? t : kHuge;
        P.ts[gi] = t;
        peer_store_ts(po, gi, t);
    }
}

// ---------------------------------------------------------------- kick, FP64
// Sink s of a split level: s < nf -> fast sink F[s]; else slow sink L[s - nf].
// Sources: slow tiles (every sink), then fast tiles (slow sinks only). Slow sinks
// apply v += aLL*dt then v += aLF*dt (kick_slow then kick_sf(fast->slow),
// src/hold.cuh:138,142); fast sinks apply v += aFL*dt (kick_sf(slow->fast), :143).
__global__ void __launch_bounds__(kKickBlock)
    k_kick_level_fp64(SoA P, const int32_t* __restrict__ F, const int32_t* __restrict__ L,
                      const hhs_partition* __restrict__ counts, double dt, double eps2,
                      PeerOut po) {
    __shared__ double sx[kKickBlock], sy[kKickBlock], sz[kKickBlock], sm[kKickBlock];
    const int nf = counts->n_fast, ns = counts->n_slow, n = nf + ns;
    if (ns == 0) return;
    const int hi = po.hi < 0 ? n : min(po.hi, n);
    if (po.lo + (int)(blockIdx.x * kKickBlock) >= hi) return;
    const int s = po.lo + blockIdx.x * kKickBlock + threadIdx.x;
    const bool active = s < hi;
    const bool slow_sink = s >= nf;
    const int g = active ? (slow_sink ? L[s - nf] : F[s]) : 0;
    const double xi = active ? P.x[g] : 0.0, yi = active ? P.y[g] : 0.0,
                 zi = active ? P.z[g] : 0.0;
    double aLx = 0, aLy = 0, aLz = 0, aFx = 0, aFy = 0, aFz = 0;
    for (int jt = 0; jt < ns; jt += kKickBlock) {
        const int j = jt + threadIdx.x;
        if (j < ns) {
            const int gj = L[j];
            sx[threadIdx.x] = P.x[gj]; sy[threadIdx.x] = P.y[gj]; sz[threadIdx.x] = P.z[gj];
            sm[threadIdx.x] = P.m[gj];
        }
        __syncthreads();
        if (active) {
            const int jn = min(kKickBlock, ns - jt);
            for (int jl = 0; jl < jn; jl++)
                kick_pair_fp64(f64_sub(sx[jl], xi), f64_sub(sy[jl], yi), f64_sub(sz[jl], zi), sm[jl],
                               aLx, aLy, aLz, eps2);
        }
        __syncthreads();
    }
    for (int jt = 0; jt < nf; jt += kKickBlock) {
        const int j = jt + threadIdx.x;
        if (j < nf) {
            const int gj = F[j];
            sx[threadIdx.x] = P.x[gj]; sy[threadIdx.x] = P.y[gj]; sz[threadIdx.x] = P.z[gj];
            sm[threadIdx.x] = P.m[gj];
        }
        __syncthreads();
        if (active && slow_sink) {
            const int jn = min(kKickBlock, nf - jt);
            for (int jl = 0; jl < jn; jl++)
                kick_pair_fp64(f64_sub(sx[jl], xi), f64_sub(sy[jl], yi), f64_sub(sz[jl], zi), sm[jl],
                               aFx, aFy, aFz, eps2);
        }
        __syncthreads();
    }
    if (!active) return;
    double vx = P.vx[g], vy = P.vy[g], vz = P.vz[g];
    vx = f64_add(vx, f64_mul(aLx, dt));
    vy = f64_add(vy, f64_mul(aLy, dt));
    vz = f64_add(vz, f64_mul(aLz, dt));
    if (slow_sink && nf > 0) {
        vx = f64_add(vx, f64_mul(aFx, dt));
        vy = f64_add(vy, f64_mul(aFy, dt));
        vz = f64_add(vz, f64_mul(aFz, dt));
    }
    P.vx[g] = vx; P.vy[g] = vy; P.vz[g] = vz;
    peer_store_v(po, g, vx, vy, vz);
}

// ---------------------------------------------------------------- kick, mixed
// Same sink/source structure. Pair terms in FP32 from double-single relative
// coordinates; per-sink sums Kahan-compensated in FP32 and applied in FP64. The slow
// and fast source sums are kept apart so the update order matches the FP64 form.
__global__ void __launch_bounds__(kKickBlock)
    k_kick_level_mixed(SoA P, const int32_t* __restrict__ F, const int32_t* __restrict__ L,
                       const hhs_partition* __restrict__ counts, double dt, float eps2,
                       PeerOut po) {
    __shared__ float4 sA[kKickBlock];  // xh, yh, zh, m
    __shared__ float4 sB[kKickBlock];  // xl, yl, zl, -
    const int nf = counts->n_fast, ns = counts->n_slow, n = nf + ns;
    if (ns == 0) return;
    const int hi = po.hi < 0 ? n : min(po.hi, n);
    if (po.lo + (int)(blockIdx.x * kKickBlock) >= hi) return;
    const int s = po.lo + blockIdx.x * kKickBlock + threadIdx.x;
    const bool active = s < hi;
    const bool slow_sink = s >= nf;
    const int g = active ? (slow_sink ? L[s - nf] : F[s]) : 0;
    DS xi{0, 0}, yi{0, 0}, zi{0, 0};
    if (active) { xi = ds_split(P.x[g]); yi = ds_split(P.y[g]); zi = ds_split(P.z[g]); }
    float acc[2][3] = {{0, 0, 0}, {0, 0, 0}}, cmp[2][3] = {{0, 0, 0}, {0, 0, 0}};
#pragma unroll 1
    for (int part = 0; part < 2; part++) {
        const int cnt = part == 0 ? ns : nf;
        const int32_t* lst = part == 0 ? L : F;
        const bool use = active && (part == 0 || slow_sink);
        for (int jt = 0; jt < cnt; jt += kKickBlock) {
            const int j = jt + threadIdx.x;
            if (j < cnt) {
                const int gj = lst[j];
                const DS a = ds_split(P.x[gj]), b = ds_split(P.y[gj]), c = ds_split(P.z[gj]);
                sA[threadIdx.x] = make_float4(a.hi, b.hi, c.hi, (float)P.m[gj]);
                sB[threadIdx.x] = make_float4(a.lo, b.lo, c.lo, 0.0f);
            }
            __syncthreads();
            if (use) {
                const int jn = min(kKickBlock, cnt - jt);
                for (int jl = 0; jl < jn; jl++) {
                    const float4 A = sA[jl], B = sB[jl];
                    const float dx = ds_diff(A.x, B.x, xi.hi, xi.lo);
                    const float dy = ds_diff(A.y, B.y, yi.hi, yi.lo);
                    const float dz = ds_diff(A.z, B.z, zi.hi, zi.lo);
                    const float d2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
                    if (d2 == 0.0f) continue;
                    const float ri = rsqrt_nr(d2);
                    const float mr3 = A.w * ri * ri * ri;
                    kahan_add(acc[part][0], cmp[part][0], dx * mr3);
                    kahan_add(acc[part][1], cmp[part][1], dy * mr3);
                    kahan_add(acc[part][2], cmp[part][2], dz * mr3);
                }
            }
            __syncthreads();
        }
    }
    if (!active) return;
    double v[3] = {P.vx[g], P.vy[g], P.vz[g]};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        v[k] += ((double)acc[0][k] - (double)cmp[0][k]) * dt;
        if (slow_sink && nf > 0) v[k] += ((double)acc[1][k] - (double)cmp[1][k]) * dt;
    }
    P.vx[g] = v[0]; P.vy[g] = v[1]; P.vz[g] = v[2];
    peer_store_v(po, g, v[0], v[1], v[2]);
}

// ---------------------------------------------------------------- standalone kicks
// kick_slow / kick_sf of the reference API: sinks sink[0..n), sources src[0..m).
__global__ void __launch_bounds__(kKickBlock)
    k_kick_pair_fp64(SoA K, double* __restrict__ ax_out, double* __restrict__ ay_out,
                     double* __restrict__ az_out, SoA S, int n, int m, double dtfac) {
    __shared__ double sx[kKickBlock], sy[kKickBlock], sz[kKickBlock], sm[kKickBlock];
    const int i = blockIdx.x * kKickBlock + threadIdx.x;
    const bool active = i < n;
    const double xi = active ? K.x[i] : 0.0, yi = active ? K.y[i] : 0.0,
                 zi = active ? K.z[i] : 0.0;
    double ax = 0, ay = 0, az = 0;
    for (int jt = 0; jt < m; jt += kKickBlock) {
        const int j = jt + threadIdx.x;
        if (j < m) {
            sx[threadIdx.x] = S.x[j]; sy[threadIdx.x] = S.y[j]; sz[threadIdx.x] = S.z[j];
            sm[threadIdx.x] = S.m[j];
        }
        __syncthreads();
        if (active) {
            const int jn = min(kKickBlock, m - jt);
            for (int jl = 0; jl < jn; jl++)
                kick_pair_fp64(f64_sub(sx[jl], xi), f64_sub(sy[jl], yi), f64_sub(sz[jl], zi), sm[jl],
                               ax, ay, az);
        }
        __syncthreads();
    }
    if (!active) return;
    if (ax_out) { ax_out[i] = ax; ay_out[i] = ay; az_out[i] = az; }
    K.vx[i] = f64_add(K.vx[i], f64_mul(ax, dtfac));
    K.vy[i] = f64_add(K.vy[i], f64_mul(ay, dtfac));
    K.vz[i] = f64_add(K.vz[i], f64_mul(az, dtfac));
}

__global__ void __launch_bounds__(kKickBlock)
    k_kick_pair_mixed(SoA K, double* __restrict__ ax_out, double* __restrict__ ay_out,
                      double* __restrict__ az_out, SoA S, int n, int m, double dtfac) {
    __shared__ float4 sA[kKickBlock], sB[kKickBlock];
    const int i = blockIdx.x * kKickBlock + threadIdx.x;
    const bool active = i < n;
    DS xi{0, 0}, yi{0, 0}, zi{0, 0};
    if (active) { xi = ds_split(K.x[i]); yi = ds_split(K.y[i]); zi = ds_split(K.z[i]); }
    float acc[3] = {0, 0, 0}, cmp[3] = {0, 0, 0};
    for (int jt = 0; jt < m; jt += kKickBlock) {
        const int j = jt + threadIdx.x;
        if (j < m) {
            const DS a = ds_split(S.x[j]), b = ds_split(S.y[j]), c = ds_split(S.z[j]);
            sA[threadIdx.x] = make_float4(a.hi, b.hi, c.hi, (float)S.m[j]);
            sB[threadIdx.x] = make_float4(a.lo, b.lo, c.lo, 0.0f);
        }
        __syncthreads();
        if (active) {
            const int jn = min(kKickBlock, m - jt);
            for (int jl = 0; jl < jn; jl++) {
                const float4 A = sA[jl], B = sB[jl];
                const float dx = ds_diff(A.x, B.x, xi.hi, xi.lo);
                const float dy = ds_diff(A.y, B.y, yi.hi, yi.lo);
                const float dz = ds_diff(A.z, B.z, zi.hi, zi.lo);
                const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                if (d2 == 0.0f) continue;
                const float ri = rsqrt_nr(d2);
                const float mr3 = A.w * ri * ri * ri;
                kahan_add(acc[0], cmp[0], dx * mr3);
                kahan_add(acc[1], cmp[1], dy * mr3);
                kahan_add(acc[2], cmp[2], dz * mr3);
            }
        }
        __syncthreads();
    }
    if (!active) return;
    const double a0 = (double)acc[0] - cmp[0], a1 = (double)acc[1] - cmp[1],
                 a2 = (double)acc[2] - cmp[2];
    if (ax_out) { ax_out[i] = a0; ay_out[i] = a1; az_out[i] = a2; }
    K.vx[i] += a0 * dtfac;
    K.vy[i] += a1 * dtfac;
    K.vz[i] += a2 * dtfac;
}

// ---------------------------------------------------------------- drift / gathers
// pos += vel*h (src/drift.cuh:24-26) over the slow list of a split level.
__global__ void k_drift_slow(SoA P, const int32_t* __restrict__ L,
                             const hhs_partition* __restrict__ counts, double h) {
    const int ns = counts->n_slow;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
        const int g = L[s];
        P.x[g] = f64_add(P.x[g], f64_mul(P.vx[g], h));
        P.y[g] = f64_add(P.y[g], f64_mul(P.vy[g], h));
        P.z[g] = f64_add(P.z[g], f64_mul(P.vz[g], h));
    }
}

__global__ void k_drift(SoA P, int n, double h) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        P.x[g] = f64_add(P.x[g], f64_mul(P.vx[g], h));
        P.y[g] = f64_add(P.y[g], f64_mul(P.vy[g], h));
        P.z[g] = f64_add(P.z[g], f64_mul(P.vz[g], h));
    }
}

// prev[parent_id[i]] <- cur[i] for pos, vel, m, timestep (src/update_system.cuh:14-23)
__global__ void k_update_system(SoA prev, SoA cur, const int32_t* __restrict__ parent, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = parent[i];
        prev.x[p] = cur.x[i]; prev.y[p] = cur.y[i]; prev.z[p] = cur.z[i];
        prev.vx[p] = cur.vx[i]; prev.vy[p] = cur.vy[i]; prev.vz[p] = cur.vz[i];
        prev.m[p] = cur.m[i];
        prev.ts[p] = cur.ts[i];
    }
}

// Copy of the split (src/split.cuh:341-356): fast[k] <- total[F[k]], slow[k] <- total[L[k]]
// for pos, vel, m, timestep, id, with parent_id = the source index.
__global__ void k_gather_split(SoA T, SoA Ls, int32_t* __restrict__ lpar, SoA Fs,
                               int32_t* __restrict__ fpar, const int32_t* __restrict__ L,
                               const int32_t* __restrict__ F,
                               const hhs_partition* __restrict__ counts) {
    const int nf = counts->n_fast, ns = counts->n_slow;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nf + ns;
         k += gridDim.x * blockDim.x) {
        const bool fast = k < nf;
        const int d = fast ? k : k - nf;
        const int g = fast ? F[d] : L[d];
        SoA& D = fast ? Fs : Ls;
        D.x[d] = T.x[g]; D.y[d] = T.y[g]; D.z[d] = T.z[g];
        D.vx[d] = T.vx[g]; D.vy[d] = T.vy[g]; D.vz[d] = T.vz[g];
        D.m[d] = T.m[g]; D.ts[d] = T.ts[g];
        D.id[d] = T.id[g];
        (fast ? fpar : lpar)[d] = g;
    }
}

inline int grid_for(int n, int block) { return (n + block - 1) / block; }
inline int grid_stride(int n, int block) {
    int g = grid_for(n, block);
    return g < 148 * 8 ? (g > 0 ? g : 1) : 148 * 8;
}

}  // namespace

hhs_status launch_timesteps(const SoA& P, const int32_t* list, int n, double eta,
                            hhs_precision prec, cudaStream_t stream, const PeerOut& po) {
    if (n <= 0) return HHS_OK;
    if (po.lo < 0 || po.n_peer < 0 || po.n_peer > kMaxPeers) return HHS_ERR_INVALID_ARG;
    const int hi = po.hi < 0 ? n : po.hi;
    if (hi > n || po.lo > hi) return HHS_ERR_INVALID_ARG;
    if (hi == po.lo) return HHS_OK;  // an empty shard
    const double eta_s2 = eta / 1.41421356237309504880;  // eta / M_SQRT2
    const int grid = grid_for(hi - po.lo, kTsBlock);
    if (prec == HHS_PREC_FP64)
        k_timesteps_fp64<<<grid, kTsBlock, 0, stream>>>(P, list, n, eta, eta_s2, po);
    else
        k_timesteps_mixed<<<grid, kTsBlock, 0, stream>>>(P, list, n, (float)(1.0 / eta_s2),
                                                         (float)(1.0 / eta), po);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

hhs_status launch_kick_level(const SoA& P, const int32_t* fast_list,
                             const int32_t* slow_list, const hhs_partition* counts,
                             int n_max, double dt, double eps2, hhs_precision prec,
                             cudaStream_t stream, const PeerOut& po) {
    if (n_max <= 0) return HHS_OK;
    if (po.lo < 0 || po.n_peer < 0 || po.n_peer > kMaxPeers) return HHS_ERR_INVALID_ARG;
    // hi >= 0: a shard whose bounds the caller took from the host copy of the counts
    const int hi = po.hi < 0 ? n_max : po.hi;
    if (hi > n_max || po.lo > hi) return HHS_ERR_INVALID_ARG;
    if (hi == po.lo) return HHS_OK;
    const int grid = grid_for(hi - po.lo, kKickBlock);
    if (prec == HHS_PREC_FP64)
        k_kick_level_fp64<<<grid, kKickBlock, 0, stream>>>(P, fast_list, slow_list, counts, dt,
                                                           eps2, po);
    else
        k_kick_level_mixed<<<grid, kKickBlock, 0, stream>>>(P, fast_list, slow_list, counts, dt,
                                                            (float)eps2, po);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

hhs_status launch_kick_pair(const SoA& sink, double* ax, double* ay, double* az,
                            const SoA& src, int n_sink, int n_src, double dtfac,
                            hhs_precision prec, cudaStream_t stream) {
    if (n_sink <= 0) return HHS_OK;
    if (prec == HHS_PREC_FP64)
        k_kick_pair_fp64<<<grid_for(n_sink, kKickBlock), kKickBlock, 0, stream>>>(
            sink, ax, ay, az, src, n_sink, n_src, dtfac);
    else
        k_kick_pair_mixed<<<grid_for(n_sink, kKickBlock), kKickBlock, 0, stream>>>(
            sink, ax, ay, az, src, n_sink, n_src, dtfac);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

hhs_status launch_drift_slow(const SoA& P, const int32_t* slow_list,
                             const hhs_partition* counts, int n_max, double h,
                             cudaStream_t stream) {
    if (n_max <= 0) return HHS_OK;
    k_drift_slow<<<grid_stride(n_max, 256), 256, 0, stream>>>(P, slow_list, counts, h);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

hhs_status launch_drift(const SoA& P, int n, double h, cudaStream_t stream) {
    if (n <= 0) return HHS_OK;
    k_drift<<<grid_stride(n, 256), 256, 0, stream>>>(P, n, h);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

hhs_status launch_update_system(const SoA& prev, const SoA& cur, const int32_t* parent_id,
                                int n, cudaStream_t stream) {
    if (n <= 0) return HHS_OK;
    k_update_system<<<grid_stride(n, 256), 256, 0, stream>>>(prev, cur, parent_id, n);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

hhs_status launch_gather_split(const SoA& total, const SoA& slow, int32_t* slow_parent,
                               const SoA& fast, int32_t* fast_parent,
                               const int32_t* slow_list, const int32_t* fast_list,
                               const hhs_partition* counts, int n_max, cudaStream_t stream) {
    if (n_max <= 0) return HHS_OK;
    k_gather_split<<<grid_stride(n_max, 256), 256, 0, stream>>>(
        total, slow, slow_parent, fast, fast_parent, slow_list, fast_list, counts);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}
