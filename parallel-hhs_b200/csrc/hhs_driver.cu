// hhs_driver.cu -- the top-level driver around the HOLD step: FP64 energy diagnostic,
// binary snapshots (checkpoint / resume) and hhs_hold, the integration loop the
// reference declares but never defines (src/hold.cuh:20-35).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <vector>

#include "hhs_ctx.h"
#include "hhs_kernels.h"
#include "hhs_pairmath.cuh"

using namespace hhs;

namespace {

constexpr int kEnBlock = 256;

// Per-sink potential sum over all j != i, FP64 with Neumaier compensation:
// rows[i] = sum_j -m_i m_j / r_ij (each pair counted twice; halved by the reduction).
// The softening length enters as r = sqrt(d2 + eps^2).
__global__ void __launch_bounds__(kEnBlock)
    k_potential_rows(const double* __restrict__ x, const double* __restrict__ y,
                     const double* __restrict__ z, const double* __restrict__ m, int n,
                     double eps2, double* __restrict__ rows) {
    __shared__ double sx[kEnBlock], sy[kEnBlock], sz[kEnBlock], sm[kEnBlock];
    const int i = blockIdx.x * kEnBlock + threadIdx.x;
    const bool act = i < n;
    const double xi = act ? x[i] : 0.0, yi = act ? y[i] : 0.0, zi = act ? z[i] : 0.0;
    const double mi = act ? m[i] : 0.0;
    double s = 0.0, c = 0.0;
    for (int t0 = 0; t0 < n; t0 += kEnBlock) {
        const int j = t0 + threadIdx.x;
        if (j < n) { sx[threadIdx.x] = x[j]; sy[threadIdx.x] = y[j]; sz[threadIdx.x] = z[j]; sm[threadIdx.x] = m[j]; }
        __syncthreads();
        if (act) {
            const int tl = min(kEnBlock, n - t0);
            for (int jl = 0; jl < tl; jl++) {
                if (t0 + jl == i) continue;
                const double dx = xi - sx[jl], dy = yi - sy[jl], dz = zi - sz[jl];
                const double d2 = dx * dx + dy * dy + dz * dz + eps2;
                if (d2 == 0.0) continue;
                const double v = -mi * sm[jl] / sqrt(d2);
                const double t = s + v;
                c += (fabs(s) >= fabs(v)) ? (s - t) + v : (v - t) + s;
                s = t;
            }
        }
        __syncthreads();
    }
    if (act) rows[i] = s + c;
}

// One CTA: Neumaier sums of the kinetic terms and the potential rows in a fixed order
// (each thread a fixed stride of elements, then the thread partials in index order).
__global__ void __launch_bounds__(kEnBlock)
    k_energy_reduce(const double* __restrict__ vx, const double* __restrict__ vy,
                    const double* __restrict__ vz, const double* __restrict__ m,
                    const double* __restrict__ rows, int n, double* __restrict__ out) {
    __shared__ double ks[kEnBlock], kc[kEnBlock], ps[kEnBlock], pc[kEnBlock];
    double s1 = 0, c1 = 0, s2 = 0, c2 = 0;
    for (int i = threadIdx.x; i < n; i += kEnBlock) {
        const double k = 0.5 * m[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
        double t = s1 + k;
        c1 += (fabs(s1) >= fabs(k)) ? (s1 - t) + k : (k - t) + s1;
        s1 = t;
        const double p = rows[i];
        t = s2 + p;
        c2 += (fabs(s2) >= fabs(p)) ? (s2 - t) + p : (p - t) + s2;
        s2 = t;
    }
    ks[threadIdx.x] = s1; kc[threadIdx.x] = c1; ps[threadIdx.x] = s2; pc[threadIdx.x] = c2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, ac = 0, b = 0, bc = 0;
        for (int k = 0; k < kEnBlock; k++) {
            const double vals[4] = {ks[k], kc[k], ps[k], pc[k]};
            for (int q = 0; q < 2; q++) {
                const double v = vals[q];
                const double t = a + v;
                ac += (fabs(a) >= fabs(v)) ? (a - t) + v : (v - t) + a;
                a = t;
            }
            for (int q = 2; q < 4; q++) {
                const double v = vals[q];
                const double t = b + v;
                bc += (fabs(b) >= fabs(v)) ? (b - t) + v : (v - t) + b;
                b = t;
            }
        }
        out[0] = a + ac;
        out[1] = 0.5 * (b + bc);
    }
}

struct SnapHeader {
    char magic[8];       // "HHSSNAP1"
    int32_t n;
    int32_t version;
    double time;
    double eta, eps, dt;
    int32_t step;
    int32_t pad[7];
};
static_assert(sizeof(SnapHeader) == 80, "snapshot header layout");

}  // namespace

// FP64 total energy of the first n particles of sys on the device. Uses the system's
// acceleration arrays as scratch (their contents are overwritten); synchronises `stream`.
extern "C" hhs_status hhs_energy(hhs_particle_system* sys, int32_t n, double eps,
                                 double* kinetic, double* potential, void* stream) {
    if (!sys || !sys->_base || n <= 0 || n > sys->n || !kinetic || !potential)
        return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* rows = sys->ax;
    double* out = sys->ay;
    k_potential_rows<<<(n + kEnBlock - 1) / kEnBlock, kEnBlock, 0, s>>>(sys->x, sys->y, sys->z,
                                                                       sys->m, n, eps * eps, rows);
    HHS_LAUNCH_CHECK();
    k_energy_reduce<<<1, kEnBlock, 0, s>>>(sys->vx, sys->vy, sys->vz, sys->m, rows, n, out);
    HHS_LAUNCH_CHECK();
    double h[2];
    HHS_CUDA_TRY(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s));
    HHS_CUDA_TRY(cudaStreamSynchronize(s));
    *kinetic = h[0];
    *potential = h[1];
    return HHS_OK;
}

extern "C" hhs_status hhs_snapshot_write(const hhs_particle_system* sys, int32_t n, double time,
                                         const hhs_params* params, double dt, int32_t step,
                                         const char* path, void* stream) {
    if (!sys || !sys->_base || n <= 0 || n > sys->n || !path) return HHS_ERR_INVALID_ARG;
    std::vector<double> buf(8 * (size_t)n);
    std::vector<int32_t> id(n);
    double* f[8];
    for (int k = 0; k < 8; k++) f[k] = buf.data() + (size_t)k * n;
    hhs_status st = hhs_particle_system_download(sys, n, f[0], f[1], f[2], f[3], f[4], f[5], f[6],
                                                 f[7], id.data(), stream);
    if (st != HHS_OK) return st;
    HHS_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    SnapHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, "HHSSNAP1", 8);
    h.n = n;
    h.version = 1;
    h.time = time;
    h.eta = params ? params->eta : 0.0;
    h.eps = params ? params->eps : 0.0;
    h.dt = dt;
    h.step = step;
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return HHS_ERR_INVALID_ARG;
    bool ok = std::fwrite(&h, sizeof(h), 1, fp) == 1 &&
              std::fwrite(buf.data(), sizeof(double), buf.size(), fp) == buf.size() &&
              std::fwrite(id.data(), sizeof(int32_t), id.size(), fp) == id.size();
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? HHS_OK : HHS_ERR_INVALID_ARG;
}

extern "C" hhs_status hhs_snapshot_read(hhs_particle_system* sys, const char* path, int32_t* n_out,
                                        double* time, int32_t* step, void* stream) {
    if (!sys || !sys->_base || !path) return HHS_ERR_INVALID_ARG;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return HHS_ERR_INVALID_ARG;
    SnapHeader h;
    if (std::fread(&h, sizeof(h), 1, fp) != 1 || std::memcmp(h.magic, "HHSSNAP1", 8) != 0 ||
        h.n <= 0) {
        std::fclose(fp);
        return HHS_ERR_INVALID_ARG;
    }
    if (h.n > sys->n) { std::fclose(fp); return HHS_ERR_CAPACITY; }
    const int n = h.n;
    std::vector<double> buf(8 * (size_t)n);
    std::vector<int32_t> id(n);
    const bool ok = std::fread(buf.data(), sizeof(double), buf.size(), fp) == buf.size() &&
                    std::fread(id.data(), sizeof(int32_t), id.size(), fp) == id.size();
    std::fclose(fp);
    if (!ok) return HHS_ERR_INVALID_ARG;
    double* f[8];
    for (int k = 0; k < 8; k++) f[k] = buf.data() + (size_t)k * n;
    hhs_status st = hhs_particle_system_upload(sys, n, f[0], f[1], f[2], f[3], f[4], f[5], f[6],
                                               f[7], id.data(), stream);
    if (st != HHS_OK) return st;
    HHS_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    if (n_out) *n_out = n;
    if (time) *time = h.time;
    if (step) *step = h.step;
    return HHS_OK;
}

// hold(...) of src/hold.cuh:20-35: integrate from stime to etime in top-level steps of dt
// (timesteps recomputed at every top step). Every snapshot_every steps (and at the end)
// the energy is evaluated on the device and, with a snapshot prefix, a snapshot
// "<prefix>_<step>.hhs" is written. The segments between diagnostics run as one
// graph-captured sequence of steps (hhs_hold_integrate).
extern "C" hhs_status hhs_hold(hhs_ctx* c, hhs_particle_system* sys, int32_t n, double stime,
                               double etime, double dt, hhs_precision prec,
                               int32_t snapshot_every, const char* snapshot_prefix,
                               hhs_run_log* log, void* stream) {
    if (!c || !sys || n <= 0 || !(dt > 0.0) || !(etime > stime)) return HHS_ERR_INVALID_ARG;
    const long long steps = std::llround((etime - stime) / dt);
    if (steps <= 0 || steps > 0x7fffffff) return HHS_ERR_INVALID_ARG;
    const int every = snapshot_every > 0 ? snapshot_every : (int)steps;
    int done = 0;
    auto diag = [&](int step) -> hhs_status {
        double k = 0, p = 0;
        hhs_status st = hhs_energy(sys, n, c->params.eps, &k, &p, stream);
        if (st != HHS_OK) return st;
        if (log && log->n_entries < log->capacity && log->time && log->energy) {
            log->time[log->n_entries] = stime + step * dt;
            log->energy[log->n_entries] = k + p;
            log->n_entries++;
        }
        if (snapshot_prefix && snapshot_prefix[0]) {
            char path[4096];
            std::snprintf(path, sizeof(path), "%s_%06d.hhs", snapshot_prefix, step);
            st = hhs_snapshot_write(sys, n, stime + step * dt, &c->params, dt, step, path, stream);
            if (st != HHS_OK) return st;
        }
        return HHS_OK;
    };
    if (log) log->n_entries = 0;
    hhs_status st = diag(0);
    while (st == HHS_OK && done < steps) {
        const int seg = (int)std::min<long long>(every, steps - done);
        st = hhs_hold_integrate(c, sys, n, dt, seg, prec, stream);
        if (st == HHS_OK) st = hhs_ctx_check(c, stream);
        done += seg;
        if (st == HHS_OK) st = diag(done);
    }
    return st;
}

// Balanced assignment of independent systems to ranks (longest-processing-time greedy on
// the N^2 pair work); identical on every rank, so the sharding needs no collective.
extern "C" hhs_status hhs_batch_partition(int32_t n_sys, const int32_t* sizes, int32_t n_ranks,
                                          int32_t* rank_of, double* load) {
    if (n_sys < 0 || n_ranks <= 0 || (n_sys > 0 && (!sizes || !rank_of)))
        return HHS_ERR_INVALID_ARG;
    for (int k = 0; k < n_sys; k++)
        if (sizes[k] < 0) return HHS_ERR_INVALID_ARG;
    std::vector<int32_t> order(n_sys);
    for (int k = 0; k < n_sys; k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t b) { return sizes[a] > sizes[b]; });
    std::vector<double> acc(n_ranks, 0.0);
    for (int32_t k : order) {
        int best = 0;
        for (int r = 1; r < n_ranks; r++)
            if (acc[r] < acc[best]) best = r;
        rank_of[k] = best;
        acc[best] += (double)sizes[k] * (double)sizes[k];
    }
    if (load)
        for (int r = 0; r < n_ranks; r++) load[r] = acc[r];
    return HHS_OK;
}
