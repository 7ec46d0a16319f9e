/*
 * hhs_oracle.c -- CPU FP64 restatement of the HOLD step of parallel-hhs.
 *
 * TEST INFRASTRUCTURE ONLY (the checker). Only the tests, the smoke check and the
 * benchmark's CPU-baseline leg load this file's library; the product never does.
 * Compiled with -O2 -ffp-contract=off -fopenmp; see hhs_oracle.h for the map from
 * each function to the reference lines it restates.
 */
#include "hhs_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_HUGE 1.e30 /* src/timestep.cuh:4 */

int oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Pair timestep of sink i against every source j != i.
 * Restates src/timestep.cuh:17-60 expression by expression:
 *   dr = x_i - x_j, dv = v_i - v_j, r = sqrt(dr.dr), vdotdr2 = (dr.dv)/dr2
 *   free-fall: tau = eta/M_SQRT2 * r * sqrt(r/(m_j+m_i)); dtau = 3*tau*vdotdr2/2
 *   fly-by:    tau = eta*r/sqrt(dv2); dtau = tau*vdotdr2*(1+(m_i+m_j)/(dv2*r))
 *   each: dtau = (dtau < 1) ? dtau : 1; tau /= (1 - dtau/2); min. */
void oracle_timesteps(int n, const double* x, const double* y, const double* z,
                      const double* vx, const double* vy, const double* vz,
                      const double* m, double eta, double* ts) {
    const double eta_s2 = eta / M_SQRT2;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; i++) {
        const double xi = x[i], yi = y[i], zi = z[i];
        const double vxi = vx[i], vyi = vy[i], vzi = vz[i];
        const double mi = m[i];
        double minval = ORACLE_HUGE;
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            const double drx = xi - x[j], dry = yi - y[j], drz = zi - z[j];
            const double dvx = vxi - vx[j], dvy = vyi - vy[j], dvz = vzi - vz[j];
            const double dr2 = drx * drx + dry * dry + drz * drz;
            const double dv2 = dvx * dvx + dvy * dvy + dvz * dvz;
            const double r = sqrt(dr2);
            const double vdotdr2 = (dvx * drx + dvy * dry + dvz * drz) / dr2;
            double tau = eta_s2 * r * sqrt(r / (m[j] + mi));
            double dtau = 3 * tau * vdotdr2 / 2;
            dtau = (dtau < 1) ? dtau : 1;
            tau /= (1 - dtau / 2);
            if (tau < minval) minval = tau;
            tau = eta * r / sqrt(dv2);
            dtau = tau * vdotdr2 * (1 + (mi + m[j]) / (dv2 * r));
            dtau = (dtau < 1) ? dtau : 1;
            tau /= (1 - dtau / 2);
            if (tau < minval) minval = tau;
        }
        ts[i] = minval;
    }
}

/* Exact exclusive prefix sum (the contract of the reference's multi-level Blelloch
 * scan, src/split.cuh:131-302 and its host recursion :438-565). */
void oracle_scan_exclusive_i32(int64_t n, const int32_t* in, int32_t* out) {
    int32_t acc = 0;
    for (int64_t i = 0; i < n; i++) {
        out[i] = acc;
        acc += in[i];
    }
}

/* Predicate ts <= pivot (src/split.cuh:114-116), exclusive scan, stable scatter
 * (src/split.cuh:335-357): fast particle i goes to scan[i], slow particle i goes to
 * i - scan[i]. N_fast = pred[N-1] + scan[N-1] (:312). If N_fast == 1 the lone fast
 * particle is folded into the slow set at slot N-1 and N_fast becomes 0 (intended
 * semantics of :321-324,361-368). order[] holds parent indices. */
int oracle_split(int n, const double* ts, double pivot, int32_t* order) {
    if (n <= 0) return 0;
    int32_t* pred = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* scan = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    for (int i = 0; i < n; i++) pred[i] = ts[i] <= pivot;
    oracle_scan_exclusive_i32(n, pred, scan);
    int n_fast = pred[n - 1] + scan[n - 1];
    if (n_fast == 1) {
        int lone = -1;
        for (int i = 0; i < n; i++) {
            if (pred[i]) lone = i;
            else order[i - scan[i]] = i;
        }
        order[n - 1] = lone;
        n_fast = 0;
    } else {
        for (int i = 0; i < n; i++) {
            if (pred[i]) order[scan[i]] = i;
            else order[n_fast + (i - scan[i])] = i;
        }
    }
    free(pred);
    free(scan);
    return n_fast;
}

/* In-place two-pointer partition of the HHS CPU integrators, restating
 * cpu_split (src/cpu_scan.h:20-50) on particle indices: a left cursor skips entries with
 * ts <= pivot, a right cursor skips entries with ts > pivot, the two are exchanged while
 * the cursors have not met. order[0..n_fast) ends as the fast set and order[n_fast..n)
 * as the slow set, both in that routine's (unstable) order. Returns n_fast. */
int oracle_split_cpu_order(int n, const double* ts, double pivot, int32_t* order) {
    for (int i = 0; i < n; i++) order[i] = i;
    if (n <= 0) return 0;
    int left = 0, right = n - 1;
    for (;;) {
        while (ts[order[left]] <= pivot && left < right) left++;
        while (ts[order[right]] > pivot && left < right) right--;
        if (left < right) {
            int32_t t = order[left];
            order[left] = order[right];
            order[right] = t;
        } else {
            break;
        }
    }
    if (ts[order[left]] <= pivot) left++;
    return left;
}

/* Direct-sum kick, restating src/kick.cuh:19-30 and :82-105 per sink:
 *   dx = x_j - x_i; d2 = dx.dx + eps2; skip d2 == 0; d = sqrt(d2); inv = 1.0/(d2*d);
 *   a += dx * (m_j * inv)           (attractive; the reference GPU kernel has the
 *                                    opposite sign, see tests/test_nbforce.cu:14-18)
 *   v += a * dtfac                  (dtfac = fac*dt of the reference call)
 * Sources are summed in index order. eps2 is the squared softening length the
 * reference keeps in nbodysystem_globals (src/particle_system.cuh:16) but never
 * applies; eps2 = 0 gives the reference expression exactly (d2 + 0 == d2). */
void oracle_kick_soft(int n_sink, const double* sx, const double* sy, const double* sz,
                      double* svx, double* svy, double* svz,
                      double* ax, double* ay, double* az,
                      int n_src, const double* px, const double* py, const double* pz,
                      const double* pm, double dtfac, double eps2) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n_sink; i++) {
        const double xi = sx[i], yi = sy[i], zi = sz[i];
        double accx = 0.0, accy = 0.0, accz = 0.0;
        for (int j = 0; j < n_src; j++) {
            const double dxx = px[j] - xi, dxy = py[j] - yi, dxz = pz[j] - zi;
            const double d2 = dxx * dxx + dxy * dxy + dxz * dxz + eps2;
            if (d2 == 0.0) continue;
            const double d = sqrt(d2);
            const double inv = 1.0 / (d2 * d);
            const double s = pm[j] * inv;
            accx = accx + dxx * s;
            accy = accy + dxy * s;
            accz = accz + dxz * s;
        }
        if (ax) { ax[i] = accx; ay[i] = accy; az[i] = accz; }
        svx[i] = svx[i] + accx * dtfac;
        svy[i] = svy[i] + accy * dtfac;
        svz[i] = svz[i] + accz * dtfac;
    }
}

void oracle_kick(int n_sink, const double* sx, const double* sy, const double* sz,
                 double* svx, double* svy, double* svz,
                 double* ax, double* ay, double* az,
                 int n_src, const double* px, const double* py, const double* pz,
                 const double* pm, double dtfac) {
    oracle_kick_soft(n_sink, sx, sy, sz, svx, svy, svz, ax, ay, az, n_src, px, py, pz, pm,
                     dtfac, 0.0);
}

/* pos += vel * (dt*fac)   (src/drift.cuh:24-26) */
void oracle_drift(int n, double* x, double* y, double* z,
                  const double* vx, const double* vy, const double* vz, double dtfac) {
    for (int i = 0; i < n; i++) {
        x[i] = x[i] + vx[i] * dtfac;
        y[i] = y[i] + vy[i] * dtfac;
        z[i] = z[i] + vz[i] * dtfac;
    }
}

/* ---------------------------------------------------------------------------- */
/* Recursive HOLD on per-level copies (src/hold.cuh:51-181)                      */

typedef struct {
    int n;
    double *x, *y, *z, *vx, *vy, *vz, *m, *ts;
    int32_t *id, *parent;
} osys;

static void osys_alloc(osys* s, int n) {
    size_t nn = (size_t)(n > 0 ? n : 1);
    s->n = n;
    double* d = (double*)malloc(sizeof(double) * nn * 8);
    s->x = d; s->y = d + nn; s->z = d + 2 * nn;
    s->vx = d + 3 * nn; s->vy = d + 4 * nn; s->vz = d + 5 * nn;
    s->m = d + 6 * nn; s->ts = d + 7 * nn;
    s->id = (int32_t*)malloc(sizeof(int32_t) * nn * 2);
    s->parent = s->id + nn;
}

static void osys_free(osys* s) {
    free(s->x);
    free(s->id);
}

/* copy parent particle order[k] into child slot k (src/split.cuh:341-356) */
static void osys_gather(osys* child, const osys* parent, const int32_t* order, int cnt) {
    for (int k = 0; k < cnt; k++) {
        int i = order[k];
        child->x[k] = parent->x[i]; child->y[k] = parent->y[i]; child->z[k] = parent->z[i];
        child->vx[k] = parent->vx[i]; child->vy[k] = parent->vy[i]; child->vz[k] = parent->vz[i];
        child->m[k] = parent->m[i]; child->ts[k] = parent->ts[i];
        child->id[k] = parent->id[i];
        child->parent[k] = i;
    }
    child->n = cnt;
}

/* prev[parent_id[k]] <- cur[k] for pos, vel, m, timestep (src/update_system.cuh:14-23) */
static void osys_update(osys* prev, const osys* cur) {
    for (int k = 0; k < cur->n; k++) {
        int p = cur->parent[k];
        prev->x[p] = cur->x[k]; prev->y[p] = cur->y[k]; prev->z[p] = cur->z[k];
        prev->vx[p] = cur->vx[k]; prev->vy[p] = cur->vy[k]; prev->vz[p] = cur->vz[k];
        prev->m[p] = cur->m[k];
        prev->ts[p] = cur->ts[k];
    }
}

static void trace_node(oracle_trace* tr, int level, int n, int nf, int calc) {
    if (!tr) return;
    if (tr->nodes && tr->count < tr->capacity) {
        oracle_node* e = &tr->nodes[tr->count];
        e->level = level; e->n = n; e->n_fast = nf; e->calc_ts = calc;
    }
    tr->count++;
    if (level > tr->max_level) tr->max_level = level;
    double ns = (double)(n - nf), nfd = (double)nf;
    tr->kick_pairs += ns * (ns - 1.0) + 2.0 * ns * nfd;
    if (calc) tr->ts_pairs += (double)n * (double)(n - 1);
}

static void hold_rec(int level, osys* total, double dt, int calc_ts, double eta,
                     double eps2, oracle_trace* tr) {
    const int n = total->n;
    if (calc_ts)
        oracle_timesteps(n, total->x, total->y, total->z, total->vx, total->vy,
                         total->vz, total->m, eta, total->ts);
    int32_t* order = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int nf = oracle_split(n, total->ts, dt, order);
    int ns = n - nf;
    trace_node(tr, level, n, nf, calc_ts);

    osys fast, slow;
    osys_alloc(&fast, nf);
    osys_alloc(&slow, ns);
    osys_gather(&fast, total, order, nf);
    osys_gather(&slow, total, order + nf, ns);
    free(order);

    if (nf == 0 && tr) tr->leaf_time += dt; /* src/hold.cuh:106-114 */

    if (nf > 0) hold_rec(level + 1, &fast, dt / 2, 0, eta, eps2, tr);
    if (ns > 0)
        oracle_drift(ns, slow.x, slow.y, slow.z, slow.vx, slow.vy, slow.vz, dt * 0.5);
    if (ns > 0) {
        /* kick_slow(slow, dt, 1.0): v += a * (1.0*dt)  (src/hold.cuh:138) */
        oracle_kick_soft(ns, slow.x, slow.y, slow.z, slow.vx, slow.vy, slow.vz, NULL, NULL,
                         NULL, ns, slow.x, slow.y, slow.z, slow.m, 1.0 * dt, eps2);
        if (nf > 0) {
            /* kick_sf(src=fast, sink=slow, 1.0, dt): v += a * (dt*1.0)  (:142) */
            oracle_kick_soft(ns, slow.x, slow.y, slow.z, slow.vx, slow.vy, slow.vz, NULL, NULL,
                             NULL, nf, fast.x, fast.y, fast.z, fast.m, dt * 1.0, eps2);
            /* kick_sf(src=slow, sink=fast, 1.0, dt)  (:143) */
            oracle_kick_soft(nf, fast.x, fast.y, fast.z, fast.vx, fast.vy, fast.vz, NULL, NULL,
                             NULL, ns, slow.x, slow.y, slow.z, slow.m, dt * 1.0, eps2);
        }
    }
    if (ns > 0)
        oracle_drift(ns, slow.x, slow.y, slow.z, slow.vx, slow.vy, slow.vz, dt * 0.5);
    if (nf > 0) hold_rec(level + 1, &fast, dt / 2, 1, eta, eps2, tr);

    osys_update(total, &fast);
    osys_update(total, &slow);
    osys_free(&fast);
    osys_free(&slow);
}

void oracle_hold_step_soft(int n, double* x, double* y, double* z,
                           double* vx, double* vy, double* vz, double* m, double* ts,
                           int32_t* id, double dt, int calc_ts, double eta, double eps2,
                           oracle_trace* trace) {
    if (n <= 0) return;
    osys top;
    top.n = n; top.x = x; top.y = y; top.z = z; top.vx = vx; top.vy = vy; top.vz = vz;
    top.m = m; top.ts = ts; top.id = id; top.parent = NULL;
    hold_rec(0, &top, dt, calc_ts, eta, eps2, trace);
}

void oracle_hold_step(int n, double* x, double* y, double* z,
                      double* vx, double* vy, double* vz, double* m, double* ts,
                      int32_t* id, double dt, int calc_ts, double eta,
                      oracle_trace* trace) {
    oracle_hold_step_soft(n, x, y, z, vx, vy, vz, m, ts, id, dt, calc_ts, eta, 0.0, trace);
}

/* Neumaier compensated accumulation */
typedef struct { double s, c; } nsum;
static inline void nsum_add(nsum* a, double v) {
    double t = a->s + v;
    if (fabs(a->s) >= fabs(v)) a->c += (a->s - t) + v;
    else a->c += (v - t) + a->s;
    a->s = t;
}

void oracle_energy(int n, const double* x, const double* y, const double* z,
                   const double* vx, const double* vy, const double* vz,
                   const double* m, double* out) {
    nsum ke = {0, 0};
    for (int i = 0; i < n; i++)
        nsum_add(&ke, 0.5 * m[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]));
    /* per-row compensated sums, then a sequential compensated sum over rows, so the
     * result does not depend on the thread count */
    double* rows = (double*)malloc(sizeof(double) * (size_t)(2 * (n > 0 ? n : 1)));
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; i++) {
        nsum row = {0, 0};
        for (int j = i + 1; j < n; j++) {
            double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            if (r > 0.0) nsum_add(&row, -m[i] * m[j] / r);
        }
        rows[2 * i] = row.s;
        rows[2 * i + 1] = row.c;
    }
    nsum pot = {0, 0};
    for (int i = 0; i < 2 * n; i++) nsum_add(&pot, rows[i]);
    free(rows);
    out[0] = ke.s + ke.c;
    out[1] = pot.s + pot.c;
}

/* ---- seeded initial conditions for the CPU-baseline leg ----------------------------
 * The benchmark's reference arm builds its Plummer sphere here, so that the process
 * timing the CPU path never maps the product library. The inputs of the two arms must
 * be the same arrays, so this follows the same published methods with the same random
 * stream and the same operation order as the product's generator (a CPU test compares
 * the two bit for bit):
 *  - SplitMix64 (Steele, Lea & Flood 2014), 53-bit uniforms on the open interval (0,1);
 *  - masses first, independent of position: equal, Salpeter dN/dm ~ m^-2.35 on
 *    [0.1,100] by inverse CDF, or 90/10 two-component (m = 1 or 10); normalised to 1;
 *  - Plummer radius by the inverted cumulative mass (Aarseth, Henon & Wielen 1974),
 *    radii beyond 10 rejected; speed by von Neumann rejection on q^2 (1-q^2)^(7/2);
 *    isotropic directions;
 *  - centre-of-mass frame, then Henon units: x *= beta, v /= sqrt(beta) with
 *    beta = -4 E (E from oracle_energy); an unbound sample stays in structural units. */
typedef struct { uint64_t s; } osm64;
static uint64_t osm64_next(osm64* g) {
    uint64_t z = (g->s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double osm64_uniform(osm64* g) {
    return ((double)(osm64_next(g) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

int oracle_plummer(int n, uint64_t seed, int mass_spectrum, double* x, double* y, double* z,
                   double* vx, double* vy, double* vz, double* m) {
    const double two_pi = 2.0 * 3.14159265358979323846;
    osm64 g = {seed};
    if (n < 2 || mass_spectrum < 0 || mass_spectrum > 2) return 1;
    double mtot = 0.0;
    for (int i = 0; i < n; i++) {
        double mi = 1.0;
        if (mass_spectrum == 1) {
            const double p = 1.0 - 2.35, a = pow(0.1, p), b = pow(100.0, p);
            mi = pow(a + osm64_uniform(&g) * (b - a), 1.0 / p);
        } else if (mass_spectrum == 2) {
            mi = osm64_uniform(&g) < 0.1 ? 10.0 : 1.0;
        }
        m[i] = mi;
        mtot += mi;
    }
    for (int i = 0; i < n; i++) m[i] /= mtot;
    for (int i = 0; i < n; i++) {
        double r, q, w;
        do {
            r = 1.0 / sqrt(pow(osm64_uniform(&g), -2.0 / 3.0) - 1.0);
        } while (!(r <= 10.0));
        const double cth = 1.0 - 2.0 * osm64_uniform(&g);
        const double phi = two_pi * osm64_uniform(&g);
        const double sth = sqrt(1.0 - cth * cth);
        x[i] = r * sth * cos(phi);
        y[i] = r * sth * sin(phi);
        z[i] = r * cth;
        do {
            q = osm64_uniform(&g);
            w = osm64_uniform(&g);
        } while (0.1 * w >= q * q * pow(1.0 - q * q, 3.5));
        const double v = q * sqrt(2.0) * pow(1.0 + r * r, -0.25);
        const double cv = 1.0 - 2.0 * osm64_uniform(&g);
        const double pv = two_pi * osm64_uniform(&g);
        const double sv = sqrt(1.0 - cv * cv);
        vx[i] = v * sv * cos(pv);
        vy[i] = v * sv * sin(pv);
        vz[i] = v * cv;
    }
    double c[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < n; i++) {
        c[0] += m[i] * x[i]; c[1] += m[i] * y[i]; c[2] += m[i] * z[i];
        c[3] += m[i] * vx[i]; c[4] += m[i] * vy[i]; c[5] += m[i] * vz[i];
    }
    for (int i = 0; i < n; i++) {
        x[i] -= c[0]; y[i] -= c[1]; z[i] -= c[2];
        vx[i] -= c[3]; vy[i] -= c[4]; vz[i] -= c[5];
    }
    double e[2];
    oracle_energy(n, x, y, z, vx, vy, vz, m, e);
    const double etot = e[0] + e[1];
    if (!(etot < 0.0)) return 0;
    const double beta = -4.0 * etot, vs = 1.0 / sqrt(beta);
    for (int i = 0; i < n; i++) {
        x[i] *= beta; y[i] *= beta; z[i] *= beta;
        vx[i] *= vs; vy[i] *= vs; vz[i] *= vs;
    }
    return 0;
}
