// hhs_ic.cpp -- seeded initial conditions for the HOLD benchmarks and tests.
//
// The reference ships no initial-condition generator (its driver is absent,
// src/hold.cuh:20-35), so this file restates the published methods it needs:
//  * Plummer sphere sampling of Aarseth, Henon & Wielen (1974, A&A 37, 183):
//    radius from the inverted cumulative mass, speed by von Neumann rejection
//    on q^2 (1-q^2)^(7/2), isotropic directions; radii beyond 10 scale radii
//    are rejected.
//  * Henon units (G = M = 1, E = -1/4): positions scaled by beta and velocities
//    by 1/sqrt(beta) with beta = -4 E_sample, which keeps the sampled virial
//    ratio and makes the FP64 direct-sum energy exactly -1/4 up to rounding.
//  * Salpeter mass function dN/dm ~ m^-2.35 on [0.1, 100] by inverse-CDF
//    sampling, independent of position; two-component 90/10 masses (m = 1 or
//    10 with probability 0.9 / 0.1); masses are normalised to a total of 1.
//  * Random numbers: SplitMix64 (Steele, Lea & Flood 2014), 53-bit uniforms in
//    the open interval (0, 1).
#include "hhs_internal.h"

#include <cmath>
#include <cstdint>
#include <vector>

namespace {

struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((double)(next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
};

const double kPi = 3.14159265358979323846;

}  // namespace

extern "C" double hhs_host_potential_energy(int n, const double* x, const double* y,
                                            const double* z, const double* m) {
    // FP64 direct sum with per-row Neumaier compensation; rows combined in order.
    std::vector<double> rows(2 * (size_t)(n > 0 ? n : 1));
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; i++) {
        double s = 0.0, c = 0.0;
        for (int j = i + 1; j < n; j++) {
            double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            double r = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (r > 0.0) {
                double v = -m[i] * m[j] / r;
                double t = s + v;
                c += (std::fabs(s) >= std::fabs(v)) ? (s - t) + v : (v - t) + s;
                s = t;
            }
        }
        rows[2 * (size_t)i] = s;
        rows[2 * (size_t)i + 1] = c;
    }
    double s = 0.0, c = 0.0;
    for (size_t k = 0; k < 2 * (size_t)n; k++) {
        double v = rows[k];
        double t = s + v;
        c += (std::fabs(s) >= std::fabs(v)) ? (s - t) + v : (v - t) + s;
        s = t;
    }
    return s + c;
}

extern "C" double hhs_host_kinetic_energy(int n, const double* vx, const double* vy,
                                          const double* vz, const double* m) {
    double s = 0.0, c = 0.0;
    for (int i = 0; i < n; i++) {
        double v = 0.5 * m[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
        double t = s + v;
        c += (std::fabs(s) >= std::fabs(v)) ? (s - t) + v : (v - t) + s;
        s = t;
    }
    return s + c;
}

extern "C" hhs_status hhs_ic_plummer(int n, uint64_t seed, int mass_spectrum, double* x,
                                     double* y, double* z, double* vx, double* vy,
                                     double* vz, double* m) {
    if (n < 2 || !x || !y || !z || !vx || !vy || !vz || !m) return HHS_ERR_INVALID_ARG;
    if (mass_spectrum < HHS_MASS_EQUAL || mass_spectrum > HHS_MASS_TWO_COMPONENT)
        return HHS_ERR_INVALID_ARG;
    SplitMix64 rng(seed);
    // masses first (independent of position: no mass segregation)
    double mtot = 0.0;
    for (int i = 0; i < n; i++) {
        double mi = 1.0;
        if (mass_spectrum == HHS_MASS_SALPETER) {
            const double a1 = 1.0 - 2.35, lo = std::pow(0.1, a1), hi = std::pow(100.0, a1);
            mi = std::pow(lo + rng.uniform() * (hi - lo), 1.0 / a1);
        } else if (mass_spectrum == HHS_MASS_TWO_COMPONENT) {
            mi = (rng.uniform() < 0.1) ? 10.0 : 1.0;
        }
        m[i] = mi;
        mtot += mi;
    }
    for (int i = 0; i < n; i++) m[i] /= mtot;

    // Plummer positions and velocities in structural units (G = M = a = 1)
    for (int i = 0; i < n; i++) {
        double r;
        do {
            r = 1.0 / std::sqrt(std::pow(rng.uniform(), -2.0 / 3.0) - 1.0);
        } while (!(r <= 10.0));
        double cz = 1.0 - 2.0 * rng.uniform();
        double ph = 2.0 * kPi * rng.uniform();
        double sz = std::sqrt(1.0 - cz * cz);
        x[i] = r * sz * std::cos(ph);
        y[i] = r * sz * std::sin(ph);
        z[i] = r * cz;
        double q, g;
        do {
            q = rng.uniform();
            g = rng.uniform();
        } while (0.1 * g >= q * q * std::pow(1.0 - q * q, 3.5));
        double v = q * std::sqrt(2.0) * std::pow(1.0 + r * r, -0.25);
        double cw = 1.0 - 2.0 * rng.uniform();
        double pw = 2.0 * kPi * rng.uniform();
        double sw = std::sqrt(1.0 - cw * cw);
        vx[i] = v * sw * std::cos(pw);
        vy[i] = v * sw * std::sin(pw);
        vz[i] = v * cw;
    }
    // centre-of-mass frame
    double c[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < n; i++) {
        c[0] += m[i] * x[i]; c[1] += m[i] * y[i]; c[2] += m[i] * z[i];
        c[3] += m[i] * vx[i]; c[4] += m[i] * vy[i]; c[5] += m[i] * vz[i];
    }
    for (int i = 0; i < n; i++) {
        x[i] -= c[0]; y[i] -= c[1]; z[i] -= c[2];
        vx[i] -= c[3]; vy[i] -= c[4]; vz[i] -= c[5];
    }
    // Henon units: E = -1/4 with the sampled virial ratio kept. A handful of particles
    // can sample an unbound system (E >= 0); it is returned in structural units.
    double e = hhs_host_kinetic_energy(n, vx, vy, vz, m) +
               hhs_host_potential_energy(n, x, y, z, m);
    if (!(e < 0.0)) return HHS_OK;
    double beta = -4.0 * e, vs = 1.0 / std::sqrt(beta);
    for (int i = 0; i < n; i++) {
        x[i] *= beta; y[i] *= beta; z[i] *= beta;
        vx[i] *= vs; vy[i] *= vs; vz[i] *= vs;
    }
    return HHS_OK;
}
