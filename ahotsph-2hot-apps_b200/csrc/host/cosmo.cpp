// cosmo.cpp -- background cosmology for the cosmological leapfrog.
//
// The reference takes a(t) and its kick and drift integrals from the
// cosmology object of the 2hot support library (the `2hot` git submodule,
// libcosmo: cosmo1_init and the a_at_t / kick_t0_t1 / drift_t0_t1 members
// that nln/integrate.c:82-135 calls), which is not vendored with the
// reference.  This file restates the published Friedmann model those
// members integrate:
//     H(a)^2 = H0^2 (Omega_r a^-4 + Omega_m a^-3 + Omega_k a^-2 + Omega_lambda
//                    + Omega_de a^(-3(1 + w0 + wa)) exp(-3 wa (1 - a))),
//     Omega_k = 1 - Omega_r - Omega_m - Omega_lambda - Omega_de,
//     t(a)   = int_0^a da / (a H),
//     kick   = int_t0^t1 dt / a    = int da / (a^2 H),
//     drift  = int_t0^t1 dt / a^2  = int da / (a^3 H),
// the factors of the canonical-momentum leapfrog (p = a^2 dx/dt) that
// CosmoIntegrate applies: v += a0^2 kick(tvel, tvel + dtv) acc,
// x = a1 (x / a0 + drift(tpos, tpos + dt) v).
//
// Numerics: the integrands are smooth in ln a, so every integral is a sum
// of 8-point Gauss-Legendre panels in ln a; t(a) comes from a table of
// t at 2049 nodes over ln a in [ln 1e-8, ln 1e3] plus one panel to the
// point, with t(1e-8) from the closed form of a matter + radiation universe
// (the other terms are below 1e-16 of H^2 there).  a(t) inverts t(a) by
// Newton steps (dt/da = 1 / (a H)) from the table's bracketing node.
#include <cmath>
#include <cstdlib>
#include <vector>

#include "nlnhost.h"

namespace {

constexpr int kGL = 8;
const double kX[kGL] = {-0.9602898564975363, -0.7966664774136267, -0.5255324099163290,
                        -0.1834346424956498, 0.1834346424956498,  0.5255324099163290,
                        0.7966664774136267,  0.9602898564975363};
const double kW[kGL] = {0.1012285362903763, 0.2223810344533745, 0.3137066458778873,
                        0.3626837833783620, 0.3626837833783620, 0.3137066458778873,
                        0.2223810344533745, 0.1012285362903763};
constexpr double kLnAMin = -18.420680743952367;  // ln 1e-8
constexpr double kLnAMax = 6.907755278982137;    // ln 1e3
constexpr int kNodes = 2049;

}  // namespace

struct nln_cosmo {
    nln_cosmo_params p;
    double Ok;
    double dlna;
    std::vector<double> t;  // t at the table nodes

    double hubble(double a) const {
        const double ai = 1.0 / a;
        double e2 = p.Omega_r * ai * ai * ai * ai + p.Omega_m * ai * ai * ai + Ok * ai * ai +
                    p.Omega_lambda;
        if (p.Omega_de != 0.0)
            e2 += p.Omega_de * std::pow(a, -3.0 * (1.0 + p.w0 + p.wa)) *
                  std::exp(-3.0 * p.wa * (1.0 - a));
        return p.H0 * std::sqrt(e2);
    }
    // int_{ln a0}^{ln a1} a^-k / H(a) dln a, in panels of at most dlna
    double integral(double a0, double a1, int k) const {
        const double l0 = std::log(a0), l1 = std::log(a1);
        const int np = std::max(1, (int)std::ceil(std::fabs(l1 - l0) / dlna));
        const double h = (l1 - l0) / np;
        double s = 0.0;
        for (int q = 0; q < np; q++) {
            const double mid = l0 + (q + 0.5) * h;
            double ps = 0.0;
            for (int g = 0; g < kGL; g++) {
                const double a = std::exp(mid + 0.5 * h * kX[g]);
                ps += kW[g] * std::pow(a, -k) / hubble(a);
            }
            s += 0.5 * h * ps;
        }
        return s;
    }
    // t(a) for a <= 1e-8: matter + radiation in closed form
    double t_small(double a) const {
        const double m = p.Omega_m, r = p.Omega_r;
        if (r <= 0.0)
            return 2.0 / (3.0 * p.H0 * std::sqrt(m)) * std::pow(a, 1.5);
        if (m <= 0.0)
            return a * a / (2.0 * p.H0 * std::sqrt(r));
        return 2.0 / (3.0 * p.H0 * m * m) *
               ((m * a - 2.0 * r) * std::sqrt(m * a + r) + 2.0 * r * std::sqrt(r));
    }
    double t_at_a(double a) const {
        const double la = std::log(a);
        if (la <= kLnAMin)
            return t_small(a);
        int i = (int)((la - kLnAMin) / dlna);
        if (i >= kNodes - 1)
            i = kNodes - 2;
        const double ai = std::exp(kLnAMin + i * dlna);
        return t[i] + integral(ai, a, 0);
    }
    double a_at_t(double tt) const {
        // bracketing node, then Newton on t(a) = tt
        int lo = 0, hi = kNodes - 1;
        if (tt <= t[0]) {
            // below the table: invert the closed form by bisection in ln a
            double l0 = kLnAMin - 40.0, l1 = kLnAMin;
            for (int it = 0; it < 200; it++) {
                const double lm = 0.5 * (l0 + l1);
                (t_small(std::exp(lm)) < tt ? l0 : l1) = lm;
            }
            return std::exp(0.5 * (l0 + l1));
        }
        while (hi - lo > 1) {
            const int mid = (lo + hi) / 2;
            (t[mid] <= tt ? lo : hi) = mid;
        }
        double a = std::exp(kLnAMin + (lo + 0.5) * dlna);
        for (int it = 0; it < 50; it++) {
            const double f = t_at_a(a) - tt;
            const double step = f * a * hubble(a);  // dt/da = 1 / (a H)
            a -= step;
            if (std::fabs(step) <= 1e-15 * a)
                break;
        }
        return a;
    }
};

extern "C" nln_cosmo *nln_cosmo_new(const nln_cosmo_params *params) {
    if (!params || !(params->H0 > 0.0) || params->Omega_m < 0.0 || params->Omega_r < 0.0 ||
        params->Omega_m + params->Omega_r <= 0.0)
        return nullptr;
    auto *c = new nln_cosmo();
    c->p = *params;
    c->Ok = 1.0 - params->Omega_r - params->Omega_m - params->Omega_lambda - params->Omega_de;
    c->dlna = (kLnAMax - kLnAMin) / (kNodes - 1);
    c->t.resize(kNodes);
    c->t[0] = c->t_small(std::exp(kLnAMin));
    for (int i = 1; i < kNodes; i++) {
        const double a0 = std::exp(kLnAMin + (i - 1) * c->dlna), a1 = std::exp(kLnAMin + i * c->dlna);
        c->t[i] = c->t[i - 1] + c->integral(a0, a1, 0);
    }
    return c;
}

extern "C" void nln_cosmo_free(nln_cosmo *c) { delete c; }

extern "C" double nln_cosmo_hubble(const nln_cosmo *c, double a) { return c->hubble(a); }

extern "C" double nln_cosmo_t_at_a(const nln_cosmo *c, double a) { return c->t_at_a(a); }

extern "C" double nln_cosmo_a_at_t(const nln_cosmo *c, double t) { return c->a_at_t(t); }

extern "C" double nln_cosmo_kick(const nln_cosmo *c, double t0, double t1) {
    return c->integral(c->a_at_t(t0), c->a_at_t(t1), 1);
}

extern "C" double nln_cosmo_drift(const nln_cosmo *c, double t0, double t1) {
    return c->integral(c->a_at_t(t0), c->a_at_t(t1), 2);
}

extern "C" void nln_cosmo_kdk(const nln_cosmo *c, double tpos, double tvel, double dt, double dtv,
                              double out[6]) {
    const double a0 = c->a_at_t(tpos);
    out[0] = a0 * a0 * nln_cosmo_kick(c, tvel, tpos);      // to the positions' time (energies)
    out[1] = a0 * a0 * nln_cosmo_kick(c, tvel, tvel + dtv);  // the velocities' kick
    out[2] = nln_cosmo_drift(c, tpos, tpos + dt);            // the positions' drift
    out[3] = 1.0 / a0;                                       // physical -> comoving
    out[4] = c->a_at_t(tpos + dt);                           // comoving -> physical
    out[5] = 1.0 / (a0 * a0);                                // kinetic energy scale
}
