// ewald_table.cpp -- FP64 table of the periodic correction to the Newtonian
// potential, with its first three derivatives, for the batched kernels'
// Ewald term and for the FP64 direct-sum measurement.
//
// The periodic Green's function is the Ewald sum of nln/ewald.c:13-64
// (alpha = 2/L, real-space images, k-space waves with |h|^2 <= 16, the
// constant pi/(alpha^2 L^3)); for a source at displacement y (source - sink)
//   Phi_per(y) = pi/(alpha^2 L^3) - sum_n erfc(alpha |y-nL|)/|y-nL|
//                - sum_{h != 0} exp(-pi^2 h^2/(alpha L)^2) cos(2 pi h.y/L) / (pi L h^2)
// and its gradient is the force of ewald() on the sink.  The table holds
//   C(y) = Phi_per(y) + 1/|y|      (the n = 0 term becomes erf(alpha r)/r)
// which is smooth in |y_k| < L.  Every derivative is analytic: radial
// terms through g'/r, (g'' - g'/r)/r^2 and (g''' - 3g''/r + 3g'/r^2)/r^3,
// plane waves through powers of k; near r = 0 the n = 0 term is summed as a
// power series in (alpha r)^2.  Real-space images are kept while
// erfc(alpha r) > 1e-17 (r < 3L), the same k-space cut as ewald().
#ifdef _OPENMP
#include <omp.h>
#endif

#include <cmath>
#include <cstdint>

#include "nlnlists.h"

namespace {

struct Rad {
    double g, gr, a2, a3;  // g, g'/r, (g''-g'/r)/r^2, (g'''-3g''/r+3g'/r^2)/r^3
};

// g(r) = -erfc(alpha r)/r
Rad rad_erfc(double r, double alpha) {
    const double c = 2.0 * alpha / std::sqrt(M_PI);
    const double E = std::erfc(alpha * r);
    const double ex = std::exp(-alpha * alpha * r * r);
    const double E1 = -c * ex;
    const double E2 = c * 2.0 * alpha * alpha * r * ex;
    const double E3 = c * 2.0 * alpha * alpha * (1.0 - 2.0 * alpha * alpha * r * r) * ex;
    const double r2 = r * r, r3 = r2 * r, r4 = r3 * r;
    double f = E / r;
    double f1 = E1 / r - E / r2;
    double f2 = E2 / r - 2.0 * E1 / r2 + 2.0 * E / r3;
    double f3 = E3 / r - 3.0 * E2 / r2 + 6.0 * E1 / r3 - 6.0 * E / r4;
    f = -f; f1 = -f1; f2 = -f2; f3 = -f3;
    Rad o;
    o.g = f;
    o.gr = f1 / r;
    o.a2 = (f2 - f1 / r) / r2;
    o.a3 = (f3 - 3.0 * f2 / r + 3.0 * f1 / r2) / r3;
    return o;
}

// g(r) = erf(alpha r)/r = c P(q), q = r^2, c = 2 alpha/sqrt(pi),
// P(q) = sum_n (-1)^n alpha^(2n) q^n / (n! (2n+1)); then g'/r = 2cP',
// a2 = 4cP'', a3 = 8cP''' (all regular at r = 0).
Rad rad_erf_series(double r, double alpha) {
    const double c = 2.0 * alpha / std::sqrt(M_PI);
    const double q = r * r, a2 = alpha * alpha;
    double P = 0, P1 = 0, P2 = 0, P3 = 0;
    double coef = 1.0;  // (-1)^n alpha^(2n) / n!
    for (int n = 0; n < 40; n++) {
        const double pn = coef / (2 * n + 1);
        P += pn * std::pow(q, n);
        if (n >= 1) P1 += pn * n * std::pow(q, n - 1);
        if (n >= 2) P2 += pn * n * (n - 1) * std::pow(q, n - 2);
        if (n >= 3) P3 += pn * n * (n - 1) * (n - 2) * std::pow(q, n - 3);
        coef *= -a2 / (n + 1);
        if (std::fabs(coef) * std::pow(q + 1e-300, n) < 1e-30 && n > 8)
            break;
    }
    Rad o;
    o.g = c * P;
    o.gr = 2.0 * c * P1;
    o.a2 = 4.0 * c * P2;
    o.a3 = 8.0 * c * P3;
    return o;
}

// g(r) = erf(alpha r)/r = 1/r - erfc(alpha r)/r, directly (alpha r >= 1)
Rad rad_erf_direct(double r, double alpha) {
    Rad e = rad_erfc(r, alpha);  // -erfc/r
    const double r2 = r * r, r3 = r2 * r;
    // 1/r: g = 1/r, g' = -1/r^2, g'' = 2/r^3, g''' = -6/r^4
    Rad o;
    o.g = 1.0 / r + e.g;
    o.gr = -1.0 / r3 + e.gr;
    o.a2 = 3.0 / (r2 * r3) + e.a2;
    o.a3 = -15.0 / (r3 * r2 * r2) + e.a3;
    return o;
}

// accumulate a radial term at displacement x into the 20 outputs
void add_radial(const Rad &R, const double x[3], double *o) {
    o[0] += R.g;
    for (int i = 0; i < 3; i++) o[1 + i] += R.gr * x[i];
    static const int H[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    for (int k = 0; k < 6; k++) {
        int i = H[k][0], j = H[k][1];
        o[4 + k] += R.a2 * x[i] * x[j] + (i == j ? R.gr : 0.0);
    }
    static const int T[10][3] = {{0, 0, 0}, {0, 0, 1}, {0, 0, 2}, {0, 1, 1}, {0, 1, 2},
                                 {0, 2, 2}, {1, 1, 1}, {1, 1, 2}, {1, 2, 2}, {2, 2, 2}};
    for (int k = 0; k < 10; k++) {
        int i = T[k][0], j = T[k][1], l = T[k][2];
        double d = 0.0;
        if (j == l) d += x[i];
        if (i == l) d += x[j];
        if (i == j) d += x[l];
        o[10 + k] += R.a3 * x[i] * x[j] * x[l] + R.a2 * d;
    }
}

void ewald_eval(double L, const double *y, double *o) {
    const double alpha = 2.0 / L;
    for (int q = 0; q < NLN_EWALD_NQ; q++) o[q] = 0.0;
    o[0] = M_PI / (alpha * alpha * L * L * L);
    // n = 0: erf(alpha r)/r
    {
        const double r = std::sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
        Rad R = (alpha * r < 1.0) ? rad_erf_series(r, alpha) : rad_erf_direct(r, alpha);
        add_radial(R, y, o);
    }
    const double rcut = 3.0 * L;
    for (int i = -4; i <= 4; i++)
        for (int j = -4; j <= 4; j++)
            for (int k = -4; k <= 4; k++) {
                if (!i && !j && !k)
                    continue;
                double x[3] = {y[0] - i * L, y[1] - j * L, y[2] - k * L};
                double r = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
                if (r > rcut)
                    continue;
                add_radial(rad_erfc(r, alpha), x, o);
            }
    // k space: -A cos(k.y), A = exp(-pi^2 h^2/(alpha L)^2)/(pi L h^2), k = 2 pi h / L
    for (int i = -4; i <= 4; i++)
        for (int j = -4; j <= 4; j++)
            for (int k = -4; k <= 4; k++) {
                const int hh = i * i + j * j + k * k;
                if (hh == 0 || hh > 16)
                    continue;
                const double A = std::exp(-M_PI * M_PI * hh / (alpha * alpha * L * L)) /
                                 (M_PI * L * hh);
                const double kv[3] = {2 * M_PI * i / L, 2 * M_PI * j / L, 2 * M_PI * k / L};
                const double ph = kv[0] * y[0] + kv[1] * y[1] + kv[2] * y[2];
                const double cs = std::cos(ph), sn = std::sin(ph);
                o[0] -= A * cs;
                for (int a = 0; a < 3; a++) o[1 + a] += A * kv[a] * sn;
                static const int H[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
                for (int m = 0; m < 6; m++) o[4 + m] += A * kv[H[m][0]] * kv[H[m][1]] * cs;
                static const int T[10][3] = {{0, 0, 0}, {0, 0, 1}, {0, 0, 2}, {0, 1, 1},
                                             {0, 1, 2}, {0, 2, 2}, {1, 1, 1}, {1, 1, 2},
                                             {1, 2, 2}, {2, 2, 2}};
                for (int m = 0; m < 10; m++)
                    o[10 + m] -= A * kv[T[m][0]] * kv[T[m][1]] * kv[T[m][2]] * sn;
            }
}

int ewald_table(double L, int n, double reach, double *out) {
    if (!(L > 0) || n < 2 || !(reach > 0) || !out)
        return -1;
    const double h = reach * L / (n - 1);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            for (int k = 0; k < n; k++) {
                const double y[3] = {i * h, j * h, k * h};
                ewald_eval(L, y, out + (((size_t)i * n + j) * n + k) * NLN_EWALD_NQ);
            }
    return 0;
}

}  // namespace

// Both libraries compile this file: libnlnhost.so exports the two entry
// points of nlnhost.h; libgravcuda.so includes it with NLN_EWALD_NO_EXPORT
// and calls ewald_table() internally.
#ifndef NLN_EWALD_NO_EXPORT
extern "C" void nln_ewald_eval(double L, const double *y, double *out) { ewald_eval(L, y, out); }
extern "C" int nln_ewald_table(double L, int n, double reach, double *out) {
    return ewald_table(L, n, reach, out);
}
#endif
