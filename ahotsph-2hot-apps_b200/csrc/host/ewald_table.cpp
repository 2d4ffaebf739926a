// ewald_table.cpp -- FP64 table of the periodic correction to the Newtonian
// potential, with its first five derivatives, for the batched kernels'
// Ewald term and for the FP64 direct-sum measurement.
//
// The periodic Green's function is the Ewald sum of nln/ewald.c:13-64
// (alpha = 2/L, real-space images, k-space waves with |h|^2 <= 16, the
// constant pi/(alpha^2 L^3)); for a source at displacement y (source - sink)
//   Phi_per(y) = pi/(alpha^2 L^3) - sum_n erfc(alpha |y-nL|)/|y-nL|
//                - sum_{h != 0} exp(-pi^2 h^2/(alpha L)^2) cos(2 pi h.y/L) / (pi L h^2)
// and its gradient is the force of ewald() on the sink.  The table holds
//   C(y) = Phi_per(y) + 1/|y|      (the n = 0 term becomes erf(alpha r)/r)
// which is smooth in |y_k| < L.
//
// Every derivative is analytic.  A radial g(r) differentiates through
// D^k g, D = (1/r) d/dr: the derivative with multi-index alpha (|alpha| = n)
// is the sum over partial pairings of its n indices, a pairing with p
// pairs contributing D^(n-p) g times the product of the paired deltas and
// of x over the unpaired indices.  For erfc(alpha r)/r the D^k follow the
// recurrence B_0 = erfc(alpha r)/r,
//   B_k = ((2k-1) B_(k-1) + (2 alpha^2)^k exp(-alpha^2 r^2) / (alpha sqrt(pi))) / r^2,
// with D^k (erfc(alpha r)/r) = (-1)^k B_k; near r = 0 the n = 0 term
// erf(alpha r)/r is summed as a power series in q = r^2 (D = 2 d/dq).
// Plane waves differentiate through powers of k.  Real-space images are
// kept while erfc(alpha r) > 1e-17 (r < 3L), the same k-space cut as
// ewald().
#ifdef _OPENMP
#include <omp.h>
#endif

#include <cmath>
#include <cstdint>

#include "nlnlists.h"

namespace {

constexpr int kMaxOrder = 5;

// Component layout (nlnlists.h): order n starts at n(n+1)(n+2)/6 and lists
// the multi-indices (ax, ay, az), ax + ay + az = n, with the sorted index
// tuples in lexicographic order, i.e. at offset (n-ax)(n-ax+1)/2 + az.
int comp_base(int n) { return n * (n + 1) * (n + 2) / 6; }
int comp_off(int n, int ax, int az) { return (n - ax) * (n - ax + 1) / 2 + az; }

// D^k g for k = 0..kMaxOrder at radius r
struct Rad {
    double d[kMaxOrder + 1];
};

// g(r) = -erfc(alpha r)/r
Rad rad_erfc(double r, double alpha) {
    const double r2 = r * r;
    const double ex = std::exp(-alpha * alpha * r2) / (alpha * std::sqrt(M_PI));
    double B = std::erfc(alpha * r) / r, p = 1.0;
    Rad o;
    o.d[0] = -B;
    for (int k = 1; k <= kMaxOrder; k++) {
        p *= 2.0 * alpha * alpha;
        B = ((2 * k - 1) * B + p * ex) / r2;
        o.d[k] = (k & 1) ? B : -B;  // -(-1)^k B_k
    }
    return o;
}

// g(r) = erf(alpha r)/r = c P(q), q = r^2, c = 2 alpha/sqrt(pi),
// P(q) = sum_n (-1)^n alpha^(2n) q^n / (n! (2n+1)); D^k g = 2^k c P^(k)(q)
// (all regular at r = 0).
Rad rad_erf_series(double r, double alpha) {
    const double c = 2.0 * alpha / std::sqrt(M_PI);
    const double q = r * r, a2 = alpha * alpha;
    double P[kMaxOrder + 1] = {};
    double coef = 1.0;  // (-1)^n alpha^(2n) / n!
    for (int n = 0; n < 40; n++) {
        const double pn = coef / (2 * n + 1);
        // k-th derivative of q^n: n!/(n-k)! q^(n-k)
        double f = 1.0;
        for (int k = 0; k <= kMaxOrder && k <= n; k++) {
            P[k] += pn * f * std::pow(q, n - k);
            f *= (n - k);
        }
        coef *= -a2 / (n + 1);
        if (std::fabs(coef) * std::pow(q + 1e-300, n) < 1e-30 && n > 10)
            break;
    }
    Rad o;
    double s = c;
    for (int k = 0; k <= kMaxOrder; k++, s *= 2.0) o.d[k] = s * P[k];
    return o;
}

// g(r) = erf(alpha r)/r = 1/r - erfc(alpha r)/r, directly (alpha r >= 1);
// D^k (1/r) = (-1)^k (2k-1)!! / r^(2k+1)
Rad rad_erf_direct(double r, double alpha) {
    Rad o = rad_erfc(r, alpha);
    const double r2 = r * r;
    double v = 1.0 / r;
    for (int k = 0; k <= kMaxOrder; k++) {
        o.d[k] += v;
        v *= -(2 * k + 1) / r2;
    }
    return o;
}

// Sum over partial pairings of the index list I[0..n): for each set of
// disjoint pairs, delta products times x over the unpaired indices times
// D^(n - pairs) g.  n <= 5, so a plain recursion is enough.
double pair_sum(const int *I, int n, const double x[3], const Rad &R, unsigned used, int pairs) {
    int first = -1;
    for (int a = 0; a < n; a++)
        if (!(used & (1u << a))) {
            first = a;
            break;
        }
    if (first < 0)
        return R.d[n - pairs];
    // `first` stays unpaired ...
    double s = x[I[first]] * pair_sum(I, n, x, R, used | (1u << first), pairs);
    // ... or pairs with a later free index of the same axis
    for (int b = first + 1; b < n; b++)
        if (!(used & (1u << b)) && I[b] == I[first])
            s += pair_sum(I, n, x, R, used | (1u << first) | (1u << b), pairs + 1);
    return s;
}

// accumulate a radial term at displacement x into all NLN_EWALD_NQ outputs
void add_radial(const Rad &R, const double x[3], double *o) {
    for (int n = 0; n <= kMaxOrder; n++)
        for (int ax = n; ax >= 0; ax--)
            for (int ay = n - ax; ay >= 0; ay--) {
                const int az = n - ax - ay;
                int I[kMaxOrder];
                int k = 0;
                for (int a = 0; a < ax; a++) I[k++] = 0;
                for (int a = 0; a < ay; a++) I[k++] = 1;
                for (int a = 0; a < az; a++) I[k++] = 2;
                o[comp_base(n) + comp_off(n, ax, az)] += pair_sum(I, n, x, R, 0u, 0);
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
    // k space: -A cos(k.y), A = exp(-pi^2 h^2/(alpha L)^2)/(pi L h^2), k = 2 pi h / L;
    // the n-th derivative is -A k^alpha times cos, -sin, -cos, sin, ... at n = 0, 1, 2, 3
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
                const double trig[4] = {cs, -sn, -cs, sn};
                for (int n = 0; n <= kMaxOrder; n++)
                    for (int ax = n; ax >= 0; ax--)
                        for (int ay = n - ax; ay >= 0; ay--) {
                            const int az = n - ax - ay;
                            const double kp = std::pow(kv[0], ax) * std::pow(kv[1], ay) *
                                              std::pow(kv[2], az);
                            o[comp_base(n) + comp_off(n, ax, az)] -= A * kp * trig[n & 3];
                        }
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
