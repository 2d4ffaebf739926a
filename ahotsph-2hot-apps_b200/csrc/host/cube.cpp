// cube.cpp -- the field of a uniform-density cube, the sink-side piece of
// background subtraction: the reference subtracts the mean density from
// the cells a walk opens and adds back, per sink, the exact field of the
// uniform cube of its near zone (nln/mac.c:688-706, with cubic_acc of
// nln/ewald_le2.c:773-1033 scaled by -rho0).
//
// Restated from the closed form of a rectangular prism's attraction (the
// potential's integrand integrated over two axes, then differenced over the
// eight corners): with u = corner - sink, r = |u|,
//   acc_x = -sum_{ijk} (-1)^(i+j+k) [ y ln(z + r) + z ln(y + r) - x atan(y z / (x r)) ]
// over the corners (x_i, y_j, z_k), i, j, k in {1, 2} (1 = low face), and
// cyclically for y and z.  FP64 throughout; the logarithms use
// ln(z + r) = ln((x^2 + y^2) / (r - z)) where z < 0 to avoid cancellation,
// and terms whose coefficient vanishes on an edge or a face are zero (their
// limit).
#include <math.h>

#include "nlnhost.h"

namespace {

// y ln(z + r): the limit 0 where y = 0 (also where z + r = 0).
double ylog(double y, double z, double r, double rho2) {
    if (y == 0.0)
        return 0.0;
    if (z >= 0.0)
        return y * log(z + r);
    if (rho2 == 0.0)
        return 0.0;
    return y * log(rho2 / (r - z));
}

// x atan(y z / (x r)): the limit 0 where x = 0 or r = 0.
double xatan(double x, double y, double z, double r) {
    if (x == 0.0 || r == 0.0)
        return 0.0;
    return x * atan(y * z / (x * r));
}

// The corner term for the x component, corner at (x, y, z) from the sink.
double corner_x(double x, double y, double z) {
    const double r = sqrt(x * x + y * y + z * z);
    return ylog(y, z, r, x * x + y * y) + ylog(z, y, r, x * x + z * z) - xatan(x, y, z, r);
}

}  // namespace

extern "C" void nln_cubic_acc(const double r[3], double a, double acc[3]) {
    // faces of the cube [-a, a]^3 relative to the sink
    const double lo[3] = {-a - r[0], -a - r[1], -a - r[2]};
    const double hi[3] = {a - r[0], a - r[1], a - r[2]};
    double s[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                const double x = i ? hi[0] : lo[0], y = j ? hi[1] : lo[1], z = k ? hi[2] : lo[2];
                const double sign = ((i + j + k) & 1) ? -1.0 : 1.0;  // (-1)^(i+j+k), 0 = low
                // the three components, each with its axis first
                s[0] += sign * corner_x(x, y, z);
                s[1] += sign * corner_x(y, z, x);
                s[2] += sign * corner_x(z, x, y);
            }
    // (with 0 for the low face, (-1)^(i+j+k) already carries the leading
    // minus of the 1-based form)
    for (int d = 0; d < 3; d++) acc[d] = s[d];
}
