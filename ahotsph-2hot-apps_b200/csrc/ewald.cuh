// ewald.cuh -- device side of the periodic correction.
//
// C(y) = Phi_Ewald(y) + 1/|y| (nln/ewald.c:13-64 minus the nearest-image
// Newtonian term) is smooth inside |y_k| < NLN_EWALD_REACH * L, so a sink
// group collects, over its list, the moments
//     M0 = sum m C(y_j),  M1 = sum m dC(y_j),  M2 = sum m ddC(y_j),  M3 = sum m dddC(y_j)
// at its centre (y_j = source centre - group centre, in the list's image)
// and each sink at offset u takes the Taylor expansion
//     phi_i = M0 - u.M1 + 1/2 u.M2.u - 1/6 M3[uuu],   a_i = M1 - M2 u + 1/2 M3[uu].
// Values at y come from an FP64-built table of C and its first three
// derivatives on the positive octant (cubic symmetry), by a third-order
// Taylor expansion about the nearest node, in FP32.
// Component order (nlnlists.h): C | x y z | xx xy xz yy yz zz |
//                                xxx xxy xxz xyy xyz xzz yyy yyz yzz zzz
#pragma once

#include "common.cuh"

struct EwTab {
    const float *t;   // n^3 x NLN_EWALD_NQ
    int n;
    float h, inv_h;
};

// v = T[d, d] (vector) for symmetric T in the 10-component order
__device__ __forceinline__ void t_dd(const float *T, float dx, float dy, float dz, float *v) {
    const float xx = dx * dx, xy = 2.f * dx * dy, xz = 2.f * dx * dz, yy = dy * dy,
                yz = 2.f * dy * dz, zz = dz * dz;
    v[0] = T[0] * xx + T[1] * xy + T[2] * xz + T[3] * yy + T[4] * yz + T[5] * zz;
    v[1] = T[1] * xx + T[3] * xy + T[4] * xz + T[6] * yy + T[7] * yz + T[8] * zz;
    v[2] = T[2] * xx + T[4] * xy + T[5] * xz + T[7] * yy + T[8] * yz + T[9] * zz;
}

// v = T[Q] (vector) for symmetric 3x3 Q given as xx xy xz yy yz zz
__device__ __forceinline__ void t_q(const float *T, const float *Q, float *v) {
    v[0] = T[0] * Q[0] + 2.f * T[1] * Q[1] + 2.f * T[2] * Q[2] + T[3] * Q[3] + 2.f * T[4] * Q[4] + T[5] * Q[5];
    v[1] = T[1] * Q[0] + 2.f * T[3] * Q[1] + 2.f * T[4] * Q[2] + T[6] * Q[3] + 2.f * T[7] * Q[4] + T[8] * Q[5];
    v[2] = T[2] * Q[0] + 2.f * T[4] * Q[1] + 2.f * T[5] * Q[2] + T[7] * Q[3] + 2.f * T[8] * Q[4] + T[9] * Q[5];
}

// M = T d (symmetric matrix xx xy xz yy yz zz)
__device__ __forceinline__ void t_d(const float *T, float dx, float dy, float dz, float *M) {
    M[0] = T[0] * dx + T[1] * dy + T[2] * dz;
    M[1] = T[1] * dx + T[3] * dy + T[4] * dz;
    M[2] = T[2] * dx + T[4] * dy + T[5] * dz;
    M[3] = T[3] * dx + T[6] * dy + T[7] * dz;
    M[4] = T[4] * dx + T[7] * dy + T[8] * dz;
    M[5] = T[5] * dx + T[8] * dy + T[9] * dz;
}

// w = H d
__device__ __forceinline__ void h_d(const float *H, float dx, float dy, float dz, float *w) {
    w[0] = H[0] * dx + H[1] * dy + H[2] * dz;
    w[1] = H[1] * dx + H[3] * dy + H[4] * dz;
    w[2] = H[2] * dx + H[4] * dy + H[5] * dz;
}

// C and its derivatives at y (20 floats, component order above).
__device__ __forceinline__ void ew_lookup(const EwTab &E, float yx, float yy, float yz,
                                          float *o) {
    const float sx = yx < 0.f ? -1.f : 1.f, sy = yy < 0.f ? -1.f : 1.f, sz = yz < 0.f ? -1.f : 1.f;
    const float ax = fabsf(yx), ay = fabsf(yy), az = fabsf(yz);
    const int nm = E.n - 1;
    const int i = min(__float2int_rn(ax * E.inv_h), nm);
    const int j = min(__float2int_rn(ay * E.inv_h), nm);
    const int k = min(__float2int_rn(az * E.inv_h), nm);
    const float dx = ax - i * E.h, dy = ay - j * E.h, dz = az - k * E.h;
    const float4 *p = reinterpret_cast<const float4 *>(E.t + (((size_t)i * E.n + j) * E.n + k) * 20);
    float t[20];
#pragma unroll
    for (int q = 0; q < 5; q++) {
        float4 v = __ldg(p + q);
        t[4 * q] = v.x;
        t[4 * q + 1] = v.y;
        t[4 * q + 2] = v.z;
        t[4 * q + 3] = v.w;
    }
    const float *G0 = t + 1, *H0 = t + 4, *T0 = t + 10;
    float Tdd[3], Td[6], Hd[3];
    t_dd(T0, dx, dy, dz, Tdd);
    t_d(T0, dx, dy, dz, Td);
    h_d(H0, dx, dy, dz, Hd);
    // C
    o[0] = t[0] + G0[0] * dx + G0[1] * dy + G0[2] * dz +
           0.5f * (Hd[0] * dx + Hd[1] * dy + Hd[2] * dz) +
           (1.f / 6.f) * (Tdd[0] * dx + Tdd[1] * dy + Tdd[2] * dz);
    // gradient
    o[1] = sx * (G0[0] + Hd[0] + 0.5f * Tdd[0]);
    o[2] = sy * (G0[1] + Hd[1] + 0.5f * Tdd[1]);
    o[3] = sz * (G0[2] + Hd[2] + 0.5f * Tdd[2]);
    // Hessian
    o[4] = H0[0] + Td[0];
    o[5] = sx * sy * (H0[1] + Td[1]);
    o[6] = sx * sz * (H0[2] + Td[2]);
    o[7] = H0[3] + Td[3];
    o[8] = sy * sz * (H0[4] + Td[4]);
    o[9] = H0[5] + Td[5];
    // third derivatives: component xyz picks up sx^nx sy^ny sz^nz
    o[10] = sx * T0[0];
    o[11] = sy * T0[1];
    o[12] = sz * T0[2];
    o[13] = sx * T0[3];
    o[14] = sx * sy * sz * T0[4];
    o[15] = sx * T0[5];
    o[16] = sy * T0[6];
    o[17] = sz * T0[7];
    o[18] = sy * T0[8];
    o[19] = sz * T0[9];
}

// Evaluate a group's correction moments M (20, FP64) at sink offset u: (phi, a).
__device__ __forceinline__ void ew_apply(const double *M, double ux, double uy, double uz,
                                         double &phi, double &axx, double &ayy, double &azz) {
    const double *M1 = M + 1, *H = M + 4, *T = M + 10;
    const double Mu0 = H[0] * ux + H[1] * uy + H[2] * uz;
    const double Mu1 = H[1] * ux + H[3] * uy + H[4] * uz;
    const double Mu2 = H[2] * ux + H[4] * uy + H[5] * uz;
    const double xx = ux * ux, xy = 2 * ux * uy, xz = 2 * ux * uz, yy = uy * uy,
                 yz = 2 * uy * uz, zz = uz * uz;
    const double T0 = T[0] * xx + T[1] * xy + T[2] * xz + T[3] * yy + T[4] * yz + T[5] * zz;
    const double T1 = T[1] * xx + T[3] * xy + T[4] * xz + T[6] * yy + T[7] * yz + T[8] * zz;
    const double T2 = T[2] * xx + T[4] * xy + T[5] * xz + T[7] * yy + T[8] * yz + T[9] * zz;
    phi = M[0] - (M1[0] * ux + M1[1] * uy + M1[2] * uz) + 0.5 * (Mu0 * ux + Mu1 * uy + Mu2 * uz) -
          (T0 * ux + T1 * uy + T2 * uz) / 6.0;
    axx = M1[0] - Mu0 + 0.5 * T0;
    ayy = M1[1] - Mu1 + 0.5 * T1;
    azz = M1[2] - Mu2 + 0.5 * T2;
}
