// interact.cuh -- one sink against one staged source record, FP32.
//
// The arithmetic is the reference's multipole recurrence
// (do_gravph_avx8, nln/do_grav_avx8.c:1779-1904; pH, nln/pgrav.cu:49-213):
// with d = sink - source and the normalised traceless moments q_l / R^l,
// order l contributes
//     eq  = t_l * (q_l contracted with d^(l-1)),   t_l = -(2l-1)!! R^l / r^(2l+1)
//     phi += c_l eq.d,          c_l = 1/2, 1/3, 1/4
//     a   += d (2l+1) c_l eq.d / r^2 - eq
// The constant -(2l-1)!! R^l is folded into the moments once per source when
// a tile is staged (stage_* below), so the inner loop only multiplies by
// powers of 1/r.  Staged record layouts (floats, 16-byte aligned):
//   P (points, 4):      x y z m
//   Q (quadrupole, 12): x y z m | Qxx Qxy Qyy Qxz Qyz Qzz | - -
//   H (order 4, 32):    x y z m | Qxx Qxy Qyy Qxz Qyz Qzz | O[7] Osum1 Osum2 |
//                       X[9] Xsum | - - -
// with Q = -3 R^2 q2, O = -15 R^3 q3, X = -105 R^4 q4 and the sums
// Qzz = -(Qxx+Qyy), Osum1 = Oxxx+Oxyy, Osum2 = Oxxy+Oyyy, Xsum = Xxyyy+Xxxxy.
#pragma once

#include "common.cuh"

constexpr int REC_P = 4, REC_Q = 12, REC_H = 32;

struct Acc4 {
    float ax, ay, az, phi;
};

// Softening laws of the monopole term.
enum Soft { SOFT_PLUMMER = 0, SOFT_NONE = 1, SOFT_MASKED = 2, SOFT_K1 = 3 };

// Staging: raw fields -> folded record.  q2[5], q3[7], q4[9] in the
// reference order (qxx qxy qyy qxz qyz; qxxx qxxy qxyy qyyy qxxz qxyz qyyz;
// qxxxx qxxxy qxxyy qxyyy qyyyy qxxxz qxxyz qxyyz qyyyz).
__device__ __forceinline__ void stage_quad(float *o, float R, const float *q2) {
    const float c2 = -3.0f * R * R;
    float Qxx = c2 * q2[0], Qxy = c2 * q2[1], Qyy = c2 * q2[2], Qxz = c2 * q2[3],
          Qyz = c2 * q2[4];
    o[4] = Qxx;
    o[5] = Qxy;
    o[6] = Qyy;
    o[7] = Qxz;
    o[8] = Qyz;
    o[9] = -(Qxx + Qyy);
    o[10] = 0.0f;
    o[11] = 0.0f;
}

__device__ __forceinline__ void stage_hexa(float *o, float R, const float *q3, const float *q4) {
    const float c3 = -15.0f * R * R * R;
    const float c4 = -105.0f * R * R * R * R;
    float O[7], X[9];
#pragma unroll
    for (int k = 0; k < 7; k++) O[k] = c3 * q3[k];
#pragma unroll
    for (int k = 0; k < 9; k++) X[k] = c4 * q4[k];
#pragma unroll
    for (int k = 0; k < 7; k++) o[12 + k] = O[k];
    o[19] = O[0] + O[2];  // Oxxx + Oxyy
    o[20] = O[1] + O[3];  // Oxxy + Oyyy
#pragma unroll
    for (int k = 0; k < 9; k++) o[21 + k] = X[k];
    o[30] = X[3] + X[1];  // Xxyyy + Xxxxy
    o[31] = 0.0f;
}

// Monopole term: its potential pm and radial coefficient kr (the term adds
// pm to phi and d * kr to the acceleration), and ri = 1/r, ri2 for the
// higher orders.
template <int SOFT>
__device__ __forceinline__ void mono_terms(float x, float y, float z, float m, float e, float &pm,
                                           float &kr, float &ri, float &ri2) {
    if (SOFT == SOFT_PLUMMER || SOFT == SOFT_NONE) {
        // nln/do_grav_avx8.c:2181-2210, e = eps^2
        float r2 = fmaf(x, x, fmaf(y, y, SOFT == SOFT_PLUMMER ? fmaf(z, z, e) : z * z));
        ri = rsqrt_fast(r2);
        ri2 = ri * ri;
        float mri = m * ri;
        pm = -mri;
        kr = -mri * ri2;
    } else if (SOFT == SOFT_MASKED) {
        // do_grav_avx8: pairs closer than e contribute nothing (nln/do_grav_avx8.c:978-990)
        float r2 = fmaf(x, x, fmaf(y, y, z * z));
        ri = (r2 >= e * e) ? rsqrt_fast(r2) : 0.0f;
        ri2 = ri * ri;
        float mri = m * ri;
        pm = -mri;
        kr = -mri * ri2;
    } else {
        // Dehnen K1 inside r < eps, e = 1/eps (nln/do_grav_avx8.c:1013-1045, nln/pgrav.cu:441-461)
        float r2 = fmaf(x, x, fmaf(y, y, z * z));
        float pf, af;
        if (r2 * e * e < 1.0f) {
            float u2 = fmaf(r2, e * e, -1.0f);
            pf = fmaf(fmaf(fmaf(-45.0f / 32.0f, u2, 3.0f / 8.0f), u2, -0.5f), u2, 1.0f) * e;
            af = fmaf(fmaf(135.0f / 16.0f, u2, -1.5f), u2, 1.0f) * e * e * e;
            ri = 0.0f;
        } else {
            ri = rsqrt_fast(r2);
            pf = ri;
            af = ri * ri * ri;
        }
        ri2 = ri * ri;
        pm = -m * pf;
        kr = -m * af;
    }
}

template <int SOFT>
__device__ __forceinline__ void mono(float x, float y, float z, float m, float e, Acc4 &a,
                                     float &ri, float &ri2) {
    float pm, kr;
    mono_terms<SOFT>(x, y, z, m, e, pm, kr, ri, ri2);
    a.phi += pm;
    a.ax = fmaf(x, kr, a.ax);
    a.ay = fmaf(y, kr, a.ay);
    a.az = fmaf(z, kr, a.az);
}

// Quadrupole contraction: Q.d and d.Q.d.
__device__ __forceinline__ void quad_vec(float x, float y, float z, const float *__restrict__ r,
                                         float &Qx, float &Qy, float &Qz, float &dQd) {
    const float4 q0 = *reinterpret_cast<const float4 *>(r + 4);  // Qxx Qxy Qyy Qxz
    const float2 q1 = *reinterpret_cast<const float2 *>(r + 8);  // Qyz Qzz
    Qx = fmaf(q0.x, x, fmaf(q0.y, y, q0.w * z));
    Qy = fmaf(q0.y, x, fmaf(q0.z, y, q1.x * z));
    Qz = fmaf(q0.w, x, fmaf(q1.x, y, q1.y * z));
    dQd = fmaf(x, Qx, fmaf(y, Qy, z * Qz));
}

// Octupole and hexadecapole contractions with d^2 and d^3 (e, h) and their
// products with d (nln/do_grav_avx8.c:1853-1898), traceless moments.
__device__ __forceinline__ void hexa_vec(float x, float y, float z, const float *__restrict__ r,
                                         float e[3], float &d3, float h[3], float &d4) {
    const float4 o0 = *reinterpret_cast<const float4 *>(r + 12);  // Oxxx Oxxy Oxyy Oyyy
    const float4 o1 = *reinterpret_cast<const float4 *>(r + 16);  // Oxxz Oxyz Oyyz S1
    const float4 o2 = *reinterpret_cast<const float4 *>(r + 20);  // S2 Xxxxx Xxxxy Xxxyy
    const float4 x0 = *reinterpret_cast<const float4 *>(r + 24);  // Xxyyy Xyyyy Xxxxz Xxxyz
    const float4 x1 = *reinterpret_cast<const float4 *>(r + 28);  // Xxyyz Xyyyz XS -
    const float third = 1.0f / 3.0f;
    float xx = 0.5f * x * x, yy = 0.5f * y * y, zz = 0.5f * z * z;
    float xy = x * y, xz = x * z, yz = y * z;
    float xxx = x * fmaf(xx, third, -zz);
    float xxz = z * fmaf(zz, -third, xx);
    float yyy = y * fmaf(yy, third, -zz);
    float yyz = z * fmaf(zz, -third, yy);
    xx -= zz;
    yy -= zz;
    e[0] = fmaf(o0.x, xx, fmaf(o0.z, yy, fmaf(o0.y, xy, fmaf(o1.x, xz, o1.y * yz))));
    e[1] = fmaf(o0.z, xy, fmaf(o0.y, xx, fmaf(o0.w, yy, fmaf(o1.z, yz, o1.y * xz))));
    e[2] = fmaf(-o1.w, xz, fmaf(-o2.x, yz, fmaf(o1.x, xx, fmaf(o1.z, yy, o1.y * xy))));
    d3 = fmaf(x, e[0], fmaf(y, e[1], z * e[2]));
    float xxy = y * xx, xyy = x * yy, xyz = xy * z;
    // X order: xxxx(o2.y) xxxy(o2.z) xxyy(o2.w) xyyy(x0.x) yyyy(x0.y) xxxz(x0.z) xxyz(x0.w)
    //          xyyz(x1.x) yyyz(x1.y), XS = xyyy + xxxy (x1.z)
    h[0] = fmaf(o2.y, xxx, fmaf(x0.x, yyy, fmaf(o2.z, xxy, fmaf(x0.z, xxz,
           fmaf(o2.w, xyy, fmaf(x0.w, xyz, x1.x * yyz))))));
    h[1] = fmaf(x0.x, xyy, fmaf(o2.z, xxx, fmaf(x0.y, yyy, fmaf(x1.y, yyz,
           fmaf(o2.w, xxy, fmaf(x0.w, xxz, x1.x * xyz))))));
    h[2] = fmaf(-o2.y, xxz, fmaf(-x1.z, xyz, fmaf(-x0.y, yyz, fmaf(x0.z, xxx,
           fmaf(x1.y, yyy, fmaf(-o2.w, xxz + yyz, fmaf(x0.w, xxy, x1.x * xyy)))))));
    d4 = fmaf(x, h[0], fmaf(y, h[1], z * h[2]));
}

// One staged record of order ORDER (0, 2, 4) against a sink at (sx, sy, sz).
// The orders' terms are summed before they reach the accumulators: with
// eq_l = r^-(2l+1) (moment contracted with d^(l-1)),
//     phi += pm + qsh eq_2.d + eq_3.d/3 + eq_4.d/4
//     a   += d (kr + r^-2 (5 qsh' eq_2.d + 7/3 eq_3.d + 9/4 eq_4.d)) - (eq_2 + eq_3 + eq_4)
// (qsh' = 1/2: the acceleration does not take the potential's sign
// convention) and eq_2 + eq_3 + eq_4 = r^-5 (Q.d + r^-2 (e + r^-2 h)).
template <int ORDER, int SOFT>
__device__ __forceinline__ void interact(const float *__restrict__ r, float sx, float sy,
                                         float sz, float e, float qsh, Acc4 &a) {
    const float4 p = *reinterpret_cast<const float4 *>(r);
    float x = sx - p.x, y = sy - p.y, z = sz - p.z;
    float ri, ri2;
    if (ORDER == 0) {
        mono<SOFT>(x, y, z, p.w, e, a, ri, ri2);
        return;
    }
    float pm, kr;
    mono_terms<SOFT>(x, y, z, p.w, e, pm, kr, ri, ri2);
    float Qx, Qy, Qz, dQd;
    quad_vec(x, y, z, r, Qx, Qy, Qz, dQd);
    const float ri5 = ri * ri2 * ri2;
    const float eqd2 = ri5 * dQd;
    float tx = Qx, ty = Qy, tz = Qz, K;
    if (ORDER >= 4) {
        float ev[3], hv[3], d3, d4;
        hexa_vec(x, y, z, r, ev, d3, hv, d4);
        const float ri7 = ri5 * ri2, ri9 = ri7 * ri2;
        const float eqd3 = ri7 * d3, eqd4 = ri9 * d4;
        a.phi = fmaf(0.25f, eqd4, fmaf(1.0f / 3.0f, eqd3, fmaf(qsh, eqd2, a.phi + pm)));
        K = fmaf(ri2, fmaf(2.25f, eqd4, fmaf(7.0f / 3.0f, eqd3, 2.5f * eqd2)), kr);
        tx = fmaf(ri2, fmaf(ri2, hv[0], ev[0]), Qx);
        ty = fmaf(ri2, fmaf(ri2, hv[1], ev[1]), Qy);
        tz = fmaf(ri2, fmaf(ri2, hv[2], ev[2]), Qz);
    } else {
        a.phi = fmaf(qsh, eqd2, a.phi + pm);
        K = fmaf(2.5f * ri2, eqd2, kr);
    }
    a.ax = fmaf(x, K, fmaf(-ri5, tx, a.ax));
    a.ay = fmaf(y, K, fmaf(-ri5, ty, a.ay));
    a.az = fmaf(z, K, fmaf(-ri5, tz, a.az));
}

// Two point records against one sink with Blackwell's paired FP32
// instructions (fma/add/mul .f32x2): the .x halves belong to one record,
// the .y halves to the other.  The records are staged as negated offsets,
// np = -(source - group centre), so d = s + np needs no negation; the
// accumulators hold +m/r and +d m/r^3 (the caller negates once per tile).
// Same Plummer arithmetic as mono<SOFT_PLUMMER>, element by element.
struct Acc2 {
    float2 nax, nay, naz, nphi;
};

__device__ __forceinline__ void mono2_plummer(float2 npx, float2 npy, float2 npz, float2 m,
                                              float2 sx, float2 sy, float2 sz, float2 e2,
                                              Acc2 &acc) {
    const float2 dx = __fadd2_rn(sx, npx), dy = __fadd2_rn(sy, npy), dz = __fadd2_rn(sz, npz);
    const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, e2)));
    const float2 ri = make_float2(rsqrt_fast(r2.x), rsqrt_fast(r2.y));
    const float2 ri2 = __fmul2_rn(ri, ri);
    const float2 mri = __fmul2_rn(m, ri);
    const float2 mri3 = __fmul2_rn(mri, ri2);
    acc.nphi = __fadd2_rn(acc.nphi, mri);
    acc.nax = __ffma2_rn(dx, mri3, acc.nax);
    acc.nay = __ffma2_rn(dy, mri3, acc.nay);
    acc.naz = __ffma2_rn(dz, mri3, acc.naz);
}

// Two order-4 records against one sink with the paired FP32 instructions,
// on a pair-interleaved tile: field f of records a (.x) and b (.y) sits at
// floats 2f, 2f+1 of the pair.  Fields: 0-2 position (group-centred), 3
// mass, 4-9 Q as in the staged record, 10 -(Xxxxx + Xxxyy), 11 -(Xyyyy +
// Xxxyy) (h_z's xxz and yyz coefficients, the traceless moment's zz-pair
// components folded in), 12-18 -O (the octupole negated), 19-20 the
// octupole sums (not negated), 21-29 X, 30 -XS, 31 unused.  Working in v = source - sink = -d with those signs folded in
// leaves no negation in the loop:
//   e'(v) = -O:vv (so v.e' = d.e), h(v) = -h(d), U = Q.v + r^-2 (e' + r^-2 h),
//   a   = v (m/r^3 - r^-2 (5/2 eq_2.d + 7/3 eq_3.d + 9/4 eq_4.d)) + r^-5 U,
//   -phi = m/r - qsh eq_2.d - eq_3.d/3 - eq_4.d/4   (accumulated negated),
// the terms of interact<4, SOFT_PLUMMER> in another order, element by element.
struct Acc2h {
    float2 ax, ay, az, nphi;
};

// The quadrupole counterpart on a pair-interleaved tile of 10 fields
// (position, mass, Q as staged): with v = -d and U = Q.v,
//   a = v (m/r^3 - 5/2 r^-2 eq_2.d) + r^-5 U,  -phi = m/r - qsh eq_2.d.
__device__ __forceinline__ void quad2_plummer(const float *__restrict__ pr, float2 nsx, float2 nsy,
                                              float2 nsz, float2 eps2, float2 nqsh, Acc2h &A);

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 splat2(float a) { return make_float2(a, a); }

__device__ __forceinline__ void hexa2_plummer(const float *__restrict__ pr, float2 nsx, float2 nsy,
                                              float2 nsz, float2 eps2, float2 nqsh, Acc2h &A) {
    const float4 *q = reinterpret_cast<const float4 *>(pr);
    float4 w = q[0];
    const float2 vx = __fadd2_rn(f2(w.x, w.y), nsx);
    const float2 vy = __fadd2_rn(f2(w.z, w.w), nsy);
    w = q[1];
    const float2 vz = __fadd2_rn(f2(w.x, w.y), nsz);
    const float2 m = f2(w.z, w.w);
    // monopole
    const float2 r2 = __ffma2_rn(vx, vx, __ffma2_rn(vy, vy, __ffma2_rn(vz, vz, eps2)));
    const float2 ri = f2(rsqrt_fast(r2.x), rsqrt_fast(r2.y));
    const float2 ri2 = __fmul2_rn(ri, ri);
    const float2 ri3 = __fmul2_rn(ri, ri2);  // shared by the monopole and the higher orders
    const float2 mri3 = __fmul2_rn(m, ri3);
    A.nphi = __ffma2_rn(m, ri, A.nphi);
    // quadrupole
    w = q[2];
    const float2 Qxx = f2(w.x, w.y), Qxy = f2(w.z, w.w);
    w = q[3];
    const float2 Qyy = f2(w.x, w.y), Qxz = f2(w.z, w.w);
    w = q[4];
    const float2 Qyz = f2(w.x, w.y), Qzz = f2(w.z, w.w);
    float2 Ux = __ffma2_rn(Qxx, vx, __ffma2_rn(Qxy, vy, __fmul2_rn(Qxz, vz)));
    float2 Uy = __ffma2_rn(Qxy, vx, __ffma2_rn(Qyy, vy, __fmul2_rn(Qyz, vz)));
    float2 Uz = __ffma2_rn(Qxz, vx, __ffma2_rn(Qyz, vy, __fmul2_rn(Qzz, vz)));
    const float2 vQv = __ffma2_rn(vx, Ux, __ffma2_rn(vy, Uy, __fmul2_rn(vz, Uz)));
    const float2 ri5 = __fmul2_rn(ri3, ri2);
    const float2 eqd2 = __fmul2_rn(ri5, vQv);
    // monomials of v (hexa_vec's, with -zz in place of zz)
    const float2 third = splat2(1.0f / 3.0f);
    float2 xx = __fmul2_rn(__fmul2_rn(splat2(0.5f), vx), vx);
    float2 yy = __fmul2_rn(__fmul2_rn(splat2(0.5f), vy), vy);
    const float2 nzz = __fmul2_rn(__fmul2_rn(splat2(-0.5f), vz), vz);
    const float2 xy = __fmul2_rn(vx, vy), xz = __fmul2_rn(vx, vz), yz = __fmul2_rn(vy, vz);
    const float2 xxx = __fmul2_rn(vx, __ffma2_rn(xx, third, nzz));
    const float2 xxz = __fmul2_rn(vz, __ffma2_rn(nzz, third, xx));
    const float2 yyy = __fmul2_rn(vy, __ffma2_rn(yy, third, nzz));
    const float2 yyz = __fmul2_rn(vz, __ffma2_rn(nzz, third, yy));
    xx = __fadd2_rn(xx, nzz);
    yy = __fadd2_rn(yy, nzz);
    // octupole (negated moments): e' and d3 = v.e'
    w = q[6];
    const float2 O0 = f2(w.x, w.y), O1 = f2(w.z, w.w);  // Oxxx Oxxy
    w = q[7];
    const float2 O2 = f2(w.x, w.y), O3 = f2(w.z, w.w);  // Oxyy Oyyy
    w = q[8];
    const float2 O4 = f2(w.x, w.y), O5 = f2(w.z, w.w);  // Oxxz Oxyz
    w = q[9];
    const float2 O6 = f2(w.x, w.y), S1 = f2(w.z, w.w);  // Oyyz, Oxxx+Oxyy
    w = q[10];
    const float2 S2 = f2(w.x, w.y), X0 = f2(w.z, w.w);  // Oxxy+Oyyy, Xxxxx
    const float2 e0 = __ffma2_rn(O0, xx, __ffma2_rn(O2, yy, __ffma2_rn(O1, xy, __ffma2_rn(O4, xz, __fmul2_rn(O5, yz)))));
    const float2 e1 = __ffma2_rn(O2, xy, __ffma2_rn(O1, xx, __ffma2_rn(O3, yy, __ffma2_rn(O6, yz, __fmul2_rn(O5, xz)))));
    const float2 e2 = __ffma2_rn(S1, xz, __ffma2_rn(S2, yz, __ffma2_rn(O4, xx, __ffma2_rn(O6, yy, __fmul2_rn(O5, xy)))));
    const float2 d3 = __ffma2_rn(vx, e0, __ffma2_rn(vy, e1, __fmul2_rn(vz, e2)));
    // hexadecapole: h(v) and d4 = v.h
    w = q[11];
    const float2 X1 = f2(w.x, w.y), X2 = f2(w.z, w.w);  // Xxxxy Xxxyy
    w = q[12];
    const float2 X3 = f2(w.x, w.y), X4 = f2(w.z, w.w);  // Xxyyy Xyyyy
    w = q[13];
    const float2 X5 = f2(w.x, w.y), X6 = f2(w.z, w.w);  // Xxxxz Xxxyz
    w = q[14];
    const float2 X7 = f2(w.x, w.y), X8 = f2(w.z, w.w);  // Xxyyz Xyyyz
    w = q[15];
    const float2 nXS = f2(w.x, w.y);
    w = q[5];
    const float2 nX02 = f2(w.x, w.y), nX42 = f2(w.z, w.w);
    const float2 xxy = __fmul2_rn(vy, xx), xyy = __fmul2_rn(vx, yy), xyz = __fmul2_rn(xy, vz);
    // each chain starts from xyz, the monomial ready first (two operations
    // from v; the others take four)
    const float2 h0 = __ffma2_rn(X0, xxx, __ffma2_rn(X3, yyy, __ffma2_rn(X1, xxy, __ffma2_rn(X5, xxz,
                      __ffma2_rn(X2, xyy, __ffma2_rn(X7, yyz, __fmul2_rn(X6, xyz)))))));
    const float2 h1 = __ffma2_rn(X3, xyy, __ffma2_rn(X1, xxx, __ffma2_rn(X4, yyy, __ffma2_rn(X8, yyz,
                      __ffma2_rn(X2, xxy, __ffma2_rn(X6, xxz, __fmul2_rn(X7, xyz)))))));
    const float2 h2 = __ffma2_rn(nX02, xxz, __ffma2_rn(nX42, yyz, __ffma2_rn(X5, xxx, __ffma2_rn(X8, yyy,
                      __ffma2_rn(X6, xxy, __ffma2_rn(X7, xyy, __fmul2_rn(nXS, xyz)))))));
    const float2 d4 = __ffma2_rn(vx, h0, __ffma2_rn(vy, h1, __fmul2_rn(vz, h2)));
    // sums of the orders
    const float2 ri7 = __fmul2_rn(ri5, ri2), ri9 = __fmul2_rn(ri7, ri2);
    const float2 eqd3 = __fmul2_rn(ri7, d3), eqd4 = __fmul2_rn(ri9, d4);
    A.nphi = __ffma2_rn(splat2(-0.25f), eqd4,
             __ffma2_rn(splat2(-1.0f / 3.0f), eqd3, __ffma2_rn(nqsh, eqd2, A.nphi)));
    const float2 Kn = __ffma2_rn(ri2, __ffma2_rn(splat2(-2.25f), eqd4,
                      __ffma2_rn(splat2(-7.0f / 3.0f), eqd3, __fmul2_rn(splat2(-2.5f), eqd2))), mri3);
    Ux = __ffma2_rn(ri2, __ffma2_rn(ri2, h0, e0), Ux);
    Uy = __ffma2_rn(ri2, __ffma2_rn(ri2, h1, e1), Uy);
    Uz = __ffma2_rn(ri2, __ffma2_rn(ri2, h2, e2), Uz);
    A.ax = __ffma2_rn(vx, Kn, __ffma2_rn(ri5, Ux, A.ax));
    A.ay = __ffma2_rn(vy, Kn, __ffma2_rn(ri5, Uy, A.ay));
    A.az = __ffma2_rn(vz, Kn, __ffma2_rn(ri5, Uz, A.az));
}

__device__ __forceinline__ void quad2_plummer(const float *__restrict__ pr, float2 nsx, float2 nsy,
                                              float2 nsz, float2 eps2, float2 nqsh, Acc2h &A) {
    const float4 *q = reinterpret_cast<const float4 *>(pr);
    float4 w = q[0];
    const float2 vx = __fadd2_rn(f2(w.x, w.y), nsx);
    const float2 vy = __fadd2_rn(f2(w.z, w.w), nsy);
    w = q[1];
    const float2 vz = __fadd2_rn(f2(w.x, w.y), nsz);
    const float2 m = f2(w.z, w.w);
    const float2 r2 = __ffma2_rn(vx, vx, __ffma2_rn(vy, vy, __ffma2_rn(vz, vz, eps2)));
    const float2 ri = f2(rsqrt_fast(r2.x), rsqrt_fast(r2.y));
    const float2 ri2 = __fmul2_rn(ri, ri);
    const float2 ri3 = __fmul2_rn(ri, ri2);  // shared by the monopole and quadrupole terms
    const float2 mri3 = __fmul2_rn(m, ri3);
    w = q[2];
    const float2 Qxx = f2(w.x, w.y), Qxy = f2(w.z, w.w);
    w = q[3];
    const float2 Qyy = f2(w.x, w.y), Qxz = f2(w.z, w.w);
    w = q[4];
    const float2 Qyz = f2(w.x, w.y), Qzz = f2(w.z, w.w);
    const float2 Ux = __ffma2_rn(Qxx, vx, __ffma2_rn(Qxy, vy, __fmul2_rn(Qxz, vz)));
    const float2 Uy = __ffma2_rn(Qxy, vx, __ffma2_rn(Qyy, vy, __fmul2_rn(Qyz, vz)));
    const float2 Uz = __ffma2_rn(Qxz, vx, __ffma2_rn(Qyz, vy, __fmul2_rn(Qzz, vz)));
    const float2 vQv = __ffma2_rn(vx, Ux, __ffma2_rn(vy, Uy, __fmul2_rn(vz, Uz)));
    const float2 ri5 = __fmul2_rn(ri3, ri2);
    const float2 eqd2 = __fmul2_rn(ri5, vQv);
    A.nphi = __ffma2_rn(nqsh, eqd2, __ffma2_rn(m, ri, A.nphi));
    const float2 Kn = __ffma2_rn(__fmul2_rn(splat2(-2.5f), ri2), eqd2, mri3);
    A.ax = __ffma2_rn(vx, Kn, __ffma2_rn(ri5, Ux, A.ax));
    A.ay = __ffma2_rn(vy, Kn, __ffma2_rn(ri5, Uy, A.ay));
    A.az = __ffma2_rn(vz, Kn, __ffma2_rn(ri5, Uz, A.az));
}
