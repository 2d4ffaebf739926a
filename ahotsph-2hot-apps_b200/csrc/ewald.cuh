// ewald.cuh -- device side of the periodic correction.
//
// C(y) = Phi_Ewald(y) + 1/|y| (nln/ewald.c:13-64 minus the nearest-image
// Newtonian term) is smooth inside |y_k| < NLN_EWALD_REACH * L, so a sink
// group collects, over its list, the moments
//     M_s[alpha] = sum_j sum_k sum_{|beta| = k} S_k,j[beta] D^(alpha+beta) C(y_j) / beta!,
// |alpha| = s = 0..4, at its centre (y_j = source centre - group centre, in
// the list's image; S_0 = m, S_1 = 0 about the centre of mass, S_2..S_4 the
// source's traceless second to fourth moments; their traces only meet the
// constant Laplacian of C).  A sink at offset u then takes the Taylor
// expansion
//     phi = sum_{|beta| <= 4} M[beta] (-u)^beta / beta!,
//     a_i = sum_{|beta| <= 3} M[e_i + beta] (-u)^beta / beta!.
// Values at y come from an FP64-built table of C and its first five
// derivatives on the positive octant (cubic symmetry), by a fourth-order
// Taylor expansion about the nearest node, in FP32.
//
// Multi-index layout (nlnlists.h): order n starts at n(n+1)(n+2)/6 and
// (ax, ay, az) sits at offset (ay+az)(ay+az+1)/2 + az within it.
#pragma once

#include "common.cuh"

namespace ew {

constexpr int kNode = 56;  // floats per table node: orders 0..5
constexpr int kNQ4 = 35;   // components of orders 0..4

__host__ __device__ constexpr int base(int n) { return n * (n + 1) * (n + 2) / 6; }
__host__ __device__ constexpr int idx(int ax, int ay, int az) {
    return base(ax + ay + az) + (ay + az) * (ay + az + 1) / 2 + az;
}
__host__ __device__ constexpr float ifact(int k) {
    return k == 0 ? 1.f : k == 1 ? 1.f : k == 2 ? 0.5f : k == 3 ? 1.f / 6.f : k == 4 ? 1.f / 24.f
                                                                                 : 1.f / 120.f;
}

}  // namespace ew

struct EwTab {
    const float *t;   // n^3 nodes x ew::kNode
    int n;
    float h, inv_h;
};

// d^beta / beta! for |beta| <= 4 (35 values, multi-index layout)
__device__ __forceinline__ void ew_monomials(float dx, float dy, float dz, float *mono) {
    float px[5], py[5], pz[5];
    px[0] = py[0] = pz[0] = 1.f;
#pragma unroll
    for (int k = 1; k < 5; k++) {
        px[k] = px[k - 1] * dx * (1.f / k);
        py[k] = py[k - 1] * dy * (1.f / k);
        pz[k] = pz[k - 1] * dz * (1.f / k);
    }
#pragma unroll
    for (int bx = 0; bx <= 4; bx++)
#pragma unroll
        for (int by = 0; by <= 4; by++)
#pragma unroll
            for (int bz = 0; bz <= 4; bz++)
                if (bx + by + bz <= 4)
                    mono[ew::idx(bx, by, bz)] = px[bx] * py[by] * pz[bz];
}

// The table node nearest |y| (the positive octant; C is even in each axis),
// the offsets of |y| from it and the octant signs of y.
struct EwNode {
    int node;              // node number: (i n + j) n + k
    float dx, dy, dz;      // |y| - node position
    float sx, sy, sz;      // signs of y's components
};

__device__ __forceinline__ EwNode ew_node(const EwTab &E, float yx, float yy, float yz) {
    EwNode r;
    r.sx = yx < 0.f ? -1.f : 1.f;
    r.sy = yy < 0.f ? -1.f : 1.f;
    r.sz = yz < 0.f ? -1.f : 1.f;
    const float ax = fabsf(yx), ay = fabsf(yy), az = fabsf(yz);
    const int nm = E.n - 1;
    const int i = min(__float2int_rn(ax * E.inv_h), nm);
    const int j = min(__float2int_rn(ay * E.inv_h), nm);
    const int k = min(__float2int_rn(az * E.inv_h), nm);
    r.dx = ax - i * E.h;
    r.dy = ay - j * E.h;
    r.dz = az - k * E.h;
    r.node = (i * E.n + j) * E.n + k;
    return r;
}

// The fifth derivatives at the node (21 floats, f5), octant signs applied,
// from the node's order-5 values V5 = V[35..55].
__device__ __forceinline__ void ew_fifth(const float *V5, const EwNode &N, float *f5) {
#pragma unroll
    for (int a0 = 0; a0 <= 5; a0++)
#pragma unroll
        for (int a1 = 0; a1 <= 5; a1++) {
            if (a0 + a1 > 5)
                continue;
            const int a2 = 5 - a0 - a1;
            const float sg = ((a0 & 1) ? N.sx : 1.f) * ((a1 & 1) ? N.sy : 1.f) *
                             ((a2 & 1) ? N.sz : 1.f);
            const int q = ew::idx(a0, a1, a2) - ew::base(5);
            f5[q] = sg * V5[q];
        }
}

// C and its derivatives of orders 0..4 at the point (35 floats, multi-index
// layout) from the node's values V (orders 0..4 in V[0..34], and 5 in
// V[35..55] when WANT5); with WANT5 also the fifth derivatives at the node
// (21 floats, f5).
template <bool WANT5>
__device__ __forceinline__ void ew_expand(const float *V, const EwNode &N, float *o, float *f5) {
    float mono[35];
    ew_monomials(N.dx, N.dy, N.dz, mono);
    // o[alpha] = sum_{|beta| <= 4 - |alpha|} V[alpha + beta] d^beta / beta!, then the octant
    // sign.  Every loop has constant bounds (guards fold after unrolling), so
    // the arrays stay in registers.
#pragma unroll
    for (int a0 = 0; a0 <= 4; a0++)
#pragma unroll
        for (int a1 = 0; a1 <= 4; a1++)
#pragma unroll
            for (int a2 = 0; a2 <= 4; a2++) {
                if (a0 + a1 + a2 > 4)
                    continue;
                float acc = 0.f;
#pragma unroll
                for (int b0 = 0; b0 <= 4; b0++)
#pragma unroll
                    for (int b1 = 0; b1 <= 4; b1++)
#pragma unroll
                        for (int b2 = 0; b2 <= 4; b2++)
                            if (a0 + a1 + a2 + b0 + b1 + b2 <= 4)
                                acc = fmaf(V[ew::idx(a0 + b0, a1 + b1, a2 + b2)],
                                           mono[ew::idx(b0, b1, b2)], acc);
                const float sg = ((a0 & 1) ? N.sx : 1.f) * ((a1 & 1) ? N.sy : 1.f) *
                                 ((a2 & 1) ? N.sz : 1.f);
                o[ew::idx(a0, a1, a2)] = sg * acc;
            }
    if (WANT5)
        ew_fifth(V + ew::base(5), N, f5);
}

// C and its derivatives at y by a fourth-order Taylor expansion about the
// nearest node of the table (ew_node + ew_expand on the node read from global
// memory).
template <bool WANT5>
__device__ __forceinline__ void ew_lookup(const EwTab &E, float yx, float yy, float yz, float *o,
                                          float *f5) {
    const EwNode N = ew_node(E, yx, yy, yz);
    const float4 *p = reinterpret_cast<const float4 *>(E.t + (size_t)N.node * ew::kNode);
    float V[WANT5 ? 56 : 36];
#pragma unroll
    for (int q = 0; q < (WANT5 ? 14 : 9); q++) {
        const float4 v = __ldg(p + q);
        V[4 * q] = v.x;
        V[4 * q + 1] = v.y;
        V[4 * q + 2] = v.z;
        V[4 * q + 3] = v.w;
    }
    ew_expand<WANT5>(V, N, o, f5);
}

// Group correction moments: orders 0..2 in FP64 (the net field is a small
// difference of O(1)-per-mass terms summed over thousands of entries), the
// u^2 and u^3 terms (orders 3, 4) in FP32.  One entry's terms of orders
// 0..2 (its mass and up to four folds) are first summed in FP32 (`cur`),
// which carries their own FP32 rounding anyway, and reach the FP64 sums once
// per entry (end_entry): one FP64 add per component and entry, not five.
struct EwMoments {
    double lo[10];
    float hi[25];
    float cur[10];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int q = 0; q < 10; q++) lo[q] = 0.0;
#pragma unroll
        for (int q = 0; q < 25; q++) hi[q] = 0.f;
#pragma unroll
        for (int q = 0; q < 10; q++) cur[q] = 0.f;
    }
    // rounded adds (never contracted with the product that forms v), so
    // every kernel that sums moments stores the same bits
    __device__ __forceinline__ void add(int q, float v) {
        if (q < 10)
            cur[q] = __fadd_rn(cur[q], v);
        else
            hi[q - 10] = __fadd_rn(hi[q - 10], v);
    }
    __device__ __forceinline__ void end_entry() {
#pragma unroll
        for (int q = 0; q < 10; q++) {
            lo[q] += (double)cur[q];
            cur[q] = 0.f;
        }
    }
    __device__ __forceinline__ double get(int q) const { return q < 10 ? lo[q] : (double)hi[q - 10]; }
    __device__ __forceinline__ void warp_sum() {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
#pragma unroll
            for (int q = 0; q < 10; q++) lo[q] += __shfl_xor_sync(0xffffffffu, lo[q], d);
#pragma unroll
            for (int q = 0; q < 25; q++) hi[q] += __shfl_xor_sync(0xffffffffu, hi[q], d);
        }
    }
};

// M_s[alpha] += sum_{|beta| = K} S[beta] D[alpha + beta] / beta!  for s = 0..SMAX,
// D = o (orders <= 4) and f5 (order 5); S in the multi-index layout of order K.
template <int K, int SMAX>
__device__ __forceinline__ void ew_fold(EwMoments &M, const float *S, const float *o, const float *f5) {
#pragma unroll
    for (int a0 = 0; a0 <= SMAX; a0++)
#pragma unroll
        for (int a1 = 0; a1 <= SMAX; a1++)
#pragma unroll
            for (int a2 = 0; a2 <= SMAX; a2++) {
                if (a0 + a1 + a2 > SMAX)
                    continue;
                float acc = 0.f;
#pragma unroll
                for (int b0 = 0; b0 <= K; b0++)
#pragma unroll
                    for (int b1 = 0; b1 <= K; b1++) {
                        if (b0 + b1 > K)
                            continue;
                        const int b2 = K - b0 - b1;
                        const int q = ew::idx(a0 + b0, a1 + b1, a2 + b2);
                        const float D = q < ew::kNQ4 ? o[q] : f5[q - ew::kNQ4];
                        acc = fmaf(S[ew::idx(b0, b1, b2) - ew::base(K)] *
                                       (ew::ifact(b0) * ew::ifact(b1) * ew::ifact(b2)),
                                   D, acc);
                    }
                M.add(ew::idx(a0, a1, a2), acc);
            }
}

// A source of mass m at the looked-up point: M_s += m D^alpha C.
__device__ __forceinline__ void ew_add_mass(EwMoments &M, float m, const float *o) {
#pragma unroll
    for (int q = 0; q < ew::kNQ4; q++) M.add(q, __fmul_rn(m, o[q]));
}

// Traceless second moment (multi-index layout xx xy xz yy yz zz) from the
// normalised quadrupole q2 = (xx, xy, yy, xz, yz) / R^2 of the cell tables.
__device__ __forceinline__ void ew_quad(float R, const float *q2, float *S2) {
    const float R2 = R * R;
    S2[0] = R2 * q2[0];
    S2[1] = R2 * q2[1];
    S2[2] = R2 * q2[3];
    S2[3] = R2 * q2[2];
    S2[4] = R2 * q2[4];
    S2[5] = -R2 * (q2[0] + q2[2]);
}

// Traceless third moment (10 components) from q3 = (xxx, xxy, xyy, yyy, xxz, xyz, yyz) / R^3.
__device__ __forceinline__ void ew_oct(float R, const float *q3, float *S3) {
    const float R3 = R * R * R;
    const float xxx = R3 * q3[0], xxy = R3 * q3[1], xyy = R3 * q3[2], yyy = R3 * q3[3],
                xxz = R3 * q3[4], xyz = R3 * q3[5], yyz = R3 * q3[6];
    S3[ew::idx(3, 0, 0) - 10] = xxx;
    S3[ew::idx(2, 1, 0) - 10] = xxy;
    S3[ew::idx(2, 0, 1) - 10] = xxz;
    S3[ew::idx(1, 2, 0) - 10] = xyy;
    S3[ew::idx(1, 1, 1) - 10] = xyz;
    S3[ew::idx(1, 0, 2) - 10] = -(xxx + xyy);
    S3[ew::idx(0, 3, 0) - 10] = yyy;
    S3[ew::idx(0, 2, 1) - 10] = yyz;
    S3[ew::idx(0, 1, 2) - 10] = -(xxy + yyy);
    S3[ew::idx(0, 0, 3) - 10] = -(xxz + yyz);
}

// Traceless fourth moment (15 components) from
// q4 = (xxxx, xxxy, xxyy, xyyy, yyyy, xxxz, xxyz, xyyz, yyyz) / R^4.
__device__ __forceinline__ void ew_hex(float R, const float *q4, float *S4) {
    const float R2 = R * R, R4 = R2 * R2;
    const float xxxx = R4 * q4[0], xxxy = R4 * q4[1], xxyy = R4 * q4[2], xyyy = R4 * q4[3],
                yyyy = R4 * q4[4], xxxz = R4 * q4[5], xxyz = R4 * q4[6], xyyz = R4 * q4[7],
                yyyz = R4 * q4[8];
    const float xxzz = -(xxxx + xxyy), yyzz = -(xxyy + yyyy);
    S4[ew::idx(4, 0, 0) - 20] = xxxx;
    S4[ew::idx(3, 1, 0) - 20] = xxxy;
    S4[ew::idx(3, 0, 1) - 20] = xxxz;
    S4[ew::idx(2, 2, 0) - 20] = xxyy;
    S4[ew::idx(2, 1, 1) - 20] = xxyz;
    S4[ew::idx(2, 0, 2) - 20] = xxzz;
    S4[ew::idx(1, 3, 0) - 20] = xyyy;
    S4[ew::idx(1, 2, 1) - 20] = xyyz;
    S4[ew::idx(1, 1, 2) - 20] = -(xxxy + xyyy);
    S4[ew::idx(1, 0, 3) - 20] = -(xxxz + xyyz);
    S4[ew::idx(0, 4, 0) - 20] = yyyy;
    S4[ew::idx(0, 3, 1) - 20] = yyyz;
    S4[ew::idx(0, 2, 2) - 20] = yyzz;
    S4[ew::idx(0, 1, 3) - 20] = -(xxyz + yyyz);
    S4[ew::idx(0, 0, 4) - 20] = -(xxzz + yyzz);
}

// Evaluate the group's correction moments at sink offset u: (phi, a), FP64.
__device__ __forceinline__ void ew_apply(const EwMoments &M, double ux, double uy, double uz,
                                         double &phi, double &axx, double &ayy, double &azz) {
    double px[5], py[5], pz[5];
    px[0] = py[0] = pz[0] = 1.0;
#pragma unroll
    for (int k = 1; k < 5; k++) {
        px[k] = px[k - 1] * (-ux) / k;
        py[k] = py[k - 1] * (-uy) / k;
        pz[k] = pz[k - 1] * (-uz) / k;
    }
    double p = 0.0, a[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int b0 = 0; b0 <= 4; b0++)
#pragma unroll
        for (int b1 = 0; b1 <= 4; b1++)
#pragma unroll
            for (int b2 = 0; b2 <= 4; b2++) {
                if (b0 + b1 + b2 > 4)
                    continue;
                const double w = px[b0] * py[b1] * pz[b2];
                p += M.get(ew::idx(b0, b1, b2)) * w;
                if (b0 + b1 + b2 <= 3) {
                    a[0] += M.get(ew::idx(b0 + 1, b1, b2)) * w;
                    a[1] += M.get(ew::idx(b0, b1 + 1, b2)) * w;
                    a[2] += M.get(ew::idx(b0, b1, b2 + 1)) * w;
                }
            }
    phi = p;
    axx = a[0];
    ayy = a[1];
    azz = a[2];
}
