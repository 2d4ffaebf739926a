// adjoint.cuh -- the hand-written adjoint of the batched evaluation (no
// counterpart in the reference): for a loss L = sum_i w_i . a_i + u_i phi_i
// on the last evaluation's sinks, dL/dx and dL/dm of every body, with the
// interaction lists held fixed.
//
// Included once, at the end of batch.cu (after step.cuh): it works on the
// plan's tables and uses the tree links of the refit.
//
// Per pair (sink i, source e) with d = x_i - X_e and rho^2 = |d|^2 + eps^2,
// the forward of interact.cuh is phi = -m/rho + qsh rho^-5 d.Q.d (Q the
// staged quadrupole, -3 R^2 q2) and a = -grad_d phi.  With H = grad grad phi
// the pair's loss term -w.grad phi + u phi has
//     dL/dx_i = -(H w + u a) =: -t,     dL/dX_e = +t,
//     dL/dm   = -(w.d rho^-3 + u rho^-1),
//     dL/dQ   = qsh [(u rho^-5 + 5 (w.d) rho^-7) d d^T - rho^-5 (w d^T + d w^T)]
// (the last w.r.t. the full symmetric matrix, Frobenius dual).  Cells pass
// their adjoints to their bodies through M = sum m_b, X = sum m_b x_b / M
// and S2 = sum m_b y_b y_b^T (y_b = x_b - X), with staged Q = -3 (S2 - tr S2/3):
//     dL/dx_b += (m_b/M) Xbar + 2 m_b S2bar y_b,
//     dL/dm_b += Mbar + Xbar.y_b/M + y_b.S2bar.y_b,      S2bar = -3 (Qbar - tr Qbar/3).
//
// Work layout: one warp per work item (group, list kind, slice), as the
// forward's queues.  Each lane holds two sinks as an f32x2 pair and one
// record of a 32-record tile; records and their running source-side sums
// pass round the 16 lanes of each half-warp (k_adjoint_points,
// k_adjoint_quads), so every record meets every sink without shared memory.
// Record sums are flushed with FP64 atomics once per tile, sink sums once
// per item.
#pragma once

namespace {

constexpr int kAdjTile = 32;

struct AdjProblem {
    const float4 *points;
    const nln_qcell *qcells;
    const nln_group *groups;
    const uint32_t *list[2];
    const Item *items[2];
    int nitems[2];
    int *counters;
    const float4 *wu;        // (wx, wy, wz, u) per sink, tree order
    double *gbody;           // 4 per body: dL/dx (3), dL/dm
    double *gcell;           // 10 per cell: Mbar, Xbar (3), Qbar (xx xy xz yy yz zz)
    int64_t nbodies;
    float eps2, qsh;
    unsigned *err;
};

// The point-list adjoint (bodies and cell monopoles), systolic.  Lane l
// holds sinks 2j and 2j+1 (j = l mod 16) and one record of the tile of 32
// in registers (half h = l / 16 takes records 16h..16h+15).
// At each of 16 steps every lane evaluates its two sinks against the record
// it holds, adds their source-side terms to the record's running sums, and
// passes record and sums to the next lane of its half (8 shuffles); after
// 16 steps every record has met all 32 sinks and its sums are back with
// their owner lane, which flushes them with FP64 atomics.  No shared memory:
// per-record shared slots cost 8-12 shared-memory wavefronts per step of
// 32 interactions and bound that form at 29.6 ms on the N = 2^20 Plummer
// case (this one: about 19 ms).  Plain FP32: the same loop with the two
// sinks as an f32x2 pair measured 9 % slower.
__global__ void __launch_bounds__(256) k_adjoint_points(AdjProblem P) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, j = lane & 15;
    const int next = (lane & 16) | ((j + 1) & 15);  // the lane this one takes its record from
    const uint32_t nb = (uint32_t)P.nbodies;
    while (true) {
        int it = 0;
        if (lane == 0)
            it = atomicAdd(&P.counters[KP], 1);
        it = __shfl_sync(FULL, it, 0);
        if (it >= P.nitems[KP])
            break;
        const Item item = P.items[KP][it];
        const nln_group G = P.groups[item.group];
        const double c[3] = {G.cen[0], G.cen[1], G.cen[2]};
        // sinks 2j, 2j+1 as pairs; a missing sink has w = u = 0 and adds nothing
        float s[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        float w[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int sk = 2 * j + h;
            if (sk < G.count) {
                const float4 p = P.points[G.first + sk];
                s[h][0] = (float)((double)p.x - c[0]);
                s[h][1] = (float)((double)p.y - c[1]);
                s[h][2] = (float)((double)p.z - c[2]);
                const float4 q = P.wu[G.first + sk];
                w[h][0] = q.x;
                w[h][1] = q.y;
                w[h][2] = q.z;
                w[h][3] = q.w;
            }
        }
        const float2 Sx = f2(s[0][0], s[1][0]), Sy = f2(s[0][1], s[1][1]), Sz = f2(s[0][2], s[1][2]);
        const float2 Wx = f2(w[0][0], w[1][0]), Wy = f2(w[0][1], w[1][1]), Wz = f2(w[0][2], w[1][2]);
        const float2 U = f2(w[0][3], w[1][3]), NU = f2(-w[0][3], -w[1][3]);
        const float2 e2 = splat2(P.eps2);
        float2 Gx = splat2(0.f), Gy = splat2(0.f), Gz = splat2(0.f);  // the sinks' sums of t
        // records are loaded a tile ahead of use and list entries two tiles
        // ahead, so a tile's loads overlap the previous tile's 16 steps
        auto entry = [&](int64_t b) -> uint32_t {
            return b + lane < item.end ? (P.list[0][b + lane] & NLN_IDX_MASK) : 0xffffffffu;
        };
        auto record = [&](uint32_t e) -> float4 {
            return e != 0xffffffffu ? __ldg(P.points + e) : make_float4(0.f, 0.f, 0.f, 0.f);
        };
        uint32_t e_cur = entry(item.begin), e_next = entry(item.begin + kAdjTile);
        float4 p_cur = record(e_cur);
        for (int64_t b0 = item.begin; b0 < item.end; b0 += kAdjTile) {
            const int nt = (int)min((int64_t)kAdjTile, item.end - b0);
            const float4 p_next = record(e_next);
            const uint32_t e_after = entry(b0 + 2 * kAdjTile);
            // this lane's record, negated position relative to the centre
            const uint32_t idx = e_cur;
            float nx = -1.0e3f, ny = -1.0e3f, nz = -1.0e3f, m = 0.f;  // massless and far: adds 0
            if (lane < nt) {
                nx = (float)(c[0] - (double)p_cur.x);
                ny = (float)(c[1] - (double)p_cur.y);
                nz = (float)(c[2] - (double)p_cur.z);
                m = p_cur.w;
            }
            e_cur = e_next;
            e_next = e_after;
            p_cur = p_next;
            float ax = 0.f, ay = 0.f, az = 0.f, am = 0.f;  // the record's sums of t, w.d/r^3 + u/r
#pragma unroll 4
            for (int k = 0; k < 16; k++) {
#pragma unroll
                for (int hh = 0; hh < 2; hh++) {
                    const float sx_ = hh ? Sx.y : Sx.x, sy_ = hh ? Sy.y : Sy.x, sz_ = hh ? Sz.y : Sz.x;
                    const float wx_ = hh ? Wx.y : Wx.x, wy_ = hh ? Wy.y : Wy.x, wz_ = hh ? Wz.y : Wz.x;
                    const float u_ = hh ? U.y : U.x;
                    const float dx = sx_ + nx, dy = sy_ + ny, dz = sz_ + nz;
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, e2.x)));
                    const float ri = rsqrt_fast(r2), ri2 = ri * ri;
                    const float mr3 = m * ri * ri2;
                    const float wd = fmaf(wx_, dx, fmaf(wy_, dy, wz_ * dz));
                    const float in = fmaf(-3.f * ri2, wd, -u_);
                    const float ex = fmaf(in, dx, wx_), ey = fmaf(in, dy, wy_), ez = fmaf(in, dz, wz_);
                    const float tx = mr3 * ex, ty = mr3 * ey, tz = mr3 * ez;
                    if (hh) { Gx.y += tx; Gy.y += ty; Gz.y += tz; } else { Gx.x += tx; Gy.x += ty; Gz.x += tz; }
                    ax += tx;
                    ay += ty;
                    az += tz;
                    am = fmaf(ri, fmaf(wd, ri2, u_), am);
                }
                nx = __shfl_sync(FULL, nx, next);
                ny = __shfl_sync(FULL, ny, next);
                nz = __shfl_sync(FULL, nz, next);
                m = __shfl_sync(FULL, m, next);
                ax = __shfl_sync(FULL, ax, next);
                ay = __shfl_sync(FULL, ay, next);
                az = __shfl_sync(FULL, az, next);
                am = __shfl_sync(FULL, am, next);
            }
            if (lane < nt) {
                if (idx < nb) {
                    double *g = P.gbody + (size_t)idx * 4;
                    atomicAdd(g + 0, (double)ax);
                    atomicAdd(g + 1, (double)ay);
                    atomicAdd(g + 2, (double)az);
                    atomicAdd(g + 3, -(double)am);
                } else {
                    double *g = P.gcell + (size_t)(idx - nb) * 10;
                    atomicAdd(g + 0, -(double)am);
                    atomicAdd(g + 1, (double)ax);
                    atomicAdd(g + 2, (double)ay);
                    atomicAdd(g + 3, (double)az);
                }
            }
        }
        // the two halves met different records: add their sink sums
        float g6[6] = {Gx.x, Gx.y, Gy.x, Gy.y, Gz.x, Gz.y};
#pragma unroll
        for (int q = 0; q < 6; q++) g6[q] += __shfl_xor_sync(FULL, g6[q], 16);
        if (lane < 16) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int sk = 2 * j + h;
                if (sk < G.count) {
                    double *g = P.gbody + (size_t)(G.first + sk) * 4;
                    atomicAdd(g + 0, -(double)g6[h]);
                    atomicAdd(g + 1, -(double)g6[2 + h]);
                    atomicAdd(g + 2, -(double)g6[4 + h]);
                }
            }
        }
    }
}

#ifndef GRAV_ADJQ_UNROLL
#define GRAV_ADJQ_UNROLL 2
#endif
constexpr int kAdjQUnroll = GRAV_ADJQ_UNROLL;

// The quadrupole-list adjoint, systolic like k_adjoint_points: each record
// (negated centre offset, mass, the six staged Q components) travels through
// the 16 lanes of its half with its ten running sums (t, w.d/r^3 + u/r and
// dL/dQ), 20 shuffles per step of 64 interactions.
__global__ void __launch_bounds__(256) k_adjoint_quads(AdjProblem P) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, j = lane & 15;
    const int next = (lane & 16) | ((j + 1) & 15);
    const float2 h = splat2(P.qsh);
    while (true) {
        int it = 0;
        if (lane == 0)
            it = atomicAdd(&P.counters[KQ], 1);
        it = __shfl_sync(FULL, it, 0);
        if (it >= P.nitems[KQ])
            break;
        const Item item = P.items[KQ][it];
        const nln_group G = P.groups[item.group];
        const double c[3] = {G.cen[0], G.cen[1], G.cen[2]};
        float s[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        float w[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
        for (int hh = 0; hh < 2; hh++) {
            const int sk = 2 * j + hh;
            if (sk < G.count) {
                const float4 p = P.points[G.first + sk];
                s[hh][0] = (float)((double)p.x - c[0]);
                s[hh][1] = (float)((double)p.y - c[1]);
                s[hh][2] = (float)((double)p.z - c[2]);
                const float4 q = P.wu[G.first + sk];
                w[hh][0] = q.x;
                w[hh][1] = q.y;
                w[hh][2] = q.z;
                w[hh][3] = q.w;
            }
        }
        const float2 Sx = f2(s[0][0], s[1][0]), Sy = f2(s[0][1], s[1][1]), Sz = f2(s[0][2], s[1][2]);
        const float2 Wx = f2(w[0][0], w[1][0]), Wy = f2(w[0][1], w[1][1]), Wz = f2(w[0][2], w[1][2]);
        const float2 U = f2(w[0][3], w[1][3]);
        const float2 e2 = splat2(P.eps2);
        float2 Gx = splat2(0.f), Gy = splat2(0.f), Gz = splat2(0.f);
        auto entry = [&](int64_t b) -> uint32_t {
            return b + lane < item.end ? (P.list[1][b + lane] & NLN_IDX_MASK) : 0xffffffffu;
        };
        uint32_t e_cur = entry(item.begin), e_next = entry(item.begin + kAdjTile);
        for (int64_t b0 = item.begin; b0 < item.end; b0 += kAdjTile) {
            const int nt = (int)min((int64_t)kAdjTile, item.end - b0);
            const uint32_t idx = e_cur;
            float r[10];  // negated offset, mass, Qxx Qxy Qyy Qxz Qyz Qzz
#pragma unroll
            for (int q = 0; q < 10; q++) r[q] = 0.f;
            r[0] = r[1] = r[2] = -1.0e3f;  // massless, momentless and far: adds 0
            if (lane < nt) {
                const nln_qcell q = P.qcells[idx];
                r[0] = (float)(c[0] - q.cen[0]);
                r[1] = (float)(c[1] - q.cen[1]);
                r[2] = (float)(c[2] - q.cen[2]);
                r[3] = q.mass;
                const float q2[5] = {q.qxx, q.qxy, q.qyy, q.qxz, q.qyz};
                float o[12];
                stage_quad(o, q.R, q2);
#pragma unroll
                for (int k = 4; k < 10; k++) r[k] = o[k];
            }
            e_cur = e_next;
            e_next = entry(b0 + 2 * kAdjTile);
            float a[10];  // the record's sums: t (3), w.d/r^3 + u/r, dL/dQ (xx xy xz yy yz zz)
#pragma unroll
            for (int q = 0; q < 10; q++) a[q] = 0.f;
#pragma unroll kAdjQUnroll
            for (int k = 0; k < 16; k++) {
#pragma unroll
                for (int hh = 0; hh < 2; hh++) {
                    const float wx = hh ? Wx.y : Wx.x, wy = hh ? Wy.y : Wy.x, wz = hh ? Wz.y : Wz.x;
                    const float u = hh ? U.y : U.x, hq = h.x;
                    const float dx = (hh ? Sx.y : Sx.x) + r[0], dy = (hh ? Sy.y : Sy.x) + r[1];
                    const float dz = (hh ? Sz.y : Sz.x) + r[2], M = r[3];
                    const float Qxx = r[4], Qxy = r[5], Qyy = r[6], Qxz = r[7], Qyz = r[8], Qzz = r[9];
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, e2.x)));
                    const float ri = rsqrt_fast(r2), ri2 = ri * ri, ri3 = ri * ri2;
                    const float ri5 = ri3 * ri2, ri7 = ri5 * ri2, ri9 = ri7 * ri2;
                    const float wd = fmaf(wx, dx, fmaf(wy, dy, wz * dz));
                    // monopole: t = m ri3 (w + (-3 ri2 (w.d) - u) d)
                    const float in = fmaf(-3.f * ri2, wd, -u);
                    const float mr3 = M * ri3;
                    float tx = mr3 * fmaf(in, dx, wx), ty = mr3 * fmaf(in, dy, wy);
                    float tz = mr3 * fmaf(in, dz, wz);
                    // quadrupole: H_q w + u a_q, and dL/dQ
                    const float Qdx = fmaf(Qxx, dx, fmaf(Qxy, dy, Qxz * dz));
                    const float Qdy = fmaf(Qxy, dx, fmaf(Qyy, dy, Qyz * dz));
                    const float Qdz = fmaf(Qxz, dx, fmaf(Qyz, dy, Qzz * dz));
                    const float Qwx = fmaf(Qxx, wx, fmaf(Qxy, wy, Qxz * wz));
                    const float Qwy = fmaf(Qxy, wx, fmaf(Qyy, wy, Qyz * wz));
                    const float Qwz = fmaf(Qxz, wx, fmaf(Qyz, wy, Qzz * wz));
                    const float P2 = fmaf(dx, Qdx, fmaf(dy, Qdy, dz * Qdz));
                    const float Qdw = fmaf(wx, Qdx, fmaf(wy, Qdy, wz * Qdz));
                    const float ri7P2 = ri7 * P2;
                    const float kd = hq * fmaf(-10.f * ri7, Qdw, fmaf(35.f * ri9 * P2, wd, 5.f * u * ri7P2));
                    const float kq = hq * fmaf(-10.f * ri7, wd, -2.f * u * ri5);
                    const float kw = -5.f * hq * ri7P2;
                    const float k2 = 2.f * hq * ri5;
                    tx += fmaf(k2, Qwx, fmaf(kd, dx, fmaf(kq, Qdx, kw * wx)));
                    ty += fmaf(k2, Qwy, fmaf(kd, dy, fmaf(kq, Qdy, kw * wy)));
                    tz += fmaf(k2, Qwz, fmaf(kd, dz, fmaf(kq, Qdz, kw * wz)));
                    // dL/dQ = h [(u ri5 + 5 (w.d) ri7) d d^T - ri5 (w d^T + d w^T)]
                    //       = P_i d_j + Bw_j d_i with P = A d + B w, Bw = B w
                    const float A = hq * fmaf(u, ri5, 5.f * wd * ri7), B = -hq * ri5;
                    const float Bwx = B * wx, Bwy = B * wy, Bwz = B * wz;
                    const float Px = fmaf(A, dx, Bwx), Py = fmaf(A, dy, Bwy), Pz = fmaf(A, dz, Bwz);
                    if (hh) {
                        Gx.y += tx;
                        Gy.y += ty;
                        Gz.y += tz;
                    } else {
                        Gx.x += tx;
                        Gy.x += ty;
                        Gz.x += tz;
                    }
                    a[0] += tx;
                    a[1] += ty;
                    a[2] += tz;
                    a[3] = fmaf(ri, fmaf(wd, ri2, u), a[3]);  // -dL/dm
                    a[4] = fmaf(Px, dx, fmaf(Bwx, dx, a[4]));
                    a[5] = fmaf(Px, dy, fmaf(Bwy, dx, a[5]));
                    a[6] = fmaf(Px, dz, fmaf(Bwz, dx, a[6]));
                    a[7] = fmaf(Py, dy, fmaf(Bwy, dy, a[7]));
                    a[8] = fmaf(Py, dz, fmaf(Bwz, dy, a[8]));
                    a[9] = fmaf(Pz, dz, fmaf(Bwz, dz, a[9]));
                }
#pragma unroll
                for (int q = 0; q < 10; q++) {
                    r[q] = __shfl_sync(FULL, r[q], next);
                    a[q] = __shfl_sync(FULL, a[q], next);
                }
            }
            if (lane < nt) {
                double *g = P.gcell + (size_t)idx * 10;
                atomicAdd(g + 0, -(double)a[3]);
                atomicAdd(g + 1, (double)a[0]);
                atomicAdd(g + 2, (double)a[1]);
                atomicAdd(g + 3, (double)a[2]);
#pragma unroll
                for (int q = 0; q < 6; q++) atomicAdd(g + 4 + q, (double)a[4 + q]);
            }
        }
        float g6[6] = {Gx.x, Gx.y, Gy.x, Gy.y, Gz.x, Gz.y};
#pragma unroll
        for (int q = 0; q < 6; q++) g6[q] += __shfl_xor_sync(FULL, g6[q], 16);
        if (lane < 16) {
#pragma unroll
            for (int hh = 0; hh < 2; hh++) {
                const int sk = 2 * j + hh;
                if (sk < G.count) {
                    double *g = P.gbody + (size_t)(G.first + sk) * 4;
                    atomicAdd(g + 0, -(double)g6[hh]);
                    atomicAdd(g + 1, -(double)g6[2 + hh]);
                    atomicAdd(g + 2, -(double)g6[4 + hh]);
                }
            }
        }
    }
}

// Bodies from their cells' adjoints: every ancestor of the body's leaf.
// A cell's centre and mass are read as the forward used them: the FP64
// centre of the quadrupole table when there is one, else the cell monopole
// of the point table.
__global__ void k_adjoint_bodies(const float4 *__restrict__ pts, const int32_t *__restrict__ leaf,
                                 const int32_t *__restrict__ parent, const nln_qcell *__restrict__ qc,
                                 const double *__restrict__ gcell, const double *__restrict__ gbody,
                                 int64_t n, float4 *__restrict__ out) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n)
        return;
    const float4 p = pts[b];
    double g[4] = {gbody[4 * b], gbody[4 * b + 1], gbody[4 * b + 2], gbody[4 * b + 3]};
    for (int32_t cidx = leaf[b]; cidx >= 0; cidx = parent[cidx]) {
        const double *A = gcell + (size_t)cidx * 10;
        if (A[0] == 0.0 && A[1] == 0.0 && A[2] == 0.0 && A[3] == 0.0 && A[4] == 0.0 &&
            A[5] == 0.0 && A[6] == 0.0 && A[7] == 0.0 && A[8] == 0.0 && A[9] == 0.0)
            continue;
        double X[3], M;
        if (qc) {
            X[0] = qc[cidx].cen[0];
            X[1] = qc[cidx].cen[1];
            X[2] = qc[cidx].cen[2];
            M = qc[cidx].mass;
        } else {
            const float4 cm = pts[n + cidx];
            X[0] = cm.x;
            X[1] = cm.y;
            X[2] = cm.z;
            M = cm.w;
        }
        if (M == 0.0)
            continue;
        const double y[3] = {(double)p.x - X[0], (double)p.y - X[1], (double)p.z - X[2]};
        // S2bar = -3 (Qbar - tr Qbar / 3)
        const double tr = (A[4] + A[7] + A[9]) / 3.0;
        const double S[6] = {-3.0 * (A[4] - tr), -3.0 * A[5], -3.0 * A[6], -3.0 * (A[7] - tr),
                             -3.0 * A[8], -3.0 * (A[9] - tr)};
        const double Sy[3] = {S[0] * y[0] + S[1] * y[1] + S[2] * y[2],
                              S[1] * y[0] + S[3] * y[1] + S[4] * y[2],
                              S[2] * y[0] + S[4] * y[1] + S[5] * y[2]};
        const double mb = p.w;
        for (int d = 0; d < 3; d++) g[d] += (mb / M) * A[1 + d] + 2.0 * mb * Sy[d];
        g[3] += A[0] + (A[1] * y[0] + A[2] * y[1] + A[3] * y[2]) / M +
                (y[0] * Sy[0] + y[1] * Sy[1] + y[2] * Sy[2]);
    }
    out[b] = make_float4((float)g[0], (float)g[1], (float)g[2], (float)g[3]);
}

}  // namespace

// Per-plan adjoint state (owned by the plan).
struct grav_adjoint_state {
    int32_t *leaf = nullptr, *parent = nullptr;
    double *gbody = nullptr, *gcell = nullptr;
    ~grav_adjoint_state() {
        for (void *p : {(void *)leaf, (void *)parent, (void *)gbody, (void *)gcell})
            if (p)
                cudaFree(p);
    }
};

void adjoint_state_free(grav_adjoint_state *A) { delete A; }

extern "C" int grav_plan_adjoint_CUDA(grav_plan *pl, const float *wu, float *grad, void *stream) {
    if (!pl || !wu || !grad)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: bad arguments");
    if (!pl->step)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: no tree links (grav_plan_set_tree_CUDA)");
    if (pl->hp.box > 0 || pl->dp.nitems[KH] > 0)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: isolated problems with monopole and "
                                  "quadrupole lists only (no order-4 cells, no periodic images)");
    if (pl->dp.nitems[KQ] > 0 && !pl->dp.qcells)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: no quadrupole table");
    if (pl->dp.qsh != 0.5f)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: the physical quadrupole potential "
                                  "(quad_phi_sign = +1) only");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t nb = pl->hp.nbodies, nc = pl->hp.ncells;
    grav_step_state *S = pl->step;
    if (!pl->adj) {
        auto *A = new grav_adjoint_state();
        // leaf of every body and parent of every cell, from the links
        std::vector<int32_t> child(nc), nchild(nc), parent(nc, -1), leaf(nb, -1);
        std::vector<int64_t> first(nc);
        std::vector<int32_t> count(nc);
        cudaError_t e = cudaMemcpy(child.data(), S->cchild, nc * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(nchild.data(), S->cnchild, nc * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(first.data(), S->cfirst, nc * 8, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(count.data(), S->ccount, nc * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            delete A;
            return gc::cuda_status(e, "grav_plan_adjoint_CUDA: links");
        }
        for (int64_t c = 0; c < nc; c++) {
            if (child[c] >= 0) {
                for (int32_t k = 0; k < nchild[c]; k++) parent[child[c] + k] = (int32_t)c;
            } else {
                for (int64_t b = first[c]; b < first[c] + count[c]; b++) leaf[b] = (int32_t)c;
            }
        }
        e = cudaMalloc((void **)&A->leaf, nb * 4);
        if (e == cudaSuccess)
            e = cudaMemcpy(A->leaf, leaf.data(), nb * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMalloc((void **)&A->parent, nc * 4);
        if (e == cudaSuccess)
            e = cudaMemcpy(A->parent, parent.data(), nc * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMalloc((void **)&A->gbody, nb * 4 * sizeof(double));
        if (e == cudaSuccess)
            e = cudaMalloc((void **)&A->gcell, nc * 10 * sizeof(double));
        if (e != cudaSuccess) {
            delete A;
            return gc::cuda_status(e, "grav_plan_adjoint_CUDA: scratch");
        }
        pl->adj = A;
    }
    grav_adjoint_state *A = pl->adj;
    GC_CHECK(cudaMemsetAsync(A->gbody, 0, nb * 4 * sizeof(double), st));
    GC_CHECK(cudaMemsetAsync(A->gcell, 0, nc * 10 * sizeof(double), st));
    GC_CHECK(cudaMemsetAsync(pl->dp.counters, 0, 4 * sizeof(int), st));
    AdjProblem P{};
    P.points = pl->dp.points;
    P.qcells = pl->dp.qcells;
    P.groups = pl->dp.groups;
    P.list[0] = pl->dp.list[KP];
    P.list[1] = pl->dp.list[KQ];
    P.items[0] = pl->dp.items[KP];
    P.items[1] = pl->dp.items[KQ];
    P.nitems[0] = pl->dp.nitems[KP];
    P.nitems[1] = pl->dp.nitems[KQ];
    P.counters = pl->dp.counters;
    P.wu = reinterpret_cast<const float4 *>(wu);
    P.gbody = A->gbody;
    P.gcell = A->gcell;
    P.nbodies = nb;
    P.eps2 = pl->dp.eps2;
    P.qsh = pl->dp.qsh;
    P.err = pl->dp.err;
    const unsigned blocks = (unsigned)pl->nsm * 4;
    if (P.nitems[0] > 0)
        k_adjoint_points<<<blocks, 256, 0, st>>>(P);
    if (P.nitems[1] > 0)
        k_adjoint_quads<<<blocks, 256, 0, st>>>(P);
    GC_CHECK(cudaGetLastError());
    k_adjoint_bodies<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(
        pl->dp.points, A->leaf, A->parent, pl->dp.qcells, A->gcell, A->gbody, nb,
        reinterpret_cast<float4 *>(grad));
    GC_CHECK(cudaGetLastError());
    return 0;
}
