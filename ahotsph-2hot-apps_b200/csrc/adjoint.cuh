// adjoint.cuh -- the hand-written adjoint of the batched evaluation (no
// counterpart in the reference): for a loss L = sum_i w_i . a_i + u_i phi_i
// on the last evaluation's sinks, dL/dx and dL/dm of every body, with the
// interaction lists held fixed.
//
// Included once, at the end of batch.cu (after step.cuh): it works on the
// plan's tables and uses the tree links of the refit.
//
// Pair terms.  With d = x_i - X_e (image shift included), rho^2 = |d|^2 +
// eps^2, a cell's term of order l = 2, 3, 4 is
//     phi_l = -g_l P_l rho^-n,   P_l = <A_l, d^l>,  n = 2l+1,  g_l = (2l-1)!!/l!,
// with A_l the trace-free l-th moment sum m (y^l) of the cell (y = x_b - X;
// the staged moments of interact.cuh are -(2l-1)!! A_l with the 1/l! of the
// contraction folded in), so a = -grad phi and H = grad grad phi follow from
// E_l = A_l.d^(l-1) and F_l = A_l.d^(l-2).  The pair's loss term
// -w.grad phi + u phi has
//     dL/dx_i = -t, dL/dX_e = +t,   t = H w + u a,
//     dL/dm   = -(w.d rho^-3 + u rho^-1),
//     dL/dA_l = g_l l sym(d^(l-1) (x) v_l),
//               v_l = rho^-n w - (n rho^-(n+2) (w.d) + u rho^-n) d / l
// (full-tensor duals: L changes by <dL/dA_l, dA_l>).
//
// Periodic correction.  A group's Taylor moments M[alpha] (ewald.cuh) give
// its sinks phi = sum M[b] (-u)^b/b!; the adjoint takes per group
// Mbar[alpha] = dL/dM[alpha] from its sinks (k_adjoint_ewald_groups, which
// also adds the sinks' own -t), then per correction entry at y = X + shift
// - c: dL/dm = Mbar.D C(y), dL/dX_l = sum N[g] D^(g+e_l) C(y) with
// N = m Mbar + the moments' convolution with Mbar, and dL/dA_K[b] =
// (1/K!) sum Mbar[a] D^(a+b) C(y) (k_adjoint_ewald_entries).  Derivatives
// of order 6, which the table does not hold, are dropped: they belong to
// the forward's order-5 terms, whose table values are constant inside a
// table cell.
//
// Cells to bodies.  M = sum m_b, X = sum m_b x_b / M, A_l = STF(sum m_b y_b^l)
// and B2 = sum m_b |y_b|^2 (the correction's trace term) give, with
// PG_l = STF(dL/dA_l) and f(y) = sum_l <PG_l, y^l> + B2bar |y|^2,
//     dL/dx_b += m_b grad f(y_b) + (m_b/M) Xbar',
//     dL/dm_b += Mbar + f(y_b) + Xbar'.y_b/M,
//     Xbar' = Xbar - 3 PG_3.A_2 - 4 PG_4.A_3
// (the moments' dependence on X; the dipole term vanishes about the centre
// of mass).  k_adjoint_cells forms PG_l and Xbar' once per cell,
// k_adjoint_bodies walks every body's ancestors.
//
// A body's pair with itself (in its own group's point list, d = 0) adds
// +t and -t to the same body and is left out of the position adjoint; its
// mass term (-u/eps) stays.
//
// Work layout: one warp per work item (group, list kind, slice), as the
// forward's queues.  Points and quadrupoles: each lane holds two sinks as
// an f32x2 pair and one record of a 32-record tile; records and their
// running source-side sums pass round the 16 lanes of each half-warp
// (k_adjoint_points, k_adjoint_quads), so every record meets every sink
// without shared memory.  Order 4: a lane holds one record and its 35
// running sums and meets the group's sinks one by one from shared memory
// (k_adjoint_hexa).  Record sums are flushed with FP64 atomics once per
// tile, sink sums once per item.
#pragma once
#include <type_traits>

namespace {

constexpr int kAdjTile = 32;
constexpr int kCellAdj = 36;  // doubles per cell: Mbar, Xbar (3), A_2, A_3, A_4 duals (6, 10, 15), B2bar
constexpr int kAdjG2 = 4, kAdjG3 = 10, kAdjG4 = 20, kAdjB2 = 35;

struct AdjProblem {
    const float4 *points;
    const nln_qcell *qcells;
    const nln_hcell *hcells;
    const nln_group *groups;
    const uint32_t *list[3];
    int64_t ntab[3];         // table sizes: list entries at or past them are skipped
    const Item *items[3];
    int nitems[3];
    int *counters;
    const float4 *wu;        // (wx, wy, wz, u) per sink, tree order
    double *gbody;           // 4 per body: dL/dx (3), dL/dm
    double *gcell;           // kCellAdj per cell
    int64_t nbodies, ngroups;
    float eps2, qsh;
    double box;
    unsigned *err;
    // periodic correction (ewald != 0)
    int ewald;
    const int64_t *cptr;
    const uint32_t *clist;
    EwTab ew;
    float ew_self, ew_trace;
    const EwStored *ewm;     // the forward's per-group moments
    double *mbar;            // 35 per group: dL/dM[alpha]
    double *gstf;            // kStfIndep per cell: the correction's trace-free moment duals
};

// Offset of the record at image code `code` relative to the group centre c,
// negated (c - (X + shift)), as the kernels below hold their records.
__device__ __forceinline__ void neg_offset(const double *X, uint32_t code, double box,
                                           const double *c, float &nx, float &ny, float &nz) {
    double sx, sy, sz;
    decode_shift(code, box, sx, sy, sz);
    nx = (float)(c[0] - (X[0] + sx));
    ny = (float)(c[1] - (X[1] + sy));
    nz = (float)(c[2] - (X[2] + sz));
}

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
            if (b + lane >= item.end)
                return 0xffffffffu;
            const uint32_t e = P.list[0][b + lane];
            return (e & NLN_IDX_MASK) < (uint32_t)P.ntab[0] && (e >> NLN_IDX_BITS) <= 26u ? e
                                                                                         : 0xffffffffu;
        };
        auto record = [&](uint32_t e) -> float4 {
            return e != 0xffffffffu ? __ldg(P.points + (e & NLN_IDX_MASK))
                                    : make_float4(0.f, 0.f, 0.f, 0.f);
        };
        uint32_t e_cur = entry(item.begin), e_next = entry(item.begin + kAdjTile);
        float4 p_cur = record(e_cur);
        for (int64_t b0 = item.begin; b0 < item.end; b0 += kAdjTile) {
            const int nt = (int)min((int64_t)kAdjTile, item.end - b0);
            const float4 p_next = record(e_next);
            const uint32_t e_after = entry(b0 + 2 * kAdjTile);
            // this lane's record, negated position relative to the centre
            const uint32_t idx = e_cur & NLN_IDX_MASK, e_prev_code = e_cur >> NLN_IDX_BITS;
            float nx = -1.0e3f, ny = -1.0e3f, nz = -1.0e3f, m = 0.f;  // massless and far: adds 0
            const bool live = lane < nt && e_cur != 0xffffffffu;
            if (live) {
                const double X[3] = {(double)p_cur.x, (double)p_cur.y, (double)p_cur.z};
                neg_offset(X, e_cur >> NLN_IDX_BITS, P.box, c, nx, ny, nz);
                m = p_cur.w;
            }
            e_cur = e_next;
            e_next = e_after;
            p_cur = p_next;
            float ax = 0.f, ay = 0.f, az = 0.f, am = 0.f;  // the record's sums of t, w.d/r^3 + u/r
            // A body against itself (d = 0: offsets of one point, exact
            // negatives) adds t on both sides of the same body; it is left
            // out, since the two FP32 sums would not cancel it exactly
            // (t = m w / eps^3).  Only tiles holding one of the group's own
            // bodies can meet it: those run the loop with the check.
            const bool own = live && (e_prev_code == NLN_SHIFT_NONE) &&
                             idx - (uint32_t)G.first < (uint32_t)G.count;
            auto steps = [&](auto self_c) {
                constexpr bool SELF = decltype(self_c)::value;
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
                        float mr3 = m * ri * ri2;
                        if (SELF && dx == 0.f && dy == 0.f && dz == 0.f)
                            mr3 = 0.f;
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
            };
            if (__any_sync(FULL, own))
                steps(std::true_type{});
            else
                steps(std::false_type{});
            if (live) {
                if (idx < nb) {
                    double *g = P.gbody + (size_t)idx * 4;
                    atomicAdd(g + 0, (double)ax);
                    atomicAdd(g + 1, (double)ay);
                    atomicAdd(g + 2, (double)az);
                    atomicAdd(g + 3, -(double)am);
                } else {
                    double *g = P.gcell + (size_t)(idx - nb) * kCellAdj;
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
            if (b + lane >= item.end)
                return 0xffffffffu;
            const uint32_t e = P.list[1][b + lane];
            return (e & NLN_IDX_MASK) < (uint32_t)P.ntab[1] && (e >> NLN_IDX_BITS) <= 26u ? e
                                                                                         : 0xffffffffu;
        };
        uint32_t e_cur = entry(item.begin), e_next = entry(item.begin + kAdjTile);
        for (int64_t b0 = item.begin; b0 < item.end; b0 += kAdjTile) {
            const int nt = (int)min((int64_t)kAdjTile, item.end - b0);
            const uint32_t idx = e_cur & NLN_IDX_MASK, code = e_cur >> NLN_IDX_BITS;
            float r[10];  // negated offset, mass, Qxx Qxy Qyy Qxz Qyz Qzz
#pragma unroll
            for (int q = 0; q < 10; q++) r[q] = 0.f;
            r[0] = r[1] = r[2] = -1.0e3f;  // massless, momentless and far: adds 0
            const bool live = lane < nt && e_cur != 0xffffffffu;
            if (live) {
                const nln_qcell q = P.qcells[idx];
                neg_offset(q.cen, code, P.box, c, r[0], r[1], r[2]);
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
            if (live) {
                double *g = P.gcell + (size_t)idx * kCellAdj;
                atomicAdd(g + 0, -(double)a[3]);
                atomicAdd(g + 1, (double)a[0]);
                atomicAdd(g + 2, (double)a[1]);
                atomicAdd(g + 3, (double)a[2]);
                // the staged Q is -3 A_2: dL/dA_2 = -3 dL/dQ
#pragma unroll
                for (int q = 0; q < 6; q++) atomicAdd(g + kAdjG2 + q, -3.0 * (double)a[4 + q]);
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

// ---- multi-indices (the layout of ewald.cuh: order L's component
// (a0, a1, a2) at (a1+a2)(a1+a2+1)/2 + a2) ----
__host__ __device__ constexpr int mi_loc(int a1, int a2) { return (a1 + a2) * (a1 + a2 + 1) / 2 + a2; }
__host__ __device__ constexpr int mi_s(int p) { return p < 1 ? 0 : p < 3 ? 1 : p < 6 ? 2 : p < 10 ? 3 : p < 15 ? 4 : 5; }
__host__ __device__ constexpr int mi_a2(int p) { return p - mi_s(p) * (mi_s(p) + 1) / 2; }
__host__ __device__ constexpr int mi_a1(int p) { return mi_s(p) - mi_a2(p); }
__host__ __device__ constexpr int mi_a0(int L, int p) { return L - mi_s(p); }
__host__ __device__ constexpr int mi_n(int L) { return (L + 1) * (L + 2) / 2; }
__host__ __device__ constexpr int fact(int k) { return k <= 1 ? 1 : k * fact(k - 1); }
// multinomial L! / (a0! a1! a2!) of component p of order L
__host__ __device__ constexpr int mi_mult(int L, int p) {
    return fact(L) / (fact(mi_a0(L, p)) * fact(mi_a1(p)) * fact(mi_a2(p)));
}
// component of order L+1 = (component p of order L) + e_k
__host__ __device__ constexpr int mi_up(int p, int k) {
    return mi_loc(mi_a1(p) + (k == 1), mi_a2(p) + (k == 2));
}
// the pair (i, k) as a component of order 2
__host__ __device__ constexpr int mi_pair(int i, int k) { return mi_loc((i == 1) + (k == 1), (i == 2) + (k == 2)); }

// Unweighted monomials d^alpha of order L from those of order L-1.
template <int L, typename T>
__device__ __forceinline__ void mono_up(const T *lo, T x, T y, T z, T *hi) {
#pragma unroll
    for (int p = 0; p < mi_n(L); p++) {
        // drop one power of the first axis the component has
        if (mi_a0(L, p) > 0)
            hi[p] = lo[mi_loc(mi_a1(p), mi_a2(p))] * x;
        else if (mi_a1(p) > 0)
            hi[p] = lo[mi_loc(mi_a1(p) - 1, mi_a2(p))] * y;
        else
            hi[p] = lo[mi_loc(0, mi_a2(p) - 1)] * z;
    }
}

// F = A_L . d^(L-2) as a symmetric 3x3 (order-2 layout); wm: monomials of
// order L-2 weighted by their multinomials (L-2)!/gamma!.
template <int L>
__device__ __forceinline__ void contract_F(const float *A, const float *wm, float *F) {
#pragma unroll
    for (int q = 0; q < 6; q++) {
        float acc = 0.f;
#pragma unroll
        for (int g = 0; g < mi_n(L - 2); g++)
            acc = fmaf(A[mi_loc(mi_a1(g) + mi_a1(q), mi_a2(g) + mi_a2(q))], wm[g], acc);
        F[q] = acc;
    }
}

// One order-l term of the pair adjoint: t += (H_l w + u a_l) and G += dL/dA_l.
// mono: unweighted monomials of order l-1; F: A_l . d^(l-2).
template <int L>
__device__ __forceinline__ void pair_term(const float *F, const float *mono, float dx, float dy,
                                          float dz, float wx, float wy, float wz, float u,
                                          float wd, float rn, float ri2, float *t, float *G) {
    constexpr float g = L == 2 ? 1.5f : L == 3 ? 2.5f : 4.375f;
    constexpr float n = 2 * L + 1, fl = L;
    const float Ex = fmaf(F[mi_pair(0, 0)], dx, fmaf(F[mi_pair(0, 1)], dy, F[mi_pair(0, 2)] * dz));
    const float Ey = fmaf(F[mi_pair(0, 1)], dx, fmaf(F[mi_pair(1, 1)], dy, F[mi_pair(1, 2)] * dz));
    const float Ez = fmaf(F[mi_pair(0, 2)], dx, fmaf(F[mi_pair(1, 2)], dy, F[mi_pair(2, 2)] * dz));
    const float Fx = fmaf(F[mi_pair(0, 0)], wx, fmaf(F[mi_pair(0, 1)], wy, F[mi_pair(0, 2)] * wz));
    const float Fy = fmaf(F[mi_pair(0, 1)], wx, fmaf(F[mi_pair(1, 1)], wy, F[mi_pair(1, 2)] * wz));
    const float Fz = fmaf(F[mi_pair(0, 2)], wx, fmaf(F[mi_pair(1, 2)], wy, F[mi_pair(2, 2)] * wz));
    const float Pv = fmaf(Ex, dx, fmaf(Ey, dy, Ez * dz));
    const float Ew = fmaf(Ex, wx, fmaf(Ey, wy, Ez * wz));
    const float rn2 = rn * ri2, rn4 = rn2 * ri2;
    const float cF = -g * fl * (fl - 1.f) * rn;
    const float al = fmaf(n * rn2, wd, u * rn);  // n rho^-(n+2) (w.d) + u rho^-n
    const float cE = g * fl * al;
    const float cd = g * n * fmaf(fl * rn2, Ew, -Pv * fmaf((n + 2.f) * rn4, wd, u * rn2));
    const float cw = g * n * Pv * rn2;
    t[0] = fmaf(cF, Fx, fmaf(cE, Ex, fmaf(cd, dx, fmaf(cw, wx, t[0]))));
    t[1] = fmaf(cF, Fy, fmaf(cE, Ey, fmaf(cd, dy, fmaf(cw, wy, t[1]))));
    t[2] = fmaf(cF, Fz, fmaf(cE, Ez, fmaf(cd, dz, fmaf(cw, wz, t[2]))));
    // dL/dA_l[alpha] = g sum_k alpha_k v_k d^(alpha - e_k)
    const float ka = -g * al / fl, kw = g * rn;
    const float vx = fmaf(ka, dx, kw * wx), vy = fmaf(ka, dy, kw * wy), vz = fmaf(ka, dz, kw * wz);
#pragma unroll
    for (int p = 0; p < mi_n(L); p++) {
        float acc = G[p];
        if (mi_a0(L, p) > 0)
            acc = fmaf((float)mi_a0(L, p) * vx, mono[mi_loc(mi_a1(p), mi_a2(p))], acc);
        if (mi_a1(p) > 0)
            acc = fmaf((float)mi_a1(p) * vy, mono[mi_loc(mi_a1(p) - 1, mi_a2(p))], acc);
        if (mi_a2(p) > 0)
            acc = fmaf((float)mi_a2(p) * vz, mono[mi_loc(mi_a1(p), mi_a2(p) - 1)], acc);
        G[p] = acc;
    }
}

// The order-4 list adjoint.  Lane l holds record l of a 32-record tile:
// its negated offset from the group centre, mass and trace-free moments
// A_2, A_3, A_4 (31 floats), with its 35 running sums (t, the mass adjoint
// and the three moment duals).  The group's sinks (w, u and their offsets)
// sit in shared memory; every lane meets them one by one, and each sink's
// t is summed over the warp's records by a butterfly and kept by the lane
// that owns the sink.
constexpr int kAdjHexaWarps = 4;

__global__ void __launch_bounds__(32 * kAdjHexaWarps) k_adjoint_hexa(AdjProblem P) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ float4 sk[kAdjHexaWarps][32][2];  // (offset xyz, u), (w xyz, -)
    const float e2 = P.eps2;
    while (true) {
        int it = 0;
        if (lane == 0)
            it = atomicAdd(&P.counters[KH], 1);
        it = __shfl_sync(FULL, it, 0);
        if (it >= P.nitems[KH])
            break;
        const Item item = P.items[KH][it];
        const nln_group G = P.groups[item.group];
        const double c[3] = {G.cen[0], G.cen[1], G.cen[2]};
        const int ns = min(G.count, 32);
        __syncwarp();
        if (lane < ns) {
            const float4 p = P.points[G.first + lane];
            const float4 q = P.wu[G.first + lane];
            sk[warp][lane][0] = make_float4((float)((double)p.x - c[0]), (float)((double)p.y - c[1]),
                                            (float)((double)p.z - c[2]), q.w);
            sk[warp][lane][1] = make_float4(q.x, q.y, q.z, 0.f);
        }
        __syncwarp();
        float tsx = 0.f, tsy = 0.f, tsz = 0.f;  // this lane's sink: sum of t over the records
        for (int64_t b0 = item.begin; b0 < item.end; b0 += kAdjTile) {
            const int nt = (int)min((int64_t)kAdjTile, item.end - b0);
            uint32_t ent = 0xffffffffu, idx = 0;
            float nx = -1.0e3f, ny = -1.0e3f, nz = -1.0e3f, m = 0.f;  // massless and far: adds 0
            float A2[6], A3[10], A4[15];
#pragma unroll
            for (int q = 0; q < 6; q++) A2[q] = 0.f;
#pragma unroll
            for (int q = 0; q < 10; q++) A3[q] = 0.f;
#pragma unroll
            for (int q = 0; q < 15; q++) A4[q] = 0.f;
            if (lane < nt) {
                ent = P.list[2][b0 + lane];
                idx = ent & NLN_IDX_MASK;
                if (idx >= (uint32_t)P.ntab[2] || (ent >> NLN_IDX_BITS) > 26u)
                    ent = 0xffffffffu;
            }
            const bool live = ent != 0xffffffffu;
            if (live) {
                const nln_hcell &h = P.hcells[idx];
                neg_offset(h.cen, ent >> NLN_IDX_BITS, P.box, c, nx, ny, nz);
                m = h.mass;
                ew_quad(h.R, h.q2, A2);
                ew_oct(h.R, h.q3, A3);
                ew_hex(h.R, h.q4, A4);
            }
            float T[3] = {0.f, 0.f, 0.f}, am = 0.f;
            float G2[6], G3[10], G4[15];
#pragma unroll
            for (int q = 0; q < 6; q++) G2[q] = 0.f;
#pragma unroll
            for (int q = 0; q < 10; q++) G3[q] = 0.f;
#pragma unroll
            for (int q = 0; q < 15; q++) G4[q] = 0.f;
            for (int j = 0; j < ns; j++) {
                const float4 s0 = sk[warp][j][0], s1 = sk[warp][j][1];
                const float dx = s0.x + nx, dy = s0.y + ny, dz = s0.z + nz;
                const float u = s0.w, wx = s1.x, wy = s1.y, wz = s1.z;
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, e2)));
                const float ri = rsqrt_fast(r2), ri2 = ri * ri, ri3 = ri * ri2;
                const float wd = fmaf(wx, dx, fmaf(wy, dy, wz * dz));
                // monopole: t = m ri3 (w + (-3 ri2 (w.d) - u) d)
                const float in = fmaf(-3.f * ri2, wd, -u);
                const float mr3 = m * ri3;
                float t[3] = {mr3 * fmaf(in, dx, wx), mr3 * fmaf(in, dy, wy), mr3 * fmaf(in, dz, wz)};
                am = fmaf(ri, fmaf(wd, ri2, u), am);
                // monomials of orders 1..3 and the weighted order 2
                const float m1[3] = {dx, dy, dz};
                float m2[6], m3[10];
                mono_up<2>(m1, dx, dy, dz, m2);
                mono_up<3>(m2, dx, dy, dz, m3);
                const float w2[6] = {m2[0], 2.f * m2[1], 2.f * m2[2], m2[3], 2.f * m2[4], m2[5]};
                const float ri5 = ri3 * ri2, ri7 = ri5 * ri2, ri9 = ri7 * ri2;
                float F[6];
                pair_term<2>(A2, m1, dx, dy, dz, wx, wy, wz, u, wd, ri5, ri2, t, G2);
                contract_F<3>(A3, m1, F);
                pair_term<3>(F, m2, dx, dy, dz, wx, wy, wz, u, wd, ri7, ri2, t, G3);
                contract_F<4>(A4, w2, F);
                pair_term<4>(F, m3, dx, dy, dz, wx, wy, wz, u, wd, ri9, ri2, t, G4);
                T[0] += t[0];
                T[1] += t[1];
                T[2] += t[2];
                // sink j's t summed over the tile's records
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    t[0] += __shfl_xor_sync(FULL, t[0], o);
                    t[1] += __shfl_xor_sync(FULL, t[1], o);
                    t[2] += __shfl_xor_sync(FULL, t[2], o);
                }
                if (lane == j) {
                    tsx += t[0];
                    tsy += t[1];
                    tsz += t[2];
                }
            }
            if (live) {
                double *g = P.gcell + (size_t)idx * kCellAdj;
                atomicAdd(g + 0, -(double)am);
                atomicAdd(g + 1, (double)T[0]);
                atomicAdd(g + 2, (double)T[1]);
                atomicAdd(g + 3, (double)T[2]);
#pragma unroll
                for (int q = 0; q < 6; q++) atomicAdd(g + kAdjG2 + q, (double)G2[q]);
#pragma unroll
                for (int q = 0; q < 10; q++) atomicAdd(g + kAdjG3 + q, (double)G3[q]);
#pragma unroll
                for (int q = 0; q < 15; q++) atomicAdd(g + kAdjG4 + q, (double)G4[q]);
            }
        }
        if (lane < ns) {
            double *g = P.gbody + (size_t)(G.first + lane) * 4;
            atomicAdd(g + 0, -(double)tsx);
            atomicAdd(g + 1, -(double)tsy);
            atomicAdd(g + 2, -(double)tsz);
        }
    }
}

// STF projection (in place) of a symmetric tensor of order L held by its
// components (the multi-index layout): subtract the trace parts.
template <typename T>
__device__ __forceinline__ void stf2(T *G) {
    const T tr = (G[mi_pair(0, 0)] + G[mi_pair(1, 1)] + G[mi_pair(2, 2)]) / (T)3;
    G[mi_pair(0, 0)] -= tr;
    G[mi_pair(1, 1)] -= tr;
    G[mi_pair(2, 2)] -= tr;
}

// the component of order L of the sorted index tuple (i1 <= i2 <= ...)
__host__ __device__ constexpr int tup3(int i, int j, int k) {
    return mi_loc((i == 1) + (j == 1) + (k == 1), (i == 2) + (j == 2) + (k == 2));
}
__host__ __device__ constexpr int tup4(int i, int j, int k, int l) {
    return mi_loc((i == 1) + (j == 1) + (k == 1) + (l == 1), (i == 2) + (j == 2) + (k == 2) + (l == 2));
}

template <typename T>
__device__ __forceinline__ void stf3(T *G) {
    T t[3];
#pragma unroll
    for (int k = 0; k < 3; k++) t[k] = G[tup3(k, 0, 0)] + G[tup3(k, 1, 1)] + G[tup3(k, 2, 2)];
    T o[10];
#pragma unroll
    for (int p = 0; p < 10; p++) {
        // the tuple of component p
        const int a0 = 3 - mi_s(p), a1 = mi_a1(p);
        const int i[3] = {0 < a0 ? 0 : (0 < a0 + a1 ? 1 : 2), 1 < a0 ? 0 : (1 < a0 + a1 ? 1 : 2),
                          2 < a0 ? 0 : (2 < a0 + a1 ? 1 : 2)};
        T s = 0;
        if (i[0] == i[1]) s += t[i[2]];
        if (i[0] == i[2]) s += t[i[1]];
        if (i[1] == i[2]) s += t[i[0]];
        o[p] = G[p] - s / (T)5;
    }
#pragma unroll
    for (int p = 0; p < 10; p++) G[p] = o[p];
}

template <typename T>
__device__ __forceinline__ void stf4(T *G) {
    T T2[6];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int q = k; q < 3; q++)
            T2[mi_pair(k, q)] = G[tup4(k, q, 0, 0)] + G[tup4(k, q, 1, 1)] + G[tup4(k, q, 2, 2)];
    const T tt = T2[mi_pair(0, 0)] + T2[mi_pair(1, 1)] + T2[mi_pair(2, 2)];
    T o[15];
#pragma unroll
    for (int p = 0; p < 15; p++) {
        const int a0 = 4 - mi_s(p), a1 = mi_a1(p);
        int i[4];
#pragma unroll
        for (int r = 0; r < 4; r++) i[r] = r < a0 ? 0 : (r < a0 + a1 ? 1 : 2);
        T s6 = 0, s3 = 0;
        // the six pairs (r, q) and the indices left over
        const int pr[6][4] = {{0, 1, 2, 3}, {0, 2, 1, 3}, {0, 3, 1, 2},
                              {1, 2, 0, 3}, {1, 3, 0, 2}, {2, 3, 0, 1}};
#pragma unroll
        for (int e = 0; e < 6; e++)
            if (i[pr[e][0]] == i[pr[e][1]])
                s6 += T2[mi_pair(i[pr[e][2]] < i[pr[e][3]] ? i[pr[e][2]] : i[pr[e][3]],
                                 i[pr[e][2]] < i[pr[e][3]] ? i[pr[e][3]] : i[pr[e][2]])];
        if (i[0] == i[1] && i[2] == i[3]) s3 += 1;
        if (i[0] == i[2] && i[1] == i[3]) s3 += 1;
        if (i[0] == i[3] && i[1] == i[2]) s3 += 1;
        o[p] = G[p] - s6 / (T)7 + s3 * tt / (T)35;
    }
#pragma unroll
    for (int p = 0; p < 15; p++) G[p] = o[p];
}

// A trace-free tensor of order L is fixed by its 2L + 1 components with at
// most one z index (a2 <= 1); the rest follow from A[a0,a1,a2] =
// -A[a0+2,a1,a2-2] - A[a0,a1+2,a2-2], in layout order.
template <int L>
__device__ __forceinline__ void stf_fill(double *A) {
#pragma unroll
    for (int p = 0; p < mi_n(L); p++)
        if (mi_a2(p) >= 2)
            A[p] = -A[mi_loc(mi_a1(p), mi_a2(p) - 2)] - A[mi_loc(mi_a1(p) + 2, mi_a2(p) - 2)];
}
constexpr int kStfIndep = 5 + 7 + 9;  // doubles per cell of the correction's moment duals

// Periodic correction, sink side: one warp per group, a lane per sink.
// Mbar[alpha] = sum_i u_i (-u_i)^alpha/alpha! + sum_k w_ik (-u_i)^(alpha-e_k)/(alpha-e_k)!
// (|alpha - e_k| <= 3, the terms the accelerations use), and each sink's
// -t with t = H w + u a of its Taylor series, plus dL/dm_i of the self term.
__global__ void k_adjoint_ewald_groups(AdjProblem P) {
    const int64_t g = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (g >= P.ngroups)
        return;
    const nln_group G = P.groups[g];
    const EwStored &E = P.ewm[g];
    double M[35];
#pragma unroll
    for (int q = 0; q < 10; q++) M[q] = E.lo[q];
#pragma unroll
    for (int q = 0; q < 25; q++) M[10 + q] = (double)E.hi[q];
    double mb[35];
#pragma unroll
    for (int q = 0; q < 35; q++) mb[q] = 0.0;
    if (lane < G.count) {
        const int64_t i = G.first + lane;
        const float4 p = P.points[i];
        const float4 q4 = P.wu[i];
        const double w[3] = {q4.x, q4.y, q4.z}, uu = q4.w;
        const double u[3] = {(double)p.x - G.cen[0], (double)p.y - G.cen[1], (double)p.z - G.cen[2]};
        double px[5], py[5], pz[5];
        px[0] = py[0] = pz[0] = 1.0;
#pragma unroll
        for (int k = 1; k < 5; k++) {
            px[k] = px[k - 1] * (-u[0]) / k;
            py[k] = py[k - 1] * (-u[1]) / k;
            pz[k] = pz[k - 1] * (-u[2]) / k;
        }
        double a[3] = {0, 0, 0}, H[6] = {0, 0, 0, 0, 0, 0};
        // every multi-index (a0, a1, a2) of order <= 4 (constant bounds, so
        // the loops unroll fully and the arrays stay in registers)
#pragma unroll
        for (int a0 = 0; a0 <= 4; a0++)
#pragma unroll
            for (int a1 = 0; a1 <= 4; a1++)
#pragma unroll
                for (int a2 = 0; a2 <= 4; a2++) {
                    const int L = a0 + a1 + a2;
                    if (L > 4)
                        continue;
                    const int q = ew::idx(a0, a1, a2);
                    const double W = px[a0] * py[a1] * pz[a2];
                    mb[q] += uu * W;
                    if (L <= 3) {
                        // the accelerations' and the Mbar's w terms at order L + 1
#pragma unroll
                        for (int k = 0; k < 3; k++) {
                            const int qk = ew::idx(a0 + (k == 0), a1 + (k == 1), a2 + (k == 2));
                            a[k] += M[qk] * W;
                            mb[qk] += w[k] * W;
                        }
                    }
                    if (L <= 2) {
#pragma unroll
                        for (int k = 0; k < 3; k++)
#pragma unroll
                            for (int l = k; l < 3; l++)
                                H[mi_pair(k, l)] +=
                                    M[ew::idx(a0 + (k == 0) + (l == 0), a1 + (k == 1) + (l == 1),
                                              a2 + (k == 2) + (l == 2))] * W;
                    }
                }
        double t[3];
#pragma unroll
        for (int k = 0; k < 3; k++)
            t[k] = H[mi_pair(k, 0)] * w[0] + H[mi_pair(k, 1)] * w[1] + H[mi_pair(k, 2)] * w[2] +
                   uu * a[k];
        double *gb = P.gbody + (size_t)i * 4;
        atomicAdd(gb + 0, -t[0]);
        atomicAdd(gb + 1, -t[1]);
        atomicAdd(gb + 2, -t[2]);
        atomicAdd(gb + 3, -uu * (double)P.ew_self);
    }
#pragma unroll
    for (int q = 0; q < 35; q++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mb[q] += __shfl_xor_sync(0xffffffffu, mb[q], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 35; q++) P.mbar[g * 35 + q] = mb[q];
    }
}

// Periodic correction, source side: one warp per group, lanes over its
// correction entries (as ewald_moments_loop).  Per entry at y = X + shift - c
// with the table values D (orders 0..5) there:
//   dL/dm = sum_a Mbar[a] D[a],   dL/dX_l = sum_{|g|<=4} N[g] D[g + e_l],
//   N[g] = m Mbar[g] + sum_K sum_{|b|=K, b<=g} A_K[b]/b! Mbar[g - b],
//   dL/dA_K[b] = (1/K!) sum_a Mbar[a] D[a + b] over the forward's terms
//                (|a| <= 3, 2, 1 for K = 2, 3, 4),
//   dL/dB2 = Mbar[0] ew_trace / 6.
__device__ __forceinline__ float ew_D(const float *o, const float *f5, int q) {
    return q < ew::kNQ4 ? o[q] : f5[q - ew::kNQ4];
}

template <int K, int SMAX>
__device__ __forceinline__ void ew_adj_moment(const float *Mb, const float *o, const float *f5,
                                              float *G) {
    constexpr float ik = 1.f / (float)fact(K);
#pragma unroll
    for (int b0 = 0; b0 <= K; b0++)
#pragma unroll
        for (int b1 = 0; b1 <= K; b1++) {
            if (b0 + b1 > K)
                continue;
            const int b2 = K - b0 - b1;
            float acc = 0.f;
#pragma unroll
            for (int a0 = 0; a0 <= SMAX; a0++)
#pragma unroll
                for (int a1 = 0; a1 <= SMAX; a1++)
#pragma unroll
                    for (int a2 = 0; a2 <= SMAX; a2++) {
                        if (a0 + a1 + a2 > SMAX)
                            continue;
                        acc = fmaf(Mb[ew::idx(a0, a1, a2)],
                                   ew_D(o, f5, ew::idx(a0 + b0, a1 + b1, a2 + b2)), acc);
                    }
            G[ew::idx(b0, b1, b2) - ew::base(K)] = acc * ik;
        }
}

// The trace-free part of a moment dual of order K, added to the cell's
// independent components (a2 <= 1): 2K + 1 atomics instead of (K+1)(K+2)/2.
template <int K>
__device__ __forceinline__ void add_indep(float *G, double *dst) {
    if (K == 2)
        stf2(G);
    else if (K == 3)
        stf3(G);
    else
        stf4(G);
    int k = 0;
#pragma unroll
    for (int p = 0; p < mi_n(K); p++)
        if (mi_a2(p) <= 1)
            atomicAdd(dst + k++, (double)G[p]);
}

// N[g] += sum_{|b| = K} S[b] / b! Mbar[g - b] for |g| <= 4
template <int K>
__device__ __forceinline__ void ew_adj_conv(const float *S, const float *Mb, float *N) {
#pragma unroll
    for (int b0 = 0; b0 <= K; b0++)
#pragma unroll
        for (int b1 = 0; b1 <= K; b1++) {
            if (b0 + b1 > K)
                continue;
            const int b2 = K - b0 - b1;
            const float sb = S[ew::idx(b0, b1, b2) - ew::base(K)] *
                             (ew::ifact(b0) * ew::ifact(b1) * ew::ifact(b2));
#pragma unroll
            for (int a0 = 0; a0 <= 4 - K; a0++)
#pragma unroll
                for (int a1 = 0; a1 <= 4 - K; a1++)
#pragma unroll
                    for (int a2 = 0; a2 <= 4 - K; a2++) {
                        if (a0 + a1 + a2 > 4 - K)
                            continue;
                        const int q = ew::idx(a0 + b0, a1 + b1, a2 + b2);
                        N[q] = fmaf(sb, Mb[ew::idx(a0, a1, a2)], N[q]);
                    }
        }
}

__global__ void __launch_bounds__(64) k_adjoint_ewald_entries(AdjProblem P) {
    const int64_t g = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    __shared__ float mb_s[2][36];  // the group's Mbar, read by every lane alike
    float *Mb = mb_s[threadIdx.x >> 5];
    if (g < P.ngroups) {
        for (int q = lane; q < 35; q += 32) Mb[q] = (float)P.mbar[g * 35 + q];
    }
    __syncwarp();
    if (g >= P.ngroups)
        return;
    const nln_group G = P.groups[g];
    const double c[3] = {G.cen[0], G.cen[1], G.cen[2]};
    const uint32_t nb = (uint32_t)P.nbodies;
    for (int64_t k = P.cptr[g] + lane; k < P.cptr[g + 1]; k += 32) {
        const uint32_t ent = P.clist[k];
        const uint32_t idx = ent & NLN_IDX_MASK;
        if (idx >= (uint32_t)P.ntab[0] || (ent >> NLN_IDX_BITS) > 26u)
            continue;
        double sx, sy, sz;
        decode_shift(ent >> NLN_IDX_BITS, P.box, sx, sy, sz);
        float o[ew::kNQ4], f5[21];
        double X[3];
        float m;
        const nln_hcell *h = nullptr;
        if (idx < nb) {
            const float4 p = P.points[idx];
            X[0] = p.x;
            X[1] = p.y;
            X[2] = p.z;
            m = p.w;
        } else {
            h = &P.hcells[idx - nb];
            X[0] = h->cen[0];
            X[1] = h->cen[1];
            X[2] = h->cen[2];
            m = h->mass;
        }
        ew_lookup<true>(P.ew, (float)(X[0] + sx - c[0]), (float)(X[1] + sy - c[1]),
                        (float)(X[2] + sz - c[2]), o, f5);
        float dm = 0.f;
#pragma unroll
        for (int q = 0; q < ew::kNQ4; q++) dm = fmaf(Mb[q], o[q], dm);
        float N[35];
#pragma unroll
        for (int q = 0; q < 35; q++) N[q] = m * Mb[q];
        if (h) {
            float S[15];
            double *gc = P.gcell + (size_t)(idx - nb) * kCellAdj;
            double *gi = P.gstf + (size_t)(idx - nb) * kStfIndep;
            float G[15];
            ew_quad(h->R, h->q2, S);
            ew_adj_conv<2>(S, Mb, N);
            ew_adj_moment<2, 3>(Mb, o, f5, G);
            add_indep<2>(G, gi);
            ew_oct(h->R, h->q3, S);
            ew_adj_conv<3>(S, Mb, N);
            ew_adj_moment<3, 2>(Mb, o, f5, G);
            add_indep<3>(G, gi + 5);
            ew_hex(h->R, h->q4, S);
            ew_adj_conv<4>(S, Mb, N);
            ew_adj_moment<4, 1>(Mb, o, f5, G);
            add_indep<4>(G, gi + 12);
            atomicAdd(gc + kAdjB2, (double)(Mb[0] * (1.f / 6.f) * P.ew_trace));
        }
        float dX[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int a0 = 0; a0 <= 4; a0++)
#pragma unroll
            for (int a1 = 0; a1 <= 4; a1++)
#pragma unroll
                for (int a2 = 0; a2 <= 4; a2++) {
                    if (a0 + a1 + a2 > 4)
                        continue;
                    const float nq = N[ew::idx(a0, a1, a2)];
                    dX[0] = fmaf(nq, ew_D(o, f5, ew::idx(a0 + 1, a1, a2)), dX[0]);
                    dX[1] = fmaf(nq, ew_D(o, f5, ew::idx(a0, a1 + 1, a2)), dX[1]);
                    dX[2] = fmaf(nq, ew_D(o, f5, ew::idx(a0, a1, a2 + 1)), dX[2]);
                }
        double *gt = h ? P.gcell + (size_t)(idx - nb) * kCellAdj : P.gbody + (size_t)idx * 4;
        if (h) {
            atomicAdd(gt + 0, (double)dm);
            atomicAdd(gt + 1, (double)dX[0]);
            atomicAdd(gt + 2, (double)dX[1]);
            atomicAdd(gt + 3, (double)dX[2]);
        } else {
            atomicAdd(gt + 0, (double)dX[0]);
            atomicAdd(gt + 1, (double)dX[1]);
            atomicAdd(gt + 2, (double)dX[2]);
            atomicAdd(gt + 3, (double)dm);
        }
    }
}

// Per cell with a non-zero adjoint: project the moment duals onto their
// trace-free parts and fold the moments' dependence on the centre of mass
// into Xbar (Xbar' = Xbar - 3 PG_3.A_2 - 4 PG_4.A_3); flag marks the cells
// the bodies' pass visits.
__global__ void k_adjoint_cells(double *__restrict__ gcell, const double *__restrict__ gstf,
                                const nln_hcell *__restrict__ hc, int64_t nc,
                                int *__restrict__ flag) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc)
        return;
    double *G = gcell + (size_t)c * kCellAdj;
    bool any = false;
    for (int q = 0; q < kCellAdj; q++) any |= G[q] != 0.0;
    const double *I = gstf ? gstf + (size_t)c * kStfIndep : nullptr;
    bool anyi = false;
    if (I)
        for (int q = 0; q < kStfIndep; q++) anyi |= I[q] != 0.0;
    flag[c] = any || anyi;
    if (!any && !anyi)
        return;
    stf2(G + kAdjG2);
    stf3(G + kAdjG3);
    stf4(G + kAdjG4);
    if (anyi) {
        // the correction's duals, already trace-free, from their independent parts
        double A2[6], A3[10], A4[15];
        int k = 0;
#pragma unroll
        for (int p = 0; p < 6; p++) A2[p] = mi_a2(p) <= 1 ? I[k++] : 0.0;
#pragma unroll
        for (int p = 0; p < 10; p++) A3[p] = mi_a2(p) <= 1 ? I[k++] : 0.0;
#pragma unroll
        for (int p = 0; p < 15; p++) A4[p] = mi_a2(p) <= 1 ? I[k++] : 0.0;
        stf_fill<2>(A2);
        stf_fill<3>(A3);
        stf_fill<4>(A4);
#pragma unroll
        for (int p = 0; p < 6; p++) G[kAdjG2 + p] += A2[p];
#pragma unroll
        for (int p = 0; p < 10; p++) G[kAdjG3 + p] += A3[p];
#pragma unroll
        for (int p = 0; p < 15; p++) G[kAdjG4 + p] += A4[p];
    }
    if (hc) {
        float A2[6], A3[10];
        const nln_hcell &h = hc[c];
        ew_quad(h.R, h.q2, A2);
        ew_oct(h.R, h.q3, A3);
        // (PG_l . A_(l-1))_i = sum_{|b| = l-1} ((l-1)!/b!) PG_l[b + e_i] A_(l-1)[b]
#pragma unroll
        for (int i = 0; i < 3; i++) {
            double s3 = 0.0, s4 = 0.0;
#pragma unroll
            for (int b = 0; b < 6; b++) s3 += (double)mi_mult(2, b) * G[kAdjG3 + mi_up(b, i)] * A2[b];
#pragma unroll
            for (int b = 0; b < 10; b++) s4 += (double)mi_mult(3, b) * G[kAdjG4 + mi_up(b, i)] * A3[b];
            G[1 + i] -= 3.0 * s3 + 4.0 * s4;
        }
    }
}

// Bodies from their cells' adjoints: every ancestor of the body's leaf.
// A cell's centre and mass are read as the forward used them: the FP64
// centre of the quadrupole (or order-4) table when there is one, else the
// cell monopole of the point table.
__global__ void k_adjoint_bodies(const float4 *__restrict__ pts, const int32_t *__restrict__ leaf,
                                 const int32_t *__restrict__ parent, const nln_qcell *__restrict__ qc,
                                 const nln_hcell *__restrict__ hc, const double *__restrict__ gcell,
                                 const int *__restrict__ flag, const double *__restrict__ gbody,
                                 int64_t n, float4 *__restrict__ out) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n)
        return;
    const float4 p = pts[b];
    double g[4] = {gbody[4 * b], gbody[4 * b + 1], gbody[4 * b + 2], gbody[4 * b + 3]};
    for (int32_t cidx = leaf[b]; cidx >= 0; cidx = parent[cidx]) {
        if (!flag[cidx])
            continue;
        const double *A = gcell + (size_t)cidx * kCellAdj;
        double X[3], M;
        if (qc) {
            X[0] = qc[cidx].cen[0];
            X[1] = qc[cidx].cen[1];
            X[2] = qc[cidx].cen[2];
            M = qc[cidx].mass;
        } else if (hc) {
            X[0] = hc[cidx].cen[0];
            X[1] = hc[cidx].cen[1];
            X[2] = hc[cidx].cen[2];
            M = hc[cidx].mass;
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
        // f(y) = sum_l <PG_l, y^l> + B2bar |y|^2 and its gradient
        double m1[3] = {y[0], y[1], y[2]}, m2[6], m3[10], m4[15];
        mono_up<2>(m1, y[0], y[1], y[2], m2);
        mono_up<3>(m2, y[0], y[1], y[2], m3);
        mono_up<4>(m3, y[0], y[1], y[2], m4);
        double f = A[kAdjB2] * (m2[0] + m2[3] + m2[5]);
        double df[3] = {2.0 * A[kAdjB2] * y[0], 2.0 * A[kAdjB2] * y[1], 2.0 * A[kAdjB2] * y[2]};
#pragma unroll
        for (int q = 0; q < 6; q++) f += (double)mi_mult(2, q) * A[kAdjG2 + q] * m2[q];
#pragma unroll
        for (int q = 0; q < 10; q++) f += (double)mi_mult(3, q) * A[kAdjG3 + q] * m3[q];
#pragma unroll
        for (int q = 0; q < 15; q++) f += (double)mi_mult(4, q) * A[kAdjG4 + q] * m4[q];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            // l = 2: 2 (PG_2 y)_i; l = 3: 3 (PG_3 . y^2)_i; l = 4: 4 (PG_4 . y^3)_i
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < 3; q++) s += 2.0 * A[kAdjG2 + mi_up(q, i)] * m1[q];
#pragma unroll
            for (int q = 0; q < 6; q++) s += 3.0 * (double)mi_mult(2, q) * A[kAdjG3 + mi_up(q, i)] * m2[q];
#pragma unroll
            for (int q = 0; q < 10; q++) s += 4.0 * (double)mi_mult(3, q) * A[kAdjG4 + mi_up(q, i)] * m3[q];
            df[i] += s;
        }
        const double mb = p.w;
        for (int d = 0; d < 3; d++) g[d] += mb * df[d] + (mb / M) * A[1 + d];
        g[3] += A[0] + f + (A[1] * y[0] + A[2] * y[1] + A[3] * y[2]) / M;
    }
    out[b] = make_float4((float)g[0], (float)g[1], (float)g[2], (float)g[3]);
}

}  // namespace

// Per-plan adjoint state (owned by the plan).
struct grav_adjoint_state {
    int32_t *leaf = nullptr, *parent = nullptr;
    int *flag = nullptr;
    double *gbody = nullptr, *gcell = nullptr, *mbar = nullptr, *gstf = nullptr;
    ~grav_adjoint_state() {
        for (void *p : {(void *)leaf, (void *)parent, (void *)flag, (void *)gbody, (void *)gcell,
                        (void *)mbar, (void *)gstf})
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
    if (pl->dp.nitems[KQ] > 0 && !pl->dp.qcells)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: no quadrupole table");
    if ((pl->dp.nitems[KH] > 0 || pl->dp.ewald) && !pl->dp.hcells)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: no order-4 table");
    if (pl->dp.qsh != 0.5f)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: the physical quadrupole potential "
                                  "(quad_phi_sign = +1) only");
    if (pl->plain)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: the mixed-precision form only "
                                  "(grav_problem.precision = 0)");
    if (pl->dp.ewald && !pl->evaluated)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: evaluate the plan first (the "
                                  "periodic correction's adjoint reads its group moments)");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t nb = pl->hp.nbodies, nc = pl->hp.ncells, ng = pl->hp.ngroups;
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
            e = cudaMalloc((void **)&A->flag, nc * 4);
        if (e == cudaSuccess)
            e = cudaMalloc((void **)&A->gbody, nb * 4 * sizeof(double));
        if (e == cudaSuccess)
            e = cudaMalloc((void **)&A->gcell, nc * kCellAdj * sizeof(double));
        if (e == cudaSuccess && pl->dp.ewald)
            e = cudaMalloc((void **)&A->mbar, ng * 35 * sizeof(double));
        if (e == cudaSuccess && pl->dp.ewald)
            e = cudaMalloc((void **)&A->gstf, nc * kStfIndep * sizeof(double));
        if (e != cudaSuccess) {
            delete A;
            return gc::cuda_status(e, "grav_plan_adjoint_CUDA: scratch");
        }
        pl->adj = A;
    }
    grav_adjoint_state *A = pl->adj;
    GC_CHECK(cudaMemsetAsync(A->gbody, 0, nb * 4 * sizeof(double), st));
    GC_CHECK(cudaMemsetAsync(A->gcell, 0, nc * kCellAdj * sizeof(double), st));
    if (A->gstf)
        GC_CHECK(cudaMemsetAsync(A->gstf, 0, nc * kStfIndep * sizeof(double), st));
    GC_CHECK(cudaMemsetAsync(pl->dp.counters, 0, 4 * sizeof(int), st));
    AdjProblem P{};
    P.points = pl->dp.points;
    P.qcells = pl->dp.qcells;
    P.hcells = pl->dp.hcells;
    P.groups = pl->dp.groups;
    for (int k = 0; k < 3; k++) {
        P.list[k] = pl->dp.list[k];
        P.ntab[k] = pl->dp.ntab[k];
        P.items[k] = pl->dp.items[k];
        P.nitems[k] = pl->dp.nitems[k];
    }
    P.counters = pl->dp.counters;
    P.wu = reinterpret_cast<const float4 *>(wu);
    P.gbody = A->gbody;
    P.gcell = A->gcell;
    P.nbodies = nb;
    P.ngroups = ng;
    P.eps2 = pl->dp.eps2;
    P.qsh = pl->dp.qsh;
    P.box = pl->dp.box;
    P.err = pl->dp.err;
    P.ewald = pl->dp.ewald;
    P.cptr = pl->dp.cptr;
    P.clist = pl->dp.clist;
    P.ew = pl->dp.ew;
    P.ew_self = pl->dp.ew_self;
    P.ew_trace = pl->dp.ew_trace;
    P.ewm = pl->ewm;
    P.mbar = A->mbar;
    P.gstf = A->gstf;
    const unsigned blocks = (unsigned)pl->nsm * 4;
    if (P.nitems[KP] > 0)
        k_adjoint_points<<<blocks, 256, 0, st>>>(P);
    if (P.nitems[KQ] > 0)
        k_adjoint_quads<<<blocks, 256, 0, st>>>(P);
    if (P.nitems[KH] > 0)
        k_adjoint_hexa<<<blocks, 32 * kAdjHexaWarps, 0, st>>>(P);
    GC_CHECK(cudaGetLastError());
    if (P.ewald && ng > 0) {
        k_adjoint_ewald_groups<<<(unsigned)((ng + 3) / 4), 128, 0, st>>>(P);
        k_adjoint_ewald_entries<<<(unsigned)((ng + 1) / 2), 64, 0, st>>>(P);
        GC_CHECK(cudaGetLastError());
    }
    if (nc > 0)
        k_adjoint_cells<<<(unsigned)((nc + 127) / 128), 128, 0, st>>>(A->gcell, A->gstf,
                                                                       pl->dp.hcells, nc, A->flag);
    k_adjoint_bodies<<<(unsigned)((nb + 127) / 128), 128, 0, st>>>(
        pl->dp.points, A->leaf, A->parent, pl->dp.qcells, pl->dp.hcells, A->gcell, A->flag,
        A->gbody, nb, reinterpret_cast<float4 *>(grad));
    GC_CHECK(cudaGetLastError());
    return 0;
}
