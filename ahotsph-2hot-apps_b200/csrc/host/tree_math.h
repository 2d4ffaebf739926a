// tree_math.h -- the arithmetic of the tree build and the MAC walk, shared
// word for word by the host builder (nlnhost.cpp, g++) and the GPU builder
// (build.cu, nvcc).  Both compile it without contracting a * b + c into
// fused multiply-adds (g++ -ffp-contract=off, nvcc -fmad=false for the
// builder), and every operation here is an IEEE-754 double operation with a
// correctly rounded result (+ - * / sqrt, floor, nearbyint), so the two
// builders produce bit-identical moments, critical radii and lists.
//
// Algorithms restated from the reference (file:line in lanl/ahotsph-2hot-apps):
//   moments and their normalisation   nln/cofm.c:96-231, 398-420, 486-562
//   AREL critical radii               nln/cofm.c:276-565, rcrit_poly/rtnewt 577-624
//   MAC acceptance order m -> q -> h  nln/mac.c:1785-1805 (DLRcritMAC)
//   leaf expansion to bodies          nln/mac.c:1817-1832
//   completeness invariant            nln/mac.c:734-735
//   image offsets                     nln/mac.c:91-111
#pragma once

#include <math.h>
#include <stdint.h>

#include "nlnlists.h"

#if defined(__CUDACC__)
#define NLN_HD __host__ __device__
#else
#define NLN_HD
#endif

// Raw moment sums of a cell about its centre: second (xx xy xz yy yz zz),
// third (xxx xxy xxz xyy xyz xzz yyy yyz yzz zzz), fourth order (xxxx xxxy
// xxxz xxyy xxyz xxzz xyyy xyyz xyzz xzzz yyyy yyyz yyzz yzzz zzzz), then
// sum m r^2, m r^4, m r^6.
#define NLN_NMOM 34

// Body terms of a cell's first pass: mass and mass-weighted offset from the
// cell's geometric centre gc (its centre of mass follows from them).
NLN_HD inline void nln_mass_terms(const float *p, float m, const double *gc, double *a) {
    const double w = m;
    a[0] += w;
    a[1] += w * ((double)p[0] - gc[0]);
    a[2] += w * ((double)p[1] - gc[1]);
    a[3] += w * ((double)p[2] - gc[2]);
}

// Body terms of the second pass (NLN_NMOM sums about the centre of mass
// cen); returns the body's r^2 from cen (bmax is the largest).
NLN_HD inline double nln_moment_terms(const float *p, float m, const double *cen, double *a) {
    const double w = m;
    const double x = (double)p[0] - cen[0];
    const double y = (double)p[1] - cen[1];
    const double z = (double)p[2] - cen[2];
    const double xx = x * x, yy = y * y, zz = z * z, r2 = xx + yy + zz;
    a[0] += w * xx; a[1] += w * x * y; a[2] += w * x * z;
    a[3] += w * yy; a[4] += w * y * z; a[5] += w * zz;
    a[6] += w * xx * x; a[7] += w * xx * y; a[8] += w * xx * z;
    a[9] += w * x * yy; a[10] += w * x * y * z; a[11] += w * x * zz;
    a[12] += w * yy * y; a[13] += w * yy * z; a[14] += w * y * zz; a[15] += w * zz * z;
    a[16] += w * xx * xx; a[17] += w * xx * x * y; a[18] += w * xx * x * z;
    a[19] += w * xx * yy; a[20] += w * xx * y * z; a[21] += w * xx * zz;
    a[22] += w * x * yy * y; a[23] += w * x * yy * z; a[24] += w * x * y * zz;
    a[25] += w * x * zz * z; a[26] += w * yy * yy; a[27] += w * yy * y * z;
    a[28] += w * yy * zz; a[29] += w * y * zz * z; a[30] += w * zz * zz;
    a[31] += w * r2;
    a[32] += w * r2 * r2;
    a[33] += w * r2 * r2 * r2;
    return r2;
}

// A cell's table records from its FP64 centre of mass, mass, bmax and raw
// moments mo (NLN_NMOM): the point-table monopole (x, y, z, m), and the
// quadrupole and order-4 records with the traceless R^-l normalisation of
// nln/cofm.c:398-420 (quadrupole), 507-522 (octupole), 523-558
// (hexadecapole).
NLN_HD inline void nln_cell_tables(const double *cen, double m, double bmax, const double *mo,
                                   float *pt, nln_qcell *q, nln_hcell *h) {
    const double x2 = mo[0], xy = mo[1], xz = mo[2], y2 = mo[3], yz = mo[4], z2 = mo[5];
    const double x3 = mo[6], x2y = mo[7], x2z = mo[8], xy2 = mo[9], xyz = mo[10], xz2 = mo[11],
                 y3 = mo[12], y2z = mo[13], yz2 = mo[14], z3 = mo[15];
    const double x4 = mo[16], x3y = mo[17], x3z = mo[18], x2y2 = mo[19], x2yz = mo[20],
                 x2z2 = mo[21], xy3 = mo[22], xy2z = mo[23], xyz2 = mo[24], xz3 = mo[25],
                 y4 = mo[26], y3z = mo[27], y2z2 = mo[28], yz3 = mo[29], z4 = mo[30];
    const double ri = bmax > 0 ? 1.0 / bmax : 0.0;
    for (int d = 0; d < 3; d++) pt[d] = (float)cen[d];
    pt[3] = (float)m;
    // quadrupole, nln/cofm.c:398-420
    const double tq = (x2 + y2 + z2) / 3.0;
    const double q2[5] = {(x2 - tq) * ri * ri, xy * ri * ri, (y2 - tq) * ri * ri, xz * ri * ri,
                          yz * ri * ri};
    // octupole, nln/cofm.c:507-522
    const double tx = (x3 + xy2 + xz2) / 5.0, ty = (x2y + y3 + yz2) / 5.0,
                 tz = (x2z + y2z + z3) / 5.0;
    const double r3 = ri * ri * ri;
    const double q3[7] = {(x3 - 3.0 * tx) * r3, (x2y - ty) * r3, (xy2 - tx) * r3,
                          (y3 - 3.0 * ty) * r3, (x2z - tz) * r3, xyz * r3, (y2z - tz) * r3};
    // hexadecapole, nln/cofm.c:523-558
    const double txx = (x4 + x2y2 + x2z2) / 7.0, txy = (x3y + xy3 + xyz2) / 7.0,
                 txz = (x3z + xy2z + xz3) / 7.0, tyy = (x2y2 + y4 + y2z2) / 7.0,
                 tyz = (x2yz + y3z + yz3) / 7.0, tzz = (x2z2 + y2z2 + z4) / 7.0;
    const double tt = 0.1 * (txx + tyy + tzz);
    const double r4 = r3 * ri;
    const double q4[9] = {(x4 - 6.0 * (txx - tt)) * r4, (x3y - 3.0 * txy) * r4,
                          (x2y2 - (txx + tyy - 2.0 * tt)) * r4, (xy3 - 3.0 * txy) * r4,
                          (y4 - 6.0 * (tyy - tt)) * r4, (x3z - 3.0 * txz) * r4,
                          (x2yz - tyz) * r4, (xy2z - txz) * r4, (y3z - 3.0 * tyz) * r4};
    (void)z2;
    (void)z3;
    (void)z4;
    (void)tzz;
    for (int d = 0; d < 3; d++) q->cen[d] = h->cen[d] = cen[d];
    q->mass = h->mass = (float)m;
    q->R = h->R = (float)bmax;
    q->B2 = h->B2 = (float)mo[31];
    q->qxx = (float)q2[0];
    q->qxy = (float)q2[1];
    q->qyy = (float)q2[2];
    q->qxz = (float)q2[3];
    q->qyz = (float)q2[4];
    q->pad[0] = q->pad[1] = 0.f;
    h->pad[0] = h->pad[1] = 0.f;
    for (int k = 0; k < 5; k++) h->q2[k] = (float)q2[k];
    for (int k = 0; k < 7; k++) h->q3[k] = (float)q3[k];
    for (int k = 0; k < 9; k++) h->q4[k] = (float)q4[k];
}

// Newton iteration on a polynomial sum_k a[k] r^k, started at x1 and stopped
// when the step is below xacc; returns x1 when it does not converge in 30
// steps (the behaviour of rtnewt, nln/cofm.c:602-624, with rcrit_poly's
// Horner evaluation, nln/cofm.c:577-596).
NLN_HD inline double nln_newton_root(const double *a, int n, double x1, double xacc) {
    double r = x1;
    for (int it = 0; it < 30; it++) {
        double p = a[n], dp = 0.0;
        for (int k = n; k > 0; k--) {
            dp = dp * r + p;
            p = p * r + a[k - 1];
        }
        if (!isfinite(p) || !isfinite(dp) || dp == 0.0)
            return x1;
        const double dx = p / dp;
        r -= dx;
        if (fabs(dx) < xacc)
            return r;
    }
    return x1;
}

// MAC parameters of the critical radii and the walk.
typedef struct nln_mac {
    double tol, rel_tol, rel_tol0, ptol_boost, bmax0;  // bmax0: half the root cube
    int p2cut, p4cut;
    double box, ewald_theta;
} nln_mac;

// AREL critical radii of one cell, nln/cofm.c:276-565 (stol_max at its
// default; ptol = tol / (1 + ptol_boost bmax / bmax0)).  A relative
// tolerance of 0 switches that criterion off (the reference would divide by
// zero, cofm.c:322-335).  rc[0..2]: monopole, quadrupole, order 4.
NLN_HD inline void nln_cell_rcrit(const nln_mac &P, int32_t count, double m, double b, double B2,
                                  double B4, double B6, double *rc) {
    rc[0] = rc[1] = rc[2] = 0.0;
    if (B2 <= 0.0 || m <= 0.0 || b <= 0.0)
        return;  // coincident bodies: every expansion is exact
    const double rel = P.rel_tol, rel0 = P.rel_tol0;
    const double boost = P.ptol_boost, bmax0 = P.bmax0;
    // larger cells get a tighter tolerance with ptol_boost (cofm.c:302)
    const double ptol = P.tol / (1.0 + (boost > 0 && bmax0 > 0 ? boost * b / bmax0 : 0.0));
    const double B3 = B2 * sqrt(B2 / m);  // lower bound, cofm.c:314
    double a[10];
    // monopole
    const double bh = 0.5 * b;
    double rmax = bh + sqrt(bh * bh + sqrt(3.0 * B2 / ptol));
    a[0] = 2 * B3; a[1] = -3 * B2; a[2] = 0; a[3] = ptol * b * b; a[4] = -2 * ptol * b;
    a[5] = ptol;
    double r_abs = nln_newton_root(a, 5, rmax, 0.01 * rmax) + 0.01 * rmax;
    double r_rel0 = 0.0, r_rel = INFINITY;
    if (rel0 > 0) {
        rmax = b + sqrt(3.0 / rel0 * B2 / m);
        a[0] = 2 * B3; a[1] = -3 * B2 + rel0 * b * b * m; a[2] = -2 * rel0 * b * m;
        a[3] = rel0 * m;
        r_rel0 = nln_newton_root(a, 3, rmax, 0.01 * rmax) + 0.01 * rmax;
    }
    if (rel > 0) {
        rmax = b + sqrt(3.0 / rel * B2 / m);
        a[0] = 2 * B3; a[1] = -3 * B2 + rel * b * b * m; a[2] = -2 * rel * b * m;
        a[3] = rel * m;
        r_rel = nln_newton_root(a, 3, rmax, 0.01 * rmax) + 0.01 * rmax;
    }
    rc[0] = fmax(fmin(r_abs, r_rel), r_rel0);
    const double m_abs = r_abs, m_rel0 = r_rel0, m_rel = r_rel;
    // quadrupole, cofm.c:442-485
    if (P.p2cut && count >= P.p2cut) {
        const double B3q = b * B2;  // upper bound, cofm.c:433
        a[0] = 3 * B4; a[1] = -4 * B3q; a[2] = 0; a[3] = 0; a[4] = ptol * b * b;
        a[5] = -2 * ptol * b; a[6] = ptol;
        r_abs = nln_newton_root(a, 6, m_abs, 0.01 * m_abs) + 0.01 * m_abs;
        r_rel0 = 0.0;
        r_rel = INFINITY;
        if (rel0 > 0) {
            a[0] = 3 * B4; a[1] = -4 * B3q; a[2] = rel0 * b * b * m; a[3] = -2 * rel0 * b * m;
            a[4] = rel0 * m;
            r_rel0 = nln_newton_root(a, 4, m_rel0, 0.01 * m_rel0) + 0.01 * m_rel0;
        }
        if (rel > 0 && isfinite(m_rel)) {
            a[0] = 3 * B4; a[1] = -4 * B3q; a[2] = rel * b * b * m; a[3] = -2 * rel * b * m;
            a[4] = rel * m;
            r_rel = nln_newton_root(a, 4, m_rel, 0.01 * m_rel) + 0.01 * m_rel;
        }
        rc[1] = fmax(fmin(r_abs, r_rel), r_rel0);
    }
    // order 4, cofm.c:489-505
    if (P.p4cut && count >= P.p4cut) {
        const double B5 = b * B4;
        for (int k = 0; k < 10; k++) a[k] = 0.0;
        a[0] = 5 * B6; a[1] = -6 * B5; a[6] = ptol * b * b; a[7] = -2 * ptol * b; a[8] = ptol;
        r_abs = nln_newton_root(a, 8, m_abs, 0.001 * m_abs) + 0.001 * m_abs;
        r_rel0 = 0.0;
        r_rel = INFINITY;
        if (rel0 > 0) {
            for (int k = 0; k < 10; k++) a[k] = 0.0;
            a[0] = 5 * B6; a[1] = -6 * B5; a[4] = rel0 * b * b * m; a[5] = -2 * rel0 * b * m;
            a[6] = rel0 * m;
            r_rel0 = nln_newton_root(a, 6, m_rel0, 0.001 * m_rel0) + 0.001 * m_rel0;
        }
        if (rel > 0 && isfinite(m_rel)) {
            for (int k = 0; k < 10; k++) a[k] = 0.0;
            a[0] = 5 * B6; a[1] = -6 * B5; a[4] = rel * b * b * m; a[5] = -2 * rel * b * m;
            a[6] = rel * m;
            r_rel = nln_newton_root(a, 6, m_rel, 0.001 * m_rel) + 0.001 * m_rel;
        }
        rc[2] = fmax(fmin(r_abs, r_rel), r_rel0);
    }
}

// Stack entries of one group's walk: at most 8 children per level are
// pending below each of at most 22 levels (21 key levels and the root).
#define NLN_WALK_STACK 256

// What the walk reads of a cell (80 bytes).
typedef struct nln_wcell {
    double cen[3];
    double bmax;
    double rc[3];      // critical radii: monopole, quadrupole, order 4
    int64_t first;
    int32_t count;
    int32_t child;     // first child cell, -1 for a leaf
    int32_t nchild;
    int32_t pad;
} nln_wcell;

NLN_HD inline uint32_t nln_shift_code(const int s[3]) {
    return (uint32_t)((s[0] + 1) * 9 + (s[1] + 1) * 3 + (s[2] + 1));
}

// Distance from y to the nearest nonzero lattice vector of the periodic cube.
// For y in the minimum-image cube (|y_k| <= L/2) that vector is a single
// step along one axis: a step along two axes i, j is no nearer since
// L^2 - 2 L |y_j| >= 0.  So the six axis steps suffice.
NLN_HD inline double nln_lattice_gap(const double y[3], double box) {
    double D2 = INFINITY;
    for (int k = 0; k < 3; k++)
        for (int a = -1; a <= 1; a += 2) {
            const double dx = y[0] - (k == 0 ? a * box : 0.0), dy = y[1] - (k == 1 ? a * box : 0.0),
                         dz = y[2] - (k == 2 ? a * box : 0.0);
            D2 = fmin(D2, dx * dx + dy * dy + dz * dz);
        }
    return sqrt(D2);
}

// The walk of one sink group (nln/mac.c:1703-1840 semantics: a cell is
// taken at the lowest order whose critical radius it clears, else opened;
// a leaf that cannot be taken expands to its bodies).  The MAC distance is
// reduced by the group radius, so every sink of the group passes the
// reference's per-sink test.
//
// Periodic boxes also get the group's correction list.  The correction
// needs every source in the same image as its Newtonian entry, but only
// near the half-box does that image depend on the walk: a cell whose
// bodies all lie strictly inside the group centre's minimum-image cube
// (|y|_inf + bmax < L/2) has every descendant entry in that same image.
// Such a cell enters the correction list whole, in place of its subtree's
// entries, once bmax + group radius <= ewald_theta x its distance to the
// correction's nearest singularity (the group's own image at a lattice
// vector); everywhere else the correction list repeats the Newtonian
// entries.  Stack entries carry that "covered" flag in bit 0.
//
// Emit receives the entries: p(e) point list (bodies: count in nb; cells:
// nm), q(e), h(e), c(e).  stack holds cap entries; returns 0, -1 when the
// group does not cover exactly the n bodies (the completeness invariant of
// nln/mac.c:734-735), -2 when the stack overflows.
template <class Emit>
NLN_HD inline int nln_walk_group(const nln_wcell *cells, const float *spos, int64_t n,
                                 const nln_group &G, const nln_mac &P, int32_t *stack, int cap,
                                 Emit &em) {
    const double box = P.box;
    const double theta = P.ewald_theta;
    const int p2 = P.p2cut, p4 = P.p4cut;
    const uint32_t nb = (uint32_t)n;
    int64_t covered = 0;
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const int32_t top = stack[--sp];
        const int32_t ci = top >> 1;
        bool ccov = (top & 1) != 0;
        const nln_wcell &c = cells[ci];
        double y[3];
        int s[3] = {0, 0, 0};
        for (int d = 0; d < 3; d++) {
            y[d] = c.cen[d] - G.cen[d];
            if (box > 0) {
                s[d] = -(int)nearbyint(y[d] / box);
                y[d] += s[d] * box;
            }
        }
        const double dist = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
        // Periodic: the cell is taken whole in the image nearest the group
        // centre.  Every sink-body displacement it implies must stay inside
        // the domain of the Ewald correction, |y_k| <= NLN_EWALD_REACH * box,
        // where the correction is smooth; otherwise the cell is opened.
        bool inside = true;
        const uint32_t sc = nln_shift_code(s);
        if (box > 0) {
            const double ym = fmax(fabs(y[0]), fmax(fabs(y[1]), fabs(y[2])));
            inside = ym + c.bmax + G.radius <= NLN_EWALD_REACH * box;
            if (!ccov && theta > 0 && c.count > 0 && ym + c.bmax < 0.5 * box * (1.0 - 1e-9) &&
                c.bmax + G.radius <= theta * nln_lattice_gap(y, box)) {
                em.c((nb + (uint32_t)ci) | (sc << NLN_IDX_BITS));
                ccov = true;
            }
        }
        const bool emit_c = box > 0 && !ccov;
        const double dd = dist - G.radius;
        if (inside && c.count > 0) {
            const bool take = dd > c.rc[0] + c.bmax ||
                              (p2 && c.count >= p2 && dd > c.rc[1] + c.bmax) ||
                              (p4 && c.count >= p4 && dd > c.rc[2] + c.bmax);
            if (take) {
                if (dd > c.rc[0] + c.bmax) {
                    em.p((nb + (uint32_t)ci) | (sc << NLN_IDX_BITS), false);
                } else if (p2 && c.count >= p2 && dd > c.rc[1] + c.bmax) {
                    em.q((uint32_t)ci | (sc << NLN_IDX_BITS));
                } else {
                    em.h((uint32_t)ci | (sc << NLN_IDX_BITS));
                }
                if (emit_c)
                    em.c((nb + (uint32_t)ci) | (sc << NLN_IDX_BITS));
                covered += c.count;
                continue;
            }
        }
        if (c.child >= 0) {
            if (sp + c.nchild > cap)
                return -2;
            for (int k = c.nchild - 1; k >= 0; k--) stack[sp++] = ((c.child + k) << 1) | (ccov ? 1 : 0);
            continue;
        }
        // leaf: expand to bodies (nln/mac.c:1817-1832)
        for (int32_t k = 0; k < c.count; k++) {
            uint32_t e;
            if (inside || box <= 0) {
                e = (uint32_t)(c.first + k) | (sc << NLN_IDX_BITS);
            } else {
                // a leaf reaching out of the correction's domain: each body its own image
                const float *x = spos + 3 * (c.first + k);
                int sb[3];
                for (int d = 0; d < 3; d++) sb[d] = -(int)nearbyint((x[d] - G.cen[d]) / box);
                e = (uint32_t)(c.first + k) | (nln_shift_code(sb) << NLN_IDX_BITS);
            }
            em.p(e, true);
            if (emit_c)
                em.c(e);
        }
        covered += c.count;
    }
    return covered == n ? 0 : -1;
}
