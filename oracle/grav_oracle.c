/*
 * grav_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity checker).
 *
 * A plain-C, double-precision restatement of the 2HOT tree-gravity
 * interaction algorithms of lanl/ahotsph-2hot-apps (nln/).  It is linked
 * only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg,
 * always as the checker; the product path never calls it.
 *
 * Pinning: every list kernel here is checked (tests/test_oracle_pin.py)
 * against the reference's own AVX kernels compiled unmodified from
 * nln/do_grav_avx8.c and nln/pgrav_vec.c into oracle/_ref (see
 * oracle/Makefile), and against the committed fixtures in tests/golden/
 * that were produced from those compiled reference kernels.  ewald() is
 * restated from nln/ewald.c; the reference file does not compile without
 * the absent 2hot headers (error.h, vop.h), so the restatement is pinned by
 * its own invariants (periodicity, the x=0 rule, symmetry) and by Ewald
 * sums of known lattices in tests/test_ewald.py.
 *
 * List format (the reference AoSoA of mac.c:117-153): blocks of 8 lanes;
 * block b holds `sz` fields, field k of lane l at f[(b*sz + k)*8 + l].
 *   fields 0..3  mass, x, y, z                       (MSZ = 4)
 *   field  4     R (= bmax)
 *   fields 5..7  qx, qy, qz (dipole; COM centres give zero)
 *   fields 8..12 qxx qxy qyy qxz qyz                 (QSZ = 13)
 *   fields 13..19 qxxx qxxy qxyy qyyy qxxz qxyz qyyz
 *   fields 20..28 qxxxx qxxxy qxxyy qxyyy qyyyy qxxxz qxxyz qxyyz qyyyz (HSZ = 29)
 * Moments are traceless and normalised by R^l (nln/cofm.c:398-420,486-562).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NL 8

/* kinds of list evaluation */
enum {
    ORC_MONO_PLUMMER = 0, /* do_gravp_avx8   nln/do_grav_avx8.c:2163-2216 */
    ORC_QUAD_PLUMMER = 1, /* do_gravpq_avx8  nln/do_grav_avx8.c:2090-2160 */
    ORC_HEXA_PLUMMER = 2, /* do_gravph_avx8  nln/do_grav_avx8.c:1779-1904 */
    ORC_MONO_MASKED = 3,  /* do_grav_avx8    nln/do_grav_avx8.c:953-1006 (r < e dropped) */
    ORC_MONO_K1 = 4,      /* do_grav_sK1_avx8 nln/do_grav_avx8.c:1047-1110 (e = 1/eps) */
    ORC_QUAD_COM = 5,     /* do_gravq_avx8   nln/do_grav_avx8.c:881-950 (no softening) */
    ORC_HEXA_COM = 6,     /* do_gravh_avx8   nln/do_grav_avx8.c:572-696 (no softening) */
    ORC_MONO_BARE = 7,    /* CUDA pM         nln/pgrav.cu:370-410 (no softening, no mask) */
    ORC_QUAD_PLUMMER_P = 8, /* do_gravpq_avx8 with the order-4 kernels' quadrupole potential
                              sign (+1, nln/do_grav_avx8.c:1846): the physical potential */
    ORC_QUAD_DIPOLE = 9   /* do_gravdq_avx8  nln/do_grav_avx8.c:378-459 (no softening, dipole
                             fields 5..7 about the record's centre; CUDA pQ1_mnss and pQQ1,
                             nln/pgrav.cu:293-368,498-572, compute the same terms) */
};

typedef struct {
    double m, x, y, z, R;
    double qx, qy, qz;
    double qxx, qxy, qyy, qxz, qyz;
    double qxxx, qxxy, qxyy, qyyy, qxxz, qxyz, qyyz;
    double qxxxx, qxxxy, qxxyy, qxyyy, qyyyy, qxxxz, qxxyz, qxyyz, qyyyz;
} orc_src;

/*
 * Dehnen K1 compensating kernel inside r < eps, as in sK1()
 * (nln/do_grav_avx8.c:1013-1045): u2 = r^2/eps^2 - 1,
 *   phi = -(1 + u2(-1/2 + u2(3/8 - 45/32 u2))) / eps
 *   a   = -(1 + u2(-3/2 + 135/16 u2)) / eps^3   (multiplies d = sink - source)
 */
static void k1_inside(double r2, double eps_inv, double *phi, double *a) {
    double u2 = r2 * eps_inv * eps_inv - 1.0;
    double t = ((-45.0 / 32.0 * u2 + 3.0 / 8.0) * u2 - 0.5) * u2 + 1.0;
    *phi = -t * eps_inv;
    t = (135.0 / 16.0 * u2 - 1.5) * u2 + 1.0;
    *a = -t * eps_inv * eps_inv * eps_inv;
}

/*
 * One sink, one source record: accumulate acc (3) and phi in double.
 * order 0: monopole, 2: + quadrupole, 4: + octupole + hexadecapole.
 * The algebra follows do_gravph_avx8 (nln/do_grav_avx8.c:1809-1898): with
 * d = sink - source and t = -1/r, each order l adds
 *   eq = t_l * (Q_l . d^(l-1)),  phi += c_l eq.d,  a += d (2l+1) rinv2 c_l eq.d - eq
 * with c_l = 1/2, 1/3, 1/4 and t_l = t_(l-1) (2l-1) rinv2 R.
 * qsign multiplies the quadrupole potential term: the reference's quad
 * kernels use -1 (do_gravpq, do_gravq: nln/do_grav_avx8.c:2150,940), its
 * order-4 CPU kernels +1 (nln/do_grav_avx8.c:1846,638).
 */
static void orc_interact(const orc_src *s, int order, double px, double py, double pz,
                         double eps2, double qsign, int dipole, double *acc, double *phi) {
    double x = px - s->x, y = py - s->y, z = pz - s->z;
    double r2 = x * x + y * y + z * z + eps2;
    double rinv = -1.0 / sqrt(r2);
    double t = rinv;
    double eqe = t * s->m;
    double rinv2 = t * t;
    t *= rinv2;
    *phi += eqe;
    eqe *= rinv2;
    acc[0] += x * eqe;
    acc[1] += y * eqe;
    acc[2] += z * eqe;
    if (order < 2)
        return;
    double R = s->R;
    if (dipole) {
        /* do_gravdq_avx8 (nln/do_grav_avx8.c:428-436): t_1 = t R,
         * eq = t_1 q, phi += eq.d, a += d 3 rinv2 eq.d - eq */
        double td = t * R;
        double e0 = td * s->qx, e1 = td * s->qy, e2 = td * s->qz;
        double ed = x * e0 + y * e1 + z * e2;
        *phi += ed;
        ed *= 3.0 * rinv2;
        acc[0] += x * ed - e0;
        acc[1] += y * ed - e1;
        acc[2] += z * ed - e2;
    }
    t *= 3.0 * rinv2 * R * R;
    double eq0 = t * (s->qxx * x + s->qxy * y + s->qxz * z);
    double eq1 = t * (s->qyy * y + s->qxy * x + s->qyz * z);
    double eq2 = t * (-(s->qxx + s->qyy) * z + s->qxz * x + s->qyz * y);
    eqe = 0.5 * (eq0 * x + eq1 * y + eq2 * z);
    *phi += qsign * eqe;
    eqe *= 5.0 * rinv2;
    acc[0] += x * eqe - eq0;
    acc[1] += y * eqe - eq1;
    acc[2] += z * eqe - eq2;
    if (order < 4)
        return;
    t *= 5.0 * rinv2 * R;
    double xx = 0.5 * x * x, xy = x * y, xz = x * z;
    double yy = 0.5 * y * y, yz = y * z, zz = 0.5 * z * z;
    double xxx = x * (xx / 3.0 - zz);
    double xxz = z * (xx - zz / 3.0);
    double yyy = y * (yy / 3.0 - zz);
    double yyz = z * (yy - zz / 3.0);
    xx -= zz;
    yy -= zz;
    eq0 = t * (s->qxxx * xx + s->qxyy * yy + s->qxxy * xy + s->qxxz * xz + s->qxyz * yz);
    eq1 = t * (s->qxyy * xy + s->qxxy * xx + s->qyyy * yy + s->qyyz * yz + s->qxyz * xz);
    eq2 = t * (-(s->qxxx + s->qxyy) * xz - (s->qxxy + s->qyyy) * yz + s->qxxz * xx
               + s->qyyz * yy + s->qxyz * xy);
    eqe = (eq0 * x + eq1 * y + eq2 * z) / 3.0;
    *phi += eqe;
    eqe *= 7.0 * rinv2;
    acc[0] += x * eqe - eq0;
    acc[1] += y * eqe - eq1;
    acc[2] += z * eqe - eq2;
    t *= 7.0 * rinv2 * R;
    double xxy = y * xx, xyy = x * yy, xyz = xy * z;
    eq0 = t * (s->qxxxx * xxx + s->qxyyy * yyy + s->qxxxy * xxy + s->qxxxz * xxz
               + s->qxxyy * xyy + s->qxxyz * xyz + s->qxyyz * yyz);
    eq1 = t * (s->qxyyy * xyy + s->qxxxy * xxx + s->qyyyy * yyy + s->qyyyz * yyz
               + s->qxxyy * xxy + s->qxxyz * xxz + s->qxyyz * xyz);
    eq2 = t * (-s->qxxxx * xxz - (s->qxyyy + s->qxxxy) * xyz - s->qyyyy * yyz + s->qxxxz * xxx
               + s->qyyyz * yyy - s->qxxyy * (xxz + yyz) + s->qxxyz * xxy + s->qxyyz * xyy);
    eqe = 0.25 * (eq0 * x + eq1 * y + eq2 * z);
    *phi += eqe;
    eqe *= 9.0 * rinv2;
    acc[0] += x * eqe - eq0;
    acc[1] += y * eqe - eq1;
    acc[2] += z * eqe - eq2;
}

static void load_lane(const float *f, long b, int sz, int l, orc_src *s) {
    const float *blk = f + (size_t)b * sz * NL;
#define FLD(k) ((k) < sz ? (double)blk[(k)*NL + l] : 0.0)
    s->m = FLD(0);
    s->x = FLD(1);
    s->y = FLD(2);
    s->z = FLD(3);
    s->R = FLD(4);
    s->qx = FLD(5);
    s->qy = FLD(6);
    s->qz = FLD(7);
    s->qxx = FLD(8);
    s->qxy = FLD(9);
    s->qyy = FLD(10);
    s->qxz = FLD(11);
    s->qyz = FLD(12);
    s->qxxx = FLD(13);
    s->qxxy = FLD(14);
    s->qxyy = FLD(15);
    s->qyyy = FLD(16);
    s->qxxz = FLD(17);
    s->qxyz = FLD(18);
    s->qyyz = FLD(19);
    s->qxxxx = FLD(20);
    s->qxxxy = FLD(21);
    s->qxxyy = FLD(22);
    s->qxyyy = FLD(23);
    s->qyyyy = FLD(24);
    s->qxxxz = FLD(25);
    s->qxxyz = FLD(26);
    s->qxyyz = FLD(27);
    s->qyyyz = FLD(28);
#undef FLD
}

/*
 * Evaluate one sink (pos0) against nblk 8-lane blocks of an AoSoA list of
 * field count sz, with the semantics of reference kernel `kind`.
 * e: eps^2 for the Plummer kinds (mac.c:235,499), eps for ORC_MONO_MASKED,
 * 1/eps for ORC_MONO_K1, ignored otherwise.  out[0..2] += acc, out[3] += phi.
 * Returns the number of lanes inside the K1 radius (the reference's ncut).
 */
int orc_list_eval(int kind, const float *f, long nblk, int sz, const float *pos0, float e,
                  double *out) {
    double acc[3] = {0, 0, 0}, phi = 0.0;
    double px = pos0[0], py = pos0[1], pz = pos0[2];
    int order = 0, ncut = 0;
    double eps2 = 0.0, qsign = 1.0;
    switch (kind) {
    case ORC_MONO_PLUMMER: eps2 = e; break;
    case ORC_QUAD_PLUMMER: eps2 = e; order = 2; qsign = -1.0; break;
    case ORC_HEXA_PLUMMER: eps2 = e; order = 4; qsign = 1.0; break;
    case ORC_QUAD_COM: order = 2; qsign = -1.0; break;
    case ORC_HEXA_COM: order = 4; qsign = 1.0; break;
    case ORC_QUAD_PLUMMER_P: eps2 = e; order = 2; qsign = 1.0; break;
    case ORC_QUAD_DIPOLE: order = 2; qsign = -1.0; break;
    default: break;
    }
    const int dipole = kind == ORC_QUAD_DIPOLE;
    for (long b = 0; b < nblk; b++) {
        for (int l = 0; l < NL; l++) {
            orc_src s;
            load_lane(f, b, sz, l, &s);
            if (kind == ORC_MONO_MASKED) {
                double x = px - s.x, y = py - s.y, z = pz - s.z;
                double r2 = x * x + y * y + z * z;
                if (r2 < (double)e * (double)e)
                    continue;
                orc_interact(&s, 0, px, py, pz, 0.0, 1.0, 0, acc, &phi);
            } else if (kind == ORC_MONO_K1) {
                double x = px - s.x, y = py - s.y, z = pz - s.z;
                double r2 = x * x + y * y + z * z;
                double ei = e;
                if (r2 < 1.0 / (ei * ei)) {
                    double kp, ka;
                    k1_inside(r2, ei, &kp, &ka);
                    phi += s.m * kp;
                    acc[0] += x * s.m * ka;
                    acc[1] += y * s.m * ka;
                    acc[2] += z * s.m * ka;
                    ncut++;
                } else {
                    orc_interact(&s, 0, px, py, pz, 0.0, 1.0, 0, acc, &phi);
                }
            } else {
                orc_interact(&s, order, px, py, pz, eps2, qsign, dipole, acc, &phi);
            }
        }
    }
    out[0] += acc[0];
    out[1] += acc[1];
    out[2] += acc[2];
    out[3] += phi;
    return ncut;
}

/*
 * MxN form: m sinks at p + i*stride (positions at float offsets 1..3, as the
 * reference passes &body.mass, nln/pgrav_vec.c:267-270) against the same
 * list; accp[i*stride + 0..3] += (ax, ay, az, phi) rounded to float, as
 * pMinteract/pQinteract/pHinteract do (nln/pgrav_vec.c:45-300).
 */
void orc_mxn_eval(int kind, const float *p, float *accp, int m, int stride, const float *f,
                  long nblk, int sz, float e) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < m; i++) {
        double out[4] = {0, 0, 0, 0};
        orc_list_eval(kind, f, nblk, sz, p + (size_t)i * stride + 1, e, out);
        for (int k = 0; k < 4; k++) accp[(size_t)i * stride + k] += (float)out[k];
    }
}

/*
 * Body-segment K1 monopole, do_gravmm_sK1_avx8 (nln/do_grav_avx8.c:1112-1201):
 * sources are runs seg[k] = {base, length} of a strided position table
 * (xyz + base*stride), all of mass pmass; e = 1/eps.  Returns the number of
 * source interactions walked (the reference's checksum against source_n).
 */
long orc_segments_k1(const float *xyz, int stride, float pmass, const uint32_t *seg, int nseg,
                     const float *pos0, float e, double *out) {
    double acc[3] = {0, 0, 0}, phi = 0.0;
    long n = 0;
    double ei = e;
    for (int k = 0; k < nseg; k++) {
        uint32_t base = seg[2 * k], len = seg[2 * k + 1];
        for (uint32_t j = 0; j < len; j++) {
            const float *q = xyz + (size_t)(base + j) * stride;
            double x = pos0[0] - (double)q[0], y = pos0[1] - (double)q[1],
                   z = pos0[2] - (double)q[2];
            double r2 = x * x + y * y + z * z;
            if (r2 < 1.0 / (ei * ei)) {
                double kp, ka;
                k1_inside(r2, ei, &kp, &ka);
                phi += pmass * kp;
                acc[0] += x * pmass * ka;
                acc[1] += y * pmass * ka;
                acc[2] += z * pmass * ka;
            } else {
                double rinv = -1.0 / sqrt(r2);
                double eqe = pmass * rinv;
                phi += eqe;
                eqe *= rinv * rinv;
                acc[0] += x * eqe;
                acc[1] += y * eqe;
                acc[2] += z * eqe;
            }
            n++;
        }
    }
    out[0] += acc[0];
    out[1] += acc[1];
    out[2] += acc[2];
    out[3] += phi;
    return n;
}

/*
 * FP64 direct sum, isolated, Plummer softening (the scalar do_grav of
 * nln/grav.c:46-79 summed over every source, self included, in double as
 * the N^2 oracle of nln/grav_n2.c:17-23,162-173 accumulates):
 *   acc_i = sum_j m_j (x_j - x_i) / (r^2 + eps2)^1.5,  phi_i = -sum_j m_j / (r^2 + eps2)^0.5
 * sinks: nsink indices into pos (xyz, 3 doubles each).  G is applied by the caller.
 */
void orc_direct(const double *pos, const double *mass, long n, double eps2, const long *sinks,
                long nsink, double *acc, double *phi) {
#pragma omp parallel for schedule(dynamic, 4)
    for (long k = 0; k < nsink; k++) {
        long i = sinks[k];
        double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
        double ax = 0, ay = 0, az = 0, ph = 0;
        for (long j = 0; j < n; j++) {
            double x = pos[3 * j] - xi, y = pos[3 * j + 1] - yi, z = pos[3 * j + 2] - zi;
            double r2 = x * x + y * y + z * z + eps2;
            if (r2 == 0.0)
                continue;
            double rinv = 1.0 / sqrt(r2);
            double mr3 = mass[j] * rinv * rinv * rinv;
            ax += x * mr3;
            ay += y * mr3;
            az += z * mr3;
            ph -= mass[j] * rinv;
        }
        acc[3 * k] = ax;
        acc[3 * k + 1] = ay;
        acc[3 * k + 2] = az;
        phi[k] = ph;
    }
}

/*
 * Periodic Green's function of a unit point mass in a cube of side L, the
 * Ewald sum of nln/ewald.c:13-64: for x = x_source - x_sink,
 *   alpha = 2/L, phi0 = pi/(alpha^2 L^3); x == 0 returns phi0 and f = 0;
 *   real space over |n_k| <= 4 with |x - nL| <= 4L:
 *     t = (erfc(alpha r)/r + 2 alpha/sqrt(pi) exp(-alpha^2 r^2)) / r^2,
 *     f += t (x - nL), phi -= erfc(alpha r)/r
 *   k space over 0 < |h|^2 <= 16:
 *     f += (2/L^2) exp(-pi^2 h^2/(alpha L)^2) sin(2 pi h.x/L)/h^2 h
 *     phi -= (1/(pi L)) exp(...) cos(2 pi h.x/L)/h^2
 * f is the force on the sink (towards the source), phi the potential.
 */
void orc_ewald(const double *x, double L, double *f, double *phi) {
    const int N = 4;
    double alpha = 2.0 / L;
    f[0] = f[1] = f[2] = 0.0;
    *phi = M_PI / (alpha * alpha * L * L * L);
    if (x[0] == 0.0 && x[1] == 0.0 && x[2] == 0.0)
        return;
    double a1 = 2.0 * alpha / sqrt(M_PI);
    double a2 = -M_PI * M_PI / (alpha * alpha * L * L);
    double a3 = 2.0 * M_PI / L;
    double a4 = 2.0 / (L * L);
    double a5 = 1.0 / (M_PI * L);
    for (int i = -N; i <= N; i++)
        for (int j = -N; j <= N; j++)
            for (int k = -N; k <= N; k++) {
                double xx = x[0] - L * i, yy = x[1] - L * j, zz = x[2] - L * k;
                double ax2 = xx * xx + yy * yy + zz * zz;
                double axx = sqrt(ax2);
                if (axx > 4.0 * L)
                    continue;
                double t1 = erfc(alpha * axx);
                double t2 = a1 * exp(-alpha * alpha * ax2);
                double t = (t1 / axx + t2) / ax2;
                f[0] += t * xx;
                f[1] += t * yy;
                f[2] += t * zz;
                *phi -= t1 / axx;
            }
    for (int i = -N; i <= N; i++)
        for (int j = -N; j <= N; j++)
            for (int k = -N; k <= N; k++) {
                double hh = (double)(i * i + j * j + k * k);
                if (hh > 16 || hh == 0)
                    continue;
                double hx = i * x[0] + j * x[1] + k * x[2];
                double t = a4 * exp(a2 * hh) * sin(a3 * hx) / hh;
                f[0] += t * i;
                f[1] += t * j;
                f[2] += t * k;
                *phi -= a5 * exp(a2 * hh) * cos(a3 * hx) / hh;
            }
}

/* Batch form of orc_ewald for n displacements (OpenMP). */
void orc_ewald_batch(const double *x, long n, double L, double *f, double *phi) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) orc_ewald(x + 3 * i, L, f + 3 * i, phi + i);
}

/*
 * FP64 Ewald-summed direct sum on a sample of sinks, EwaldForces of
 * nln/grav_n2.c:97-196 (FP64 accumulation, no softening, x = b.pos - q.pos,
 * G applied by the caller).  With eps2 > 0 the nearest-image Newtonian term
 * of each pair is replaced by its Plummer-softened form, so the oracle has
 * the same short-range force law as the tree code it checks.
 */
void orc_direct_ewald(const double *pos, const double *mass, long n, double L, double eps2,
                      const long *sinks, long nsink, double *acc, double *phi) {
#pragma omp parallel for schedule(dynamic, 1)
    for (long k = 0; k < nsink; k++) {
        long i = sinks[k];
        double ax = 0, ay = 0, az = 0, ph = 0;
        for (long j = 0; j < n; j++) {
            double x[3], f[3], p;
            for (int d = 0; d < 3; d++) x[d] = pos[3 * j + d] - pos[3 * i + d];
            orc_ewald(x, L, f, &p);
            if (eps2 > 0.0) {
                double y[3];
                for (int d = 0; d < 3; d++) y[d] = x[d] - L * nearbyint(x[d] / L);
                double r2 = y[0] * y[0] + y[1] * y[1] + y[2] * y[2];
                if (r2 > 0.0) {
                    double r = sqrt(r2), rs2 = r2 + eps2, rs = sqrt(rs2);
                    double dk = 1.0 / (r2 * r) - 1.0 / (rs2 * rs);
                    for (int d = 0; d < 3; d++) f[d] -= y[d] * dk;
                    p += 1.0 / r - 1.0 / rs;
                } else {
                    p -= 1.0 / sqrt(eps2);
                }
            }
            ax += mass[j] * f[0];
            ay += mass[j] * f[1];
            az += mass[j] * f[2];
            ph += mass[j] * p;
        }
        acc[3 * k] = ax;
        acc[3 * k + 1] = ay;
        acc[3 * k + 2] = az;
        phi[k] = ph;
    }
}

/*
 * Grouped evaluation over whole-tree lists, the way nln/mac.c's leaf loop
 * applies one list to every sink below a node (mac.c:549-676): group g owns
 * sinks [sink_first[g], +sink_count[g]) of pos (xyz floats) and list blocks
 * [blk_first[g], +blk_count[g]) of f.  out (4 doubles per sink) accumulates.
 */
void orc_groups_eval(int kind, const float *f, int sz, const long *blk_first,
                     const long *blk_count, const long *sink_first, const int *sink_count,
                     long ngroups, const float *pos, float e, double *out) {
#pragma omp parallel for schedule(dynamic, 4)
    for (long g = 0; g < ngroups; g++) {
        const float *fb = f + (size_t)blk_first[g] * sz * NL;
        for (int s = 0; s < sink_count[g]; s++) {
            long i = sink_first[g] + s;
            orc_list_eval(kind, fb, blk_count[g], sz, pos + 3 * i, e, out + 4 * i);
        }
    }
}

/*
 * FP64 gradient of L = sum_i w_i.a_i + u_i phi_i for the Plummer-softened
 * direct sum over all pairs, the self pair included as the tree's lists
 * include it (it adds -m_i / eps to phi_i and nothing to a_i): dL/dx (3 per
 * body), dL/dm.  With d = x_i - x_j, rho^2 = |d|^2 + eps2, the pair adds to
 * body i -(m_j)[rho^-3 w_i - 3 rho^-5 (w_i.d) d - u_i rho^-3 d] and the
 * opposite to body j, and dL/dm_j -= rho^-3 w_i.d + u_i rho^-1 (sink i,
 * source j); the self pair adds -u_i / eps to dL/dm_i.
 */
void orc_direct_grad(long n, const double *x, const double *m, const double *w, const double *u,
                     double eps2, double *gx, double *gm) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long i = 0; i < n; i++) {
        double g[3] = {0, 0, 0};
        double gmi = 0;
        for (long j = 0; j < n; j++) {
            if (j == i)
                continue;
            /* sink i, source j */
            double d[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
            double rho2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + eps2;
            double ri = 1.0 / sqrt(rho2), ri3 = ri * ri * ri, ri5 = ri3 * ri * ri;
            double wd = w[3 * i] * d[0] + w[3 * i + 1] * d[1] + w[3 * i + 2] * d[2];
            for (int k = 0; k < 3; k++)
                g[k] -= m[j] * (ri3 * w[3 * i + k] - 3.0 * ri5 * wd * d[k] - u[i] * ri3 * d[k]);
            /* sink j, source i: the same pair seen from j; dL/dm_i from sink j */
            double dj[3] = {-d[0], -d[1], -d[2]};
            double wdj = w[3 * j] * dj[0] + w[3 * j + 1] * dj[1] + w[3 * j + 2] * dj[2];
            for (int k = 0; k < 3; k++)
                g[k] += m[i] * (ri3 * w[3 * j + k] - 3.0 * ri5 * wdj * dj[k] - u[j] * ri3 * dj[k]);
            gmi -= ri3 * wdj + u[j] * ri;
        }
        if (eps2 > 0.0)
            gmi -= u[i] / sqrt(eps2);
        for (int k = 0; k < 3; k++) gx[3 * i + k] = g[k];
        gm[i] = gmi;
    }
}

/*
 * ---- FP64 evaluation of fixed lists of every kind, periodic boxes included ----
 *
 * The general form of orc_lists_eval64: point (kind 0), quadrupole (1) and
 * order-4 (2) lists and the periodic correction list (3), with the image
 * shift of every entry.  Cells' moments come from their bodies in FP64:
 * mass M, centre of mass X and the symmetric trace-free (STF) parts A_l of
 * the raw moments sum m y^l (y = x - X), l = 2, 3, 4, held as full tensors
 * of 3^l entries.  A cell of order L adds to its monopole term the exact
 * harmonic terms of the Taylor series of 1/|d - y| (d = sink - source),
 *     phi_l = -g_l <A_l, d^l> rho^-(2l+1),   g_l = (2l-1)!! / l!,
 *     a_l   = g_l (l A_l.d^(l-1) rho^-(2l+1) - (2l+1) <A_l, d^l> rho^-(2l+3) d),
 * with the Plummer rho^2 = |d|^2 + eps2 of the list kernels (nln/cofm.c
 * normalises the same STF moments by R^l, :398-420, 486-562; the order-4
 * kernel do_gravph_avx8, nln/do_grav_avx8.c:1779-1904, evaluates these
 * terms in its own variables).  Correction-list entries (point-table
 * records: a body, or a cell n + c standing for all of its bodies) add, for
 * every body b of the entry, m_b C(y) to phi and m_b grad C(y) to a, with
 * y = x_b + shift - x_sink and C(y) = Phi(y) + 1/|y| the periodic Green's
 * function of orc_ewald less the nearest-image Newtonian term (C(0) its
 * limit); every sink then adds -m_i (C(0) - pi/(alpha^2 L^3)), the self
 * term the Ewald sum leaves out.  This is the exact sum the list kernels'
 * cell moments and Taylor series approximate.
 */
#define ORC_IDX_MASK ((1u << 27) - 1u)

typedef struct {
    double M, X[3];
    double A[3][81]; /* A_2, A_3, A_4 as full tensors, index i1*3^(l-1) + ... + il */
} orc_momx;

static const int orc_pow3[5] = {1, 3, 9, 27, 81};

/* STF part of the full symmetric tensor T of order l (2..4) into A. */
static void stf_project(int l, const double *T, double *A) {
    if (l == 2) {
        double tr = (T[0] + T[4] + T[8]) / 3.0;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) A[3 * i + j] = T[3 * i + j] - (i == j ? tr : 0.0);
    } else if (l == 3) {
        double t[3];
        for (int k = 0; k < 3; k++) t[k] = T[9 * k + 0] + T[9 * k + 4] + T[9 * k + 8];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                for (int k = 0; k < 3; k++)
                    A[9 * i + 3 * j + k] = T[9 * i + 3 * j + k] -
                                           ((i == j ? t[k] : 0.0) + (i == k ? t[j] : 0.0) +
                                            (j == k ? t[i] : 0.0)) / 5.0;
    } else {
        double t2[9], tt = 0.0;
        for (int k = 0; k < 3; k++)
            for (int q = 0; q < 3; q++)
                t2[3 * k + q] = T[27 * k + 9 * q + 0] + T[27 * k + 9 * q + 4] + T[27 * k + 9 * q + 8];
        tt = t2[0] + t2[4] + t2[8];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                for (int k = 0; k < 3; k++)
                    for (int q = 0; q < 3; q++) {
                        double s6 = (i == j ? t2[3 * k + q] : 0.0) + (i == k ? t2[3 * j + q] : 0.0) +
                                    (i == q ? t2[3 * j + k] : 0.0) + (j == k ? t2[3 * i + q] : 0.0) +
                                    (j == q ? t2[3 * i + k] : 0.0) + (k == q ? t2[3 * i + j] : 0.0);
                        double s3 = (i == j && k == q ? 1.0 : 0.0) + (i == k && j == q ? 1.0 : 0.0) +
                                    (i == q && j == k ? 1.0 : 0.0);
                        A[27 * i + 9 * j + 3 * k + q] =
                            T[27 * i + 9 * j + 3 * k + q] - s6 / 7.0 + s3 * tt / 35.0;
                    }
    }
}

/* Mass, centre of mass and the trace-free moments up to order `order`
   (0 or 1: none; 2: A_2; 4: A_2..A_4) of a cell's bodies. */
static void cell_momx_upto(const double *x, const double *m, long first, int count, int order,
                           orc_momx *o) {
    double M = 0, s[3] = {0, 0, 0};
    for (long b = first; b < first + count; b++) {
        M += m[b];
        for (int d = 0; d < 3; d++) s[d] += m[b] * x[3 * b + d];
    }
    o->M = M;
    for (int d = 0; d < 3; d++) o->X[d] = M > 0 ? s[d] / M : 0.0;
    double T[81];
    for (int l = 2; l <= order; l++) {
        memset(T, 0, sizeof(T));
        for (long b = first; b < first + count; b++) {
            double y[3] = {x[3 * b] - o->X[0], x[3 * b + 1] - o->X[1], x[3 * b + 2] - o->X[2]};
            for (int t = 0; t < orc_pow3[l]; t++) {
                double p = m[b];
                for (int k = 0, r = t; k < l; k++, r /= 3) p *= y[r % 3];
                T[t] += p;
            }
        }
        stf_project(l, T, o->A[l - 2]);
    }
}

static void cell_momx(const double *x, const double *m, long first, int count, orc_momx *o) {
    cell_momx_upto(x, m, first, count, 4, o);
}

/* Monopole plus orders 2..order of a cell at X (M, A) on a sink at s. */
static void termx(const double *s, const double *X, double M, const orc_momx *c, int order,
                  double eps2, double *a, double *phi) {
    const double d[3] = {s[0] - X[0], s[1] - X[1], s[2] - X[2]};
    const double rho2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + eps2;
    const double ri = 1.0 / sqrt(rho2), ri2 = ri * ri;
    *phi -= M * ri;
    for (int k = 0; k < 3; k++) a[k] -= M * d[k] * ri * ri2;
    static const double g[5] = {0, 0, 1.5, 2.5, 4.375};
    for (int l = 2; l <= order; l++) {
        const double *A = c->A[l - 2];
        double P = 0.0, E[3] = {0, 0, 0};
        for (int t = 0; t < orc_pow3[l]; t++) {
            /* t = i1 * 3^(l-1) + rest: E_i1 takes the rest's monomial */
            double mono = 1.0;
            int r = t;
            for (int k = 0; k < l - 1; k++, r /= 3) mono *= d[r % 3];
            const int i1 = r % 3;
            E[i1] += A[t] * mono;
            P += A[t] * mono * d[i1];
        }
        const int n = 2 * l + 1;
        const double rn = pow(ri, n), rn2 = rn * ri2;
        *phi -= g[l] * P * rn;
        for (int k = 0; k < 3; k++) a[k] += g[l] * (l * E[k] * rn - n * P * rn2 * d[k]);
    }
}

static void decode_shift64(unsigned code, double box, double *sh) {
    sh[0] = ((int)(code / 9) - 1) * box;
    sh[1] = ((int)(code / 3 % 3) - 1) * box;
    sh[2] = ((int)(code % 3) - 1) * box;
}

/* C(0) = lim_{y->0} Phi(y) + 1/|y| of orc_ewald's sum (the n = 0 real-space
   term erfc(alpha r)/r - 1/r tends to -2 alpha/sqrt(pi)). */
double orc_ewald_c0(double L) {
    const int N = 4;
    double alpha = 2.0 / L;
    double phi = M_PI / (alpha * alpha * L * L * L) + 2.0 * alpha / sqrt(M_PI);
    double a2 = -M_PI * M_PI / (alpha * alpha * L * L), a5 = 1.0 / (M_PI * L);
    for (int i = -N; i <= N; i++)
        for (int j = -N; j <= N; j++)
            for (int k = -N; k <= N; k++) {
                double r = L * sqrt((double)(i * i + j * j + k * k));
                if (r == 0.0 || r > 4.0 * L)
                    continue;
                phi -= erfc(alpha * r) / r;
            }
    for (int i = -N; i <= N; i++)
        for (int j = -N; j <= N; j++)
            for (int k = -N; k <= N; k++) {
                double hh = (double)(i * i + j * j + k * k);
                if (hh > 16 || hh == 0)
                    continue;
                phi -= a5 * exp(a2 * hh) / hh;
            }
    return phi;
}

/* One body of mass mb at y (source + shift - sink) through the correction C. */
static void corr_body(const double *y, double mb, double L, double c0, double *a, double *phi) {
    if (y[0] == 0.0 && y[1] == 0.0 && y[2] == 0.0) {
        *phi += mb * c0;
        return;
    }
    double f[3], p;
    orc_ewald(y, L, f, &p);
    const double r2 = y[0] * y[0] + y[1] * y[1] + y[2] * y[2], r = sqrt(r2);
    *phi += mb * (p + 1.0 / r);
    for (int k = 0; k < 3; k++) a[k] += mb * (f[k] - y[k] / (r2 * r));
}

/* Lists of one group, as the arrays of the general evaluators. */
typedef struct {
    long n, ncells;
    const double *x, *m;
    const long *cfirst;
    const int *ccount;
    const long *ptr[4];
    const unsigned *list[4];
    double eps2, box;
    int ewald;
    double c0, self;
} orc_lx;

/* (a, phi) of sink i over group g's lists; moms: every cell's moments. */
static void sink_lists(const orc_lx *P, const orc_momx *moms, long g, long i, double *a,
                       double *phi) {
    const double *s = P->x + 3 * i;
    for (int kind = 0; kind < 3; kind++) {
        if (!P->ptr[kind])
            continue;
        for (long e = P->ptr[kind][g]; e < P->ptr[kind][g + 1]; e++) {
            const unsigned ent = P->list[kind][e], idx = ent & ORC_IDX_MASK;
            double sh[3], X[3];
            decode_shift64(ent >> 27, P->box, sh);
            if (kind == 0 && (long)idx < P->n) {
                for (int k = 0; k < 3; k++) X[k] = P->x[3 * (long)idx + k] + sh[k];
                termx(s, X, P->m[idx], NULL, 0, P->eps2, a, phi);
            } else {
                const orc_momx *c = &moms[kind == 0 ? (long)idx - P->n : (long)idx];
                for (int k = 0; k < 3; k++) X[k] = c->X[k] + sh[k];
                termx(s, X, c->M, c, kind == 0 ? 0 : kind == 1 ? 2 : 4, P->eps2, a, phi);
            }
        }
    }
    if (P->ewald && P->ptr[3]) {
        for (long e = P->ptr[3][g]; e < P->ptr[3][g + 1]; e++) {
            const unsigned ent = P->list[3][e], idx = ent & ORC_IDX_MASK;
            double sh[3];
            decode_shift64(ent >> 27, P->box, sh);
            long b0 = idx, b1 = (long)idx + 1;
            if ((long)idx >= P->n) {
                b0 = P->cfirst[idx - P->n];
                b1 = b0 + P->ccount[idx - P->n];
            }
            for (long b = b0; b < b1; b++) {
                double y[3];
                for (int k = 0; k < 3; k++) y[k] = P->x[3 * b + k] + sh[k] - s[k];
                corr_body(y, P->m[b], P->box, P->c0, a, phi);
            }
        }
        *phi -= P->m[i] * P->self;
    }
}

static void lx_init(orc_lx *P, long n, const double *x, const double *m, long ncells,
                    const long *cfirst, const int *ccount, const long *const *ptr,
                    const unsigned *const *list, double eps2, double box, int ewald) {
    P->n = n;
    P->ncells = ncells;
    P->x = x;
    P->m = m;
    P->cfirst = cfirst;
    P->ccount = ccount;
    for (int k = 0; k < 4; k++) {
        P->ptr[k] = ptr[k];
        P->list[k] = list[k];
    }
    P->eps2 = eps2;
    P->box = box;
    P->ewald = ewald && box > 0.0;
    P->c0 = P->ewald ? orc_ewald_c0(box) : 0.0;
    P->self = P->ewald ? P->c0 - M_PI / (4.0 / (box * box) * box * box * box) : 0.0;
}

/*
 * out (4 doubles per body, tree order) = (a, phi) of every sink over its
 * group's lists of every kind (ptr[k] / list[k] NULL for a kind without
 * lists; k = 0 P, 1 Q, 2 H, 3 correction, the last only with ewald and
 * box > 0).
 */
void orc_lists_eval64x(long n, const double *x, const double *m, long ncells, const long *cfirst,
                       const int *ccount, long ngroups, const long *gfirst, const int *gcount,
                       const long *const *ptr, const unsigned *const *list, double eps2,
                       double box, int ewald, double *out) {
    orc_lx P;
    lx_init(&P, n, x, m, ncells, cfirst, ccount, ptr, list, eps2, box, ewald);
    orc_momx *mom = (orc_momx *)malloc(sizeof(orc_momx) * (size_t)(ncells > 0 ? ncells : 1));
#pragma omp parallel for schedule(dynamic, 64)
    for (long c = 0; c < ncells; c++) cell_momx(x, m, cfirst[c], ccount[c], &mom[c]);
#pragma omp parallel for schedule(dynamic, 4)
    for (long g = 0; g < ngroups; g++) {
        for (int k = 0; k < gcount[g]; k++) {
            long i = gfirst[g] + k;
            double a[3] = {0, 0, 0}, phi = 0;
            sink_lists(&P, mom, g, i, a, &phi);
            for (int d = 0; d < 3; d++) out[4 * i + d] = a[d];
            out[4 * i + 3] = phi;
        }
    }
    free(mom);
}

/*
 * The entries of every kind that depend on the selected bodies sel[0..nsel)
 * (nsel <= 64), as orc_fd_hits: 3 longs per hit (group, kind 0..3,
 * position) and the mask of the selected bodies it depends on.  Point and
 * correction entries are point-table records (bodies, cells n + c);
 * quadrupole and order-4 entries are cells.
 */
long orc_fd_hits_x(long n, long ncells, const int *cparent, long ngroups, const long *const *ptr,
                   const unsigned *const *list, int nsel, const long *sel, const long *body_leaf,
                   long cap, long *hits, unsigned long long *hmask) {
    if (nsel > 64)
        return -1;
    unsigned long long *mask = (unsigned long long *)calloc((size_t)(n + ncells), 8);
    for (int s = 0; s < nsel; s++) {
        unsigned long long bit = 1ull << s;
        mask[sel[s]] |= bit;
        for (long c = body_leaf[sel[s]]; c >= 0; c = cparent[c]) mask[n + c] |= bit;
    }
    long nh = 0;
    for (long g = 0; g < ngroups; g++) {
        for (int kind = 0; kind < 4; kind++) {
            if (!ptr[kind])
                continue;
            for (long e = ptr[kind][g]; e < ptr[kind][g + 1]; e++) {
                long idx = (long)(list[kind][e] & ORC_IDX_MASK) + (kind == 1 || kind == 2 ? n : 0);
                if (!mask[idx])
                    continue;
                if (hits && nh < cap) {
                    hits[3 * nh] = g;
                    hits[3 * nh + 1] = kind;
                    hits[3 * nh + 2] = e;
                    hmask[nh] = mask[idx];
                }
                nh++;
            }
        }
    }
    free(mask);
    return nh;
}

/*
 * The part of L = sum_i w_i.a_i + u_i phi_i (orc_lists_eval64x's sums,
 * fixed lists) that depends on body j = sel[s], as orc_fd_partial_loss:
 * every hit carrying bit s over its group's sinks other than j (for a
 * correction entry only body j's own term, the entry's other bodies being
 * constant), plus sink j over its own group's whole lists.
 */
double orc_fd_partial_loss_x(int s, long j, long n, const double *x, const double *m, long ncells,
                             const long *cfirst, const int *ccount, long ngroups,
                             const long *gfirst, const int *gcount, const long *body_group,
                             const long *const *ptr, const unsigned *const *list, long nhits,
                             const long *hits, const unsigned long long *hmask, const double *w,
                             const double *u, double eps2, double box, int ewald) {
    orc_lx P;
    lx_init(&P, n, x, m, ncells, cfirst, ccount, ptr, list, eps2, box, ewald);
    const unsigned long long bit = 1ull << s;
    double L = 0.0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : L)
    for (long h = 0; h < nhits; h++) {
        if (!(hmask[h] & bit))
            continue;
        const long g = hits[3 * h], kind = hits[3 * h + 1], e = hits[3 * h + 2];
        const unsigned ent = list[kind][e], idx = ent & ORC_IDX_MASK;
        double sh[3];
        decode_shift64(ent >> 27, box, sh);
        orc_momx mo;
        double X[3], M = 0.0;
        int order = 0, corr = kind == 3;
        if (corr) {
            if (!P.ewald)
                continue;
            for (int k = 0; k < 3; k++) X[k] = x[3 * j + k] + sh[k];
            M = m[j];
        } else if (kind == 0 && (long)idx < n) {
            for (int k = 0; k < 3; k++) X[k] = x[3 * (long)idx + k] + sh[k];
            M = m[idx];
        } else {
            const long c = kind == 0 ? (long)idx - n : (long)idx;
            order = kind == 0 ? 0 : kind == 1 ? 2 : 4;
            cell_momx_upto(x, m, cfirst[c], ccount[c], order, &mo);
            for (int k = 0; k < 3; k++) X[k] = mo.X[k] + sh[k];
            M = mo.M;
        }
        for (int k = 0; k < gcount[g]; k++) {
            long i = gfirst[g] + k;
            if (i == j)
                continue;
            double a[3] = {0, 0, 0}, phi = 0;
            if (corr) {
                double y[3] = {X[0] - x[3 * i], X[1] - x[3 * i + 1], X[2] - x[3 * i + 2]};
                corr_body(y, M, box, P.c0, a, &phi);
            } else {
                termx(x + 3 * i, X, M, &mo, order, eps2, a, &phi);
            }
            L += w[3 * i] * a[0] + w[3 * i + 1] * a[1] + w[3 * i + 2] * a[2] + u[i] * phi;
        }
    }
    /* sink j over its own lists, cells' moments from the bodies */
    const long g = body_group[j];
    double a[3] = {0, 0, 0}, phi = 0;
    orc_momx *moms = (orc_momx *)calloc((size_t)(ncells > 0 ? ncells : 1), sizeof(orc_momx));
    char *done = (char *)calloc((size_t)(ncells > 0 ? ncells : 1), 1);
    for (int kind = 0; kind < 3; kind++) {
        if (!ptr[kind])
            continue;
        for (long e = ptr[kind][g]; e < ptr[kind][g + 1]; e++) {
            const unsigned idx = list[kind][e] & ORC_IDX_MASK;
            if (kind == 0 && (long)idx < n)
                continue;
            const long c = kind == 0 ? (long)idx - n : (long)idx;
            const int need = kind == 0 ? 1 : kind == 1 ? 2 : 4;
            if (done[c] < need) {
                cell_momx_upto(x, m, cfirst[c], ccount[c], need, &moms[c]);
                done[c] = (char)need;
            }
        }
    }
    orc_lx Q = P;
    Q.ewald = 0;
    sink_lists(&Q, moms, g, j, a, &phi);
    if (P.ewald && ptr[3]) {
        double lc = 0.0;
        const long e0 = ptr[3][g], e1 = ptr[3][g + 1];
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : lc)
        for (long e = e0; e < e1; e++) {
            const unsigned ent = list[3][e], idx = ent & ORC_IDX_MASK;
            double sh[3];
            decode_shift64(ent >> 27, box, sh);
            long b0 = idx, b1 = (long)idx + 1;
            if ((long)idx >= n) {
                b0 = cfirst[idx - n];
                b1 = b0 + ccount[idx - n];
            }
            double ae[3] = {0, 0, 0}, pe = 0.0;
            for (long b = b0; b < b1; b++) {
                double y[3];
                for (int k = 0; k < 3; k++) y[k] = x[3 * b + k] + sh[k] - x[3 * j + k];
                corr_body(y, m[b], box, P.c0, ae, &pe);
            }
            lc += w[3 * j] * ae[0] + w[3 * j + 1] * ae[1] + w[3 * j + 2] * ae[2] + u[j] * pe;
        }
        L += lc - u[j] * m[j] * P.self;
    }
    free(moms);
    free(done);
    L += w[3 * j] * a[0] + w[3 * j + 1] * a[1] + w[3 * j + 2] * a[2] + u[j] * phi;
    return L;
}

/*
 * CosmoIntegrate of nln/integrate.c:82-135 on n bodies held as float4
 * records: pos (x, y, z, m), vel (vx, vy, vz, -), acc (ax, ay, az, phi).
 * f: the step's six factors {a0^2 kick(tvel, tpos), a0^2 kick(tvel,
 * tvel + dtv), drift(tpos, tpos + dt), 1/a0, a(tpos + dt), 1/a0^2} of the
 * cosmology (the integrals are the caller's).  As the reference: the
 * centred velocity in FP64 for the energies, the new velocity stored to
 * float, the position converted to comoving, drifted and converted back,
 * each stored to float; ke += m |vc|^2 / a0^2, pe += m phi (the reference
 * halves both when it returns them).
 */
void orc_cosmo_integrate(long n, float *pos, float *vel, const float *acc, const double *f,
                         double *ke, double *pe) {
    double k = 0.0, p = 0.0;
    const double a0 = 1.0 / f[3];
    for (long i = 0; i < n; i++) {
        float *x = pos + 4 * i, *v = vel + 4 * i;
        const float *a = acc + 4 * i;
        double vc[3];
        for (int d = 0; d < 3; d++) vc[d] = v[d] + f[0] * a[d];
        k += x[3] * (vc[0] * vc[0] + vc[1] * vc[1] + vc[2] * vc[2]) / (a0 * a0);
        p += x[3] * a[3];
        for (int d = 0; d < 3; d++) v[d] = (float)(v[d] + f[1] * a[d]);
        for (int d = 0; d < 3; d++) x[d] = (float)(f[3] * x[d]);
        for (int d = 0; d < 3; d++) x[d] = (float)(x[d] + f[2] * v[d]);
        for (int d = 0; d < 3; d++) x[d] = (float)(f[4] * x[d]);
    }
    *ke = k;
    *pe = p;
}
