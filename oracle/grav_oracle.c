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
 * ---- FP64 evaluation of fixed batched index lists (the adjoint's checker) ----
 *
 * The batched lists (include/nlnlists.h): bodies 0..n-1 in tree order, the
 * point table's records n + c are cell c's monopoles, quadrupole-list
 * entries are cells.  Isolated trees only (image code 13).  Every cell's
 * moments are taken in FP64 from its bodies: mass M, centre of mass X and
 * the traceless Q = -3 (S2 - tr(S2)/3 I), S2 = sum m (x - X)(x - X)^T, so
 * that a quadrupole cell adds phi += 1/2 rho^-5 d.Q.d and
 * a += 5/2 rho^-7 (d.Q.d) d - rho^-5 Q d to its monopole term (the physical
 * quadrupole potential, sign +1, of do_gravpq_avx8's arithmetic,
 * nln/do_grav_avx8.c:2090-2160 with the order-4 kernels' sign, :1846);
 * d = sink - source, rho^2 = |d|^2 + eps2.  Order-4 lists are not covered.
 */
typedef struct {
    double M, X[3], Q[6]; /* Q: xx xy xz yy yz zz */
} orc_mom;

static void cell_moments(const double *x, const double *m, long first, int count, orc_mom *o) {
    double M = 0, s[3] = {0, 0, 0};
    for (long b = first; b < first + count; b++) {
        M += m[b];
        for (int d = 0; d < 3; d++) s[d] += m[b] * x[3 * b + d];
    }
    o->M = M;
    for (int d = 0; d < 3; d++) o->X[d] = M > 0 ? s[d] / M : 0.0;
    double S[6] = {0, 0, 0, 0, 0, 0};
    for (long b = first; b < first + count; b++) {
        double y0 = x[3 * b] - o->X[0], y1 = x[3 * b + 1] - o->X[1], y2 = x[3 * b + 2] - o->X[2];
        S[0] += m[b] * y0 * y0; S[1] += m[b] * y0 * y1; S[2] += m[b] * y0 * y2;
        S[3] += m[b] * y1 * y1; S[4] += m[b] * y1 * y2; S[5] += m[b] * y2 * y2;
    }
    double tr = (S[0] + S[3] + S[5]) / 3.0;
    o->Q[0] = -3.0 * (S[0] - tr); o->Q[1] = -3.0 * S[1]; o->Q[2] = -3.0 * S[2];
    o->Q[3] = -3.0 * (S[3] - tr); o->Q[4] = -3.0 * S[4]; o->Q[5] = -3.0 * (S[5] - tr);
}

/* One sink at s against a point (quad = 0) or a quadrupole cell (quad = 1). */
static void term64(const double *s, const double *X, double M, const double *Q, int quad,
                   double eps2, double *a, double *phi) {
    double d0 = s[0] - X[0], d1 = s[1] - X[1], d2 = s[2] - X[2];
    double rho2 = d0 * d0 + d1 * d1 + d2 * d2 + eps2;
    double ri = 1.0 / sqrt(rho2), ri2 = ri * ri, ri3 = ri * ri2;
    *phi -= M * ri;
    a[0] -= M * d0 * ri3;
    a[1] -= M * d1 * ri3;
    a[2] -= M * d2 * ri3;
    if (!quad)
        return;
    double q0 = Q[0] * d0 + Q[1] * d1 + Q[2] * d2;
    double q1 = Q[1] * d0 + Q[3] * d1 + Q[4] * d2;
    double q2 = Q[2] * d0 + Q[4] * d1 + Q[5] * d2;
    double P2 = d0 * q0 + d1 * q1 + d2 * q2;
    double ri5 = ri3 * ri2, ri7 = ri5 * ri2;
    *phi += 0.5 * ri5 * P2;
    a[0] += 2.5 * ri7 * P2 * d0 - ri5 * q0;
    a[1] += 2.5 * ri7 * P2 * d1 - ri5 * q1;
    a[2] += 2.5 * ri7 * P2 * d2 - ri5 * q2;
}

#define ORC_IDX_MASK ((1u << 27) - 1u)

/* (X, M, Q) of point-table record idx (body, or cell monopole) from mom[]. */
static void point_source(unsigned idx, long n, const double *x, const double *m, const orc_mom *mom,
                         const double **X, double *M) {
    if ((long)idx < n) {
        *X = x + 3 * (long)idx;
        *M = m[idx];
    } else {
        *X = mom[idx - n].X;
        *M = mom[idx - n].M;
    }
}

/*
 * Full FP64 evaluation: out (4 doubles per body, tree order) = (a, phi) of
 * every sink over its group's point and quadrupole lists, all cells'
 * moments recomputed from x, m.  Returns 0, or -1 on an image code other
 * than 13 (periodic lists are not covered).
 */
int orc_lists_eval64(long n, const double *x, const double *m, long ncells, const long *cfirst,
                     const int *ccount, long ngroups, const long *gfirst, const int *gcount,
                     const long *pptr, const unsigned *plist, const long *qptr,
                     const unsigned *qlist, double eps2, double *out) {
    orc_mom *mom = (orc_mom *)malloc(sizeof(orc_mom) * (size_t)(ncells > 0 ? ncells : 1));
#pragma omp parallel for schedule(dynamic, 64)
    for (long c = 0; c < ncells; c++) cell_moments(x, m, cfirst[c], ccount[c], &mom[c]);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(| : bad)
    for (long g = 0; g < ngroups; g++) {
        for (int k = 0; k < gcount[g]; k++) {
            long i = gfirst[g] + k;
            double a[3] = {0, 0, 0}, phi = 0;
            for (long e = pptr[g]; e < pptr[g + 1]; e++) {
                if ((plist[e] >> 27) != 13u) { bad = 1; continue; }
                const double *X; double M;
                point_source(plist[e] & ORC_IDX_MASK, n, x, m, mom, &X, &M);
                term64(x + 3 * i, X, M, NULL, 0, eps2, a, &phi);
            }
            if (qptr)
                for (long e = qptr[g]; e < qptr[g + 1]; e++) {
                    if ((qlist[e] >> 27) != 13u) { bad = 1; continue; }
                    const orc_mom *c = &mom[qlist[e] & ORC_IDX_MASK];
                    term64(x + 3 * i, c->X, c->M, c->Q, 1, eps2, a, &phi);
                }
            for (int d = 0; d < 3; d++) out[4 * i + d] = a[d];
            out[4 * i + 3] = phi;
        }
    }
    free(mom);
    return bad ? -1 : 0;
}

/*
 * The entries that depend on the selected bodies sel[0..nsel) (nsel <= 64):
 * every (group, kind, position) whose list entry is a selected body or a
 * cell containing one.  cparent: parent cell of each cell (-1 at a root).
 * hits: 3 longs per hit (group, kind 0 = point / 1 = quadrupole, position),
 * hmask: the selected bodies it depends on (bit s for sel[s]).  Returns the
 * number of hits (filled when hits != NULL and cap allows), -1 for nsel > 64.
 */
long orc_fd_hits(long n, long ncells, const int *cparent, long ngroups, const long *pptr,
                 const unsigned *plist, const long *qptr, const unsigned *qlist, int nsel,
                 const long *sel, const long *body_leaf, long cap, long *hits,
                 unsigned long long *hmask) {
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
        for (int kind = 0; kind < 2; kind++) {
            const long *ptr = kind ? qptr : pptr;
            const unsigned *list = kind ? qlist : plist;
            if (!ptr)
                continue;
            for (long e = ptr[g]; e < ptr[g + 1]; e++) {
                long idx = (long)(list[e] & ORC_IDX_MASK) + (kind ? n : 0);
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
 * The part of L = sum_i w_i.a_i + u_i phi_i (FP64, fixed lists) that depends
 * on body j = sel[s]: every hit carrying bit s, over its group's sinks other
 * than j, plus sink j against its own group's whole lists.  The other terms
 * of L do not change when x_j or m_j does, so central differences of this
 * partial sum are those of L.  Cell moments come from the bodies (x, m),
 * so the caller perturbs x[3j + d] or m[j] and calls it twice.
 */
double orc_fd_partial_loss(int s, long j, long n, const double *x, const double *m, long ncells,
                           const long *cfirst, const int *ccount, long ngroups,
                           const long *gfirst, const int *gcount, const long *body_group,
                           const long *pptr, const unsigned *plist, const long *qptr,
                           const unsigned *qlist, long nhits, const long *hits,
                           const unsigned long long *hmask, const double *w, const double *u,
                           double eps2) {
    const unsigned long long bit = 1ull << s;
    double L = 0.0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : L)
    for (long h = 0; h < nhits; h++) {
        if (!(hmask[h] & bit))
            continue;
        long g = hits[3 * h], kind = hits[3 * h + 1], e = hits[3 * h + 2];
        unsigned idx = (kind ? qlist[e] : plist[e]) & ORC_IDX_MASK;
        orc_mom mo;
        const double *X;
        double M;
        if (!kind && (long)idx < n) {
            X = x + 3 * (long)idx;
            M = m[idx];
        } else {
            long c = kind ? (long)idx : (long)idx - n;
            cell_moments(x, m, cfirst[c], ccount[c], &mo);
            X = mo.X;
            M = mo.M;
        }
        for (int k = 0; k < gcount[g]; k++) {
            long i = gfirst[g] + k;
            if (i == j)
                continue;
            double a[3] = {0, 0, 0}, phi = 0;
            term64(x + 3 * i, X, M, mo.Q, (int)kind, eps2, a, &phi);
            L += w[3 * i] * a[0] + w[3 * i + 1] * a[1] + w[3 * i + 2] * a[2] + u[i] * phi;
        }
    }
    /* sink j over its own lists */
    long g = body_group[j];
    double a[3] = {0, 0, 0}, phi = 0;
    for (long e = pptr[g]; e < pptr[g + 1]; e++) {
        unsigned idx = plist[e] & ORC_IDX_MASK;
        if ((long)idx < n) {
            term64(x + 3 * j, x + 3 * (long)idx, m[idx], NULL, 0, eps2, a, &phi);
        } else {
            orc_mom mo;
            cell_moments(x, m, cfirst[idx - n], ccount[idx - n], &mo);
            term64(x + 3 * j, mo.X, mo.M, NULL, 0, eps2, a, &phi);
        }
    }
    if (qptr)
        for (long e = qptr[g]; e < qptr[g + 1]; e++) {
            orc_mom mo;
            long c = qlist[e] & ORC_IDX_MASK;
            cell_moments(x, m, cfirst[c], ccount[c], &mo);
            term64(x + 3 * j, mo.X, mo.M, mo.Q, 1, eps2, a, &phi);
        }
    L += w[3 * j] * a[0] + w[3 * j + 1] * a[1] + w[3 * j + 2] * a[2] + u[j] * phi;
    return L;
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
