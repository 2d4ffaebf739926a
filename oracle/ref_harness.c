/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Bulk drivers around the reference's own CPU kernels, which oracle/Makefile
 * compiles unmodified from nln/do_grav_avx8.c and nln/pgrav_vec.c into
 * oracle/_ref/libnlnref.so.  This file holds no force arithmetic: it only
 * calls the reference functions the way nln/mac.c does (one call per sink
 * over a list suffix, mac.c:549-676) so that tests and the CPU baseline can
 * run them over many sinks and many lists.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef float vsf __attribute__((vector_size(32)));
typedef void (*ref_grav_f)(const vsf *, const vsf *, const float *, float *, float *, float *,
                           const float *, int *);

/* prototypes of the reference kernels (nln/physics.h:357-440) */
void do_gravp_avx8(const vsf *, const vsf *, const float *, float *, float *, float *,
                   const float *, int *);
void do_gravpq_avx8(const vsf *, const vsf *, const float *, float *, float *, float *,
                    const float *, int *);
void do_gravph_avx8(const vsf *, const vsf *, const float *, float *, float *, float *,
                    const float *, int *);
void do_grav_avx8(const vsf *, const vsf *, const float *, float *, float *, float *,
                  const float *, int *);
void do_grav_sK1_avx8(const vsf *, const vsf *, const float *, float *, float *, float *,
                      const float *, int *);
void do_gravq_avx8(const vsf *, const vsf *, const float *, float *, float *, float *,
                   const float *, int *);
void do_gravdq_avx8(const vsf *, const vsf *, const float *, float *, float *, float *,
                    const float *, int *);
void do_gravh_avx8(const vsf *, const vsf *, const float *, float *, float *, float *,
                   const float *, int *);
void do_gravmm_sK1_avx8(const float *xyz, const int stride, const float pmass, const void *mm,
                        const int mm_n, const int source_n, const float *pos0, float *mass0,
                        float *acc, float *phi0, const float *e, int *ncut);
void pMinteract(const float *p, float *accp, const int m, const int stride, const vsf *f,
                const int n);
void pQinteract(const float *p, float *accp, const int m, const int stride, const vsf *f,
                const int n);
void pHinteract(const float *p, float *accp, const int m, const int stride, const vsf *f,
                const int n);

/* kind numbering shared with oracle/grav_oracle.c */
static ref_grav_f pick(int kind) {
    switch (kind) {
    case 0: return do_gravp_avx8;
    case 1: return do_gravpq_avx8;
    case 2: return do_gravph_avx8;
    case 3: return do_grav_avx8;
    case 4: return do_grav_sK1_avx8;
    case 5: return do_gravq_avx8;
    case 6: return do_gravh_avx8;
    case 9: return do_gravdq_avx8;
    default: return NULL;
    }
}

/* One sink against nblk 8-lane blocks (f must be 32-byte aligned). */
int ref_list_eval(int kind, const float *f, long nblk, int sz, const float *pos0, float e,
                  float *out) {
    ref_grav_f fn = pick(kind);
    if (!fn)
        return -1;
    float mtot = 0.0f;
    int ncut = 0;
    float acc[3] = {0, 0, 0}, phi = 0.0f;
    fn((const vsf *)f, (const vsf *)(f + (size_t)nblk * sz * 8), pos0, &mtot, acc, &phi, &e,
       &ncut);
    out[0] += acc[0];
    out[1] += acc[1];
    out[2] += acc[2];
    out[3] += phi;
    return ncut;
}

/*
 * Grouped evaluation, the way mac.c's leaf loop and mxn_* fall-backs run the
 * CPU kernels: group g owns sinks [sink_first[g], sink_first[g]+sink_count[g])
 * of the position table pos (xyz, 3 floats per sink) and the list blocks
 * [blk_first[g], blk_first[g]+blk_count[g]) of f.  out (4 floats per sink)
 * is accumulated.  OpenMP over groups: one host thread per group at a time.
 */
void ref_groups_eval(int kind, const float *f, int sz, const long *blk_first,
                     const long *blk_count, const long *sink_first, const int *sink_count,
                     long ngroups, const float *pos, float e, float *out, int nthreads) {
    ref_grav_f fn = pick(kind);
    if (!fn)
        return;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (long g = 0; g < ngroups; g++) {
        const float *fb = f + (size_t)blk_first[g] * sz * 8;
        const float *fe = fb + (size_t)blk_count[g] * sz * 8;
        for (int s = 0; s < sink_count[g]; s++) {
            long i = sink_first[g] + s;
            float mtot = 0.0f;
            int ncut = 0;
            float acc[3] = {0, 0, 0}, phi = 0.0f;
            fn((const vsf *)fb, (const vsf *)fe, pos + 3 * i, &mtot, acc, &phi, &e, &ncut);
            out[4 * i + 0] += acc[0];
            out[4 * i + 1] += acc[1];
            out[4 * i + 2] += acc[2];
            out[4 * i + 3] += phi;
        }
    }
}

/* The MxN CPU kernels of nln/pgrav_vec.c, called as mac.c:1094,1246 do. */
void ref_pinteract(int kind, const float *p, float *accp, int m, int stride, const float *f,
                   long nblk) {
    if (kind == 0)
        pMinteract(p, accp, m, stride, (const vsf *)f, (int)nblk);
    else if (kind == 1)
        pQinteract(p, accp, m, stride, (const vsf *)f, (int)nblk);
    else if (kind == 2)
        pHinteract(p, accp, m, stride, (const vsf *)f, (int)nblk);
}

/*
 * do_gravmm_sK1_avx8 over body segments.  The reference kernel reads one
 * segment past the end (mm[mm_n], do_grav_avx8.c:1149), so this copies the
 * segments into a buffer with a zeroed sentinel.
 */
long ref_segments_k1(const float *xyz, int stride, float pmass, const uint32_t *seg, int nseg,
                     long source_n, const float *pos0, float e, float *out) {
    uint32_t *mm = (uint32_t *)calloc((size_t)(nseg + 1) * 2, sizeof(uint32_t));
    memcpy(mm, seg, (size_t)nseg * 2 * sizeof(uint32_t));
    float mtot = 0.0f, acc[3] = {0, 0, 0}, phi = 0.0f;
    int ncut = 0;
    do_gravmm_sK1_avx8(xyz, stride, pmass, mm, nseg, (int)source_n, pos0, &mtot, acc, &phi, &e,
                       &ncut);
    free(mm);
    out[0] += acc[0];
    out[1] += acc[1];
    out[2] += acc[2];
    out[3] += phi;
    return ncut;
}

/* the reference's periodic Green's function (nln/ewald.c:13-64) */
void ewald(double *x, double L, double *f, double *phi);

/* ewald() of nln/ewald.c at n displacements x (3 doubles each), OpenMP. */
void ref_ewald_batch(const double *x, long n, double L, double *f, double *phi) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) {
        double xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
        ewald(xi, L, f + 3 * i, phi + i);
    }
}

/*
 * The reference's own periodic scheme (images in the walk plus the
 * order-8 local expansion of FixCubeEwaldLE), for comparison
 * with other periodic evaluations: n bodies in a cube of side L centred on
 * the origin (positions in [-L/2, L/2)), G = 1.
 *   - every body in each of the (2 nimage + 1)^3 images of the box
 *     (SetGravOffset, nln/mac.c:91-111) summed directly in FP64 with the
 *     Plummer softening eps2 on every pair, the sink's own body in its own
 *     image included as the lists include it (phi -= m/eps, no force):
 *     the limit the reference's tree walk over those images approximates;
 *   - then FixCubeEwaldLE (nln/main.c:1811-1859) with subtract_background
 *     = 0: the lattice beyond those images from the compiled
 *     nln/ewald_le2.c (calculate_cartesian_moments, ewald_background,
 *     ewald_le), scaled by L G rho and L^2 G rho as there.
 * acc: 3 doubles per sink, phi: one, for the bodies sinks[0..nsink).
 */
typedef struct {
    float mass;
    float pos[3];
} le_body; /* the layout of oracle/ref_stubs/physics.h's body */
void calculate_cartesian_moments(le_body *btab, int nobj, double L, float *Q, int msb);
void ewald_background(const float xx[3], float mass, double phicorr, double acc[3], double *phi);
void ewald_le(const float xx[3], double acc[3], double *phi, float *Q, int nimage);

void ref_periodic_le(long n, const float *pos, const float *mass, double L, int nimage,
                     double eps2, const long *sinks, long nsink, double *acc, double *phi) {
    le_body *bt = (le_body *)malloc(sizeof(le_body) * (size_t)n);
    double mtot = 0.0;
    for (long i = 0; i < n; i++) {
        bt[i].mass = mass[i];
        for (int d = 0; d < 3; d++) bt[i].pos[d] = pos[3 * i + d];
        mtot += mass[i];
    }
    static float Q[1716];
    calculate_cartesian_moments(bt, (int)n, L, Q, 0);
    const double grho = mtot / (L * L * L);
    double phicorr = 0.0;
    for (int i = -nimage; i <= nimage; i++)
        for (int j = -nimage; j <= nimage; j++)
            for (int k = -nimage; k <= nimage; k++)
                if (i || j || k)
                    phicorr += 1.0 / sqrt((double)(i * i + j * j + k * k));
#pragma omp parallel for schedule(dynamic, 1)
    for (long s = 0; s < nsink; s++) {
        const long i = sinks[s];
        double a[3] = {0, 0, 0}, p = 0.0;
        for (int ii = -nimage; ii <= nimage; ii++)
            for (int jj = -nimage; jj <= nimage; jj++)
                for (int kk = -nimage; kk <= nimage; kk++) {
                    const double off[3] = {ii * L, jj * L, kk * L};
                    for (long j = 0; j < n; j++) {
                        double d[3];
                        for (int c = 0; c < 3; c++)
                            d[c] = (double)pos[3 * j + c] + off[c] - (double)pos[3 * i + c];
                        const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + eps2;
                        if (r2 <= 0.0)
                            continue;
                        const double ri = 1.0 / sqrt(r2), mr3 = mass[j] * ri * ri * ri;
                        p -= mass[j] * ri;
                        for (int c = 0; c < 3; c++) a[c] += mr3 * d[c];
                    }
                }
        float r[3];
        double f[3], ph;
        for (int c = 0; c < 3; c++) r[c] = (float)(pos[3 * i + c] / L);
        ewald_background(r, mass[i], phicorr, f, &ph);
        for (int c = 0; c < 3; c++) a[c] += f[c] * L * grho;
        p += ph * L * L * grho;
        ewald_le(r, f, &ph, Q, nimage);
        for (int c = 0; c < 3; c++) a[c] += f[c] * L * grho;
        p += ph * L * L * grho;
        for (int c = 0; c < 3; c++) acc[3 * s + c] = a[c];
        phi[s] = p;
    }
    free(bt);
}
