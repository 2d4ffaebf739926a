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
