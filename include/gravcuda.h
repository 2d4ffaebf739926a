/*
 * gravcuda.h -- the C ABI of libgravcuda.so, the B200 (sm_100a) drop-in for
 * the CUDA entry points that nln/mac.c and nln/main.c call through the
 * reference's nln/gravcuda.h (declarations at nln/gravcuda.h:13-69).
 *
 * Part 1 keeps every reference entry point with its name, arguments and
 * meaning.  Part 2 adds status-returning variants, the Plummer-softened
 * list kernels the reference only has on the CPU, and the batched
 * index-list path (all sink groups of a step in one persistent launch,
 * mixed precision, Ewald correction).
 *
 * Conventions kept from the reference:
 *   - sinks are bodies of the table registered by WalkInitSinkCUDA, read at
 *     float offsets 1..3 of each record of `stride` floats (body.pos,
 *     nln/physics.h:33-44); results are ADDED to offsets 7..10 (acc, phi)
 *     at WalkTerminateSinkCUDA, unscaled by G (nln/mac.c:273-276 scales);
 *   - lists are the reference AoSoA 8-lane blocks (nln/mac.c:117-153),
 *     source_n a multiple of 8, zero-mass padding lanes;
 *   - list kernels accumulate d = sink - source with the monopole potential
 *     -m/r, and the quadrupole potential sign of the CPU kernel they stand
 *     in for (-1 for the quadrupole kernels, nln/do_grav_avx8.c:2150,940;
 *     +1 for the order-4 kernels, nln/do_grav_avx8.c:1846,638).
 * Errors: by default an error prints a message and aborts, as the
 * reference's Error() does (nln/pgrav.cu:1047-1052); gravcuda_set_error_mode(1)
 * makes every entry point record the error and return instead
 * (gravcuda_status() reads it).
 */
#ifndef GRAVCUDA_H
#define GRAVCUDA_H

#include <stddef.h>
#include <stdint.h>

#include "nlnhost.h"
#include "nlnlists.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The reference's body-run type (nln/segment.h:16-19). */
#ifndef SEGMENT_DEFINED
#define SEGMENT_DEFINED
typedef struct {
    unsigned int base;
    unsigned int length;
} segment;
#endif

/* ================================================================ Part 1 */

/* Select device 0 and report it (nln/cuda.cu:13-47; caller passes NULL, nln/main.c:228). */
void CUDA_Init(void *device_prop);
/* Release every library resource (declared but never defined in the reference, nln/gravcuda.h:15). */
void CUDA_Finalize(void);
/* Sinks handled per thread by the list kernels (nln/pgrav.cu:1022). */
int vecwidthCUDA(void);
/* A free queue slot 0..31 or -1; *inuse receives the busy count (nln/pgrav.cu:814-853,1024). */
int qallocCUDA(int *inuse);

/*
 * Cell table for grav_qns_CUDA: ncells records of `stride` floats in the
 * hexacell layout of nln/physics.h:140-157 as built with DIPOLE (mass 0,
 * pos 1..3, bmax 5, dipole 12..14, quadrupole 15..19).  The reference copied
 * wrong fields here (nln/pgrav.cu:890-904); this maps the hexacell fields as
 * named.  Replaces nln/pgrav.cu:878-913.
 */
void WalkInitSrcCUDA(float *qtab, int stride, int64_t nobj);
/* Free the cell table; safe when never initialised (called unconditionally, nln/main.c:953). */
void WalkTerminateSrcCUDA(void);
/* Copy sink positions (floats 1..3 of each record) to the device, zero the accumulators (nln/pgrav.cu:915-967). */
void WalkInitSinkCUDA(float *btab, int stride, int64_t nobj);
/* Wait for all queued work, ADD (ax, ay, az, phi) into floats 7..10 of each record (nln/pgrav.cu:969-1020). */
void WalkTerminateSinkCUDA(float *btab, int stride, int64_t nobj);

/*
 * n sinks starting at p (a pointer into the registered sink table; sink
 * index (p - btab)/stride) against the AoSoA list f of source_n sources of
 * sz floats each, on queue slot q (nln/pgrav.cu:1026-1087).  accp is
 * ignored (results accumulate on the device).  routine:
 *   "pM"     monopole, no softening              (CUDA pM,  nln/pgrav.cu:370-410)
 *   "pQ"     quadrupole, no softening            (do_gravq_avx8, nln/do_grav_avx8.c:881-950)
 *   "pH"     order 4, no softening               (do_gravh_avx8, nln/do_grav_avx8.c:572-696)
 *   "pM_sK1" monopole, Dehnen K1, e = 1/eps      (CUDA pM_sK1, nln/pgrav.cu:412-468)
 *   "pMp"    monopole, Plummer, e = eps^2        (do_gravp_avx8,  nln/do_grav_avx8.c:2163-2216)
 *   "pQp"    quadrupole, Plummer, e = eps^2      (do_gravpq_avx8, nln/do_grav_avx8.c:2090-2160)
 *   "pHp"    order 4, Plummer, e = eps^2         (do_gravph_avx8, nln/do_grav_avx8.c:1779-1904)
 *   "pMs"    monopole, contributions with r < e dropped (do_grav_avx8, nln/do_grav_avx8.c:953-1006)
 * The list is copied before return, so the caller may reuse f at once.
 */
void grav_mn_CUDA(const char *routine, const float *p, float *accp, const int n, const int stride,
                  const float *f, const int source_n, const int sz, const float e, int *ncut,
                  int q);
/*
 * m sinks from body `base` against seg_n body runs of the sink table, all
 * of mass mmass, K1 softening with e = 1/eps; routine "pMM_sK1"
 * (nln/pgrav.cu:575-637, 1089-1147).
 */
void grav_mns_CUDA(const char *routine, const int base, const int m, const segment *seg,
                   const int seg_n, const int source_n, const float mmass, float e, int *ncut,
                   int q);
/*
 * Batched body-run p-p, many sink groups in one launch: sink i of
 * [sink_base, sink_base+m) belongs to group ss_index[i]; group g owns body
 * runs seg[ss_seg[g].base .. +ss_seg[g].length), offsets relative to
 * source_base, source_n[g] bodies in all; routine "pMM_mnss_sK1"
 * (nln/pgrav.cu:713-790, 1202-1295).  A group whose runs do not add up to
 * source_n[g] is an error (the reference printed it, nln/pgrav.cu:779-789).
 */
void grav_mnss_CUDA(const char *routine, const int sink_base, const int m,
                    const uint16_t *ss_index, const segment *ss_seg, const int ss_len,
                    const segment *seg, const int seg_len, const int source_base,
                    const int *source_n, const float mmass, float e, int *ncut, int q);
/*
 * m sinks from `base` against the cells source_list[0..source_n) of the
 * table registered by WalkInitSrcCUDA: monopole, dipole and quadrupole, no
 * softening, the quadrupole potential with do_gravdq_avx8's sign; routine
 * "pQQ1" (nln/pgrav.cu:498-572, 1149-1200; the reference kernel was dead and
 * read the wrong bound and fields; this one reads the list as named).
 */
void grav_qns_CUDA(const char *routine, const int base, const int m, const int *source_list,
                   const int source_n, int q);
/*
 * Sink i of [base, base+m) against the run seg[i] of the packed QSZ AoSoA
 * buffer source (source_n records): monopole, dipole (fields 5..7) and
 * quadrupole, no softening, the arithmetic of do_gravdq_avx8
 * (nln/do_grav_avx8.c:378-459); routine "pQ1_qnss" (nln/pgrav.cu:293-368,
 * 1297-1358).
 */
void grav_qnss_CUDA(const char *routine, const int base, const int m, const segment *seg,
                    const float *source, const int source_n, int q);

/* ================================================================ Part 2 */

/* Error reporting: mode 0 = print and abort (reference behaviour), 1 = record and return. */
void gravcuda_set_error_mode(int mode);
/* Last recorded status (0 = success) and its message; gravcuda_clear_status() resets both. */
int gravcuda_status(void);
const char *gravcuda_status_string(void);
void gravcuda_clear_status(void);

/* grav_mn_CUDA returning the status instead of aborting. */
int grav_mn_status_CUDA(const char *routine, const float *p, const int n, const int stride,
                        const float *f, const int source_n, const int sz, const float e, int q);

/* Synchronise the queue and copy the device accumulators (4 floats per sink) to out, without clearing. */
int gravcuda_peek_accumulators(float *out, int64_t first, int64_t count);

/*
 * Where the drop-in calls' time went since the last WalkInitSinkCUDA, in
 * seconds: [0] copying lists out of the caller's memory into page-locked
 * staging, [1] waiting for a free staging buffer, [2] waiting for room in
 * the submitter's queue (grav_mn_CUDA returns after the staging copy; a
 * submitter thread issues the device copy and the launch), [3] the
 * submitter's CUDA calls, [4] the drain at WalkTerminateSinkCUDA; [5] the
 * number of grav_mn_CUDA calls.
 */
void gravcuda_dropin_phases(double out[6]);

/*
 * ---- batched index-list evaluation ----
 * A step's problem: bodies in tree order and cell monopoles in one point
 * table, quadrupole and order-4 cell tables, sink groups, and per-group
 * CSR index lists into those tables, as built by nlnhost.h.  All pointers
 * are host pointers for grav_groups_upload_CUDA and device pointers for
 * grav_groups_eval_dev_CUDA.
 */
typedef struct grav_problem {
    int64_t nbodies;            /* bodies = sinks, tree order */
    int64_t ncells;
    int64_t ngroups;
    const float *points;        /* (nbodies + ncells) x float4 (x, y, z, m) */
    const nln_qcell *qcells;    /* ncells records, or NULL when no quadrupole lists */
    const nln_hcell *hcells;    /* ncells records, or NULL when no order-4 lists (required
                                   with ewald: the correction uses every cell's moments) */
    const nln_group *groups;    /* ngroups records */
    const int64_t *pptr, *qptr, *hptr;  /* ngroups + 1 each */
    const uint32_t *plist, *qlist, *hlist;  /* entries: index | image << 27 (nlnlists.h) */
    double eps2;                /* Plummer softening eps^2 (all interactions) */
    double box;                 /* periodic cube side; 0 = isolated */
    float quad_phi_sign;        /* +1 physical; -1 reproduces do_gravpq's potential */
    int ewald;                  /* periodic only: 1 = add the Ewald correction */
    const int64_t *cptr;        /* ewald: ngroups + 1 offsets of the correction list */
    const uint32_t *clist;      /* ewald: point-table records | image << 27; cells enter as
                                   nbodies + cell index and take the order-4 table's moments */
    int lists_in_host;          /* 1: the lists are page-locked host memory (cudaHostAlloc) that
                                   the kernels read in place over PCIe, overlapping the transfer
                                   with the evaluation; their entries are then checked as they
                                   are read (a bad one sets the device error word) and the
                                   point list's interactions are counted as bodies.  The plan
                                   reads them at every evaluation: keep them alive and unchanged
                                   until grav_plan_free.  0: copied to the device at upload. */
    /* Run-packed lists (nlnlists.h), read by grav_groups_CUDA only: when zlist[k] is set
       (k = 0 P, 1 Q, 2 H, 3 correction) the call copies these ngroups + 1 word offsets and
       words instead of the plain list, which it then does not read (may be NULL), and unpacks
       them on the device; the plain offsets (pptr, qptr, hptr, cptr) are still required.  A
       group that does not unpack to its plain length fails the call with status -2. */
    const int64_t *zptr[4];
    const uint32_t *zlist[4];
    /* Arithmetic of the list kernels (grav_groups_upload_CUDA and grav_groups_CUDA):
       0 = mixed (default): sinks and sources as FP32 offsets from each group's FP64
       centre, compensated tile sums; 1 = plain FP32, the form the reference's lists
       compute in (absolute FP32 coordinates, nln/mac.c:1421-1561; plain sums), kept
       for comparison.  grav_groups_eval_dev_CUDA always runs the mixed form. */
    int precision;
} grav_problem;

typedef struct grav_plan grav_plan;

/* Tile shapes of the batched kernels (the autotuner's search space). */
typedef struct grav_tuning {
    int warps_per_block;        /* 4, 8 or 16 */
    int chunk_p;                /* max point records per work item (split long lists) */
    int chunk_q;                /* max quadrupole cells per work item */
    int chunk_h;                /* max order-4 cells per work item */
    int blocks_per_sm;          /* persistent grid = blocks_per_sm x SM count (0: as many as fit) */
    int ewald_n;                /* Ewald table nodes per axis (0: 32) */
    int ewald_side;             /* periodic: where the Ewald correction moments run.  > 0: on a
                                   side stream beside the list kernels, in this many two-warp
                                   blocks per SM; -k (k = 1, 2, 4): on the evaluation's stream
                                   between the list kernels and the finish pass, with the SMs to
                                   themselves, in blocks of k warps; 0: automatic (2 while the
                                   correction list is under 1.5 % of the order-4 interactions,
                                   else -2).  The results are the same either way. */
} grav_tuning;

/*
 * Copy a problem to the device and build its work queue (items sorted by
 * cost, longest first).  tuning may be NULL for defaults.  The plan owns
 * device copies of every table and its scratch; free with grav_plan_free.
 */
int grav_groups_upload_CUDA(const grav_problem *host_problem, const grav_tuning *tuning,
                            grav_plan **plan);
/* Evaluate on a stream (cudaStream_t passed as void*; NULL = legacy default). */
int grav_groups_eval_CUDA(grav_plan *plan, void *stream);
/* Copy (ax, ay, az, phi) per body, tree order, float4, to host memory (synchronising). */
int grav_groups_download_CUDA(grav_plan *plan, float *acc_phi);
/* Device pointer of the plan's output (nbodies x float4), for callers that keep results resident. */
float *grav_plan_output(grav_plan *plan);
/* Interaction counts of the plan: body-body, monopole, quadrupole, order-4 (over all sinks). */
void grav_plan_counts(const grav_plan *plan, int64_t out[4]);
/* Kernel launches per evaluation. */
int grav_plan_launches(const grav_plan *plan);
/*
 * Rebuild a plan's work queue for new tile shapes (warps per block, blocks
 * per SM, list chunks; a chunk <= 0 is chosen automatically) without
 * re-uploading its tables: the autotuner's step.  Synchronises the device;
 * a captured step graph is dropped and recaptured on its next call.
 * grav_plan_get_tuning returns the shapes in use (automatic chunks resolved).
 */
int grav_plan_retune_CUDA(grav_plan *plan, const grav_tuning *tuning);
int grav_plan_get_tuning(const grav_plan *plan, grav_tuning *out);
/* Record CUDA events around each kernel of every evaluation (on its stream). */
int grav_plan_set_timing(grav_plan *plan, int on);
/* Milliseconds of the last evaluation's kernels: order-4, quadrupole, point, finish (synchronising). */
int grav_plan_kernel_ms(grav_plan *plan, float ms[4]);
void grav_plan_free(grav_plan *plan);

/*
 * ---- the tree and lists built on the GPU ----
 * grav_plan_build_CUDA: build the tree, FP64 moments, critical radii, sink
 * groups and interaction lists of n bodies on the device and return a plan
 * that evaluates them, ready for grav_groups_eval_CUDA, the time step and
 * the adjoint (the tree links are set).  params are nlnhost.h's (emit_aosoa
 * and nthreads are ignored); bodies: device, n x float4 (x, y, z, m) in any
 * order, 16-byte aligned, not kept.  Bodies in [0, box)^3 when params->box >
 * 0.  The tables and lists are bit-identical to nln_tree_build +
 * nln_tree_walk on the same bodies (both builders share their arithmetic
 * and sum in the same order without fused multiply-adds), so a plan built
 * either way evaluates to the same forces.  Synchronises the device.
 * grav_plan_order: device int64 per body, tree position -> input index
 * (results are in tree order); NULL for plans uploaded from the host.
 * grav_plan_build_phases: seconds of this thread's last build: sort, cells,
 * moments and tables, sink groups, walk (both passes), the list offsets and
 * allocations between the passes, plus the whole call.
 */
int grav_plan_build_CUDA(const nln_params *params, const float *bodies, int64_t n, double eps2,
                         float quad_phi_sign, int ewald, const grav_tuning *tuning,
                         grav_plan **plan);
const int64_t *grav_plan_order(const grav_plan *plan);
void grav_plan_build_phases(double seconds[7]);

/*
 * One call from positions to forces: copy the bodies (host, n x float4
 * (x, y, z, m), any order; page-locked memory copies fastest) to the
 * device, build the tree and lists there (grav_plan_build_CUDA), evaluate,
 * and copy (ax, ay, az, phi) per body back to acc_phi (host, n x float4) in
 * the bodies' own order.  Device buffers come from the memory pool of
 * grav_groups_CUDA (kept reserved until grav_groups_release_CUDA).
 * grav_build_eval_phases: seconds of this thread's last call: bodies to the
 * device, build, evaluation and results back, release.
 */
int grav_build_eval_CUDA(const nln_params *params, const float *bodies, int64_t n, double eps2,
                         float quad_phi_sign, int ewald, float *acc_phi);
void grav_build_eval_phases(double seconds[4]);

/*
 * The plan's problem as it evaluates it: sizes and parameters, device
 * pointers to its tables and lists (points, qcells, hcells, groups, plist,
 * qlist, hlist, clist; NULL where absent) and host pointers to the list
 * offsets (pptr, qptr, hptr, cptr), valid until grav_plan_free.
 */
int grav_plan_problem(const grav_plan *plan, grav_problem *out);

/*
 * One-call end-to-end form: upload, evaluate, download, free.  acc_phi:
 * host, nbodies x 4 floats, tree order.  Unless lists_in_host is set, the
 * lists are copied group range by group range (one per 2 GiB of words
 * copied, at most 16, the first split in four; the environment variable
 * GRAV_E2E_CHUNKS sets the count) on a copy stream while the kernels
 * evaluate the ranges already copied.  Run-packed lists (zptr/zlist) are
 * copied as packed words and unpacked on the device before each range's
 * kernels: about 4x fewer bytes over the host link.  List entries are
 * checked by the kernels as they read them, and a bad one (or a packed
 * group of the wrong length) fails the call with status -2 after the
 * evaluation.  Lists in page-locked host memory overlap best.  The call's
 * device buffers come from a memory
 * pool that keeps freed memory reserved for the next call, until
 * grav_groups_release_CUDA or CUDA_Finalize.
 */
int grav_groups_CUDA(const grav_problem *host_problem, float *acc_phi);

/* Return the memory grav_groups_CUDA keeps reserved between calls on the current device. */
void grav_groups_release_CUDA(void);

/*
 * Wall-clock seconds of the phases of this thread's last grav_groups_CUDA
 * call: [0] host checks and work queue, [1] device allocation and table
 * upload, [2] list copies overlapped with the evaluation, [3] download,
 * [4] release of the device buffers.
 */
void grav_groups_CUDA_phases(double seconds[5]);

/*
 * FP64 direct sum at nsink sample sinks, the accuracy reference of every
 * reported force error.  Isolated (box = 0): Plummer-softened sum over all
 * bodies, self included.  Periodic (box > 0): the Ewald-summed direct sum of
 * EwaldForces (nln/grav_n2.c:97-196, pair term ewald() of nln/ewald.c:13-64)
 * with the nearest-image Newtonian term softened by eps2.  points: host
 * (x, y, z, m) float4 per body; sinks: host indices; out: host, 4 doubles
 * (ax, ay, az, phi) per sample; G not applied.
 */
int grav_direct_fp64_CUDA(const float *points, int64_t n, const int64_t *sinks, int64_t nsink,
                          double eps2, double box, double *out);

/*
 * The FP32 CUDA-core peak of the current device, measured: a grid of
 * independent FMA chains (8 per thread, 2048 threads per SM), once as scalar
 * FMAs and once as paired f32x2 FMAs, timed with CUDA events, best of five
 * launches after one warm-up each, the larger rate in TFLOP/s (2 flops per
 * FMA).  The roofline denominator of the interaction kernels; about
 * 74 TFLOP/s on a B200 at 1965 MHz (148 SMs x 128 lanes x 2 flops x clock).
 */
int grav_fp32_peak_CUDA(double *tflops);

/*
 * ---- the time step on the device ----
 * Between host rebuilds of the tree and lists, bodies move on the device
 * and the plan's cell tables are refitted from them.
 *
 * grav_plan_set_tree_CUDA: the tree's links (host arrays over the plan's
 * ncells cells, as nlnhost.h's nln_cell_ranges and nln_cell_links give them:
 * body range, first child or -1, child count, depth).
 * grav_plan_refit_CUDA: recompute every cell record (monopole, quadrupole,
 * order-4) from the plan's current body positions, deepest cells first
 * (leaves from their bodies in FP64, parents by parallel-axis shifts of
 * their children, as nln/cofm.c mpole_add); lists and sink groups are kept.
 * grav_plan_bodies: device pointer of the body table (x, y, z, m float4,
 * tree order), which the integrator updates in place.
 * grav_plan_integrate_CUDA: Integrate() of nln/integrate.c:16-59 on the
 * last evaluation's (acc, phi): params (device, 3 doubles) = {dt, dtv,
 * dtsync = tpos - tvel}; for each body ke += m |v + dtsync a|^2, pe += m phi
 * (added into energy, device, 2 doubles), then v += dtv a, x += dt v.
 * vel: device, float4 (vx, vy, vz, unused) per body, tree order.
 * grav_plan_set_integrator_CUDA: kind 0 (default) is the Integrate above;
 * kind 1 is CosmoIntegrate of nln/integrate.c:82-135: params (device, 6
 * doubles) = {a0^2 kick(tvel, tpos), a0^2 kick(tvel, tvel + dtv),
 * drift(tpos, tpos + dt), 1/a0, a(tpos + dt), 1/a0^2} (nlnhost.h
 * nln_cosmo_kdk); ke += m |v + p0 a|^2 p5, pe += m phi, v += p1 a,
 * x = p4 (p3 x + p2 v) with positions rounded to FP32 after each factor as
 * the reference does.  It applies to later integrate and step calls.
 * grav_plan_step_CUDA: one step = zero energy, evaluate, integrate, refit.
 * With use_graph the step is captured once into a CUDA graph on `stream`
 * (a created stream, not the legacy default) and replayed by later calls
 * with the same pointers; params and energy are read and written through
 * their device pointers, so update params between launches.
 */
int grav_plan_set_tree_CUDA(grav_plan *plan, const int64_t *cell_first, const int32_t *cell_count,
                            const int32_t *cell_child, const int32_t *cell_nchild,
                            const int32_t *cell_level);
int grav_plan_refit_CUDA(grav_plan *plan, void *stream);
float *grav_plan_bodies(grav_plan *plan);
int grav_plan_integrate_CUDA(grav_plan *plan, float *vel, const double *params, double *energy,
                             void *stream);
int grav_plan_set_integrator_CUDA(grav_plan *plan, int kind);
int grav_plan_step_CUDA(grav_plan *plan, float *vel, const double *params, double *energy,
                        void *stream, int use_graph);

/*
 * ---- adjoint (no counterpart in the reference) ----
 * For a loss L = sum_i w_i . a_i + u_i phi_i on the plan's last evaluation,
 * dL/dx and dL/dm of every body with the lists held fixed: the pair terms'
 * tidal-tensor-vector products on the sink and source sides, the mass and
 * trace-free moment adjoints (orders 2, 3, 4) of every listed cell, the
 * periodic correction's adjoint through each group's Taylor moments and each
 * correction entry's table lookup, then the moments' chain rule to the
 * cell's bodies (centre of mass, trace-free moments, the second-moment
 * trace).  wu: device float4 (wx, wy, wz, u) per body, tree order; grad:
 * device float4 (dL/dx, dL/dy, dL/dz, dL/dm) per body, tree order.  Needs
 * the tree links (grav_plan_set_tree_CUDA), the physical quadrupole
 * potential (quad_phi_sign = +1), the mixed-precision form and, for the
 * periodic correction, an evaluation enqueued before it (its group moments
 * are read).  Every list kind and periodic image shift is covered; the
 * correction's derivatives of order 6 (beyond its table) are dropped.
 * Enqueued on `stream`.
 */
int grav_plan_adjoint_CUDA(grav_plan *plan, const float *wu, float *grad, void *stream);

/*
 * ---- evaluation without allocation (no counterpart in the reference) ----
 * grav_groups_eval_dev_CUDA evaluates a problem whose tables and lists are
 * already in device memory (every grav_problem pointer a device pointer,
 * 16-byte aligned tables; acc_phi: device, nbodies x float4, tree order)
 * and allocates no device memory at all: no cudaMalloc/cudaFree and no
 * allocating library call.  It is for callers that cannot allocate on the
 * device: a code whose memory is owned by another allocator's pool (a
 * framework caching allocator holding the device, where an outside
 * cudaMalloc can fail or fragment the pool), and a time-step loop on a
 * stream it must not stall, where cudaFree would synchronise the whole
 * device.
 *
 * All scratch -- queue counters, error word, work items, a checked copy of
 * the groups, slot offsets and the per-item partial sums -- lives in one
 * file-scope device array of GRAV_DEV_SCRATCH_BYTES (16 MiB), enough for
 * about 5,200 groups with three list kinds (about 100,000 bodies at 20 per
 * group); larger problems are rejected with an error naming the limit.  The
 * queue counters and the error word must be zero when the kernels start:
 * every call zeroes them on its stream first, and writes every work item,
 * group copy, slot offset and partial sum it reads, so the scratch's earlier
 * contents never matter.  One work item per group and list kind (no list
 * splitting, no cost sort); isolated problems, or periodic ones without the
 * Ewald correction (ewald must be 0: its table is a per-plan allocation).
 *
 * The scratch is one per device, so calls that overlap on a device (other
 * host threads, other streams) race on it and must be serialised by the
 * caller.  The first call on each device (with that device current) looks
 * up the scratch's address with cudaGetSymbolAddress, reads the device's SM
 * count and sets kernel attributes.  The call enqueues on `stream`
 * (cudaStream_t as void*; NULL = legacy default) and waits for that stream
 * before it returns, on success and on every error after its first
 * enqueue, so no work of a returned call still uses the scratch.  It returns 0, -1 for a rejected problem, or -2 when a
 * kernel flagged an error (a bad group, list offset or entry, a lost copy).
 *
 * Precondition the call cannot check: grav_problem carries no list lengths,
 * so the last offset of each list (pptr, qptr, hptr [ngroups]) must not
 * exceed the number of entries in the matching device list (plist, qlist,
 * hlist).  The kernels check that offsets start at 0 or above and never
 * decrease, and that every entry they read lies inside its table, but a
 * final offset past the end of a list makes them read past that buffer.
 */
#define GRAV_DEV_SCRATCH_BYTES (16u << 20)
int grav_groups_eval_dev_CUDA(const grav_problem *device_problem, float *acc_phi, void *stream);

#ifdef __cplusplus
}
#endif
#endif
