/*
 * nlnhost.h -- host-side tree build, moments, MAC walk and list packing that
 * feed the interaction-list kernels of gravcuda.h.
 *
 * This is the caller side of the drop-in boundary: it stands in for the
 * pieces of 2HOT that produce interaction lists, all of which stay on the
 * host as plain C/C++:
 *   - key sort + oct-tree build   (libtree BuildTree, not vendored; used at nln/main.c:900-914)
 *   - FP64 moments, normalisation (nln/cofm.c:96-231 CofmFromDaugh, 247-574 CellFromCofm)
 *   - AREL critical radii         (nln/cofm.c:276-565, rcrit_poly/rtnewt 577-624)
 *   - MAC walk + list appends     (nln/mac.c:1774-1844 DLRcritMAC, append macros 1421-1561)
 *   - periodic image offsets      (nln/mac.c:91-111 SetGravOffset)
 * Lists are emitted in two forms from one walk: the reference AoSoA 8-lane
 * blocks (Mvec/Qvec/Hvec of nln/mac.c:117-153) for grav_mn_CUDA and the
 * reference CPU kernels, and index lists into device-resident cell and point
 * tables for the batched kernels (grav_groups_CUDA).
 */
#ifndef NLNHOST_H
#define NLNHOST_H

#include <stdint.h>

#include "nlnlists.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nln_params {
    int leaf_max;     /* bodies per leaf cell (1..65535); reference leaf_max_n, main.c:541 */
    int group_max;    /* sinks per sink group (1..64) */
    int p2cut;        /* quad_ncut: cells with >= p2cut bodies carry quadrupoles (0: none) */
    int p4cut;        /* hexa_ncut: cells with >= p4cut bodies carry order-4 moments (0: none) */
    double tol;       /* errtol, absolute acceleration tolerance (mac_s.tol) */
    double rel_tol;   /* frac_tol  (0: relative criterion off) */
    double rel_tol0;  /* frac_tol0 (0: floor criterion off) */
    double box;       /* periodic cube side L with bodies in [0,L)^3; 0 = isolated */
    int nthreads;     /* host threads (0: all) */
    int emit_aosoa;   /* 1: also pack the reference AoSoA lists */
    double ewald_theta; /* periodic: opening angle of the correction list -- a cell wholly
                           inside the group's minimum-image cube stands for its subtree there
                           once bmax + group radius <= ewald_theta x its distance to the
                           nearest other lattice image of the group centre (0: the correction
                           list repeats the Newtonian entries) */
    double ptol_boost;  /* ptol_boost: cell tolerance tol / (1 + ptol_boost bmax / bmax0),
                           bmax0 half the root cube (nln/cofm.c:302; 0: off) */
} nln_params;

typedef struct nln_tree nln_tree;

/*
 * Sort bodies into key order, build the oct-tree, compute FP64 moments and
 * critical radii.  pos: xyz of body i at pos[i*stride + 0..2] (floats),
 * mass at mass[i*mstride].  Returns NULL on bad arguments (message via
 * nln_last_error()).
 */
nln_tree *nln_tree_build(const float *pos, int stride, const float *mass, int mstride, int64_t n,
                         const nln_params *p);
void nln_tree_free(nln_tree *t);
const char *nln_last_error(void);

/* Walk every sink group against the source tree and build its lists. */
int nln_tree_walk(nln_tree *t);

/* Sizes. */
int64_t nln_nbodies(const nln_tree *t);
int64_t nln_ncells(const nln_tree *t);
int64_t nln_ngroups(const nln_tree *t);

/*
 * Array accessors (owned by the tree, valid until nln_tree_free).
 * order:  tree position -> original body index
 * points: float4 (x, y, z, m): bodies [0, n) then cell monopoles [n, n+ncells)
 */
const int64_t *nln_order(const nln_tree *t);
const float *nln_points(const nln_tree *t);
const nln_qcell *nln_qcells(const nln_tree *t);
const nln_hcell *nln_hcells(const nln_tree *t);
const nln_group *nln_groups(const nln_tree *t);

/*
 * CSR lists per group: uint32 entries [ptr[g], ptr[g+1]); kind 0 = points,
 * 1 = Q, 2 = H, 3 = the periodic correction list (point-table records:
 * bodies, and cells as n + cell index, whose moments are the order-4 table's).
 */
const int64_t *nln_list_ptr(const nln_tree *t, int kind);
const void *nln_list_data(const nln_tree *t, int kind);
int64_t nln_list_len(const nln_tree *t, int kind);

/*
 * Interaction counts over all sinks: [0] body-body, [1] monopole cells,
 * [2] quadrupole cells, [3] order-4 cells.
 */
void nln_counts(const nln_tree *t, int64_t out[4]);

/*
 * Reference AoSoA lists (when emit_aosoa): per group and kind (0 = M with
 * MSZ 4, 1 = Q with QSZ 13, 2 = H with HSZ 29) a run of 8-lane blocks.
 * blk_ptr has ngroups+1 entries; data has blk_ptr[ngroups]*sz*8 floats.
 * Positions are absolute (centre + image shift), moments as in the cell
 * tables, dipole fields zero.
 */
const int64_t *nln_aosoa_ptr(const nln_tree *t, int kind);
const float *nln_aosoa_data(const nln_tree *t, int kind);

/*
 * The same AoSoA blocks for a subset of groups gids[0..ngsel), packed from
 * the index lists (so emit_aosoa is not needed).  With data == NULL only
 * blk_ptr (ngsel + 1 entries) is filled; returns the total block count.
 */
int64_t nln_aosoa_subset(const nln_tree *t, const int64_t *gids, int64_t ngsel, int kind,
                         int64_t *blk_ptr, float *data);

/* Body range of every cell: bodies [first[c], first[c] + count[c]) in tree order. */
void nln_cell_ranges(const nln_tree *t, int64_t *first, int32_t *count);

/*
 * A batch of independent systems as one tree-like object: the members'
 * bodies one after another (member i's at the sum of the earlier members'
 * counts, in each member's tree order), then all their cells; groups,
 * lists, cell links and interaction counts are renumbered so that every
 * list still refers only to its own member.  Members must be isolated and
 * walked; they are not modified and may be freed afterwards.  Every
 * accessor works on the result (nln_order maps into the concatenation of
 * the members' original bodies); nln_tree_walk refuses it.  Free with
 * nln_tree_free.  NULL (see nln_last_error) on bad members or when bodies
 * plus cells exceed 27-bit list indices.
 */
nln_tree *nln_tree_merge(nln_tree *const *trees, int ntrees);

/*
 * Tree links of every cell: first child (-1 for a leaf), number of children
 * (children are consecutive cells) and depth (root 0).  Children always
 * follow their parent in the cell array.
 */
void nln_cell_links(const nln_tree *t, int32_t *child, int32_t *nchild, int32_t *level);

/*
 * Refit: new body positions (tree order, xyz floats) with the same tree and
 * lists; every cell's centre of mass, moments and bmax (and the point,
 * quadrupole and order-4 tables) are recomputed from the bodies in FP64.
 * Critical radii and lists are kept.  Returns 0, or -1 for bad arguments.
 */
int nln_tree_refit(nln_tree *t, const float *pos);

/* Body positions in tree order (xyz floats), the sink positions the lists were built for. */
const float *nln_sorted_pos(const nln_tree *t);

/*
 * Run-pack the walked lists (format in nlnlists.h) of every kind (0 P,
 * 1 Q, 2 H, 3 correction), group by group in parallel, and keep them beside
 * the plain lists.  Returns 0, or -1 when the tree has no lists.
 * nln_packed_ptr: ngroups + 1 word offsets per group (NULL before packing);
 * nln_packed_data / nln_packed_len: the words.
 */
int nln_tree_pack(nln_tree *t);
const int64_t *nln_packed_ptr(const nln_tree *t, int kind);
const uint32_t *nln_packed_data(const nln_tree *t, int kind);
int64_t nln_packed_len(const nln_tree *t, int kind);

/*
 * The periodic correction C(y) = Phi_Ewald(y) + 1/|y| and its first five
 * derivatives (NLN_EWALD_NQ doubles, layout of nlnlists.h) at one
 * displacement y = source - sink in a cube of side L, from the Ewald sum of
 * nln/ewald.c:13-64 (same alpha = 2/L and k-space cut), differentiated
 * analytically.  Its gradient plus y/|y|^3 is ewald()'s force.
 */
void nln_ewald_eval(double L, const double *y, double *out);
/* The same on an n^3 grid over [0, reach*L]^3 (node (i,j,k) at (i,j,k)*reach*L/(n-1)). */
int nln_ewald_table(double L, int n, double reach, double *out);

/*
 * Acceleration at r (relative to the cube's centre) from a cube of half-side
 * a and unit density, G = 1, pointing toward the cube: the field that the
 * reference's background subtraction adds back per sink for its near zone,
 * scaled by -rho0 (cubic_acc, nln/ewald_le2.c:773-1033; nln/mac.c:688-706).
 * FP64, valid inside and outside the cube.
 */
void nln_cubic_acc(const double r[3], double a, double acc[3]);

/*
 * ---- snapshots and checkpoints in the SDF format ----
 * The reference writes bodies as outbody records (nln/physics.h:49-58:
 * mass, x y z, vx vy vz, with SAVE_ACC also ax ay az phi, int64 ident;
 * packed) with the descriptor OUTBODYDESC (nln/physics.h:62-110) and header
 * scalars (version, npart, iter, tpos, tvel, ..., nln/output.c:217-330)
 * into an SDF file: an ASCII header of C-like declarations ending
 * "# SDF-EOH", then the little-endian records.  nln_sdf_write writes one
 * (acc_phi: NULL for the plain record, else 4 floats per body (ax, ay, az,
 * phi)); header entries are (key, type, value) with the NLN_SDF_* types.
 * nln_sdf_read reads one back: its header entries, the record count, and
 * the bodies (nln_sdf_bodies; any output pointer may be NULL).  Errors:
 * -1 / NULL with a message in nln_sdf_error().
 */
#define NLN_SDF_INT 0
#define NLN_SDF_INT64 1
#define NLN_SDF_FLOAT 2
#define NLN_SDF_DOUBLE 3
typedef struct nln_sdf nln_sdf;
int nln_sdf_write(const char *path, int64_t n, const float *mass, const float *pos,
                  const float *vel, const float *acc_phi, const int64_t *ident, int nkeys,
                  const char *const *keys, const int *types, const double *values);
nln_sdf *nln_sdf_read(const char *path);
int64_t nln_sdf_count(const nln_sdf *s);
int nln_sdf_has_acc(const nln_sdf *s);
int nln_sdf_nkeys(const nln_sdf *s);
const char *nln_sdf_key(const nln_sdf *s, int k, int *type, double *value);
int nln_sdf_bodies(const nln_sdf *s, float *mass, float *pos, float *vel, float *acc_phi,
                   int64_t *ident);
void nln_sdf_free(nln_sdf *s);
const char *nln_sdf_error(void);

/*
 * ---- background cosmology (the cosmological leapfrog's factors) ----
 * The reference integrates comoving runs with CosmoIntegrate
 * (nln/integrate.c:82-135), which takes a(t) and the integrals
 * kick(t0, t1) = int dt / a and drift(t0, t1) = int dt / a^2 from the 2hot
 * library's cosmology object.  nln_cosmo integrates the Friedmann equation
 *   H^2 = H0^2 (Omega_r a^-4 + Omega_m a^-3 + Omega_k a^-2 + Omega_lambda
 *               + Omega_de a^(-3(1+w0+wa)) exp(-3 wa (1-a))),
 *   Omega_k = 1 - Omega_r - Omega_m - Omega_lambda - Omega_de,
 * in the run's time unit (H0 in its inverse), t = 0 at a = 0.
 * nln_cosmo_kdk: CosmoIntegrate's factors for a step from positions at tpos
 * and velocities at tvel: out = {a0^2 kick(tvel, tpos), a0^2 kick(tvel,
 * tvel + dtv), drift(tpos, tpos + dt), 1/a0, a(tpos + dt), 1/a0^2},
 * a0 = a(tpos) -- the params of the cosmological integrator
 * (grav_plan_set_integrator_CUDA).  nln_cosmo_new returns NULL for
 * H0 <= 0 or no matter or radiation.
 */
typedef struct nln_cosmo_params {
    double H0;
    double Omega_m, Omega_r, Omega_lambda;
    double Omega_de, w0, wa; /* a w0 + wa (1 - a) dark-energy fluid */
} nln_cosmo_params;
typedef struct nln_cosmo nln_cosmo;
nln_cosmo *nln_cosmo_new(const nln_cosmo_params *params);
void nln_cosmo_free(nln_cosmo *c);
double nln_cosmo_hubble(const nln_cosmo *c, double a);
double nln_cosmo_t_at_a(const nln_cosmo *c, double a);
double nln_cosmo_a_at_t(const nln_cosmo *c, double t);
double nln_cosmo_kick(const nln_cosmo *c, double t0, double t1);
double nln_cosmo_drift(const nln_cosmo *c, double t0, double t1);
void nln_cosmo_kdk(const nln_cosmo *c, double tpos, double tvel, double dt, double dtv,
                   double out[6]);

#ifdef __cplusplus
}
#endif
#endif
