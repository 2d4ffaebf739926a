/*
 * nlnlists.h -- record layouts shared by the host list builder (nlnhost.h)
 * and the batched device kernels (gravcuda.h).
 *
 * The reference packs each list as copies of cell fields into 8-lane AoSoA
 * blocks (nln/mac.c:117-153).  At N = 2^24 per-group copies do not fit, so
 * the batched path instead keeps one table of cells and one table of points
 * resident on the device and hands the kernels index lists into them.
 */
#ifndef NLNLISTS_H
#define NLNLISTS_H

#include <stdint.h>

/* Cell record layouts of the device tables (little-endian, 16-byte multiples). */
typedef struct nln_qcell {      /* 64 bytes */
    double cen[3];              /* FP64 expansion centre (centre of mass) */
    float mass, R;              /* R = bmax normalises the moments */
    float qxx, qxy, qyy, qxz, qyz;
    float B2;                   /* sum m |x - cen|^2 (the trace the quadrupole drops) */
    float pad[2];
} nln_qcell;

typedef struct nln_hcell {      /* 128 bytes */
    double cen[3];
    float mass, R;
    float q2[5];                /* qxx qxy qyy qxz qyz              / R^2 */
    float q3[7];                /* qxxx qxxy qxyy qyyy qxxz qxyz qyyz / R^3 */
    float q4[9];                /* qxxxx qxxxy qxxyy qxyyy qyyyy qxxxz qxxyz qxyyz qyyyz / R^4 */
    float B2;                   /* sum m |x - cen|^2 */
    float pad[2];
} nln_hcell;


/*
 * Periodic boxes: a source is used whole in the image nearest the sink
 * group's centre, and every sink-source displacement stays inside
 * |y_k| <= NLN_EWALD_REACH * box, the domain of the Ewald correction table.
 */
#define NLN_EWALD_REACH 0.625

/*
 * Ewald correction table: per node, NLN_EWALD_NQ values of
 * C(y) = Phi_Ewald(y) + 1/|y| and its derivatives of orders 0..5, in the order
 *   C | dC/dx dC/dy dC/dz | xx xy xz yy yz zz | xxx xxy xxz xyy xyz xzz yyy yyz yzz zzz |
 *   xxxx xxxy ... zzzz (15) | xxxxx xxxxy ... zzzzz (21)
 * (order n starts at n(n+1)(n+2)/6; its components are the sorted index
 * tuples i <= j <= ... in lexicographic order, multi-index (ax, ay, az) at
 * offset (n-ax)(n-ax+1)/2 + az)
 * on an n^3 grid over the positive octant [0, NLN_EWALD_REACH * L]^3
 * (the cubic lattice makes C even in each coordinate).
 */
#define NLN_EWALD_NQ 56

/*
 * List entries (points, quadrupole and order-4 cells alike): the record
 * index in its table | image code << 27, where the image code is
 * (sx+1)*9 + (sy+1)*3 + (sz+1) for the periodic shift (sx, sy, sz) in box
 * units; 13 = no shift.  Point-table records below the body count are
 * bodies, the rest cell monopoles.
 */
#define NLN_SHIFT_NONE 13u
#define NLN_IDX_BITS 27
#define NLN_IDX_MASK ((1u << NLN_IDX_BITS) - 1u)

/*
 * Run-packed lists: a shorter form of a list for the host-to-device copy.
 * Entries of a group's list that continue the entry before them (index + 1,
 * same image code) are folded into run words: a word whose image code is
 * NLN_RUN_CODE stands for the entries e+1, e+2, ..., e+n after the entry e
 * that precedes it, n = word & NLN_IDX_MASK (n >= 1).  A run word follows
 * an entry word of its own group (never starts a group's list, never
 * follows another run word), and each group's packed list unpacks to
 * exactly its plain list.  Leaves expanded into bodies make long runs of the point list
 * (about 17x fewer words on a clustered 128^3 box); cell lists pack about 3x.
 */
#define NLN_RUN_CODE 31u

typedef struct nln_group {      /* 40 bytes */
    double cen[3];              /* FP64 group centre (centre of mass of its sinks) */
    int64_t first;              /* first sink, in tree order */
    int32_t count;              /* sinks */
    float radius;               /* max sink distance from cen */
} nln_group;

#endif
