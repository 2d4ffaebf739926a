/*
 * TEST INFRASTRUCTURE ONLY.  Stand-in for the 2hot library's vop.h (the
 * un-vendored 2hot submodule): the component-wise vector macros as
 * nln/ewald.c uses them, over NDIM components.
 *   VS(a, op)          a[k] op                 e.g. VS(f, = 0)
 *   VV(a, op b)        a[k] op b[k]            e.g. VV(f, += t * xx)
 *   VVV(a, op b, op c) a[k] op b[k] op c[k]    e.g. VVV(xx, = x, -L * i)
 *   Dot(a, b)          sum_k a[k] b[k]
 */
#ifndef ORACLE_STUB_VOP_H
#define ORACLE_STUB_VOP_H
#ifndef NDIM
#define NDIM 3
#endif
#define VS(a, op) do { for (int vop_k = 0; vop_k < NDIM; vop_k++) (a)[vop_k] op; } while (0)
#define VV(a, b) do { for (int vop_k = 0; vop_k < NDIM; vop_k++) (a)[vop_k] b[vop_k]; } while (0)
#define VVV(a, b, c) \
    do { for (int vop_k = 0; vop_k < NDIM; vop_k++) (a)[vop_k] b[vop_k] c[vop_k]; } while (0)
#define Dot(a, b) ((a)[0] * (b)[0] + (a)[1] * (b)[1] + (a)[2] * (b)[2])
#endif
