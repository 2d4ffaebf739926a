/*
 * TEST INFRASTRUCTURE ONLY.  Stand-in for nln/physics.h when nln/ewald_le2.c
 * is compiled into the reference checker: the reference header pulls in the
 * 2hot tree, key and timer headers, which are not vendored.  ewald_le2.c
 * reads a body's mass and position only; this body holds those (the
 * harness fills it), and NDIM and the vector macros come from vop.h.
 */
#ifndef ORACLE_STUB_PHYSICS_H
#define ORACLE_STUB_PHYSICS_H
#include "vop.h"
typedef struct {
    float mass;
    float pos[NDIM];
} body;
#endif
