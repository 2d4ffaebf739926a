/*
 * TEST INFRASTRUCTURE ONLY.  Stand-in for the 2hot library's mpmy.h (its
 * MPI layer): one process, so a combine leaves the buffer as it is.
 */
#ifndef ORACLE_STUB_MPMY_H
#define ORACLE_STUB_MPMY_H
#define MPMY_DOUBLE 0
#define MPMY_SUM 0
#define MPMY_Combine(in, out, n, type, op) ((void)(in), (void)(out), (void)(n), 0)
#endif
