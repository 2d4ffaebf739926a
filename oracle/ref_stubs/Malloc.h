/*
 * TEST INFRASTRUCTURE ONLY.  Stand-in for the 2hot library's Malloc.h (the
 * un-vendored 2hot submodule), just enough for nln/ewald_le2.c to compile
 * unmodified into the reference checker: the allocator calls it makes.
 */
#ifndef ORACLE_STUB_MALLOC_H
#define ORACLE_STUB_MALLOC_H
#include <stdlib.h>
#define Calloc(n, size) calloc((n), (size))
#define Free(p) free(p)
#endif
