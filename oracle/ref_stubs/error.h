/*
 * TEST INFRASTRUCTURE ONLY.  Stand-in for the 2hot library's error.h (the
 * un-vendored 2hot submodule), just enough for nln/ewald.c to compile
 * unmodified into the reference checker: ewald.c includes it but calls
 * nothing from it.
 */
#ifndef ORACLE_STUB_ERROR_H
#define ORACLE_STUB_ERROR_H
#include <stdio.h>
#include <stdlib.h>
#define Error(...) (fprintf(stderr, __VA_ARGS__), abort())
#endif
