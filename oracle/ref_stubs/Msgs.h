/*
 * TEST INFRASTRUCTURE ONLY.  Stand-in for the 2hot library's Msgs.h: its
 * debug-message macro, which the checker leaves silent.
 */
#ifndef ORACLE_STUB_MSGS_H
#define ORACLE_STUB_MSGS_H
#define Msgf(args) ((void)0)
#endif
