/* Declaration-only stand-in for SuiteSparse <umfpack.h>: the constants the
 * reference's hot-path sources name.  The oracle never calls UMFPACK (the
 * sparse solve is done by SciPy SuperLU in oracle/sparse.py).  Test
 * infrastructure only. */
#ifndef ORACLE_STUB_UMFPACK_H
#define ORACLE_STUB_UMFPACK_H
#define UMFPACK_A 0
#define UMFPACK_At 1
#define UMFPACK_Aat 2
#endif
