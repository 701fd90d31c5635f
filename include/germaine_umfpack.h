/*
 * germaine_umfpack.h -- the UMFPACK calls of GERMAINE's per-frequency
 * drivers, served by the B200 engine (libgermaine_umfpack.so, built over
 * libgermaine_gpu.so).
 *
 * The reference links SuiteSparse UMFPACK (src/Makefile:32-35, -lumfpack)
 * and calls exactly these six functions, always in this sequence per
 * frequency (src/AC/forward_shot_AC.c:41-120, src/AC/grad_obj_AC.c,
 * src/AC/obj_AC.c, src/AC/hessian_AC.c, src/AC/hessian_shin_AC.c and the
 * SH/TE twins):
 *
 *   umfpack_zi_triplet_to_col -> umfpack_zi_symbolic -> umfpack_zi_numeric
 *   -> umfpack_zi_free_symbolic -> umfpack_zi_solve (per shot, UMFPACK_A or
 *   UMFPACK_Aat) -> umfpack_zi_free_numeric
 *
 * A build of the unmodified drivers against this header (as "umfpack.h")
 * and this library runs its factorisations and solves on the GPU.  The
 * names, argument lists, sys codes and status codes are UMFPACK's public
 * interface (SuiteSparse UMFPACK user guide, "zi" = int indices, split
 * real/imaginary double arrays); what the library accepts is narrower:
 *
 *  - umfpack_zi_symbolic accepts square matrices whose sparsity pattern is
 *    contained in the 9-point stencil of an NX x NY grid (the impedance
 *    matrices of src/AC/init_A_AC_9p_pml.c, src/SH/init_A_SH_9p_pml.c,
 *    src/TE/init_A_TE_9p_pml.c).  NX is read from column 0, whose rows are
 *    {0, 1, NX, NX+1}; any other pattern returns
 *    UMFPACK_ERROR_invalid_matrix.  The ordering is the engine's geometric
 *    nested dissection, not AMD/COLAMD.
 *  - umfpack_zi_numeric factorises with threshold partial pivoting at
 *    UMFPACK's default relative tolerance 0.1, restricted to row exchanges
 *    inside each front's 32-pivot blocks (the smallest fronts, at the
 *    leaves of the tree, keep static pivots); a pivot that is still tiny is
 *    replaced and returns UMFPACK_WARNING_singular_matrix, like UMFPACK's
 *    zero-pivot warning.
 *  - umfpack_zi_solve supports sys = UMFPACK_A, UMFPACK_At (conjugate
 *    transpose) and UMFPACK_Aat (array transpose); the partial systems
 *    (L, U, P...) return UMFPACK_ERROR_invalid_system.  Every solve ends
 *    with FP64 iterative refinement to a relative residual of 1e-10 on the
 *    device, using the values given to umfpack_zi_numeric; the Ap, Ai, Ax,
 *    Az arguments of the solve are not read.
 *  - Control is ignored (NULL is fine, as the reference passes).  If Info
 *    is non-NULL, Info[UMFPACK_STATUS] receives the status; no other Info
 *    entry is written.
 *  - Environment: GM_UMFPACK_DEVICE (CUDA device, default 0) and
 *    GM_UMFPACK_PRECISION ("fp64", the default, or "c64" for complex64
 *    fronts with FP64 refinement).
 *
 * Complex arrays follow UMFPACK's zi convention: real parts in Xx, imaginary
 * parts in Xz; when both imaginary pointers of a call (Tz and Az, or Xz and
 * Bz) are NULL, the real-part arrays hold interleaved (packed) complex
 * values instead.
 *
 * gm_umfpack_last_error() (no counterpart in UMFPACK) returns the message
 * of the last failure on the calling thread.
 */
#ifndef GERMAINE_UMFPACK_H
#define GERMAINE_UMFPACK_H

#ifdef __cplusplus
extern "C" {
#endif

/* sys argument of umfpack_zi_solve */
#define UMFPACK_A   0   /* A x = b */
#define UMFPACK_At  1   /* A^H x = b (conjugate transpose) */
#define UMFPACK_Aat 2   /* A^T x = b (array transpose) */

/* status codes */
#define UMFPACK_OK                            0
#define UMFPACK_WARNING_singular_matrix       1
#define UMFPACK_ERROR_out_of_memory          -1
#define UMFPACK_ERROR_invalid_Numeric_object -3
#define UMFPACK_ERROR_invalid_Symbolic_object -4
#define UMFPACK_ERROR_argument_missing       -5
#define UMFPACK_ERROR_n_nonpositive          -6
#define UMFPACK_ERROR_invalid_matrix         -8
#define UMFPACK_ERROR_different_pattern     -11
#define UMFPACK_ERROR_invalid_system        -13
#define UMFPACK_ERROR_internal_error       -911

/* Info / Control array sizes and the status slot of Info */
#define UMFPACK_INFO    90
#define UMFPACK_CONTROL 20
#define UMFPACK_STATUS   0

/* src/AC/forward_shot_AC.c:41 -- triplets to compressed sparse columns,
 * duplicates summed, rows ascending within each column.  Map (optional,
 * nz entries) receives the position in Ai/Ax of each triplet. */
int umfpack_zi_triplet_to_col(int n_row, int n_col, int nz, const int Ti[], const int Tj[],
                              const double Tx[], const double Tz[], int Ap[], int Ai[],
                              double Ax[], double Az[], int Map[]);

/* src/AC/forward_shot_AC.c:58 -- pattern analysis (grid detection). */
int umfpack_zi_symbolic(int n_row, int n_col, const int Ap[], const int Ai[], const double Ax[],
                        const double Az[], void **Symbolic, const double Control[], double Info[]);

/* src/AC/forward_shot_AC.c:61 -- numeric factorisation on the GPU. */
int umfpack_zi_numeric(const int Ap[], const int Ai[], const double Ax[], const double Az[],
                       void *Symbolic, void **Numeric, const double Control[], double Info[]);

/* src/AC/forward_shot_AC.c:88, src/TE/grad_obj_TE.c:149 -- one solve. */
int umfpack_zi_solve(int sys, const int Ap[], const int Ai[], const double Ax[], const double Az[],
                     double Xx[], double Xz[], const double Bx[], const double Bz[], void *Numeric,
                     const double Control[], double Info[]);

/* src/AC/forward_shot_AC.c:62 and :120 */
void umfpack_zi_free_symbolic(void **Symbolic);
void umfpack_zi_free_numeric(void **Numeric);

/* No counterpart in UMFPACK: message of the last failure on this thread. */
const char *gm_umfpack_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
