/* Test shim: declarations of the two LAPACK SVD entry points that the
 * reference's gains_calibration_run.c names, so that file compiles for the
 * oracle without LAPACKE.  The oracle drivers call only the reference's
 * normal-equation, SUQ-product and gain-update actors; the SVD step is taken
 * by numpy.linalg.svd in the tests (shim/lapack_stub.c only reports failure). */
#ifndef ORACLE_SHIM_LAPACKE_H
#define ORACLE_SHIM_LAPACKE_H
void LAPACK_sgesvd(char *jobu, char *jobvt, int *m, int *n, float *a, int *lda, float *s, float *u, int *ldu,
                   float *vt, int *ldvt, float *work, int *lwork, int *info);
void LAPACK_dgesvd(char *jobu, char *jobvt, int *m, int *n, double *a, int *lda, double *s, double *u, int *ldu,
                   double *vt, int *ldvt, double *work, int *lwork, int *info);
#endif
