/* Test shim: inert definitions of the LAPACK SVD symbols declared in
 * shim/lapacke.h (the oracle never calls the reference's SVD actor; numpy's
 * SVD stands in for it).  Both report an illegal-argument status. */
#include "lapacke.h"

void LAPACK_sgesvd(char *jobu, char *jobvt, int *m, int *n, float *a, int *lda, float *s, float *u, int *ldu,
                   float *vt, int *ldvt, float *work, int *lwork, int *info)
{
    (void)jobu; (void)jobvt; (void)m; (void)n; (void)a; (void)lda; (void)s; (void)u; (void)ldu;
    (void)vt; (void)ldvt; (void)lwork;
    if (work) work[0] = 1.0f;
    *info = -1;
}

void LAPACK_dgesvd(char *jobu, char *jobvt, int *m, int *n, double *a, int *lda, double *s, double *u, int *ldu,
                   double *vt, int *ldvt, double *work, int *lwork, int *info)
{
    (void)jobu; (void)jobvt; (void)m; (void)n; (void)a; (void)lda; (void)s; (void)u; (void)ldu;
    (void)vt; (void)ldvt; (void)lwork;
    if (work) work[0] = 1.0;
    *info = -1;
}
