/*
 * Test infrastructure (oracle build only): link-time wrappers around the
 * LAPACK routines with CHARACTER arguments that the reference calls on the
 * DMRG path (src/wrapper/eig.cpp:74,97,115,124 and src/wrapper/svd.cpp:57,77
 * of mcbapo/mpsdyn).  Linked with -Wl,--wrap=<name>, every call from the
 * reference lands here first.  Two defects of those call sites are repaired
 * without touching the reference sources:
 *
 * 1. Hidden string lengths.  The reference declares the Fortran routines
 *    without the trailing length argument that gfortran passes for every
 *    CHARACTER dummy.  The bundled OpenBLAS LAPACK is gfortran code; when it
 *    forwards those arguments (sibling calls) it reads the missing lengths
 *    from the caller's stack and corrupts it.  Observed here as intermittent
 *    SIGSEGV inside zhetrd -> zlatrd -> zgemv.  The wrappers pass length 1.
 *
 * 2. Workspace queries into a double.  wrapper::eig passes `double workT`
 *    (8 bytes) as the COMPLEX*16 WORK argument of the size query
 *    (lwork == -1); LAPACK stores 16 bytes there.  The wrappers give LAPACK a
 *    16-byte slot and copy the real part (the requested size) back.
 */
#include <stddef.h>

extern void __real_zhetrd_(char *uplo, int *n, double *a, int *lda, double *d,
                           double *e, double *tau, double *work, int *lwork,
                           int *info, size_t uplo_len);
extern void __real_zungtr_(char *uplo, int *n, double *a, int *lda,
                           double *tau, double *work, int *lwork, int *info,
                           size_t uplo_len);
extern void __real_zstedc_(char *compz, int *n, double *d, double *e,
                           double *z, int *ldz, double *work, int *lwork,
                           double *rwork, int *lrwork, int *iwork, int *liwork,
                           int *info, size_t compz_len);
extern void __real_zgesvd_(char *jobu, char *jobvt, int *m, int *n, double *a,
                           int *lda, double *s, double *u, int *ldu,
                           double *vt, int *ldvt, double *work, int *lwork,
                           double *rwork, int *info, size_t jobu_len,
                           size_t jobvt_len);

void __wrap_zhetrd_(char *uplo, int *n, double *a, int *lda, double *d,
                    double *e, double *tau, double *work, int *lwork,
                    int *info) {
  if (*lwork == -1) {
    double slot[2] = {0.0, 0.0};
    __real_zhetrd_(uplo, n, a, lda, d, e, tau, slot, lwork, info, 1);
    work[0] = slot[0];
    return;
  }
  __real_zhetrd_(uplo, n, a, lda, d, e, tau, work, lwork, info, 1);
}

void __wrap_zungtr_(char *uplo, int *n, double *a, int *lda, double *tau,
                    double *work, int *lwork, int *info) {
  if (*lwork == -1) {
    double slot[2] = {0.0, 0.0};
    __real_zungtr_(uplo, n, a, lda, tau, slot, lwork, info, 1);
    work[0] = slot[0];
    return;
  }
  __real_zungtr_(uplo, n, a, lda, tau, work, lwork, info, 1);
}

void __wrap_zstedc_(char *compz, int *n, double *d, double *e, double *z,
                    int *ldz, double *work, int *lwork, double *rwork,
                    int *lrwork, int *iwork, int *liwork, int *info) {
  if (*lwork == -1) {
    double slot[2] = {0.0, 0.0};
    __real_zstedc_(compz, n, d, e, z, ldz, slot, lwork, rwork, lrwork, iwork,
                   liwork, info, 1);
    work[0] = slot[0];
    return;
  }
  __real_zstedc_(compz, n, d, e, z, ldz, work, lwork, rwork, lrwork, iwork,
                 liwork, info, 1);
}

void __wrap_zgesvd_(char *jobu, char *jobvt, int *m, int *n, double *a,
                    int *lda, double *s, double *u, int *ldu, double *vt,
                    int *ldvt, double *work, int *lwork, double *rwork,
                    int *info) {
  __real_zgesvd_(jobu, jobvt, m, n, a, lda, s, u, ldu, vt, ldvt, work, lwork,
                 rwork, info, 1, 1);
}
