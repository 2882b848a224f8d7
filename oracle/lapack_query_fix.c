/*
 * Test infrastructure (oracle build only): link-time wrappers around three
 * LAPACK routines called by the reference's wrapper::eig
 * (src/wrapper/eig.cpp:74,97,115 of mcbapo/mpsdyn).
 *
 * That code passes `double workT` (8 bytes) as the WORK argument of the
 * workspace-size query (lwork == -1).  WORK is COMPLEX*16, so LAPACK stores
 * 16 bytes there and overwrites the caller's stack.  Built with -O2 the
 * reference crashes at its first dense local eigensolve.  With
 * `-Wl,--wrap=zhetrd_` etc. every call from the reference lands here first;
 * a query gets a 16-byte slot and only its real part (the size LAPACK asks
 * for) is copied back.  Real calls pass straight through.  The reference
 * sources stay untouched.
 */

extern void __real_zhetrd_(char *uplo, int *n, double *a, int *lda, double *d,
                           double *e, double *tau, double *work, int *lwork,
                           int *info);
extern void __real_zungtr_(char *uplo, int *n, double *a, int *lda,
                           double *tau, double *work, int *lwork, int *info);
extern void __real_zstedc_(char *compz, int *n, double *d, double *e,
                           double *z, int *ldz, double *work, int *lwork,
                           double *rwork, int *lrwork, int *iwork, int *liwork,
                           int *info);

void __wrap_zhetrd_(char *uplo, int *n, double *a, int *lda, double *d,
                    double *e, double *tau, double *work, int *lwork,
                    int *info) {
  if (*lwork == -1) {
    double slot[2] = {0.0, 0.0};
    __real_zhetrd_(uplo, n, a, lda, d, e, tau, slot, lwork, info);
    work[0] = slot[0];
    return;
  }
  __real_zhetrd_(uplo, n, a, lda, d, e, tau, work, lwork, info);
}

void __wrap_zungtr_(char *uplo, int *n, double *a, int *lda, double *tau,
                    double *work, int *lwork, int *info) {
  if (*lwork == -1) {
    double slot[2] = {0.0, 0.0};
    __real_zungtr_(uplo, n, a, lda, tau, slot, lwork, info);
    work[0] = slot[0];
    return;
  }
  __real_zungtr_(uplo, n, a, lda, tau, work, lwork, info);
}

void __wrap_zstedc_(char *compz, int *n, double *d, double *e, double *z,
                    int *ldz, double *work, int *lwork, double *rwork,
                    int *lrwork, int *iwork, int *liwork, int *info) {
  if (*lwork == -1) {
    double slot[2] = {0.0, 0.0};
    __real_zstedc_(compz, n, d, e, z, ldz, slot, lwork, rwork, lrwork, iwork,
                   liwork, info);
    work[0] = slot[0];
    return;
  }
  __real_zstedc_(compz, n, d, e, z, ldz, work, lwork, rwork, lrwork, iwork,
                 liwork, info);
}
