/* ORACLE build helper (test infrastructure only).
 * The reference's runtime (common/dgemm/bl_dgemm_util.c:5-58) references the BLAS
 * routines dcopy_/daxpy_ from two helpers that no code path calls.  This image has no
 * BLAS, so these two small definitions satisfy the linker for the reference build. */
void dcopy_(const int *n, const double *x, const int *incx, double *y, const int *incy) {
  for (int i = 0; i < *n; ++i) y[i * *incy] = x[i * *incx];
}
void daxpy_(const int *n, const double *a, const double *x, const int *incx, double *y, const int *incy) {
  for (int i = 0; i < *n; ++i) y[i * *incy] += *a * x[i * *incx];
}
