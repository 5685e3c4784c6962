/* Stand-in for the four MKL cblas routines the reference intel/ CPU path
 * calls (cblas_ddot, cblas_daxpy, cblas_dcopy, cblas_dscal).  Used only to
 * compile that reference path from its own sources as a test oracle; the
 * implementations in cblas_seq.c are plain sequential loops, so the
 * reduction order of cblas_ddot is the natural left-to-right order. */
#ifndef XS_ORACLE_MKL_SHIM_H
#define XS_ORACLE_MKL_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif
double cblas_ddot(const int n, const double *x, const int incx, const double *y, const int incy);
void cblas_daxpy(const int n, const double a, const double *x, const int incx, double *y, const int incy);
void cblas_dcopy(const int n, const double *x, const int incx, double *y, const int incy);
void cblas_dscal(const int n, const double a, double *x, const int incx);
#ifdef __cplusplus
}
#endif
#endif
