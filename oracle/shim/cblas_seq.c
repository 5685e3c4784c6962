/* Sequential BLAS-1 used by the compiled reference oracle (see mkl.h). */
#include "mkl.h"
double cblas_ddot(const int n, const double *x, const int incx, const double *y, const int incy)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s += x[i * incx] * y[i * incy];
    return s;
}
void cblas_daxpy(const int n, const double a, const double *x, const int incx, double *y, const int incy)
{
    for (int i = 0; i < n; i++) y[i * incy] += a * x[i * incx];
}
void cblas_dcopy(const int n, const double *x, const int incx, double *y, const int incy)
{
    for (int i = 0; i < n; i++) y[i * incy] = x[i * incx];
}
void cblas_dscal(const int n, const double a, double *x, const int incx)
{
    for (int i = 0; i < n; i++) x[i * incx] *= a;
}
