/* C entry point over the reference's own ICT (hip/Precond/ict_l.cpp:196-201,
 * ict_csr_A_l: row norms then the left-looking threshold factorization),
 * which oracle/Makefile compiles from the reference sources into
 * oracle/_ref.  Test oracle only. */
template <typename T>
void ict_csr_A_l(int n, int *ptr, T *val, int *col, int *lPtr, T *lVal, int *lCol, T smallNum, T droptol, int maxfil);
extern "C" void ref_ict_csr_A_l(int n, int *ptr, double *val, int *col, int *lPtr, double *lVal, int *lCol,
                                double smallNum, double droptol, int maxfil)
{
    ict_csr_A_l<double>(n, ptr, val, col, lPtr, lVal, lCol, smallNum, droptol, maxfil);
}
