/* C entry point over the reference's own IC(0) (hip/Precond/ic0.cpp:72-81,
 * ic0_csr_A), which oracle/Makefile compiles from the reference sources
 * into oracle/_ref.  Test oracle only. */
template <typename T>
void ic0_csr_A(int n, int *ptr, T *val, int *col, int *lPtr, T *lVal, int *lCol, T smallNum, T droptol);
extern "C" void ref_ic0_csr_A(int n, int *ptr, double *val, int *col, int *lPtr, double *lVal, int *lCol,
                              double smallNum, double droptol)
{
    ic0_csr_A<double>(n, ptr, val, col, lPtr, lVal, lCol, smallNum, droptol);
}
