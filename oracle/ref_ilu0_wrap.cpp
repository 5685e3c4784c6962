/* C entry point over the reference's own CPU ILU(0) (hip/Precond/
 * ilut_diag_in_csr.cpp:347-405, `ilu0_simple`), which oracle/Makefile
 * compiles from the reference sources into oracle/_ref.  Test oracle only. */
template <typename T> void ilu0_simple(T *luval, T *val, int *rows, int *cols, int n, int *uptr);
extern "C" void ref_ilu0_simple(double *luval, double *val, int *rows, int *cols, int n, int *uptr)
{
    ilu0_simple<double>(luval, val, rows, cols, n, uptr);
}
