/* C entry points over the reference's own CPU ILU(0) (hip/Precond/
 * ilut_diag_in_csr.cpp:347-405, `ilu0_simple`) and Saad ILUT (:20-251,
 * `ilutp_final`), which oracle/Makefile compiles from the reference sources
 * into oracle/_ref.  Test oracle only. */
template <typename T> void ilu0_simple(T *luval, T *val, int *rows, int *cols, int n, int *uptr);
extern "C" void ref_ilu0_simple(double *luval, double *val, int *rows, int *cols, int n, int *uptr)
{
    ilu0_simple<double>(luval, val, rows, cols, n, uptr);
}

template <typename T>
void ilutp_final(T *luval, T *val, int *rows, int *cols, int n, T *diag, int lfil, int *lucols, int *lurows, int *uptr,
                 T permtol, T droptol, int *iperm, int *ipermn);
/* the call of hip/HostMatrix/HostMatrixCSR.cpp:230-237 (seqilut): luval and
 * lucols hold (2*lfil+2)*n entries */
extern "C" void ref_ilutp_final(double *luval, double *val, int *rows, int *cols, int n, double *diag, int lfil,
                                int *lucols, int *lurows, int *uptr, double droptol)
{
    ilutp_final<double>(luval, val, rows, cols, n, diag, lfil, lucols, lurows, uptr, 0, droptol, nullptr, nullptr);
}
