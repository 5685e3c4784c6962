/*
 * xsolver_b200 — B200 (sm_100a) preconditioned Krylov solve path behind the
 * xsolver C API.
 *
 * Three groups of entry points, all exported with C linkage from
 * libxsolver_b200.so:
 *
 *  1. The reference's setter-style API (hip/xsolver_c.h:37-49).  The
 *     reference declares these with C++ linkage and one C++ reference
 *     parameter (usediter); here they are extern "C" with a pointer, and
 *     C++ callers additionally get inline forwarders with the reference's
 *     exact signatures (same names, argument meaning and defaults).
 *  2. The Fortran-style cpu_/gpu_ entry points of the reference's cuda/
 *     backend (cuda/DeviceMatrix.h:121-169, cuda/mpicudasolver-C-v1.cu:165-1391,
 *     intel/HostMatrix.h:187-222).  Their C++ reference parameters are
 *     pointers at the ABI level; C callers pass pointers.
 *  3. Extensions with no reference counterpart: status-returning twins,
 *     precision control (mixed-precision iterative refinement), ParILU/ParILUT
 *     parameters, the adjoint, and a few kernel-level calls on device
 *     pointers used by tests and benchmarks.
 *
 * Errors: the reference prints and calls exit(0) on bad input; this library
 * never exits.  Every call records a status readable with
 * xsolver_last_error(); the xs_* twins return it directly.
 */
#ifndef XSOLVER_B200_C_H
#define XSOLVER_B200_C_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* status codes                                                        */
/* ------------------------------------------------------------------ */
enum xs_status {
    XS_OK = 0,
    XS_ERR_INVALID = 1,       /* bad argument (size, pointer, string)          */
    XS_ERR_CUDA = 2,          /* a CUDA runtime call failed                     */
    XS_ERR_NOMEM = 3,         /* device allocation failed                       */
    XS_ERR_NO_DIAG = 4,       /* a row has no diagonal entry (ILU/Jacobi)       */
    XS_ERR_TRSV_TIMEOUT = 5,  /* sync-free solve gave up waiting on a row       */
    XS_ERR_BREAKDOWN = 6,     /* Krylov breakdown (non-finite scalar)           */
    XS_ERR_NAN = 7,           /* non-finite input or residual                   */
    XS_ERR_ORDER = 8,         /* calls out of order (e.g. pc before ksp)        */
    XS_ERR_ELL_WIDTH = 9,     /* ELL width outside the supported range          */
    XS_ERR_UNSUPPORTED = 10,  /* combination not provided (e.g. CSC format)     */
    XS_ERR_CAPACITY = 11,     /* a fixed per-row capacity was exceeded          */
    XS_ERR_NO_GPU = 12        /* no CUDA device visible                         */
};

/* ------------------------------------------------------------------ */
/* 1. reference setter-style API (hip/xsolver_c.h:37-49)               */
/* ------------------------------------------------------------------ */

/* hip/xsolver_c.cpp:41-102.  CSR with n rows; rowptr[0] selects 0- or
 * 1-based indexing.  advanced_pam[3] = {distribute (must be 0: one GPU),
 * SpMV format (0 CSR, 1 ELL; 2 = CSC is CPU-only in the reference), gpu
 * (ignored: always the GPU)}.  distribute = 1 or CSC records
 * XS_ERR_UNSUPPORTED and leaves the previous matrix in place, as does a
 * pattern that fails validation (XS_ERR_INVALID).  The arrays are copied:
 * unlike the reference, which borrows them until xsolver_free(), the caller
 * may release them when the call returns. */
void xsolver_mat_setup(int nInterior, int *rowptr, int *colidx, double *val, int *advanced_pam);
/* hip/xsolver_c.cpp:103-130: "bicgstab", "cg", "igcr" (case variants as in
 * the reference), plus "gcr", "gmres", "fgmres", "cgm"/"pcg", and the
 * single-reduction "icg", "icgm", "ibicgstab" of intel/mpisolver-C-v1.cpp
 * (left open at hip/xsolver_c.cpp:127). */
void xsolver_ksp_settype(char *fmt);
/* hip/xsolver_c.cpp:131-133 */
void xsolver_ksp_set_absolute_tol(double absolute_tol);
/* hip/xsolver_c.cpp:134-149.  *usediter and resvec (>= maxiter+1 entries)
 * must stay valid until xsolver_solve returns.  resvec[0] = ||r0||,
 * resvec[k+1] = ||r_k|| (absolute), *usediter = iterations used. */
void xsolver_ksp_setoption(double tol, int maxiter, int *usediter, double *resvec, int restart);
/* hip/xsolver_c.cpp:150-263: "jacobi", "ilu0", "ic0", "ilut" (GPU ParILUT),
 * "ilu0_mkl"/"ilut_mkl" (mapped to ilu0/ilut as the reference does on GPU),
 * plus "parilu" and "none".  "ic0" needs a structurally symmetric pattern
 * (XS_ERR_UNSUPPORTED at solve otherwise).  "ict" (incomplete Cholesky with
 * threshold, the reference's CPU-only ICT: it exits for it on GPU) and
 * "ilup"/"ilut_saad" (Saad's ILUT, the reference's CPU "ilut") are factored
 * on the host by the reference's sequential algorithms and applied by the
 * GPU triangular solves.  Must follow xsolver_ksp_settype. */
void xsolver_pc_settype(char *fmt);
/* hip/xsolver_c.cpp:268-273.  For "ilut": max_fill is the ParILUT fill
 * factor, tol its drop tolerance; for "ilup": Saad ILUT's entries per row
 * part (lfil) and drop tolerance (defaults 20, 1e-5). */
void xsolver_pc_setilut(double tol, int max_fill);
/* hip/xsolver_c.cpp:264-267.  For "ict" (ignored otherwise): drop tolerance
 * and kept entries per row (defaults 1e-8, 100; max_fill is clamped to n-1).
 * As in the reference, the pivot substitute uses the fixed scale 1e-4. */
void xsolver_pc_setict(double tol, int max_fill);
/* hip/xsolver_c.cpp:274-292.  sol holds x0 on entry, the solution on exit. */
void xsolver_solve(double *rhs, double *sol);
/* hip/xsolver_c.cpp:308-333 */
void xsolver_free(void);

/* status of the last call of any entry point on this thread's default handle */
int xsolver_last_error(void);
const char *xsolver_error_string(int status);

/* ------------------------------------------------------------------ */
/* 3a. extensions to the setter API                                    */
/* ------------------------------------------------------------------ */
/* Mixed precision.  outer must be "fp64".  inner "fp64" (plain FP64 solve)
 * or "fp32" (FP64 iterative refinement around an FP32 inner solve of the
 * selected ksp type).  factor "fp64", "fp32", "bf16" or "fp16": storage of
 * the ILU factor values (dinv is kept in FP32/FP64). */
void xsolver_set_precision(const char *outer, const char *inner, const char *factor);
/* inner relative tolerance and iteration cap of the refinement's inner
 * solve.  A step whose outer residual is already within 1/inner_rtol of the
 * target solves only to 0.25 * target / ||r|| (never tighter than inner_rtol,
 * never looser than 0.5). */
void xsolver_set_inner(double inner_rtol, int inner_maxiter);
/* ParILU sweep count (default 20, hip/Precond/precon_gpuilu0.cpp:5) */
void xsolver_pc_setparilu(int sweeps);
/* ParILUT: fill factor (default 3), sweeps (default 10), drop tolerance
 * (default 0, no reference counterpart) */
void xsolver_pc_setparilut(double fill, int sweeps, double droptol);
/* triangular solve mode: 0 exact sync-free (default), k > 0 k Jacobi sweeps
 * per triangle (the reference GPU path's approximate solve) */
void xsolver_pc_set_trsv(int mode);
/* 1 (default for the gpu_* entry points) reproduces the reference GMRES
 * update with i instead of i+1 columns on convergence; 0 uses i+1. */
void xsolver_set_compat(int reference_quirks);

/* Adjoint of the last xsolver_solve: given dLdx (n), solve A^T lambda = dLdx
 * with the transposed SpMV and transposed triangular solves, then
 * dLdb = lambda and dLdA_vals[k] = -lambda_i * x_j for each stored entry
 * k = (i, j) of A (in A's CSR order).  Any output may be NULL.
 * The backward solve uses the forward solver type, tolerance and maxiter.
 * XS_ERR_ORDER when there is no solution to differentiate through: no
 * solve yet, the last solve ended with an error, or the values changed
 * since (xs_mat_update / gpu_mat_update). */
void xsolver_adjoint(double *dLdx, double *dLdb, double *dLdA_vals);

/* ------------------------------------------------------------------ */
/* 3b. status-returning handle API                                     */
/* ------------------------------------------------------------------ */
typedef struct xs_handle_s *xs_handle_t;

int xs_create(xs_handle_t *h);
int xs_destroy(xs_handle_t h);
int xs_mat_setup(xs_handle_t h, int n, const int *rowptr, const int *colidx, const double *val, int format);
/* new values for the pattern given to xs_mat_setup, in the caller's entry
 * order (cpu_mat_update + gpu_mat_update for a handle, intel/HostMatrix.h:196-200,
 * cuda/DeviceMatrix.h:145-148); the preconditioner is rebuilt on the next solve */
int xs_mat_update(xs_handle_t h, const double *val);
int xs_ksp_settype(xs_handle_t h, const char *fmt);
int xs_ksp_setoption(xs_handle_t h, double tol, int maxiter, int *usediter, double *resvec, int restart);
int xs_ksp_set_absolute_tol(xs_handle_t h, double absolute_tol);
int xs_pc_settype(xs_handle_t h, const char *fmt);
/* ParILUT ("ilut") fill and drop tolerance, and Saad ILUT ("ilup") lfil and
 * drop tolerance */
int xs_pc_setilut(xs_handle_t h, double tol, int max_fill);
/* ICT drop tolerance (> 0) and kept entries per row */
int xs_pc_setict(xs_handle_t h, double tol, int max_fill);
int xs_pc_setparilu(xs_handle_t h, int sweeps);
int xs_pc_setparilut(xs_handle_t h, double fill, int sweeps, double droptol);
int xs_pc_set_trsv(xs_handle_t h, int mode);
int xs_set_precision(xs_handle_t h, const char *outer, const char *inner, const char *factor);
int xs_set_inner(xs_handle_t h, double inner_rtol, int inner_maxiter);
int xs_set_compat(xs_handle_t h, int reference_quirks);
/* Mixed-precision BiCGSTAB: 1 (default) keeps one FP32 BiCGSTAB iteration
 * running across the refinement steps (at each step x += d in FP64, the FP64
 * residual b - A x replaces the inner residual, and the iteration continues
 * with its search directions); 0 restarts the inner solve at every step on
 * r/||r|| (classic iterative refinement, as for the other methods). */
int xs_set_refinement_mode(xs_handle_t h, int carry_krylov);
/* host rhs/sol (sol = x0 on entry) */
int xs_solve(xs_handle_t h, const double *rhs, double *sol);
/* device-resident rhs/sol (device pointers, n doubles each) */
int xs_solve_device(xs_handle_t h, const double *d_rhs, double *d_sol);
/* nrhs independent right-hand sides stored contiguously (column i at
 * rhs + i*n); host pointers; sol holds every column's x0 on entry.  New
 * entry point beside hip/xsolver_c.cpp:274-292 (xsolver_solve, one
 * right-hand side).  With PCG ("cg"/"cgm") and no, Jacobi or an ILU-family
 * preconditioner applied by exact triangular solves in FP64, 2..16 columns
 * iterate together (one pass over the matrix and one triangular-solve
 * dependency chain serve all of them; every column keeps its own scalars
 * and stops where its own solve would); otherwise the columns are solved
 * one after another.  usediter/resvec of the handle receive the last
 * system's values; xs_batch_iterations gives every column's count. */
int xs_solve_batch(xs_handle_t h, int nrhs, const double *rhs, double *sol);
/* iterations of each column of the last batched solve or adjoint (nrhs
 * must equal that call's nrhs) */
int xs_batch_iterations(xs_handle_t h, int nrhs, int *iters);
/* 1 (default): xs_solve_batch / xs_adjoint_batch iterate eligible columns
 * together; 0: always one after another.  Environment XS_BATCH. */
int xs_set_batch_kernels(int enable);
int xs_adjoint(xs_handle_t h, const double *dLdx, double *dLdb, double *dLdA_vals);
/* batch adjoint: nrhs forward solutions (host, contiguous) and gradients
 * (dLdb: nrhs*n, dLdA_vals: nrhs*nnz, each column after the other); the
 * transposed solves iterate together under the conditions of
 * xs_solve_batch. */
int xs_adjoint_batch(xs_handle_t h, int nrhs, const double *x, const double *dLdx, double *dLdb, double *dLdA_vals);
/* timing of the last solve, in milliseconds (CUDA events around the solve
 * on the handle's stream): setup = preconditioner construction */
int xs_last_timing(xs_handle_t h, double *setup_ms, double *solve_ms, int *iterations, double *final_relres);
/* the CUDA stream (cudaStream_t) all of the handle's work is ordered on */
int xs_get_stream(xs_handle_t h, void **stream);
/* kernels launched by the last solve (captured graph nodes replayed + direct
 * launches) */
int xs_last_launches(xs_handle_t h, long long *count);
/* number of refinement (outer) steps of the last mixed-precision solve */
int xs_last_outer_steps(xs_handle_t h, int *outer_steps);

/* ------------------------------------------------------------------ */
/* 2. reference cuda/ + intel/ Fortran-style API                       */
/* ------------------------------------------------------------------ */
/* intel/HostMatrix.h:187-195 (also cuda/HostMatrix.h): "diag + off-diagonal"
 * matrix; 0- or 1-based (offdiag_row_offset[0] selects); borrowed host
 * pointers, read by gpu_mat_setup / gpu_mat_update as in the reference.
 * nHalo must be 0 (one GPU).  nSizes, when > 0, is the number of
 * off-diagonal entries: row offsets that decrease or pass it are refused
 * (XS_ERR_INVALID) at gpu_mat_setup. */
void cpu_mat_setup(int *nInterior, int *nHalo, int *nSizes, double *diag_val, double *offdiag_val,
                   int *offdiag_row_offset, int *offdiag_col_index);
/* intel/HostMatrix.h:196-200: new values, same pattern */
void cpu_mat_update(double *diag_val, double *offdiag_val);
/* cuda/DeviceMatrix.h:121-126: upload the matrix set by cpu_mat_setup */
void gpu_mat_setup(void);
/* cuda/DeviceMatrix.h:127-144: "ELL"; num_nz in (0, 32] is rounded up to 16
 * or 32 as in the reference (the kernel itself uses the true max row length) */
void gpu_mat_format(char *fmt, int *num_nz);
/* cuda/DeviceMatrix.h:145-148: re-upload values after cpu_mat_update */
void gpu_mat_update(void);
/* cuda/DeviceMatrix.h:149-152 */
void gpu_mat_free(void);
/* cuda/DeviceMatrix.h:153-158: "Jacobi", plus "ILU0", "ParILU", "ParILUT" */
void gpu_preconditioner_setup(char *fmt);
/* cuda/DeviceMatrix.h:159-165 */
void gpu_preconditioner_update(char *fmt);
/* cuda/DeviceMatrix.h:166-168 */
void gpu_preconditioner_free(char *fmt);
/* cuda/mpicudasolver-C-v1.cu:165 / :380 / :588.  resvec[k] = ||r_k||/||r_0||
 * (relative, intel convention), *usediter = index of the last iteration. */
void gpu_cg_solve(double *rhs, double *sol, double *tol, int *maxiter, double *sol_init, int *usediter, double *resvec);
void gpu_cgm_solve(double *rhs, double *sol, double *tol, int *maxiter, double *sol_init, int *usediter, double *resvec);
void gpu_bicgstab_solve(double *rhs, double *sol, double *tol, int *maxiter, double *sol_init, int *usediter,
                        double *resvec);
/* The single-reduction CG variants of the reference's CPU path, on the GPU
 * with the configured preconditioner: intel/mpisolver-C-v1.cpp:104 (icg,
 * CG on M^-1 A with tao from a recurrence) and :273 (icgm, PCG with the five
 * dot products of an iteration taken together); same arguments and
 * conventions as gpu_cg_solve.  Handles select them with
 * xs_ksp_settype(h, "icg" / "icgm"). */
void gpu_icg_solve(double *rhs, double *sol, double *tol, int *maxiter, double *sol_init, int *usediter, double *resvec);
void gpu_icgm_solve(double *rhs, double *sol, double *tol, int *maxiter, double *sol_init, int *usediter, double *resvec);
/* intel/mpisolver-C-v1.cpp:484 (ibicgstab: right-preconditioned BiCGSTAB
 * with the six dot products of an iteration taken together); arguments as
 * gpu_cg_solve; handles: xs_ksp_settype(h, "ibicgstab"). */
void gpu_ibicgstab_solve(double *rhs, double *sol, double *tol, int *maxiter, double *sol_init, int *usediter,
                         double *resvec);
/* cuda/mpicudasolver-C-v1.cu:939 / :1074 / :1221 / :1391 */
void gpu_gcr_solve(double *rhs, double *sol, int *restart, double *tol, int *maxiter, double *sol_init, int *usediter,
                   double *resvec);
void gpu_igcr_solve(double *rhs, double *sol, int *restart, double *tol, int *maxiter, double *sol_init, int *usediter,
                    double *resvec);
void gpu_gmres_solve(double *rhs, double *sol, int *restart, double *tol, int *maxiter, double *sol_init,
                     int *usediter, double *resvec);
void gpu_fgmres_solve(double *rhs, double *sol, int *restart, double *tol, int *maxiter, double *sol_init,
                      int *usediter, double *resvec);

/* ------------------------------------------------------------------ */
/* 3c. kernel-level entry points on device pointers (tests/benchmarks) */
/* ------------------------------------------------------------------ */
/* A plan holds a device copy of a CSR matrix (and optionally its ELL form
 * and ILU factors) with the analysis the kernels need.  All d_* pointers are
 * device pointers; every call is ordered on the plan's stream and returns
 * after enqueueing unless stated. */
typedef struct xs_plan_s *xs_plan_t;
/* copy a host CSR (0-based) to the device and analyse it */
int xs_plan_create(xs_plan_t *p, int n, const int *rowptr, const int *colidx, const double *val);
int xs_plan_destroy(xs_plan_t p);
/* build the ELL form (width = max row length) */
int xs_plan_build_ell(xs_plan_t p, int *width);
/* y = A x (format 0 CSR, 1 ELL; precision 0 FP64, 1 FP32 values+vectors) */
int xs_plan_spmv(xs_plan_t p, int format, int precision, const void *d_x, void *d_y);
/* y = A^T x (FP64, CSR of A^T built on first use) */
int xs_plan_spmv_t(xs_plan_t p, const double *d_x, double *d_y);
/* ILU factorisation on the device: kind 0 exact ILU(0) (sync-free, same
 * operation order as the reference CPU ILU(0)), 1 ParILU (sweeps),
 * 2 ParILUT (fill, sweeps, droptol); on the host, applied on the device:
 * 4 Saad ILUT (fill = lfil >= 1, droptol), 5 ICT (fill = kept entries per
 * row, droptol > 0) */
int xs_plan_factor(xs_plan_t p, int kind, int sweeps, double fill, double droptol);
/* copy the factors to the host in the seqilu0 layout (L strict lower, dinv,
 * U' = dinv-row-scaled strict upper).  Pass NULL arrays to query nnzL/nnzU. */
/* Host threshold factorizations without a device (no handle): Saad ILUT
 * (hip/Precond/ilut_diag_in_csr.cpp:20-251 split as hip/HostMatrix/
 * HostMatrixCSR.cpp:230-268) and ICT (hip/Precond/ict_l.cpp:112-212
 * converted as hip/HostMatrix/HostMatrixCSR.cpp:327-384) of a sorted
 * 0-based CSR matrix, in the layout of xs_plan_get_factors.  lci/lv and
 * uci/uv hold at least n*lfil (ILUT) or n*min(maxfil, n-1) (ICT) entries;
 * lrp/urp n+1, dinv n.  ICT: XS_ERR_NO_DIAG for a row without a diagonal. */
int xs_host_ilut(int n, const int *rp, const int *ci, const double *v, int lfil, double droptol, int *nnzL, int *nnzU,
                 int *lrp, int *lci, double *lv, double *dinv, int *urp, int *uci, double *uv);
int xs_host_ict(int n, const int *rp, const int *ci, const double *v, int maxfil, double droptol, int *nnzL, int *nnzU,
                int *lrp, int *lci, double *lv, double *dinv, int *urp, int *uci, double *uv);
int xs_plan_get_factors(xs_plan_t p, int *nnzL, int *nnzU, int *lrp, int *lci, double *lv, double *dinv, int *urp,
                        int *uci, double *uv);
/* combined LU values over A's pattern (exact ILU(0) / ParILU only) */
int xs_plan_get_lu_values(xs_plan_t p, double *luv);
/* factor storage precision for the solves below: 0 FP64, 1 FP32, 2 BF16, 3 FP16 */
int xs_plan_set_factor_precision(xs_plan_t p, int prec);
/* triangular solve mode of the plan's LU solves: 0 exact sync-free, k > 0
 * k Jacobi sweeps per triangle */
int xs_plan_set_trsv(xs_plan_t p, int mode);
/* z = (L D U')^{-1} x with sync-free solves (vec_prec 0 FP64 / 1 FP32) */
int xs_plan_lusolve(xs_plan_t p, int vec_prec, const void *d_x, void *d_z);
/* k (1..16) LU solves at once on device vectors stored interleaved by row
 * (entry (i, c) at i*k + c), FP64, exact triangular solves: each column's
 * result is bitwise the one xs_plan_lusolve gives for that column alone.
 * No counterpart in the reference; the batched solves of xs_solve_batch use
 * it.  XS_ERR_UNSUPPORTED for Jacobi-sweep mode. */
int xs_plan_lusolve_batch(xs_plan_t p, int k, const double *x, double *z);
/* z = (L D U')^{-T} x */
int xs_plan_lusolve_t(xs_plan_t p, const double *d_x, double *d_z);
/* wait for the plan's stream; returns the device status word (e.g. a
 * sync-free timeout) */
int xs_plan_sync(xs_plan_t p);
/* the CUDA stream (cudaStream_t) the plan's work is ordered on: a caller
 * that orders its own work on it (or waits on it with events) needs no
 * xs_plan_sync between calls.  The plan owns the stream: it stays valid
 * until xs_plan_destroy, which synchronises and destroys it, so nothing may
 * be recorded on it (events, allocator stream uses) after that call. */
int xs_plan_get_stream(xs_plan_t p, void **stream);
/* Testing hook for the bounded waits: with enable != 0, the first dependency
 * of the L-solve row at `position` is redirected to the row itself, a value
 * that no thread ever publishes, so the next L solve waits out its limit
 * (about a second) and reports XS_ERR_TRSV_TIMEOUT through xs_plan_sync;
 * enable = 0 restores the dependency. */
int xs_plan_debug_break_dependency(xs_plan_t p, int position, int enable);
/* number of dependency levels of L and U */
int xs_plan_levels(xs_plan_t p, int *levelsL, int *levelsU);
/* average device time in ms of `reps` repetitions of op (0 CSR SpMV FP64,
 * 1 ELL SpMV FP64, 2 CSR SpMV FP32, 3 L solve, 4 U solve, 5 LU solve,
 * 6 ELL SpMV FP32) on internal buffers, timed with CUDA events on the plan's
 * stream; flushes L2 between repetitions when flush_l2 != 0 */
int xs_plan_time_op(xs_plan_t p, int op, int reps, int flush_l2, double *ms);
/* algorithmic bytes of op (counted once per array element) */
int xs_plan_op_bytes(xs_plan_t p, int op, double *bytes);

/* Matrix Market coordinate files (host only, no GPU needed), replacing the
 * reference's reader hip/Tool/ReadMatrix/csr_mmio_highlevel.h:8-233
 * (mmio_info / mmio_data).  xs_mm_info gives the sizes, with nnz counted
 * after the symmetric expansion; xs_mm_read fills rowptr[m+1],
 * colidx[nnz], val[nnz] and, if diag is not NULL, diag[m] (the value of
 * entry (i, i) as written).  With reference_quirks != 0 the result is the
 * reference reader's: general files store -value; symmetric / hermitian
 * files store value at (i, j) and (j, i); columns within a row keep the
 * file's order.  reference_quirks = 0 keeps general files' values as
 * written.  Real, double and integer fields; complex, pattern and
 * skew-symmetric files give XS_ERR_UNSUPPORTED; malformed files, symmetric
 * files that are not square and entry counts the file cannot hold give
 * XS_ERR_INVALID. */
int xs_mm_info(const char *path, int *m, int *n, int *nnz, int *symmetric);
int xs_mm_read(const char *path, int reference_quirks, int *rowptr, int *colidx, double *val, double *diag);

/* Host-only dependency analysis of a strictly triangular CSR pattern (no
 * GPU needed): level[i] = 1 + max level of the rows row i depends on, perm =
 * rows sorted by (level, row) — the position order of the sync-free solve. */
int xs_tri_levels(int n, const int *rowptr, const int *colidx, int upper, int *level, int *perm, int *nlevels);

/* Host-only box analysis of a strictly triangular CSR pattern (no GPU
 * needed; no counterpart in the reference: it is the schedule the exact
 * triangular solves use in place of hip/Precond/gpuparilu.cpp:257-364's
 * row-per-thread flags on grid-shaped patterns).  Finds a grid nx*ny*nz = n
 * on which every dependency lies within 2 steps per direction, the smallest
 * shear (x' = x + a*y + b*z, y' = y + c*z) that makes every dependency point
 * to smaller or equal sheared coordinates, and cuts the sheared grid into
 * boxes of tx*ty*tz.  info[12] = {fits, nx, ny, nz, a, b, c, boxes, internal
 * levels, halo entries, largest box, largest halo}; when fits is 0 nothing
 * else is written.  Optional outputs (NULL to skip): perm[n] (position ->
 * row: boxes in wavefront order, then internal level, then row order),
 * prp[n+1], pci[nnz] (each dependency as a shared-memory slot: [0, rows of
 * the box) the box's own positions, then its halo), tile_pos[boxes+1],
 * tile_lvl[boxes+1], lvl_ptr[levels+1], halo_ptr[boxes+1],
 * halo_row[halo entries]. */
int xs_tri_tiles(int n, const int *rowptr, const int *colidx, int upper, int tx, int ty, int tz, int *info, int *perm,
                 int *prp, int *pci, int *tile_pos, int *tile_lvl, int *lvl_ptr, int *halo_ptr, int *halo_row);

/* LU solve that allocates nothing (no counterpart in the reference).
 * z = (L D U')^{-1} x with the factors in the seqilu0 layout (L strict lower
 * CSR with unit diagonal implied, dinv = 1/u_ii, U' = dinv-row-scaled strict
 * upper CSR; natural row order, columns sorted), all device pointers, FP64,
 * enqueued on `stream` (a cudaStream_t, NULL = default stream).  Every call
 * waits for `stream` (cudaStreamSynchronize) before it returns and reads the
 * kernels' error word back to the host: XS_ERR_TRSV_TIMEOUT when a row's
 * dependency was not ready within 1 s.  For callers that cannot allocate
 * device memory (a pool or allocator that owns all of it, a fixed memory
 * budget after start-up, buffers handed in by the caller only): the scratch
 * lives in a fixed 4 MiB __device__ array that every GPU loading the library
 * holds until exit.  n must be <= 262144 (XS_ERR_CAPACITY otherwise); when
 * n > 0 every pointer must be non-NULL, also the column and value arrays of
 * a factor without entries (XS_ERR_INVALID otherwise).  Calls that overlap
 * on the GPU share that array and race: serialise them.  The first call on a
 * device looks up the array's address and keeps it; make it before any
 * stream capture, and do not let calls span a cudaDeviceReset of that
 * device.  Result bitwise equal to xs_plan_lusolve on the same factors. */
int xs_lusolve_noalloc(int n, const int *lrp, const int *lci, const double *lv, const double *dinv, const int *urp,
                       const int *uci, const double *uv, const double *x, double *z, void *stream);

/* Launch tuning of the sync-free triangular solves, process-wide.
 * chunk_rows > 0 selects the chunked kernel: contiguous row
 * chunks of that size, one block per chunk, dependencies inside a chunk
 * through shared memory (<= 24576 so the FP64 chunk fits in 192 KiB);
 * 0 (default) selects the level-ordered kernel with blocks_per_sm persistent blocks
 * per SM (0 = one block per 128 rows).  backoff_ns caps the exponential
 * back-off between polls of a pending row (>= 8: the sleep is also the
 * yield point a waiting lane needs so that a producer lane of its own warp
 * runs).  Defaults 2 / 128 / 0; environment XS_TRSV_BLOCKS_PER_SM,
 * XS_TRSV_BACKOFF_NS, XS_TRSV_CHUNK_ROWS override them at first use.  The
 * layout is fixed when a preconditioner is built: set before factorising. */
int xs_set_trsv_tuning(int blocks_per_sm, int backoff_ns, int chunk_rows);
/* Vector updates of the Krylov iterations fused into the preconditioner
 * pass that first reads their result (BiCGSTAB's p = omega (p - alpha u) + r
 * and s = r - gamma u formed in the first L pass of the Jacobi-sweep apply
 * that reads them, when L has an ELL copy): 1 (default) fuses, 0 runs them
 * as separate kernels.  Same results either way.  Environment XS_VEC_FUSE
 * sets it at first use. */
int xs_set_vector_fusion(int enable);
/* BiCGSTAB with an ILU-family preconditioner applied by Jacobi sweeps, the
 * operator and both triangles in diagonal-slot ELL storage: 1 runs each
 * solve's iterations as one persistent cooperative kernel (the
 * phases of an iteration separated by grid barriers, the loop on the
 * device) instead of replaying a CUDA graph of ~11 kernels per iteration;
 * 0 (default) replays the graph.  The arithmetic per element is the same; the dot
 * products' block partials follow the persistent grid, so results agree to
 * rounding.  Needs vector fusion on.  Environment XS_PERSIST. */
int xs_set_persistent_iteration(int enable);
/* Box-scheduled exact triangular solves (see xs_tri_tiles): enable = 1
 * (default) uses them for triangles of at least min_rows rows (default
 * 65536, at least 8) whose pattern fits a grid, with boxes of tx*ty*tz
 * sheared grid steps (default 16*16*8, halved along the longest side until
 * a box's staged data fits in shared memory; triangles averaging at least 20
 * entries per row, such as ParILUT fill of 27-point operators, start from
 * 8*4*2 instead unless a box size was set here or by XS_TRSV_TILES, since a
 * box size set either way applies to every triangle); 0 keeps the level-ordered
 * solve (the other arguments are then ignored).  Results are bitwise
 * identical either way.  Environment XS_TRSV_TILES ("0" or "tx,ty,tz") and
 * XS_TRSV_TILE_MIN_ROWS set it at first use.  Fixed when a preconditioner is
 * built: set before factorising. */
int xs_set_trsv_tiles(int enable, int tx, int ty, int tz, int min_rows);
/* Exact LU solves of systems with at most max_rows rows, whose solution
 * vector fits in one SM's shared memory (FP64: 25600 rows), run in one CTA
 * that walks the dependency levels with a block barrier between them
 * (bitwise the same result as the sync-free solve, without its cross-SM
 * hand-off per level).  0 disables it; default: no row limit beyond the
 * shared-memory one.  Environment XS_TRSV_BLOCK_ROWS sets it at first use. */
int xs_set_trsv_block_rows(int max_rows);
/* Single-CTA LU solve form: 1 (default) copies whole dependency levels, in
 * batches of up to 512 rows and 2048 entries, into shared memory with
 * asynchronous copies one batch ahead, so a level reads shared memory only;
 * 0 loads each row's data from global memory one level ahead.  Same result
 * either way.  Environment XS_LU_STAGED sets it at first use. */
int xs_set_trsv_block_staging(int enable);
/* Exact ILU(0) factorisation: 1 on the box schedule of the L solve when L
 * has boxes (entries staged in shared memory, one halo wait per box,
 * barriers between the box's levels), 0 (default; faster as measured) the
 * level-ordered lane groups.  Same factors either way.  Environment
 * XS_ILU_TILES sets it at first use. */
int xs_set_ilu_tiles(int enable);
/* Jacobi-sweep preconditioner apply: 1 computes sweeps 2 and 3 of each
 * narrow diagonal-slot triangle in one pass (each row recomputes the
 * second-sweep values of its neighbours; same result, about half the DRAM
 * traffic, more L2 traffic), 0 (default) runs them as separate passes.
 * Environment XS_SWEEP_FUSE sets it at first use. */
int xs_set_sweep_fusion(int enable);
/* Programmatic dependent launch for the kernels of the Krylov iterations
 * (SpMV, vector updates, Jacobi sweeps): 1 (default) lets a kernel start
 * while its predecessor drains (each waits on the hardware dependency before
 * touching the predecessor's results), 0 serialises them fully.  Results are
 * identical either way.  Environment XS_PDL sets it at first use; graphs
 * captured earlier keep the mode they were captured with. */
int xs_set_launch_overlap(int enable);
/* Column storage of ELL copies (the ELL SpMV and the Jacobi-sweep triangle
 * copies).  index_bits 0 (default): diagonal slots when every entry lies on
 * one of at most 32 diagonals with at most 25% padding (stencil matrices):
 * no index per entry, one presence mask per row; otherwise as 16.
 * 16: each column as a 16-bit offset from its row whenever every
 * |col - row| <= 32767, else as 32.  32: 32-bit columns.  Environment
 * XS_ELL_DIAGONAL=0 / XS_ELL_INDEX16=0 turn the first two off at first use.
 * Applies to copies built later. */
int xs_set_ell_index_bits(int index_bits);

/* library identification */
const char *xs_version(void);
int xs_device_count(void);

#ifdef __cplusplus
} /* extern "C" */
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus

/* C++ forwarders with the reference's exact signatures */
inline void xsolver_ksp_setoption(double tol, int maxiter, int &usediter, double *resvec, int restart = 0)
{
    xsolver_ksp_setoption(tol, maxiter, &usediter, resvec, restart);
}
#endif

#endif /* XSOLVER_B200_C_H */
