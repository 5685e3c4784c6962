"""include/xsolver_c.h as a reference caller uses it: a C program and a C++
program (the reference's C++ setter signature, int &usediter) compile
against the header with warnings as errors, link against the in-tree
libxsolver_b200.so and run.  Without a GPU the compute entry points report
XS_ERR_NO_GPU; the host-only Matrix Market reader works either way."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "xsolver_b200")

C_SRC = r"""
#include <stdio.h>
#include "xsolver_c.h"
int main(int argc, char **argv)
{
    xs_handle_t h = NULL;
    int rc = xs_create(&h);
    int m = 0, n = 0, nnz = 0, sym = 0;
    int rm = xs_mm_info(argv[1], &m, &n, &nnz, &sym);
    int rp[4], ci[8];
    double v[8], d[3];
    int rr = xs_mm_read(argv[1], 1, rp, ci, v, d);
    printf("%d %d %d %d %d %d %d %g %g %s\n", rc, rm, m, n, nnz, sym, rr, v[0], d[2],
           xsolver_error_string(XS_ERR_NO_GPU));
    if (h) xs_destroy(h);
    (void)argc;
    return 0;
}
"""

CXX_SRC = r"""
#include <cstdio>
#include "xsolver_c.h"
int main()
{
    int rowptr[3] = {0, 1, 2}, colidx[2] = {0, 1}, pam[3] = {0, 0, 1};
    double val[2] = {2.0, 4.0}, rhs[2] = {1.0, 1.0}, sol[2] = {0.0, 0.0}, resvec[11];
    int usediter = -1;
    xsolver_mat_setup(2, rowptr, colidx, val, pam);
    int e_setup = xsolver_last_error();
    xsolver_ksp_settype((char *)"bicgstab");
    xsolver_ksp_setoption(1e-10, 10, usediter, resvec);  // the reference's int & signature
    xsolver_pc_settype((char *)"jacobi");
    xsolver_solve(rhs, sol);
    int e_solve = xsolver_last_error();
    xsolver_free();
    std::printf("%d %d %.17g %.17g\n", e_setup, e_solve, sol[0], sol[1]);
    return 0;
}
"""

MTX = "%%MatrixMarket matrix coordinate real symmetric\n3 3 4\n1 1 4\n2 1 -1\n2 2 4\n3 3 2.5\n"


def _build(compiler, std, src, out, tmp_path):
    path = tmp_path / ("prog.c" if compiler == "gcc" else "prog.cpp")
    path.write_text(src)
    cmd = [compiler, f"-std={std}", "-Wall", "-Wextra", "-Werror", f"-I{INC}", str(path), "-o", str(out),
           f"-L{LIBDIR}", "-lxsolver_b200", f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


@pytest.mark.skipif(shutil.which("gcc") is None or shutil.which("g++") is None, reason="no host compiler")
def test_header_from_c_and_cxx(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libxsolver_b200.so")):
        pytest.skip("library not built")
    mtx = tmp_path / "a.mtx"
    mtx.write_text(MTX)
    _build("gcc", "c99", C_SRC, tmp_path / "c_prog", tmp_path)
    out = subprocess.run([str(tmp_path / "c_prog"), str(mtx)], check=True, capture_output=True, text=True).stdout.split()
    rc, rm, m, n, nnz, sym, rr = (int(t) for t in out[:7])
    assert rc in (0, 12)  # XS_OK with a GPU, XS_ERR_NO_GPU without
    assert (rm, m, n, nnz, sym, rr) == (0, 3, 3, 5, 1, 0)  # symmetric file: one off-diagonal mirrored
    assert float(out[7]) == 4.0 and float(out[8]) == 2.5
    assert " ".join(out[9:]) == "no CUDA device"

    _build("g++", "c++17", CXX_SRC, tmp_path / "cxx_prog", tmp_path)
    out = subprocess.run([str(tmp_path / "cxx_prog")], check=True, capture_output=True, text=True).stdout.split()
    e_setup, e_solve = int(out[0]), int(out[1])
    if e_setup == 12:  # no GPU: every entry point reports it, the solution is untouched
        assert e_solve == 12 and float(out[2]) == 0.0
    else:  # a GPU: diag(2, 4) x = 1
        assert (e_setup, e_solve) == (0, 0)
        assert abs(float(out[2]) - 0.5) < 1e-12 and abs(float(out[3]) - 0.25) < 1e-12
