/* C entry points over the reference's Matrix Market reader
 * (hip/Tool/ReadMatrix/csr_mmio_highlevel.h:8-233, mmio_info / mmio_data),
 * which oracle/Makefile compiles from the reference header into oracle/_ref.
 * Test oracle only. */
#include "csr_mmio_highlevel.h"
extern "C" int ref_mmio_info(int *m, int *n, int *nnz, int *sym, char *path)
{
    return mmio_info(m, n, nnz, sym, path);
}
extern "C" int ref_mmio_data(int *rowptr, int *colidx, double *val, double *diag, char *path)
{
    return mmio_data(rowptr, colidx, val, diag, path, 0.0);
}
