"""Matrix Market reader (xs_mm_info / xs_mm_read) against the restated
reference reader and the reference's own compiled reader
(hip/Tool/ReadMatrix/csr_mmio_highlevel.h), on files written here."""
import numpy as np
import pytest

import oracle
from xsolver_b200 import stencils as st
from xsolver_b200.mtx import read_mtx


def _write(path, text):
    path.write_text(text)
    return str(path)


def _stencil_file(path, A, symmetric=False, seed=0):
    """A as a coordinate file, entries in a shuffled order (lower triangle
    only for a symmetric file)."""
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    keep = rows >= A.colidx if symmetric else np.ones(A.nnz, bool)
    idx = np.flatnonzero(keep)
    np.random.default_rng(seed).shuffle(idx)
    kind = "symmetric" if symmetric else "general"
    lines = [f"%%MatrixMarket matrix coordinate real {kind}", "% written by the test", f"{A.n} {A.n} {len(idx)}"]
    lines += [f"{rows[k] + 1} {A.colidx[k] + 1} {float(A.val[k])!r}" for k in idx]
    return _write(path, "\n".join(lines) + "\n")


def _cases(tmp_path):
    yield _write(tmp_path / "g.mtx", "%%MatrixMarket matrix coordinate real general\n% c\n\n3 3 5\n"
                 "1 1 4.0\n3 1 -1.5\n2 2 5e0\n1 3 2\n3 3 6.25\n")
    yield _write(tmp_path / "s.mtx", "%%MatrixMarket matrix coordinate real symmetric\n4 4 6\n"
                 "1 1 4\n2 1 -1\n2 2 4\n3 2 -1\n3 3 4\n4 4 1e-3\n")
    yield _write(tmp_path / "i.mtx", "%%MatrixMarket matrix coordinate integer general\r\n2 2 3\r\n1 1 7\r\n"
                 "2 1 -2\r\n2 2 9\r\n")
    yield _write(tmp_path / "h.mtx", "%%MatrixMarket matrix coordinate real hermitian\n3 3 4\n"
                 "1 1 2.5\n3 1 0.125\n2 2 1\n3 3 3\n")
    yield _stencil_file(tmp_path / "p.mtx", st.poisson2d_5pt(12))
    yield _stencil_file(tmp_path / "ps.mtx", st.varcoef3d_7pt(5, 2), symmetric=True, seed=1)
    yield _stencil_file(tmp_path / "c.mtx", st.convdiff3d_27pt(4, pe=5.0), seed=2)


def test_reader_equals_restated_reference(tmp_path):
    for path in _cases(tmp_path):
        A, d, sym = read_mtx(path)
        m, n, rp, ci, v, do, so = oracle.read_mtx(path)
        assert (A.n, bool(so)) == (m, sym), path
        assert np.array_equal(A.rowptr, rp) and np.array_equal(A.colidx, ci), path
        assert np.array_equal(A.val, v) and np.array_equal(d, do), path


@pytest.mark.skipif(oracle.ref_mmio() is None, reason="compiled reference reader not present")
def test_restated_reader_equals_compiled_reference(tmp_path):
    for path in _cases(tmp_path):
        a, b = oracle.read_mtx(path), oracle.ref_read_mtx(path)
        for x, y in zip(a, b):
            assert np.array_equal(x, y) if isinstance(x, np.ndarray) else x == y, path


def test_general_values_negated_unless_quirks_off(tmp_path):
    A = st.poisson2d_5pt(9)
    path = _stencil_file(tmp_path / "q.mtx", A, seed=3)
    Aq, _, _ = read_mtx(path)
    Ap, _, _ = read_mtx(path, reference_quirks=False)
    assert np.array_equal(Aq.val, -Ap.val)
    assert abs(Ap.to_scipy() - A.to_scipy()).max() == 0.0  # same matrix, file column order


@pytest.mark.parametrize("text,code", [
    ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n", 10),
    ("%%MatrixMarket matrix coordinate pattern general\n1 1 1\n1 1\n", 10),
    ("%%MatrixMarket matrix coordinate real skew-symmetric\n2 2 1\n2 1 1\n", 10),
    ("%%MatrixMarket matrix array real general\n1 1\n1\n", 1),
    ("1 1 1\n1 1 1\n", 1),
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n3 1 1\n", 1),
    ("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n2 2 1\n", 1),
    ("%%MatrixMarket matrix coordinate real symmetric\n2 3 2\n1 1 1\n3 2 1\n", 1),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1000000000000\n1 1 1\n", 1),
])
def test_reader_refuses_bad_files(tmp_path, text, code):
    from xsolver_b200._lib import XsError

    path = _write(tmp_path / "bad.mtx", text)
    with pytest.raises(XsError) as e:
        read_mtx(path)
    assert e.value.code == code


def test_missing_file(tmp_path):
    from xsolver_b200._lib import XsError

    with pytest.raises(XsError) as e:
        read_mtx(str(tmp_path / "none.mtx"))
    assert e.value.code == 1


@pytest.mark.gpu
def test_reference_driver_flow_on_a_file(cuda, tmp_path):
    """hip/main_solve_base.cpp's flow on a written file: the reader's
    (negated) matrix, b = 1, x0 = 0, BiCGSTAB + ILUT, rtol 1e-4."""
    from xsolver_b200.mtx import solve_mtx

    path = _stencil_file(tmp_path / "d.mtx", st.convdiff3d_27pt(12, pe=5.0), seed=4)
    x, S = solve_mtx(path)
    A, _, _ = read_mtx(path)
    r = np.ones(A.n) - A.to_scipy() @ x
    assert np.linalg.norm(r) / np.sqrt(A.n) < 1e-4 * 1.01
    assert S.usediter < 300
