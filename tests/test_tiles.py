"""Box schedule of the exact triangular solves (host analysis, no GPU).

The box-scheduled solve replaces row-per-thread dependency flags
(hip/Precond/gpuparilu.cpp:257-364) on grid-shaped patterns.  Its
correctness rests on the host analysis alone: every dependency of a row must
be either a row of the same box at a smaller internal level (a shared-memory
slot written before the barrier that ends that level) or a halo value from a
box earlier in the ticket order (so no CTA waits on a box that is not yet
taken), and each row's dependency slots must name exactly the row's
entries, in the accumulation order of the CPU reference's LUsolve
(L: increasing column; U: decreasing column).  These tests rebuild every
dependency from the layout and compare."""
import ctypes as C

import numpy as np
import pytest

from xsolver_b200 import stencils as st

_ip = C.POINTER(C.c_int)


def _lib():
    from xsolver_b200 import _lib

    return _lib.lib()


def _tri(A, upper):
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    keep = A.colidx > rows if upper else A.colidx < rows
    rp = np.zeros(A.n + 1, np.int32)
    np.cumsum(np.bincount(rows[keep], minlength=A.n), out=rp[1:])
    return rp, np.ascontiguousarray(A.colidx[keep].astype(np.int32))


def tiles(n, rp, ci, upper, t=(16, 16, 16)):
    L = _lib()
    info = np.zeros(12, np.int32)
    p = lambda a: a.ctypes.data_as(_ip)  # noqa: E731
    assert L.xs_tri_tiles(n, p(rp), p(ci), int(upper), *t, p(info), *([None] * 8)) == 0
    if not info[0]:
        return None
    nt, nl, nh = int(info[7]), int(info[8]), int(info[9])
    out = dict(perm=np.zeros(n, np.int32), prp=np.zeros(n + 1, np.int32), pci=np.zeros(max(len(ci), 1), np.int32),
               tile_pos=np.zeros(nt + 1, np.int32), tile_lvl=np.zeros(nt + 1, np.int32),
               lvl_ptr=np.zeros(nl + 1, np.int32), halo_ptr=np.zeros(nt + 1, np.int32),
               halo_row=np.zeros(max(nh, 1), np.int32))
    assert L.xs_tri_tiles(n, p(rp), p(ci), int(upper), *t, p(info), *(p(out[k]) for k in
                          ("perm", "prp", "pci", "tile_pos", "tile_lvl", "lvl_ptr", "halo_ptr", "halo_row"))) == 0
    out["info"] = info.copy()
    return out


def check_schedule(n, rp, ci, upper, T):
    perm, prp, pci = T["perm"], T["prp"], T["pci"]
    assert np.array_equal(np.sort(perm), np.arange(n))
    pos_of = np.empty(n, np.int64)
    pos_of[perm] = np.arange(n)
    nt = len(T["tile_pos"]) - 1
    # internal level of every position
    lev_of = np.empty(n, np.int64)
    for t in range(nt):
        for l in range(T["tile_lvl"][t], T["tile_lvl"][t + 1]):
            lev_of[T["lvl_ptr"][l]:T["lvl_ptr"][l + 1]] = l
    assert T["lvl_ptr"][T["tile_lvl"][nt]] == n
    max_rows = max_halo = 0
    for t in range(nt):
        p0, p1 = T["tile_pos"][t], T["tile_pos"][t + 1]
        h0, h1 = T["halo_ptr"][t], T["halo_ptr"][t + 1]
        rows, halo = p1 - p0, T["halo_row"][h0:h1]
        max_rows, max_halo = max(max_rows, rows), max(max_halo, h1 - h0)
        assert np.all(pos_of[halo] < p0), "halo from a later box"
        for p in range(p0, p1):
            r = perm[p]
            deps = ci[rp[r]:rp[r + 1]]
            if upper:
                deps = deps[::-1]
            slots = pci[prp[p]:prp[p + 1]]
            assert len(slots) == len(deps)
            for s, d in zip(slots, deps):
                if s < rows:
                    assert perm[p0 + s] == d
                    assert lev_of[p0 + s] < lev_of[p], "same-box dependency not at a lower level"
                else:
                    assert s - rows < h1 - h0 and halo[s - rows] == d
    assert max_rows == T["info"][10] and max_halo == T["info"][11]


@pytest.mark.parametrize("upper", [False, True])
def test_7pt_grid_found_without_shear(upper):
    A = st.poisson3d_7pt(20)
    rp, ci = _tri(A, upper)
    T = tiles(A.n, rp, ci, upper, (8, 8, 8))
    assert T is not None
    assert list(T["info"][1:7]) == [20, 20, 20, 0, 0, 0]
    assert T["info"][7] == 27  # 3 x 3 x 3 boxes
    check_schedule(A.n, rp, ci, upper, T)


@pytest.mark.parametrize("upper", [False, True])
def test_27pt_grid_needs_a_shear(upper):
    A = st.convdiff3d_27pt(12)
    rp, ci = _tri(A, upper)
    T = tiles(A.n, rp, ci, upper, (8, 8, 8))
    assert T is not None
    nx, ny, nz, a, b, c = T["info"][1:7]
    assert (nx, ny, nz) == (12, 12, 12)
    assert (a, b, c) == (1, 2, 1)
    check_schedule(A.n, rp, ci, upper, T)


def test_2d_grid():
    A = st.poisson2d_5pt(40)
    rp, ci = _tri(A, False)
    T = tiles(A.n, rp, ci, False, (8, 8, 8))
    assert T is not None and list(T["info"][1:4]) == [40, 40, 1]
    check_schedule(A.n, rp, ci, False, T)


@pytest.mark.parametrize("upper", [False, True])
def test_parilut_fill_reach_two(upper):
    """ParILUT factors of the 27-point operator carry fill several grid
    steps away (up to 5 along x after 5 sweeps); the grid and a shear are
    still found."""
    import oracle

    A = st.convdiff3d_27pt(20)
    F = oracle.parilut(A, fill=2.0, sweeps=5, droptol=1e-4)
    rp, ci = (F.urp, F.uci) if upper else (F.lrp, F.lci)
    rp, ci = np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32)
    T = tiles(A.n, rp, ci, upper, (8, 8, 8))
    assert T is not None and list(T["info"][1:4]) == [20, 20, 20]
    check_schedule(A.n, rp, ci, upper, T)


def test_unstructured_pattern_is_refused():
    rng = np.random.default_rng(0)
    n = 5000
    rows, cols = [], []
    for i in range(1, n):
        for j in rng.choice(i, min(i, 4), replace=False):
            rows.append(i)
            cols.append(j)
    order = np.lexsort((cols, rows))
    rows, cols = np.array(rows)[order], np.array(cols)[order].astype(np.int32)
    rp = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(rows, minlength=n), out=rp[1:])
    assert tiles(n, rp, np.ascontiguousarray(cols), False) is None


def test_wrapping_neighbour_is_refused_or_scheduled_safely():
    """A 7-point pattern plus one coupling across the grid's x boundary
    (row (0, y, z) to row (nx-1, y-1, z)): whatever grid is chosen, every
    dependency must still respect the box order."""
    A = st.poisson3d_7pt(12)
    rp, ci = _tri(A, False)
    rows = np.repeat(np.arange(A.n), np.diff(rp))
    extra_r = np.array([12 * 5])
    extra_c = extra_r - 1
    r2 = np.concatenate([rows, extra_r])
    c2 = np.concatenate([ci, extra_c])
    o = np.lexsort((c2, r2))
    r2, c2 = r2[o], c2[o]
    c2 = np.unique(np.stack([r2, c2]), axis=1)
    r2, c2 = c2[0], c2[1].astype(np.int32)
    rp2 = np.zeros(A.n + 1, np.int32)
    np.cumsum(np.bincount(r2, minlength=A.n), out=rp2[1:])
    T = tiles(A.n, rp2, np.ascontiguousarray(c2), False, (4, 4, 4))
    if T is not None:
        check_schedule(A.n, rp2, np.ascontiguousarray(c2), False, T)


def device_rule_slots(n, rp, ci, upper, T):
    """The slots the device pass (`k_tile_entries`) writes, restated in
    numpy from the per-row data alone: each row's box and position and each
    box's sorted halo list.  A dependency d of the row at position p in box
    t gets its position minus the box's first when d lies in box t, else the
    box's row count plus the index of d in the box's halo list; entries in
    the accumulation order (L: increasing column, U: decreasing)."""
    perm, prp = T["perm"].astype(np.int64), T["prp"].astype(np.int64)
    tile_pos, halo_ptr, halo_row = T["tile_pos"].astype(np.int64), T["halo_ptr"].astype(np.int64), T["halo_row"]
    nt = len(tile_pos) - 1
    pos_of = np.empty(n, np.int64)
    pos_of[perm] = np.arange(n)
    box_of_pos = np.repeat(np.arange(nt), np.diff(tile_pos))
    box_of_row = np.empty(n, np.int64)
    box_of_row[perm] = box_of_pos
    m = int(prp[-1])
    p = np.repeat(np.arange(n), np.diff(prp))  # position of each staged entry
    j = np.arange(m) - prp[p]  # its index within the row
    r = perm[p]
    e = (rp[r + 1] - 1 - j) if upper else (rp[r] + j)
    d = ci[e].astype(np.int64)
    t = box_of_row[r]
    p0 = tile_pos[t]
    rows = tile_pos[t + 1] - p0
    nh = int(halo_ptr[-1])
    halo_box = np.repeat(np.arange(nt), np.diff(halo_ptr))
    keys = halo_box * n + halo_row[:nh].astype(np.int64)  # sorted: boxes in order, each list sorted
    same = box_of_row[d] == t
    slot = np.where(same, pos_of[d] - p0, rows + np.searchsorted(keys, t * n + d) - halo_ptr[t])
    return slot


@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("case", ["7pt", "27pt", "parilut"])
def test_device_entry_rule_matches_host_layout(case, upper):
    """The solve's per-entry slots are written on the device from per-row
    data (the host layout keeps only each row's box and position and the
    halo lists); that rule reproduces, entry for entry, the slots the host
    layout writes itself, and every halo lookup finds its row."""
    if case == "parilut":
        import oracle

        A = st.convdiff3d_27pt(16)
        F = oracle.parilut(A, fill=2.0, sweeps=5, droptol=1e-4)
        rp, ci = (F.urp, F.uci) if upper else (F.lrp, F.lci)
        rp, ci = np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32)
        n, box = A.n, (8, 4, 2)
    else:
        A = st.poisson3d_7pt(24) if case == "7pt" else st.convdiff3d_27pt(14)
        rp, ci = _tri(A, upper)
        n, box = A.n, (8, 8, 4)
    T = tiles(n, rp, ci, upper, box)
    assert T is not None
    slot = device_rule_slots(n, rp.astype(np.int64), ci, upper, T)
    assert np.array_equal(slot, T["pci"][:len(slot)].astype(np.int64))
    # per entry: its box's row count and halo length; halo slots stay inside the list
    nt = len(T["tile_pos"]) - 1
    box_of_pos = np.repeat(np.arange(nt), np.diff(T["tile_pos"]))
    box = box_of_pos[np.repeat(np.arange(n), np.diff(T["prp"]))]
    rows, nh = np.diff(T["tile_pos"])[box], np.diff(T["halo_ptr"])[box]
    assert np.all(slot < rows + nh)
