"""Grid-stencil detection (gpu_index_compress = 3) on host CSR arrays: which
matrices may be stored without column indices, with which line and plane
strides and in which row order. Runs on the CPU (XAMG_b200_stencil_layout
touches no GPU)."""
import numpy as np
import pytest

BOX27, STAR7 = 0, 1


def grid_matrix(nx, ny, nz, offsets):
    """Rows of an nx*ny*nz grid with the (dz, dy, dx) offsets that stay
    inside the grid, sorted by column."""
    row, col = [0], []
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                c = []
                for dz, dy, dx in offsets:
                    if 0 <= x + dx < nx and 0 <= y + dy < ny and 0 <= z + dz < nz:
                        c.append((z + dz) * nx * ny + (y + dy) * nx + x + dx)
                col.extend(sorted(c))
                row.append(len(col))
    return np.array(row, np.uint32), np.array(col, np.uint32)


def diag_first(row, col):
    col = col.copy()
    for i in range(len(row) - 1):
        a, b = int(row[i]), int(row[i + 1])
        c = list(col[a:b])
        if i in c:
            c.remove(i)
            c = [i] + c
        col[a:b] = c
    return col


BOX = [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)]
STAR = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]


def test_generated_matrices(xamg):
    """The diffusion generators store each row's diagonal first, the
    reference's cube generator sorts its rows."""
    row, col, _ = xamg.generate_diffusion(27, 13, 11, 9, 1.0, 1.0, 0)
    assert xamg.stencil_layout(row, col) == (BOX27, 13, 143, 1)
    row, col, _ = xamg.generate_diffusion(7, 12, 10, 9, 1.0, 1.0, 0)
    assert xamg.stencil_layout(row, col) == (STAR7, 12, 120, 1)
    row, col, _ = xamg.generate_cube(10, 12, 9)
    pat, S, S2, _ = xamg.stencil_layout(row, col)
    assert (pat, S, S2) == (STAR7, 10, 120)


@pytest.mark.parametrize("dims", [(3, 3, 3), (5, 4, 6), (17, 3, 8), (4, 9, 5)])
def test_box_and_star_shapes(xamg, dims):
    nx, ny, nz = dims
    row, col = grid_matrix(nx, ny, nz, BOX)
    assert xamg.stencil_layout(row, col) == (BOX27, nx, nx * ny, 0)
    assert xamg.stencil_layout(row, diag_first(row, col)) == (BOX27, nx, nx * ny, 1)
    row, col = grid_matrix(nx, ny, nz, STAR)
    assert xamg.stencil_layout(row, col) == (STAR7, nx, nx * ny, 0)
    assert xamg.stencil_layout(row, diag_first(row, col)) == (STAR7, nx, nx * ny, 1)


def test_subsets_of_the_box(xamg):
    """A 19-point stencil (no corners) uses a subset of the box's slots."""
    nine = [o for o in BOX if sum(map(abs, o)) <= 2]
    row, col = grid_matrix(7, 6, 5, nine)
    assert xamg.stencil_layout(row, col) == (BOX27, 7, 42, 0)


def test_rejected(xamg):
    # a row not sorted by column
    row, col = grid_matrix(6, 5, 4, BOX)
    c = col.copy()
    a = int(row[70])
    c[a], c[a + 1] = c[a + 1], c[a]
    assert xamg.stencil_layout(row, c)[0] == -1
    # rows in both orders (some diagonal first, some sorted)
    c = diag_first(row, col)
    a, b = int(row[70]), int(row[71])
    c[a:b] = col[a:b]
    assert xamg.stencil_layout(row, c)[0] == -1
    # an entry off the stencil
    row2, col2 = grid_matrix(6, 5, 4, STAR)
    r, cl = [0], []
    for i in range(len(row2) - 1):
        cs = list(col2[row2[i]:row2[i + 1]])
        if i == 50:
            cs = sorted(set(cs) | {119})
        cl.extend(cs)
        r.append(len(cl))
    assert xamg.stencil_layout(np.array(r, np.uint32), np.array(cl, np.uint32))[0] == -1
    # a random sparse matrix
    rng = np.random.default_rng(0)
    n = 500
    r, cl = [0], []
    for i in range(n):
        cs = sorted(set(rng.integers(0, n, 6).tolist()) | {i})
        cl.extend(cs)
        r.append(len(cl))
    assert xamg.stencil_layout(np.array(r, np.uint32), np.array(cl, np.uint32))[0] == -1
    # tiny
    assert xamg.stencil_layout(np.array([0, 1], np.uint32), np.array([0], np.uint32))[0] == -1


def covers(row, col, pat, S, S2):
    """Every offset of the matrix is dz*S2 + dy*S + dx with a slot in the
    pattern, and the strides keep ascending offsets in (dz, dy, dx) order."""
    if S < 3 or S2 < 2 * S + 3:
        return False
    for i in range(len(row) - 1):
        for c in col[row[i]:row[i + 1]]:
            o = int(c) - i
            dz = int(np.round(o / S2))
            r = o - dz * S2
            dy = int(np.round(r / S))
            dx = r - dy * S
            if max(abs(dz), abs(dy), abs(dx)) > 1:
                return False
            if pat == STAR7 and abs(dz) + abs(dy) + abs(dx) > 1:
                return False
    return True


@pytest.mark.parametrize("case", ["2d9", "nx2", "nx3"])
def test_other_shapes_are_covered_when_accepted(xamg, case):
    """Grids the detection is not aimed at (a 2-D nine-point stencil, lines of
    two or three points) may still be accepted under some strides; then every
    entry must lie on a slot of the reported pattern and strides (which is
    all the kernel needs to compute the right columns)."""
    if case == "2d9":
        row, col = grid_matrix(8, 7, 1, [o for o in BOX if o[0] == 0])
    elif case == "nx2":
        row, col = grid_matrix(2, 5, 6, BOX)
    else:
        row, col = grid_matrix(3, 4, 5, BOX)
    pat, S, S2, _ = xamg.stencil_layout(row, col)
    if pat != -1:
        assert covers(row, col, pat, S, S2)
