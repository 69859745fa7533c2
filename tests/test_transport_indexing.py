"""Index arithmetic of the temperature transport's column walk and of the
link-parallel face pre-fill, restated on the CPU (no GPU): every shared-memory
entry a thread stages or looks up lies inside its staged plane, and the fill's
thread index covers every (boundary cell, inward link) of the visited faces
exactly once. The constants and formulas mirror thermal_exact.cu
(thermal_column, update_pair) and d3q27_inplace.cuh (face_fill_cell)."""
from __future__ import annotations

import itertools

import pytest

# thermal_exact.cu
MZ, MY = 32, 8
MTZ = MZ // 2
MTHREADS = MTZ * MY
PZ = MZ + 4
ROW_PAIRS = PZ // 2
PAIRS = ROW_PAIRS * (MY + 2)
PLANE = PZ * (MY + 2)


def test_staged_pairs_fit_the_plane():
    assert PAIRS <= 2 * MTHREADS
    seen = set()
    for tid in range(MTHREADS):
        for e in range(2):
            p = tid + e * MTHREADS
            if p >= PAIRS:
                continue
            row, j = divmod(p, ROW_PAIRS)
            idx = row * PZ + 2 * j
            assert idx % 2 == 0 and 0 <= idx and idx + 1 < PLANE
            seen.update((idx, idx + 1))
    assert seen == set(range(PLANE))  # every staged entry is written by exactly one pair


def test_lookups_stay_inside_the_plane():
    """The two cells' own entries, their six face neighbours and the eight
    trilinear corners of a near lane (lower corner at offset -1 or 0 on each
    axis, a far lane reads its own entry) are inside the staged plane."""
    for ty, tx in itertools.product(range(MY), range(MTZ)):
        ci = (ty + 1) * PZ + 2 * tx + 2
        assert ci % 2 == 0
        for k in range(2):
            c = ci + k
            for n in (c, c + 1, c - 1, c + PZ, c - PZ):
                assert 0 <= n < PLANE
            for dy, dz in itertools.product((-1, 0), (-1, 0)):
                b = c + dy * PZ + dz
                for corner in (b, b + 1, b + PZ, b + PZ + 1):
                    assert 0 <= corner < PLANE
        # the z-neighbour pairs of update_pair: c+1, c+2 (lane 1's +z) and c-1
        assert 0 <= ci - 1 and ci + 2 < PLANE


@pytest.mark.parametrize("nx", [1, 4, 12, 37, 128])
def test_column_ring_slots(nx):
    """Planes x-1, x, x+1 (read) and x+2 (written) take four distinct ring
    slots at every plane of a column; plane -1 maps to slot 3."""
    for x in range(nx):
        slots = [(x + d) & 3 for d in (-1, 0, 1, 2)]
        assert len(set(slots)) == 4


def _face_area(dims, face):
    nx, ny, nz = dims
    axis = face // 2
    return (ny * nz, nx * nz, nx * ny)[axis]


def _fill_link(dims, faces, i):
    """face_fill_cell's decode of link index i: (x, y, z, q) or None."""
    nx, ny, nz = dims
    face = -1
    area = 0
    for fc in range(6):
        if face >= 0 or not (faces >> fc) & 1:
            continue
        n = _face_area(dims, fc)
        if i < 9 * n:
            face, area = fc, n
        else:
            i -= 9 * n
    if face < 0:
        return None
    s, r = divmod(i, area)
    hi = face & 1
    inward = 0 if hi else 2
    if face < 2:
        x = nx - 1 if hi else 0
        y, z = divmod(r, nz)
        q = inward * 9 + s
    elif face < 4:
        y = ny - 1 if hi else 0
        x, z = divmod(r, nz)
        q = (s // 3) * 9 + inward * 3 + s % 3
    else:
        z = nz - 1 if hi else 0
        x, y = divmod(r, ny)
        q = (s // 3) * 9 + (s % 3) * 3 + inward
    return x, y, z, q


@pytest.mark.parametrize("dims,faces", [((5, 3, 7), 0x3F), ((12, 10, 70), 0b100011), ((4, 4, 4), 0b010010),
                                        ((1, 2, 3), 0x3F)])
def test_fill_links_cover_each_face_link_once(dims, faces):
    nx, ny, nz = dims
    count = sum(9 * _face_area(dims, f) for f in range(6) if (faces >> f) & 1)
    got = [_fill_link(dims, faces, i) for i in range(count + 64)]
    assert all(g is None for g in got[count:])
    links = got[:count]
    # each visited face contributes its cells x its nine inward directions, once
    want = []
    for f in range(6):
        if not (faces >> f) & 1:
            continue
        axis, hi = f // 2, f & 1
        comp = -1 if hi else 1  # the direction's component along the face axis (pulls across the face)
        for x, y, z in itertools.product(range(nx), range(ny), range(nz)):
            if (x, y, z)[axis] != ((nx, ny, nz)[axis] - 1 if hi else 0):
                continue
            for q in range(27):
                c = (q // 9 - 1, (q // 3) % 3 - 1, q % 3 - 1)
                if c[axis] == comp:
                    want.append((f, x, y, z, q))
    faces_of = []
    for i, link in enumerate(links):
        assert link is not None
        x, y, z, q = link
        assert 0 <= x < nx and 0 <= y < ny and 0 <= z < nz and 0 <= q < 27
        faces_of.append(link)
    assert len(faces_of) == len(want)
    # per face the decoded tuples are distinct and match the expected set
    start = 0
    for f in range(6):
        if not (faces >> f) & 1:
            continue
        n = 9 * _face_area(dims, f)
        block = faces_of[start:start + n]
        start += n
        assert len(set(block)) == n
        assert set(block) == {(x, y, z, q) for (ff, x, y, z, q) in want if ff == f}


# ---- th_sample's interior test (thermal_exact.cu): x0 < n - 1, overflow-free
INT_MAX, INT_MIN = 2 ** 31 - 1, -2 ** 31


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 3, 5), (12, 10, 70), (128, 128, 128)])
def test_sample_interior_test_keeps_every_corner_inside(dims):
    """Saturated conversions (a non-finite or huge position gives INT_MAX /
    INT_MIN) never pass the interior test, and every accepted lower corner
    keeps all eight corners inside the brick."""
    nx, ny, nz = dims
    cells = nx * ny * nz
    probe = lambda n: sorted({INT_MIN, -1, 0, max(0, n - 2), n - 1, n, INT_MAX})
    for x0, y0, z0 in itertools.product(probe(nx), probe(ny), probe(nz)):
        inside = 0 <= x0 < nx - 1 and 0 <= y0 < ny - 1 and 0 <= z0 < nz - 1
        if x0 in (INT_MIN, INT_MAX) or y0 in (INT_MIN, INT_MAX) or z0 in (INT_MIN, INT_MAX):
            assert not inside
        if inside:
            b = (x0 * ny + y0) * nz + z0
            assert b >= 0 and b + ny * nz + nz + 1 < cells


# ---- the per-block halo source table against th_neighbour's per-entry rule
PERIODIC, DIRICHLET, NEUMANN, ADIABATIC = 2, 4, 5, 3


def _entry_rule(kinds, dims, x, y, z):
    """th_neighbour without the querying cell: periodic axes wrap first, then
    the first face crossed in the order x, y, z decides; ('cell', x, y, z) or
    ('face', f)."""
    n = dims
    p = [x, y, z]
    for a in range(3):
        if (p[a] < 0 or p[a] >= n[a]) and kinds[2 * a + (0 if p[a] < 0 else 1)] == PERIODIC:
            p[a] %= n[a]
    for a in range(3):
        if p[a] < 0:
            return ("face", 2 * a)
        if p[a] >= n[a]:
            return ("face", 2 * a + 1)
    return ("cell", *p)


def _table_rule(kinds, dims, x, y, z):
    """resolve_x, then resolve_yz (the column kernel's split)."""
    nx, ny, nz = dims
    if not 0 <= x < nx:
        if kinds[0 if x < 0 else 1] != PERIODIC:
            return ("face", 0 if x < 0 else 1)
        x %= nx
    if (y < 0 or y >= ny) and kinds[2 if y < 0 else 3] == PERIODIC:
        y %= ny
    if (z < 0 or z >= nz) and kinds[4 if z < 0 else 5] == PERIODIC:
        z %= nz
    if 0 <= y < ny and 0 <= z < nz:
        return ("cell", x, y, z)
    return ("face", 2 if y < 0 else (3 if y >= ny else (4 if z < 0 else 5)))


@pytest.mark.parametrize("kinds", [(DIRICHLET, NEUMANN, PERIODIC, PERIODIC, ADIABATIC, DIRICHLET),
                                   (PERIODIC, PERIODIC, ADIABATIC, NEUMANN, DIRICHLET, PERIODIC),
                                   (PERIODIC, PERIODIC, PERIODIC, PERIODIC, PERIODIC, PERIODIC),
                                   (ADIABATIC,) * 6])
@pytest.mark.parametrize("dims", [(3, 2, 5), (5, 9, 4)])
def test_source_table_matches_the_entry_rule(kinds, dims):
    nx, ny, nz = dims
    # every staged coordinate the column walk can touch: planes -1..nx, rows
    # -1..ny+8 (a partial last tile), z from -2 to nz+33
    for x, y, z in itertools.product(range(-1, nx + 1), range(-1, ny + 9), range(-2, nz + 34)):
        assert _table_rule(kinds, dims, x, y, z) == _entry_rule(kinds, dims, x, y, z), (x, y, z)
