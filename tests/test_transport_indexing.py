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
