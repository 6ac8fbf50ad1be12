"""Mesh generation and `.bin` mesh I/O for box-shaped hex and tet meshes.

Node and element ordering follow the reference's voxel mesher
(python/py_diff_pd/common/hex_mesh.py:8-68): nodes are numbered with the x index outermost
(`(i * ny + j) * nz + k` for a full box), and the 8 corners of a hex are listed in
(ii, jj, kk) lexicographic order.  The `.bin` layout is the one `Mesh::Initialize` reads
(cpp/core/src/mesh/mesh.cpp:4-31, file_helper.cpp:169-184): int vertex_dim, int element_dim,
then a row-major (rows, cols, data) matrix of vertices (3 x n doubles) and of elements
(k x m ints).

The reference has no hex -> tet splitter; `hex_to_tet5` adds the standard five-tetrahedron
split with alternating cell parity so that shared faces use matching diagonals.
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np


def generate_hex_mesh(voxels, dx: float, origin=(0.0, 0.0, 0.0)):
    """Voxel occupancy array -> (vertices (n, 3) float64, hexes (m, 8) int32, cell_ijk (m, 3))."""
    voxels = np.asarray(voxels).astype(bool)
    origin = np.asarray(origin, dtype=np.float64)
    cx, cy, cz = voxels.shape
    used = np.zeros((cx + 1, cy + 1, cz + 1), dtype=bool)
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                used[a:a + cx, b:b + cy, c:c + cz] |= voxels
    index = np.full(used.shape, -1, dtype=np.int64)
    ii, jj, kk = np.nonzero(used)          # C order == x outermost, z innermost
    index[ii, jj, kk] = np.arange(ii.size)
    verts = np.stack([origin[0] + dx * ii, origin[1] + dx * jj, origin[2] + dx * kk], axis=1).astype(np.float64)
    ci, cj, ck = np.nonzero(voxels)
    hexes = np.empty((ci.size, 8), dtype=np.int64)
    col = 0
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                hexes[:, col] = index[ci + a, cj + b, ck + c]
                col += 1
    return verts, hexes.astype(np.int32), np.stack([ci, cj, ck], axis=1)


# Local corner index = a*4 + b*2 + c for corner (a, b, c) of the unit cube.
_EVEN_CENTRAL = (0, 3, 5, 6)            # corners with even bit parity
_ODD_CENTRAL = (1, 2, 4, 7)


def _corner_tets(central):
    others = [c for c in range(8) if c not in central]
    tets = [list(central)]
    for o in others:
        nbrs = [o ^ 1, o ^ 2, o ^ 4]     # the three cube neighbours, all in the central set
        tets.append([o] + nbrs)
    return tets


def hex_to_tet5(verts, hexes, cell_ijk):
    """Split every hex into 5 tets; cells with odd (i+j+k) use the mirrored split."""
    verts = np.asarray(verts, dtype=np.float64)
    tets = []
    even = _corner_tets(_EVEN_CENTRAL)
    odd = _corner_tets(_ODD_CENTRAL)
    parity = np.asarray(cell_ijk).sum(axis=1) % 2
    for h, p in zip(np.asarray(hexes), parity):
        for t in (odd if p else even):
            tet = [int(h[c]) for c in t]
            x0, x1, x2, x3 = (verts[v] for v in tet)
            if np.dot(np.cross(x1 - x0, x2 - x0), x3 - x0) < 0:
                tet[1], tet[2] = tet[2], tet[1]
            tets.append(tet)
    return np.asarray(tets, dtype=np.int32)


def write_bin(path, verts, elems):
    verts = np.asarray(verts, dtype=np.float64)
    elems = np.asarray(elems, dtype=np.int32)
    k = elems.shape[1]
    with open(path, "wb") as f:
        f.write(struct.pack("ii", 3, k))
        f.write(struct.pack("ii", 3, verts.shape[0]))
        f.write(np.ascontiguousarray(verts.T).tobytes())
        f.write(struct.pack("ii", k, elems.shape[0]))
        f.write(np.ascontiguousarray(elems.T).astype(np.int32).tobytes())


def read_bin(path):
    data = Path(path).read_bytes()
    vdim, edim = struct.unpack_from("ii", data, 0)
    if vdim != 3 or edim not in (4, 8):
        raise RuntimeError(f"Corrupted mesh file: {path}")
    r, c = struct.unpack_from("ii", data, 8)
    if r != 3:
        raise RuntimeError("Inconsistent mesh matrix size.")
    off = 16
    verts = np.frombuffer(data, dtype=np.float64, count=r * c, offset=off).reshape(r, c).T.copy()
    off += 8 * r * c
    r2, c2 = struct.unpack_from("ii", data, off)
    off += 8
    if r2 != edim:
        raise RuntimeError("Inconsistent mesh matrix size.")
    elems = np.frombuffer(data, dtype=np.int32, count=r2 * c2, offset=off).reshape(r2, c2).T.copy()
    return verts, elems
