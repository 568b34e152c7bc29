"""HEALPix RING-scheme 8-neighbour table on the GPU (the get_all_neighbours call
of polyspec/weighting.py:118, :138, which the reference takes from healpy).

Geometry (Gorski et al. 2005): 12 base faces, face f centred on ring
JRLL[f] * Nside at azimuth JPLL[f] * pi/4, each an Nside x Nside lattice of pixels
(x, y) with x towards the face's east corner and y towards its west corner.  The
neighbours of (x, y) are (x + dx, y + dy) with (dx, dy) in the order SW (-1, 0),
W (-1, 1), NW (0, 1), N (1, 1), NE (1, 0), E (1, -1), SE (0, -1), S (-1, -1)
(healpy's order); one that falls outside the face lies on the adjacent face of
that 3 x 3 cell, reached by wrapping (x, y) modulo Nside and one of the eight
lattice symmetries (flip x, flip y, swap), or on no face (-1) where three faces
meet.  The adjacent face and symmetry of each (cell, face) do not depend on
Nside: ``face_tables`` derives them once from the faces' shared lattice vertices
at Nside = 4 (a vertex is keyed exactly by its ring and azimuth index), and
``ps_healpix_neighbours`` applies them to every pixel, one thread per face pixel.
"""
import ctypes
from functools import lru_cache

import numpy as np
import torch

from . import _lib

JRLL = np.array([2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4])
JPLL = np.array([1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7])
OFFSETS = [(-1, 0), (-1, 1), (0, 1), (1, 1), (1, 0), (1, -1), (0, -1), (-1, -1)]


def _vertex_key(n, f, x, y):
    jr = JRLL[f] * n - x - y
    nr = n if n <= jr <= 3 * n else (jr if jr < n else 4 * n - jr)
    t = (JPLL[f] * nr + x - y) % (8 * nr) if nr > 0 else 0
    return (int(jr), int(t))


def _transform(n, bits, x, y):
    if bits & 1:
        x = n - 1 - x
    if bits & 2:
        y = n - 1 - y
    if bits & 4:
        x, y = y, x
    return x, y


@lru_cache(maxsize=None)
def face_tables(n0=4):
    """(face[9][12], bits[9][12]): for each 3 x 3 cell (cx + 3 cy, cx/cy = 0 below, 1 inside,
    2 above the face) and face, the adjacent face (-1: none) and the symmetry bits
    (1: flip x, 2: flip y, 4: swap, applied in that order) mapping wrapped lattice
    coordinates of the cell into that face."""
    holders = {}
    for f in range(12):
        for x in range(n0):
            for y in range(n0):
                for dx in (0, 1):
                    for dy in (0, 1):
                        holders.setdefault(_vertex_key(n0, f, x + dx, y + dy), set()).add((f, x, y))
    verts = {'S': (0, 0), 'E': (1, 0), 'W': (0, 1), 'N': (1, 1)}
    edge_of = {(-1, 0): ('W', 'S'), (0, 1): ('N', 'W'), (1, 0): ('E', 'N'), (0, -1): ('S', 'E')}
    corner_of = {(-1, 1): 'W', (1, 1): 'N', (1, -1): 'E', (-1, -1): 'S'}
    face = -np.ones((9, 12), dtype=np.int32)
    bits = np.zeros((9, 12), dtype=np.int32)
    samples = {}
    for f in range(12):
        for x in range(n0):
            for y in range(n0):
                key = {c: _vertex_key(n0, f, x + d[0], y + d[1]) for c, d in verts.items()}
                edge_nb = {}
                for o, (a, b) in edge_of.items():
                    s = (holders[key[a]] & holders[key[b]]) - {(f, x, y)}
                    edge_nb[o] = s.pop() if s else None
                touching = set(v for v in edge_nb.values() if v is not None)
                for dx, dy in OFFSETS:
                    X, Y = x + dx, y + dy
                    if 0 <= X < n0 and 0 <= Y < n0:
                        continue
                    if (dx, dy) in edge_of:
                        nb = edge_nb[(dx, dy)]
                    else:
                        s = holders[key[corner_of[(dx, dy)]]] - {(f, x, y)} - touching
                        nb = s.pop() if s else None
                    cell = (0 if X < 0 else 2 if X >= n0 else 1) + 3 * (0 if Y < 0 else 2 if Y >= n0 else 1)
                    samples.setdefault((cell, f), []).append(((X % n0, Y % n0), nb))
    for (cell, f), ss in samples.items():
        targets = set(nb[0] if nb else -1 for _, nb in ss)
        if targets == {-1}:
            continue
        assert len(targets) == 1, "a cell must map to one face"
        g = targets.pop()
        ok = [b for b in range(8) if all(nb is not None and _transform(n0, b, *xy) == nb[1:] for xy, nb in ss)]
        assert ok, "no lattice symmetry maps cell %d of face %d" % (cell, f)
        face[cell, f], bits[cell, f] = g, ok[0]
    return face, bits


_TABLES = {}


def neighbours(nside, device):
    """[Npix, 8] int32 RING neighbours (SW, W, NW, N, NE, E, SE, S; -1: none) on `device`."""
    key = (int(nside), str(device))
    if key in _TABLES:
        return _TABLES[key]
    face, bits = face_tables()
    d_tab = torch.as_tensor(np.concatenate([face.ravel(), bits.ravel()]), device=device)
    out = torch.empty((12 * nside * nside, 8), dtype=torch.int32, device=device)
    _lib.call("ps_healpix_neighbours", int(nside), ctypes.c_void_p(d_tab.data_ptr()),
              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.current_stream().synchronize()
    _TABLES[key] = out
    return out
