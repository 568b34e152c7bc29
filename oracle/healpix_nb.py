"""ORACLE (test infrastructure only): HEALPix RING-scheme 8-neighbours by brute
force, and the reference's neighbour-average inpainting restated in numpy.

The reference calls healpy.get_all_neighbours (polyspec/weighting.py:118, :138),
which is not installed here, so the neighbour lists are derived from the pixel
geometry instead and their order follows healpy's documented convention
(SW, W, NW, N, NE, E, SE, S; -1 where a pixel has only 7 neighbours):

* each base face f (Gorski et al. 2005: 12 faces, face-centre ring jrll[f] * Nside
  and azimuth jpll[f] * pi/4) is a lattice of Nside x Nside pixels (x, y); pixel
  (x, y) has the lattice vertices S = (x, y), E = (x+1, y), W = (x, y+1) and
  N = (x+1, y+1);
* a vertex is identified across faces by an exact integer key: its ring
  jr = jrll Nside - x - y, and its azimuth index jpll nr + x - y modulo 8 nr (nr the
  ring's pixel count scale: jr in the north cap, 4 Nside - jr in the south cap,
  Nside in the belt; one key per pole);
* the neighbour across an edge of p is the other pixel holding both vertices of
  that edge (SE: S, E; NE: E, N; NW: N, W; SW: W, S), the neighbour at a corner is
  a pixel holding that vertex of p and sharing no edge with p (S, E, N, W corners);
  where three faces meet no such pixel exists and the slot is -1.

Parity of this ordering with healpy itself is unpinned (healpy is absent); the
tests check the neighbour relation's symmetry and its count of 7-neighbour pixels.

inpaint_map restates polyspec/weighting.py:87-146 line by line, including the
reference's np.average weights ``this_map[neighbors] != 0 + 1e-30`` (a comparison
with 1e-30, so in effect equal weights) and numpy's reading of index -1 as the
last pixel.  The neighbour array is C-ordered [8, n], as healpy builds it from its
eight per-direction outputs; the layout matters because numpy then adds the eight
values of a pixel in order (an F-ordered array would be summed pairwise).
"""
import numpy as np

JRLL = np.array([2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4])
JPLL = np.array([1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7])


def xyf2ring(nside, f, x, y):
    """RING index of face pixel (x, y) of face f (integer arrays)."""
    n = nside
    npix, ncap = 12 * n * n, 2 * n * (n - 1)
    jr = JRLL[f] * n - x - y - 1
    nr = np.where(jr < n, jr, np.where(jr > 3 * n, 4 * n - jr, n))
    kshift = np.where((jr >= n) & (jr <= 3 * n), (jr - n) & 1, 0)
    nbefore = np.where(jr < n, 2 * nr * (nr - 1),
                       np.where(jr > 3 * n, npix - 2 * (nr + 1) * nr, ncap + (jr - n) * 4 * n))
    jp = (JPLL[f] * nr + x - y + 1 + kshift) // 2
    jp = np.where(jp > 4 * nr, jp - 4 * nr, jp)
    jp = np.where(jp < 1, jp + 4 * nr, jp)
    return nbefore + jp - 1


def vertex_key(nside, f, x, y):
    """Exact integer key of lattice vertex (x, y) of face f."""
    n = nside
    jr = JRLL[f] * n - x - y
    nr = np.where(jr < n, jr, np.where(jr > 3 * n, 4 * n - jr, n))
    t = JRLL[f] * 0 + JPLL[f] * nr + x - y
    t = np.where(nr > 0, np.mod(t, np.maximum(8 * nr, 1)), 0)
    return jr.astype(np.int64) * (64 * n + 8) + t


def all_neighbours(nside):
    """[Npix, 8] RING neighbours in the order SW, W, NW, N, NE, E, SE, S (-1: none)."""
    n = nside
    f, y, x = np.meshgrid(np.arange(12), np.arange(n), np.arange(n), indexing='ij')
    f, x, y = f.ravel(), x.ravel(), y.ravel()
    pix = xyf2ring(n, f, x, y)
    corners = {'S': (0, 0), 'E': (1, 0), 'W': (0, 1), 'N': (1, 1)}
    vk = {c: vertex_key(n, f, x + d[0], y + d[1]) for c, d in corners.items()}
    holders = {}
    for c in corners:
        for p, k in zip(pix, vk[c]):
            holders.setdefault(int(k), set()).add(int(p))
    npix = 12 * n * n
    key_of = {c: np.empty(npix, dtype=np.int64) for c in corners}
    for c in corners:
        key_of[c][pix] = vk[c]
    out = -np.ones((npix, 8), dtype=np.int64)
    edges = {'SW': ('W', 'S'), 'NW': ('N', 'W'), 'NE': ('E', 'N'), 'SE': ('S', 'E')}
    slots = ['SW', 'W', 'NW', 'N', 'NE', 'E', 'SE', 'S']
    for p in range(npix):
        edge_nb = {}
        for e, (a, b) in edges.items():
            s = (holders[int(key_of[a][p])] & holders[int(key_of[b][p])]) - {p}
            assert len(s) <= 1
            edge_nb[e] = s.pop() if s else -1
        touching = set(v for v in edge_nb.values() if v >= 0)
        for k, slot in enumerate(slots):
            if slot in edges:
                out[p, k] = edge_nb[slot]
            else:
                s = holders[int(key_of[slot][p])] - {p} - touching
                assert len(s) <= 1
                out[p, k] = s.pop() if s else -1
    return out


def inpaint_map(input_map, inpainting_mask, nside, pol, n_average=50, neighbours=None):
    """polyspec/weighting.py:87-146 with the neighbour lists of all_neighbours."""
    nb_all = all_neighbours(nside) if neighbours is None else neighbours
    tmp_map = input_map.copy()
    inpainting_filt = (inpainting_mask == 1)
    if np.sum(inpainting_filt) == 0:
        return tmp_map
    for field in range(1 + 2 * pol):
        this_map = tmp_map[field].copy()
        if np.sum(this_map) == 0:
            continue
        this_map[inpainting_filt[field]] = 0
        inpaint_pix = np.where((tmp_map[field] == 0) & inpainting_filt[field])[0]
        while True:
            neighbors = np.ascontiguousarray(nb_all[inpaint_pix].T)
            this_map[inpaint_pix] = np.average(this_map[neighbors], weights=this_map[neighbors] != 0 + 1e-30, axis=0)
            next_inpaint = np.where((this_map == 0) & inpainting_filt[field])[0]
            if len(next_inpaint) == 0:
                break
            if len(next_inpaint) == len(inpaint_pix):
                print("# Inpainting field %d failed!" % field)
                break
            inpaint_pix = next_inpaint
        for i in range(n_average):
            inpaint_pix = np.where(inpainting_filt[field])[0]
            neighbors = np.ascontiguousarray(nb_all[inpaint_pix].T)
            this_map[inpaint_pix] = np.average(this_map[neighbors], axis=0)
        tmp_map[field] = this_map
    return tmp_map
