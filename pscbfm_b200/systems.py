"""Synthetic BFM systems: the standard bond set and seeded polymer generators.

The reference ships no input systems for this path (its golden
``tests/*.bfm`` files are absent), so every benchmark and test system is
generated here from a seed:

* ``saw_chains``      linear chains grown as self-avoiding walks (dilute
                      melts, e.g. 128 chains x 64 on 128^3);
* ``ordered_melt``    a dense volume-fraction-0.5 melt built as a serpentine
                      crystal (e.g. 4096 chains x 256 on 256^3) that the
                      sweep itself melts;
* ``star_comb``       3-arm stars with side chains (branched, >2 colours
                      possible after cross-links);
* ``add_crosslinks``  extra bonds between close monomers, giving odd cycles
                      and therefore 3 or more colours.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from itertools import permutations, product

import numpy as np


def bond_vectors_108() -> np.ndarray:
    """The 108 bond vectors of the standard BFM bond set: all permutations
    and sign changes of (2,0,0), (2,1,0), (2,1,1), (3,0,0), (3,1,0), (2,2,1)."""
    vecs = set()
    for base in [(2, 0, 0), (2, 1, 0), (2, 1, 1), (3, 0, 0), (3, 1, 0), (2, 2, 1)]:
        for perm in permutations(base):
            for signs in product((1, -1), repeat=3):
                vecs.add(tuple(int(p * s) for p, s in zip(perm, signs)))
    out = np.array(sorted(vecs), dtype=np.int32)
    assert out.shape == (108, 3)
    return out


def allowed_table(vectors: np.ndarray) -> np.ndarray:
    """512-entry table, index (dx&7)|(dy&7)<<3|(dz&7)<<6 (the reference's
    linearizeBondVectorIndex, UpdaterGPUScBFM_AB_Type.cu:871-889)."""
    t = np.zeros(512, dtype=bool)
    for dx, dy, dz in vectors:
        t[(dx & 7) | ((dy & 7) << 3) | ((dz & 7) << 6)] = True
    return t


BONDS_108 = bond_vectors_108()
ALLOWED_108 = allowed_table(BONDS_108)

_CUBE = np.array([(a, b, c) for c in (0, 1) for b in (0, 1) for a in (0, 1)], dtype=np.int64)


@dataclass
class System:
    box: tuple
    pos: np.ndarray                  # (n,3) int32 absolute (unfolded) corner positions
    deg: np.ndarray                  # (n,) uint8
    nbr: np.ndarray                  # (n,8) uint32
    allowed: np.ndarray = field(default_factory=lambda: ALLOWED_108.copy())
    chains: list = field(default_factory=list)   # (first id, length) of linear chains
    attributes: np.ndarray | None = None
    name: str = ""
    periodic: tuple = (True, True, True)

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    def volume_fraction(self) -> float:
        return 8.0 * self.n / float(np.prod(self.box))

    def bonds(self):
        """Undirected bond list (i < j)."""
        out = []
        for i in range(self.n):
            for j in self.nbr[i, : self.deg[i]]:
                if i < j:
                    out.append((i, int(j)))
        return out

    def mean_degree(self) -> float:
        return float(self.deg.mean()) if self.n else 0.0


def _empty_topology(n):
    return np.zeros(n, np.uint8), np.zeros((n, 8), np.uint32)


def _connect(deg, nbr, i, j):
    if deg[i] >= 8 or deg[j] >= 8:
        raise ValueError("more than 8 bonds on a monomer")
    nbr[i, deg[i]] = j
    deg[i] += 1
    nbr[j, deg[j]] = i
    deg[j] += 1


class _Occupancy:
    """2x2x2 cube occupation on a periodic box, for growing walks."""

    def __init__(self, box):
        self.box = np.array(box, dtype=np.int64)
        self.cells = np.zeros(tuple(box), dtype=bool)

    def _idx(self, p):
        c = (np.asarray(p, dtype=np.int64)[None, :] + _CUBE) % self.box
        return c[:, 0], c[:, 1], c[:, 2]

    def free(self, p) -> bool:
        return not self.cells[self._idx(p)].any()

    def set(self, p, v=True):
        self.cells[self._idx(p)] = v


def saw_chains(n_chains: int, chain_len: int, box=(128, 128, 128), seed: int = 12345, max_tries: int = 200,
               alternate_ab: bool = True) -> System:
    """Linear chains grown monomer by monomer as self-avoiding walks with
    bonds drawn uniformly from the 108-vector set; a chain that gets stuck is
    removed and regrown from a new random start."""
    rng = np.random.default_rng(seed)
    occ = _Occupancy(box)
    n = n_chains * chain_len
    pos = np.zeros((n, 3), np.int64)
    deg, nbr = _empty_topology(n)
    bvec = BONDS_108.astype(np.int64)
    for c in range(n_chains):
        first = c * chain_len
        for _ in range(max_tries):
            start = rng.integers(0, box, size=3)
            if not occ.free(start):
                continue
            occ.set(start)
            pos[first] = start
            ok = True
            for k in range(1, chain_len):
                prev = pos[first + k - 1]
                placed = False
                for b in rng.permutation(108):
                    cand = prev + bvec[b]
                    if occ.free(cand):
                        occ.set(cand)
                        pos[first + k] = cand
                        placed = True
                        break
                if not placed:
                    for q in range(k):
                        occ.set(pos[first + q], False)
                    ok = False
                    break
            if ok:
                break
        else:
            raise RuntimeError("could not place chain %d" % c)
        for k in range(1, chain_len):
            _connect(deg, nbr, first + k - 1, first + k)
    attrs = None
    if alternate_ab:
        attrs = np.array([1 + (i // chain_len) % 2 for i in range(n)], dtype=np.int32)
    return System(tuple(int(b) for b in box), pos.astype(np.int32), deg, nbr,
                  chains=[(c * chain_len, chain_len) for c in range(n_chains)], attributes=attrs,
                  name=f"saw_{n_chains}x{chain_len}_L{box[0]}")


def open_box_chains(n_chains: int, chain_len: int, box=(32, 32, 32), seed: int = 12345,
                    periodic=(False, False, False), max_tries: int = 200) -> System:
    """Linear self-avoiding chains in a box whose axes marked False are
    walls: along those axes every cube corner lies in 0 .. L-2.  Grown like
    saw_chains, with positions outside the walls refused."""
    rng = np.random.default_rng(seed)
    occ = _Occupancy(box)
    lo = np.array([0 if not p else -(1 << 30) for p in periodic], dtype=np.int64)
    hi = np.array([box[a] - 2 if not periodic[a] else (1 << 30) for a in range(3)], dtype=np.int64)

    def fits(q):
        return bool((q >= lo).all() and (q <= hi).all()) and occ.free(q)

    n = n_chains * chain_len
    pos = np.zeros((n, 3), np.int64)
    deg, nbr = _empty_topology(n)
    bvec = BONDS_108.astype(np.int64)
    for c in range(n_chains):
        first = c * chain_len
        for _ in range(max_tries):
            start = np.array([rng.integers(0, box[a] - 1 if not periodic[a] else box[a]) for a in range(3)])
            if not fits(start):
                continue
            occ.set(start)
            pos[first] = start
            ok = True
            for k in range(1, chain_len):
                prev = pos[first + k - 1]
                placed = False
                for bi in rng.permutation(108):
                    cand = prev + bvec[bi]
                    if fits(cand):
                        occ.set(cand)
                        pos[first + k] = cand
                        placed = True
                        break
                if not placed:
                    for q in range(k):
                        occ.set(pos[first + q], False)
                    ok = False
                    break
            if ok:
                break
        else:
            raise RuntimeError("could not place chain %d" % c)
        for k in range(1, chain_len):
            _connect(deg, nbr, first + k - 1, first + k)
    return System(tuple(int(b) for b in box), pos.astype(np.int32), deg, nbr,
                  chains=[(c * chain_len, chain_len) for c in range(n_chains)],
                  name=f"open_{n_chains}x{chain_len}_L{box[0]}", periodic=tuple(bool(p) for p in periodic))


def ordered_melt(L: int = 256, chain_len: int | None = None) -> System:
    """Volume fraction 0.5 on an L^3 box: monomers on the sites (2i, 2j, 4k),
    chains run along x with (2,0,0) bonds and turn into the next row with a
    (0,2,0) bond (a serpentine of chain_len / (L/2) rows).  For L = 256 and
    chain_len = 256 this is 4096 chains x 256 = 1,048,576 monomers."""
    per_row = L // 2
    if chain_len is None:
        chain_len = 2 * per_row
    if chain_len % per_row:
        raise ValueError("chain_len must be a multiple of L/2")
    rows_per_chain = chain_len // per_row
    rows_per_layer = L // 2
    if rows_per_layer % rows_per_chain:
        raise ValueError("L/2 rows per layer must be divisible by the rows per chain")
    layers = L // 4
    n_rows = rows_per_layer * layers
    n_chains = n_rows // rows_per_chain
    n = n_chains * chain_len
    # row r -> (j, k); monomer index = chain*chain_len + local
    chain = np.repeat(np.arange(n_chains), chain_len)
    local = np.tile(np.arange(chain_len), n_chains)
    row_in_chain = local // per_row
    idx_in_row = local % per_row
    row = chain * rows_per_chain + row_in_chain
    j = row % rows_per_layer
    k = row // rows_per_layer
    x_idx = np.where(row_in_chain % 2 == 0, idx_in_row, per_row - 1 - idx_in_row)
    pos = np.stack([2 * x_idx, 2 * j, 4 * k], axis=1).astype(np.int32)
    deg = np.zeros(n, np.uint8)
    nbr = np.zeros((n, 8), np.uint32)
    ids = np.arange(n)
    inner = local < chain_len - 1
    a = ids[inner]
    b = a + 1
    # neighbour order: previous first, then next (the order LeMonADE lists a linear chain)
    has_prev = local > 0
    nbr[has_prev, 0] = (ids - 1)[has_prev]
    deg[has_prev] = 1
    nbr[a, deg[a]] = b
    deg[a] += 1
    return System((L, L, L), pos, deg, nbr, chains=[(c * chain_len, chain_len) for c in range(n_chains)],
                  attributes=(1 + (chain % 2)).astype(np.int32), name=f"melt_{n_chains}x{chain_len}_L{L}")


def star_comb(n_stars: int, arm_len: int = 64, side_every: int = 8, side_len: int = 16, box=(128, 128, 128),
              seed: int = 7, max_tries: int = 200) -> System:
    """3-arm stars (a core monomer plus three arms of arm_len) carrying a side
    chain of side_len on every side_every-th backbone monomer, grown as
    self-avoiding walks.  Attribute 1 (A) backbone, 2 (B) side chains."""
    rng = np.random.default_rng(seed)
    occ = _Occupancy(box)
    bvec = BONDS_108.astype(np.int64)
    pos_l, attr_l, bonds = [], [], []

    def grow_from(parent_id, length, attr, placed):
        ids = []
        prev = parent_id
        for _ in range(length):
            for b in rng.permutation(108):
                cand = pos_l[prev] + bvec[b]
                if occ.free(cand):
                    occ.set(cand)
                    pos_l.append(cand)
                    attr_l.append(attr)
                    me = len(pos_l) - 1
                    bonds.append((prev, me))
                    placed.append(me)
                    ids.append(me)
                    prev = me
                    break
            else:
                return None
        return ids

    for s in range(n_stars):
        for _ in range(max_tries):
            mark = (len(pos_l), len(bonds))
            placed = []
            core = rng.integers(0, box, size=3)
            if not occ.free(core):
                continue
            occ.set(core)
            pos_l.append(core)
            attr_l.append(1)
            placed.append(len(pos_l) - 1)
            ok = True
            core_id = len(pos_l) - 1
            for _arm in range(3):
                arm = grow_from(core_id, arm_len, 1, placed)
                if arm is None:
                    ok = False
                    break
                for q, mid in enumerate(arm):
                    if (q + 1) % side_every == 0:
                        if grow_from(mid, side_len, 2, placed) is None:
                            ok = False
                            break
                if not ok:
                    break
            if ok:
                break
            for p in placed:
                occ.set(pos_l[p], False)
            del pos_l[mark[0]:]
            del attr_l[mark[0]:]
            del bonds[mark[1]:]
        else:
            raise RuntimeError("could not place star %d" % s)
    n = len(pos_l)
    deg, nbr = _empty_topology(n)
    for a, b in bonds:
        _connect(deg, nbr, a, b)
    return System(tuple(int(b) for b in box), np.array(pos_l, dtype=np.int32), deg, nbr,
                  attributes=np.array(attr_l, dtype=np.int32), name=f"starcomb_{n_stars}_L{box[0]}")


def add_crosslinks(sys: System, n_links: int, seed: int = 3) -> System:
    """Add up to n_links bonds between monomers that are not yet bonded but
    whose separation is already a valid bond vector (this closes cycles, so
    the colouring may need 3 or more colours)."""
    rng = np.random.default_rng(seed)
    pos = sys.pos.astype(np.int64)
    box = np.array(sys.box)
    wrapped = pos % box
    lookup = {tuple(p): i for i, p in enumerate(wrapped)}
    deg = sys.deg.copy()
    nbr = sys.nbr.copy()
    added = 0
    for i in rng.permutation(sys.n):
        if added >= n_links:
            break
        if deg[i] >= 8:
            continue
        for b in rng.permutation(108):
            q = tuple((wrapped[i] + BONDS_108[b]) % box)
            j = lookup.get(q)
            if j is None or j == i or deg[j] >= 8 or j in set(nbr[i, : deg[i]].tolist()):
                continue
            d = pos[j] - pos[i]
            d = (d + box // 2) % box - box // 2  # minimum image
            if not sys.allowed[(d[0] & 7) | ((d[1] & 7) << 3) | ((d[2] & 7) << 6)]:
                continue
            if np.any(np.abs(d) > 3):
                continue
            # unfold j next to i so the stored bond is the short one
            if not np.array_equal(pos[j] - pos[i], d):
                continue
            _connect(deg, nbr, int(i), int(j))
            added += 1
            break
    return System(sys.box, sys.pos.copy(), deg, nbr, sys.allowed.copy(), list(sys.chains), sys.attributes,
                  sys.name + f"_x{added}")


def chain_observables(pos: np.ndarray, chains) -> tuple[float, float]:
    """Mean squared end-to-end distance R_e^2 and radius of gyration R_g^2
    over linear chains (first id, length) of unfolded positions."""
    p = np.asarray(pos, dtype=np.float64)
    re2, rg2 = [], []
    for first, length in chains:
        c = p[first:first + length]
        re2.append(float(((c[-1] - c[0]) ** 2).sum()))
        rg2.append(float(((c - c.mean(axis=0)) ** 2).sum(axis=1).mean()))
    return float(np.mean(re2)), float(np.mean(rg2))


def _grid_path(L):
    """Sites (2i, 2j, 2k) of an L^3 box in a boustrophedon order: rows along
    x alternate direction, layers alternate as a whole, so consecutive sites
    are one grid step (a (2,0,0)-type bond) apart and no step wraps."""
    g = L // 2
    i = np.arange(g)
    layer = []
    for j in range(g):
        row = i if j % 2 == 0 else i[::-1]
        layer.append(np.stack([row, np.full(g, j), np.zeros(g, np.int64)], axis=1))
    layer = np.concatenate(layer)
    out = []
    for k in range(g):
        lay = (layer if k % 2 == 0 else layer[::-1]).copy()
        lay[:, 2] = k
        out.append(lay)
    return 2 * np.concatenate(out)


def _topology_from_bonds(n, bonds):
    """deg/nbr from a bond list, partner slots in the order _connect would
    fill them (bond by bond, first end then second end)."""
    bonds = np.asarray(bonds, np.int64).reshape(-1, 2)
    ends = np.empty((2 * len(bonds), 2), np.int64)
    ends[0::2, 0], ends[0::2, 1] = bonds[:, 0], bonds[:, 1]
    ends[1::2, 0], ends[1::2, 1] = bonds[:, 1], bonds[:, 0]
    order = np.argsort(ends[:, 0], kind="stable")
    node = ends[order, 0]
    first = np.searchsorted(node, node, side="left")
    rank = np.arange(len(node)) - first
    if len(rank) and rank.max() >= 8:
        raise ValueError("more than 8 bonds on a monomer")
    deg = np.zeros(n, np.uint8)
    nbr = np.zeros((n, 8), np.uint32)
    nbr[node, rank] = ends[order, 1]
    np.add.at(deg, node, 1)
    return deg, nbr


def _with_side_chains(L, path, used, idx, seqs, side_every, side_len):
    """Side chains of side_len monomers on every side_every-th monomer of each
    backbone sequence (a chain, or a star arm from the core outwards): each
    starts on the grid site above (or below) its anchor and follows the path
    over free sites; an anchor with no free run gets none.  Returns
    (path indices of all monomers, bonds of the side chains)."""
    n_sites = len(path)
    where = np.full((L // 2,) * 3, -1, np.int64)
    where[path[:, 0] // 2, path[:, 1] // 2, path[:, 2] // 2] = np.arange(n_sites)
    steps = np.arange(side_len)
    extra, bonds = [], []
    nxt = len(idx)
    for seq in seqs:
        for q in range(side_every - 1, len(seq), side_every):
            anchor = int(seq[q])
            ci, cj, ck = path[idx[anchor]] // 2
            found = None
            for dk in (1, -1):
                kk = ck + dk
                if 0 <= kk < L // 2:
                    s0 = int(where[ci, cj, kk])
                    for sgn in (1, -1):
                        run = s0 + sgn * steps
                        if run.min() >= 0 and run.max() < n_sites and not used[run].any():
                            found = run
                            break
                if found is not None:
                    break
            if found is None:
                continue
            used[found] = True
            extra.append(found)
            bonds.append((anchor, nxt))
            bonds.extend((nxt + t, nxt + t + 1) for t in range(side_len - 1))
            nxt += side_len
    allidx = np.concatenate([idx] + extra) if extra else idx
    return allidx, np.array(bonds, np.int64).reshape(-1, 2)


def star_comb_melt(L: int = 1024, arm_len: int = 64, side_every: int = 8, side_len: int = 16) -> System:
    """Dense melt of 3-arm star-combs: a core and three arms of arm_len
    backbone monomers, a side chain of side_len = 2 * side_every monomers on
    every side_every-th backbone monomer (attribute 1 backbone and core,
    2 side chains).  For L = 1024 this is 115,600 stars x 577 = 66,701,200
    monomers at volume fraction 0.497.

    Construction (every bond a vector of the 108 set, no two cubes overlap):
    monomer cubes sit on the grid (2i, 2j, 4k) of L/2 x L/2 sites in L/4
    layers.  A layer is cut into blocks of arm_len x 3 grid sites, one arm
    each: the backbone runs along one row of the block from its right end
    (index 0) to its left end, and the side chain of backbone index q (with
    (q + 1) % side_every == 0) fills the side_every x 2 sites beside the
    backbone indices q-side_every+1 .. q, starting next to its anchor and
    turning back in the far row.  Blocks pair up across rows (6 rows: the
    lower block's backbone on its top row, the upper block's on its bottom
    row), so the first backbone monomers of both meet at the corner of a
    grid cell at the right end of the block column.  The cores sit in the
    empty half-layers between grid layers (z = 4g + 2), over that corner;
    a core reaches the first backbone monomers of both blocks in the layer
    below and in the layer above with (+-1, +-1, +-2) bonds.  Along z, the
    blocks of a block column are taken in order (layer by layer, lower block
    first) three at a time: star s owns blocks 3s, 3s+1, 3s+2, which lie in
    layers g and g+1 for g = floor(3s/2), and its core sits in the half-layer
    between them (a different one for every star).  Rows of the layer beyond
    the last whole 6-row pair, and blocks beyond the last whole star of a
    column, stay empty."""
    if side_len != 2 * side_every or arm_len % side_every:
        raise ValueError("side chains must be 2 * side_every long and side_every must divide arm_len")
    G = L // 2
    if L % 4 or G % arm_len:
        raise ValueError("L / 2 must be a multiple of the arm length")
    A, E, S = arm_len, side_every, side_len
    ncol, npair, nz = G // A, G // 6, L // 4
    per_col = (2 * nz) // 3
    if npair < 1 or per_col < 1:
        raise ValueError("box too small for one star")
    arm_size = A + (A // E) * S
    size = 1 + 3 * arm_size
    # one arm in block coordinates: grid dx from the block's left column,
    # row rel. to the backbone row (0), adjacent side row (1), far row (2)
    q = np.arange(A)
    a_gx = [A - 1 - q]
    a_row = [np.zeros(A, np.int64)]
    anchors = np.arange(E - 1, A, E)
    t = np.arange(S)
    for qa in anchors:
        x0 = A - 1 - qa
        a_gx.append(x0 + np.where(t < E, t, 2 * E - 1 - t))
        a_row.append(np.where(t < E, 1, 2))
    a_gx = np.concatenate(a_gx)
    a_row = np.concatenate(a_row)
    # local bonds of one arm (ids relative to the arm's first monomer)
    ab = [np.stack([q[:-1], q[1:]], axis=1)]
    for c, qa in enumerate(anchors):
        first = A + c * S
        ab.append(np.array([[qa, first]]))
        ab.append(np.stack([first + t[:-1], first + t[1:]], axis=1))
    ab = np.concatenate(ab)
    # star template for even and odd star index: (layer offset dk, block row b) of each arm
    arm_blocks = {0: ((0, 0), (0, 1), (1, 0)), 1: ((0, 1), (1, 0), (1, 1))}

    def template(par):
        gx = np.zeros(size, np.int64)
        gy = np.zeros(size, np.int64)
        dk = np.zeros(size, np.int64)
        for a, (k, b) in enumerate(arm_blocks[par]):
            sl = slice(1 + a * arm_size, 1 + (a + 1) * arm_size)
            gx[sl] = a_gx
            # lower block (b = 0): backbone on row 2 of rows 0..2, sides on 1, 0;
            # upper block (b = 1): backbone on row 3, sides on 4, 5
            gy[sl] = np.where(b == 0, 2 - a_row, 3 + a_row)
            dk[sl] = k
        return gx, gy, dk

    tmpl = {par: template(par) for par in (0, 1)}
    bonds1 = [np.array([[0, 1 + a * arm_size] for a in range(3)])]
    for a in range(3):
        bonds1.append(ab + 1 + a * arm_size)
    bonds1 = np.concatenate(bonds1)          # (size - 1, 2) local bonds of one star
    n_stars = npair * ncol * per_col
    n = n_stars * size
    pp, jj, ss = np.meshgrid(np.arange(npair), np.arange(ncol), np.arange(per_col), indexing="ij")
    pp, jj, ss = pp.reshape(-1), jj.reshape(-1), ss.reshape(-1)
    g = (3 * ss) // 2
    pos = np.empty((n_stars, size, 3), np.int32)
    for par in (0, 1):
        sel = np.flatnonzero(ss % 2 == par)
        gx, gy, dk = tmpl[par]
        pos[sel, :, 0] = 2 * (A * jj[sel, None] + gx[None, :])
        pos[sel, :, 1] = 2 * (6 * pp[sel, None] + gy[None, :])
        pos[sel, :, 2] = 4 * (g[sel, None] + dk[None, :])
    pos[:, 0, 0] = 2 * A * jj + 2 * A - 1
    pos[:, 0, 1] = 12 * pp + 5
    pos[:, 0, 2] = 4 * g + 2
    pos = pos.reshape(n, 3)
    # topology of one star, then offset per star
    deg1 = np.zeros(size, np.uint8)
    nbr1 = np.zeros((size, 8), np.uint32)
    for x, y in bonds1:                      # partner slots in bond order, as _connect fills them
        nbr1[x, deg1[x]] = y
        deg1[x] += 1
        nbr1[y, deg1[y]] = x
        deg1[y] += 1
    deg = np.tile(deg1, n_stars)
    nbr = np.empty((n_stars, size, 8), np.uint32)
    off = (np.arange(n_stars, dtype=np.uint64) * np.uint64(size)).astype(np.uint32)
    valid = np.arange(8)[None, :] < deg1[:, None]
    nbr[:] = np.where(valid[None], nbr1[None] + off[:, None, None], 0)
    nbr = nbr.reshape(n, 8)
    attr1 = np.ones(size, np.int32)
    for a in range(3):
        attr1[1 + a * arm_size + A:1 + (a + 1) * arm_size] = 2
    return System((L, L, L), pos, deg, nbr, attributes=np.tile(attr1, n_stars),
                  name=f"starcomb_melt_{n_stars}x{size}_L{L}")


def ensemble_system(L: int, n_per_molecule: int, phi: float, star: bool = False, seed: int = 0, side_every: int = 0,
                    side_len: int = 0) -> System:
    """One system of a batched ensemble: linear chains of n_per_molecule
    monomers, or 3-arm stars (a core and three arms of (n-1)//3), placed
    along a grid path through the L^3 box (L a multiple of 8) at volume
    fraction about phi (8 sites per monomer), with gaps between molecules so
    that the density is even.  At least one molecule is placed.  With
    side_every > 0, combs: a side chain of side_len monomers on every
    side_every-th backbone monomer where there is room (attribute 2; the
    backbone is attribute 1 and its monomers keep the ids 0 .. n_backbone-1,
    molecule by molecule)."""
    rng = np.random.default_rng(seed)
    path = _grid_path(L)
    n_sites = len(path)
    arm = max(1, (n_per_molecule - 1) // 3) if star else 0
    size = 1 + 3 * arm if star else n_per_molecule
    combs = side_every > 0 and side_len > 0
    target = max(size, int(round(phi * L ** 3 / 8)))
    if combs:
        target = max(size, int(round(target / (1.0 + side_len / side_every))))
    gap = max(0, int(round(size * (1.0 - min(phi, 0.999)) / max(phi, 1e-3))))
    cursor = int(rng.integers(0, max(1, gap + 1)))
    count = target // size
    if not star:
        starts = cursor + np.arange(count) * (size + gap)
        starts = starts[starts + size <= n_sites]
        if starts.size == 0:
            starts = np.array([0])
        idx = (starts[:, None] + np.arange(size)[None, :]).reshape(-1)
        nb = idx.size
        q = np.arange(nb) % size
        a = np.flatnonzero(q < size - 1)
        bonds = np.stack([a, a + 1], axis=1)
        chains = [(c * size, size) for c in range(nb // size)]
        kind = "linear"
        if combs:
            used = np.zeros(n_sites, bool)
            used[idx] = True
            seqs = [np.arange(c * size, (c + 1) * size) for c in range(nb // size)]
            idx, side = _with_side_chains(L, path, used, idx, seqs, side_every, side_len)
            bonds = np.concatenate([bonds, side])
            chains = []
            kind = f"comb{side_every}x{side_len}_"
        n = idx.size
        pos = path[idx]
        deg, nbr = _topology_from_bonds(n, bonds)
        attrs = np.where(np.arange(n) < nb, 1, 2).astype(np.int32)
        name = f"{kind}linear{size}_phi{n * 8 / L ** 3:.2f}_L{L}" if combs else f"linear{size}_phi{n * 8 / L ** 3:.2f}_L{L}"
        return System((L, L, L), pos.astype(np.int32), deg, nbr, chains=chains, attributes=attrs, name=name)
    where = np.full((L // 2,) * 3, -1, np.int64)
    where[path[:, 0] // 2, path[:, 1] // 2, path[:, 2] // 2] = np.arange(n_sites)
    used = np.zeros(n_sites, bool)
    mols = []

    def free_run(start, length):
        while start + length <= n_sites:
            u = np.flatnonzero(used[start:start + length])
            if u.size == 0:
                return start
            start += int(u[-1]) + 1
        return -1

    steps = np.arange(arm)
    while len(mols) < max(1, count):
        s0 = free_run(cursor, 2 * arm + 1)
        found = None
        while s0 >= 0 and found is None:
            c = s0 + arm
            ci, cj, ck = path[c] // 2
            for dk in (1, -1):
                kk = ck + dk
                if kk < 0 or kk >= L // 2:
                    continue
                qq = int(where[ci, cj, kk])
                for sgn in (1, -1):
                    idx3 = qq + sgn * steps
                    if idx3.min() < 0 or idx3.max() >= n_sites or used[idx3].any():
                        continue
                    if np.any((idx3 >= s0) & (idx3 <= s0 + 2 * arm)):
                        continue
                    found = idx3
                    break
                if found is not None:
                    break
            if found is None:
                s0 = free_run(s0 + 1, 2 * arm + 1)
        if found is None:
            break
        c = s0 + arm
        order = np.concatenate([[c], np.arange(c - 1, s0 - 1, -1), np.arange(c + 1, s0 + 2 * arm + 1), found])
        used[order] = True
        mols.append(order)
        cursor = s0 + 2 * arm + 1 + gap
    if not mols:
        raise ValueError("no molecule fits the box")
    idx = np.concatenate(mols)
    nb = idx.size
    # per star: core -> arm k's first monomer, then along each arm
    base = (np.arange(len(mols)) * size)[:, None]
    tmpl = []
    for k in range(3):
        first = 1 + k * arm
        tmpl.append((0, first))
        tmpl.extend((first + t, first + t + 1) for t in range(arm - 1))
    tmpl = np.array(tmpl, np.int64)
    bonds = (base[:, :, None] + tmpl[None, :, :]).reshape(-1, 2)
    name = f"star{size}_phi{nb * 8 / L ** 3:.2f}_L{L}"
    if combs:
        seqs = [c * size + 1 + k * arm + np.arange(arm) for c in range(len(mols)) for k in range(3)]
        idx, side = _with_side_chains(L, path, used, idx, seqs, side_every, side_len)
        bonds = np.concatenate([bonds, side])
        name = f"starcomb{size}_{side_every}x{side_len}_phi{idx.size * 8 / L ** 3:.2f}_L{L}"
    n = idx.size
    pos = path[idx]
    deg, nbr = _topology_from_bonds(n, bonds)
    attrs = np.where(np.arange(n) < nb, 1, 2).astype(np.int32)
    return System((L, L, L), pos.astype(np.int32), deg, nbr, attributes=attrs, name=name)


def ensemble(n_systems: int, seed: int = 12345, boxes=(32, 48, 64, 96, 128), n_range=(16, 512), phi_range=(0.1, 0.5),
             star_fraction: float = 0.5):
    """A batched ensemble: per system a box edge drawn from boxes, monomers
    per molecule log-uniform in n_range, volume fraction uniform in
    phi_range, linear chains or 3-arm stars; returns (systems, parameters)."""
    rng = np.random.default_rng(seed)
    out, params = [], []
    for s in range(n_systems):
        L = int(rng.choice(boxes))
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        phi = float(rng.uniform(*phi_range))
        star = bool(rng.random() < star_fraction)
        n = min(n, (L // 2) ** 3 // 3)
        out.append(ensemble_system(L, n, phi, star, seed=seed + 1 + s))
        params.append({"L": L, "n": n, "phi": phi, "star": star})
    return out, params
