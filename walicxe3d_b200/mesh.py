"""Host-side block tree: bID arithmetic and mesh construction.

bIDs follow the reference's numbering (source/amr.f90:637-997,
source/init.f90:733-756): level-by-level, x fastest, 1-based.  The tree
stays on the host (as in the reference, where amr.f90 owns it); this module
builds block lists for problem setups -- uniform root grids and zone
refinement with the face-neighbour proximity rule of checkProximity
(source/amr.f90:1109-1265) -- and orders the slots along a Morton curve so
neighbouring blocks sit close together in HBM.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .config import NCELLS, Config


@dataclass
class BlockTree:
    nbroot: tuple
    maxlev: int
    leaves: set = field(default_factory=set)

    def __post_init__(self):
        self.nb = {}
        self.minid = {}
        acc = 0
        for lev in range(1, self.maxlev + 1):
            n = tuple(r << (lev - 1) for r in self.nbroot)
            self.nb[lev] = n
            self.minid[lev] = acc + 1
            acc += n[0] * n[1] * n[2]
        self.maxid = acc

    # --- bID arithmetic (amr.f90:637-997) ---------------------------------
    def level(self, bid: int) -> int:
        for lev in range(self.maxlev, 0, -1):
            if bid >= self.minid[lev]:
                return lev
        raise ValueError(bid)

    def coords(self, bid: int) -> tuple:
        """0-based block coordinates at the block's level."""
        lev = self.level(bid)
        nx, ny, _ = self.nb[lev]
        loc = bid - self.minid[lev]
        return lev, (loc % nx, (loc // nx) % ny, loc // (nx * ny))

    def bid(self, lev: int, x: tuple) -> int:
        nx, ny, _ = self.nb[lev]
        return self.minid[lev] + x[0] + nx * (x[1] + ny * x[2])

    def father(self, bid: int) -> int:
        lev, x = self.coords(bid)
        if lev == 1:
            return -1
        return self.bid(lev - 1, tuple(v // 2 for v in x))

    def children(self, bid: int) -> list:
        """Natural order: x, then y, then z (amr.f90:882-909)."""
        lev, x = self.coords(bid)
        return [self.bid(lev + 1, (2 * x[0] + (c & 1), 2 * x[1] + ((c >> 1) & 1), 2 * x[2] + (c >> 2)))
                for c in range(8)]

    def neighbour_region(self, bid: int, face: int):
        """Same-level block across a face (0..5 = LEFT..TOP) or None."""
        lev, x = self.coords(bid)
        ax, side = face // 2, face % 2
        y = list(x)
        y[ax] += 1 if side else -1
        if y[ax] < 0 or y[ax] >= self.nb[lev][ax]:
            return None
        return self.bid(lev, tuple(y))

    # --- construction ------------------------------------------------------
    def roots(self):
        self.leaves = set(range(1, self.nb[1][0] * self.nb[1][1] * self.nb[1][2] + 1))
        return self

    def refine(self, bid: int):
        self.leaves.discard(bid)
        self.leaves.update(self.children(bid))

    def active_cover(self, nid: int) -> int:
        """The active block covering same-level region nid, if it or an
        ancestor is a leaf; -1 when the region is refined further."""
        b = nid
        while b != -1:
            if b in self.leaves:
                return b
            b = self.father(b)
        return -1

    def balance(self):
        """Refine until every face neighbour differs by at most one level
        (the face proximity rule of checkProximity, amr.f90:1109-1265)."""
        changed = True
        while changed:
            changed = False
            for b in sorted(self.leaves, key=self.level, reverse=True):
                if b not in self.leaves:
                    continue
                lev = self.level(b)
                for f in range(6):
                    n = self.neighbour_region(b, f)
                    if n is None:
                        continue
                    cov = self.active_cover(n)
                    if cov != -1 and self.level(cov) < lev - 1:
                        self.refine(cov)
                        changed = True
        return self

    def refine_where(self, pred, to_level: int):
        """refineZone-style (amr.f90:1269-1425): level by level, refine
        leaves for which pred(level, lo, hi) is true, then rebalance."""
        for lev in range(1, to_level):
            for b in sorted(self.leaves):
                if self.level(b) == lev:
                    lo, hi = self.bounds(b)
                    if pred(lev, lo, hi):
                        self.refine(b)
            self.balance()
        return self

    def bounds(self, bid: int):
        lev, x = self.coords(bid)
        n = self.nb[lev]
        lo = np.array([x[d] / n[d] for d in range(3)])
        hi = np.array([(x[d] + 1) / n[d] for d in range(3)])
        return lo, hi

    def hilbert_key(self, bid: int) -> int:
        """Position along a 3-D Hilbert curve of the block's low corner at the
        finest level, on the smallest power-of-two cube that holds the finest
        grid (the curve of getHilbertKey, amr.f90:2031-2061).  Computed with
        Skilling's transpose method (J. Skilling, "Programming the Hilbert
        curve", AIP Conf. Proc. 707, 381 (2004)): undo the excess work of the
        Gray-code walk axis by axis, Gray-encode, then interleave the bits."""
        lev, x = self.coords(bid)
        s = self.maxlev - lev
        X = [v << s for v in x]
        nmax = max(self.nb[self.maxlev])
        bits = max(1, (nmax - 1).bit_length())
        q = 1 << (bits - 1)
        while q > 1:
            p = q - 1
            for i in range(3):
                if X[i] & q:
                    X[0] ^= p
                else:
                    t = (X[0] ^ X[i]) & p
                    X[0] ^= t
                    X[i] ^= t
            q >>= 1
        for i in range(1, 3):
            X[i] ^= X[i - 1]
        t = 0
        q = 1 << (bits - 1)
        while q > 1:
            if X[2] & q:
                t ^= q - 1
            q >>= 1
        for i in range(3):
            X[i] ^= t
        h = 0
        for b in range(bits - 1, -1, -1):
            for i in range(3):
                h = (h << 1) | ((X[i] >> b) & 1)
        return h

    def hilbert_order(self) -> list:
        """Leaves sorted along the Hilbert curve (the order in which the
        reference deals blocks out to processes, HilbertOrder amr.f90:1930)."""
        return sorted(self.leaves, key=self.hilbert_key)

    def morton_order(self) -> list:
        """Leaves sorted along a Morton curve of their low corner at the
        finest level."""
        def key(b):
            lev, x = self.coords(b)
            s = self.maxlev - lev
            xs = [v << s for v in x]
            k = 0
            for bit in range(24):
                for d in range(3):
                    k |= ((xs[d] >> bit) & 1) << (3 * bit + d)
            return k
        return sorted(self.leaves, key=key)


def cell_centres(cfg: Config, tree: BlockTree, bids) -> np.ndarray:
    """Cell-centre coordinates (code units) of the 16^3 physical cells of each
    block: array [nb, 3, 16, 16, 16] indexed [.., k, j, i] (amr.f90:1037-1065)."""
    out = np.empty((len(bids), 3, NCELLS, NCELLS, NCELLS))
    idx = np.arange(NCELLS) + 0.5
    for n, b in enumerate(bids):
        lev, x = tree.coords(b)
        dx = cfg.dx(lev)
        cx = (x[0] * NCELLS + idx) * dx[0]
        cy = (x[1] * NCELLS + idx) * dx[1]
        cz = (x[2] * NCELLS + idx) * dx[2]
        out[n, 0] = cx[None, None, :]
        out[n, 1] = cy[None, :, None]
        out[n, 2] = cz[:, None, None]
    return out
