"""Central-difference divergence of B on a single-level mesh: the quantity
the field-CD scheme (Toth 2000; brio-wu/flux_cd.f90:52-86) keeps constant."""
import numpy as np

from walicxe3d_b200.config import NCELLS


def assemble(prob, a):
    """[nb, 16, 16, 16] block array ([k][j][i] per block) -> one global
    [z][y][x] array of a single-level mesh."""
    n = prob.cfg.nbroot
    g = np.zeros((n[2] * NCELLS, n[1] * NCELLS, n[0] * NCELLS))
    for s, b in enumerate(prob.local_blocks):
        _, x = prob.tree.coords(int(b))
        g[x[2] * NCELLS:(x[2] + 1) * NCELLS, x[1] * NCELLS:(x[1] + 1) * NCELLS,
          x[0] * NCELLS:(x[0] + 1) * NCELLS] = a[s]
    return g


def central_divergence(prob, U):
    """(B_x(i+1)-B_x(i-1))/2dx + ... on every cell whose six face neighbours
    are inside the domain."""
    dx, dy, dz = prob.cfg.dx(1)
    bx, by, bz = (assemble(prob, U[:, e]) for e in (5, 6, 7))
    c = slice(1, -1)
    return ((bx[c, c, 2:] - bx[c, c, :-2]) / (2.0 * dx) + (by[c, 2:, c] - by[c, :-2, c]) / (2.0 * dy) +
            (bz[2:, c, c] - bz[:-2, c, c]) / (2.0 * dz))
