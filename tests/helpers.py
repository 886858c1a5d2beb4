"""Shared helpers of the test suite (tolerances, tree builders, comparisons)."""
import numpy as np

GAMMA = 5.0 / 3.0


def per_cell_rel(g, o):
    """Per-cell relative error of primitive planes d,u,v,w,p (5 x n).

    Velocities are compared relative to |v| + c_s (c_s = sqrt(gamma p / d)),
    because a relative error of a velocity component near 0 is meaningless."""
    g, o = np.asarray(g)[:5], np.asarray(o)[:5]
    cs = np.sqrt(GAMMA * np.abs(o[4]) / np.abs(o[0]))
    scale = np.abs(o).copy()
    scale[1:4] += cs
    return np.abs(g - o) / np.maximum(scale, 1e-300)


def leaf_mask(tree, level):
    return ~tree.split_mask(level)


def l1_rel(a, b, vol=None):
    """L1 = sum |a-b| dV / sum |b| dV."""
    a, b = np.asarray(a), np.asarray(b)
    if vol is None:
        vol = np.ones_like(b)
    return float(np.sum(np.abs(a - b) * vol) / np.sum(np.abs(b) * vol))


def same_tree_fields(tree_a, tree_b, levels, which=0):
    return all(np.array_equal(tree_a.get_fields(l, which), tree_b.get_fields(l, which)) for l in levels)


def rank_of_octs(tree, level, partition):
    """Owner rank of every oct of a level, from the position of its level-lcoarse
    ancestor (finer octs inherit their owner, as in the reference's Hilbert-key
    partition): `partition(ix, iy, iz)` on the integer ancestor coordinates."""
    n = 1 << (tree.lcoarse - 1)
    xyz = tree.oct_xyz(level).reshape(-1, 3)
    ijk = np.floor(xyz * n).astype(np.int64)
    return np.asarray(partition(ijk[:, 0], ijk[:, 1], ijk[:, 2]), dtype=np.int32)


def assign_ranks(tree, partition, levels=None):
    """Tag every oct of levels 1..lmax (or `levels`) with its owner rank."""
    for l in (range(1, tree.lmax + 1) if levels is None else levels):
        if tree.noct(l):
            tree.set_cpu(l, rank_of_octs(tree, l, partition))


# partitions of the 8^3-oct level-lcoarse grid used by the multi-rank tests; the
# off-centre cuts of "slabs" and "quadrants" cross the coarse-fine boundaries of
# trees refined in spheres about the box centre, so fine->coarse corrections go
# from one rank to another (central cuts only meet fine octs across faces)
PARTITIONS = {
    "halves": (2, lambda i, j, k: (i >= 4).astype(np.int32)),
    "slabs": (2, lambda i, j, k: (i >= 5).astype(np.int32)),
    "quadrants": (4, lambda i, j, k: ((i >= 5) + 2 * (j >= 3)).astype(np.int32)),
    "stripes3": (3, lambda i, j, k: ((i + j + k) % 3).astype(np.int32)),
}
