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
