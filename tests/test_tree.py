"""The product's tree builder reproduces the reference's construction (order, positions, links)."""
import numpy as np
import pytest

from emma_b200 import OctTree
from emma_b200 import configs
import oracle

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (no reference checkout)")


def _compare(mine, ref, levels):
    for l in levels:
        assert mine.noct(l) == ref.noct(l), l
        assert np.array_equal(mine.oct_xyz(l), ref.oct_xyz(l)), l
        tm, tr = mine.topology(l), ref.topology(l)
        for a, b in zip(tm, tr):
            assert np.array_equal(a, b), l


@needs_ref
def test_uniform_tree_matches_reference():
    mine = OctTree(4, 4)
    ref = oracle.RefTree(4, 4, ngridmax=1000)
    _compare(mine, ref, range(2, 5))


@needs_ref
@pytest.mark.parametrize("base,radii", [(4, (0.3, 0.15)), (3, (0.35,)), (5, (0.2, 0.1))])
def test_refined_tree_matches_reference(base, radii):
    lmax = base + len(radii)
    mine = OctTree(base, lmax)
    ref = oracle.RefTree(base, lmax, ngridmax=sum(8 ** (l - 1) for l in range(1, lmax + 1)))
    for i, r in enumerate(radii):
        pred = lambda c, r=r: np.linalg.norm(c - 0.5, axis=1) < r
        mine.refine_where(base + i, pred)
        ref.refine_where(base + i, pred)
    _compare(mine, ref, range(2, lmax + 1))


def test_sedov_geometry_counts():
    """The Sedov tree with the stated radii (level 6 base, r<0.25 -> 7, r<0.125 -> 8)."""
    t = configs.sedov().build()
    n = [t.noct(l) for l in range(6, 9)]
    cells = 8 * sum(n)
    leaves = sum(int((~t.split_mask(l)).sum()) for l in range(6, 9))
    assert n[0] == 32768
    assert cells == 538240 and leaves == 503728, (n, cells, leaves)


def test_refinement_respects_2to1():
    t = OctTree(3, 4)
    mark = np.zeros(8 * t.noct(3), np.int8)
    mark[0] = 1
    t.refine(3, mark)  # a single refined cell: its face neighbours are level-3 cells, allowed
    t2 = OctTree(3, 5)
    m2 = np.zeros(8 * t2.noct(3), np.int8)
    m2[0] = 1
    t2.refine(3, m2)
    m3 = np.ones(8 * t2.noct(4), np.int8)  # refining every level-4 cell needs level-4 neighbours
    with pytest.raises(RuntimeError):
        t2.refine(4, m3)
