"""Brick planning on the host (no GPU): every level of every configuration is
covered by brick tiles whose staged slots pass the planner's own checks."""
import ctypes

import pytest

from emma_b200 import configs
from emma_b200._lib import lib


def plan_stats(cfg, tree):
    nl = cfg.lmax - cfg.lcoarse + 1
    st = (ctypes.c_longlong * (5 * nl))()
    rc = lib().emma_hydro_plan_stats(tree.firstoct, cfg.lcoarse, cfg.lmax, cfg.trans, st)
    return rc, [list(st[5 * i:5 * i + 5]) for i in range(nl)]


@pytest.mark.parametrize("cfg", [configs.sod(level=5), configs.small_amr(), configs.small_amr(base=3, radii=(0.35, 0.2)),
                                 configs.random_uniform(level=3), configs.sedov(), configs.cosmo(base=5, lmax=8)],
                         ids=["sod", "amr4", "amr3", "uniform3", "sedov", "cosmo5"])
def test_every_level_plans(cfg):
    t = cfg.build()
    rc, stats = plan_stats(cfg, t)
    assert rc == 0, lib().emma_hydro_last_error()
    for i, (octs, tiles, max_staged, staged, leaf) in enumerate(stats):
        l = cfg.lcoarse + i
        assert octs == t.noct(l)
        if octs == 0:
            continue
        assert tiles >= 1 and max_staged >= 8
        # a complete level is tiled by full 4x4x2 bricks of 136 staged octs each
        if octs == 8 ** (l - 1) and l >= 3:
            assert tiles * 32 == octs and max_staged == 136 and staged == 136 * tiles
        assert staged <= tiles * 4 * 64


def test_fully_refined_tree_plans():
    """Every cell of the base level refined: the finer level is complete too and
    both are tiled by full 4x4x2 bricks."""
    from emma_b200 import OctTree
    t = OctTree(3, 4)
    t.refine_where(3, lambda c: c[:, 0] >= 0)
    st = (ctypes.c_longlong * 10)()
    assert lib().emma_hydro_plan_stats(t.firstoct, 3, 4, 0, st) == 0
    assert list(st[0:2]) == [64, 2] and list(st[5:7]) == [512, 16]


def test_transmissive_boundary_with_refinement_plans():
    """With transmissive boundaries (the reference's HYDROTEST build) coarser
    neighbours are interpolated (coarse2fine_hydro2); the planner lists the coarse
    cells and their slope neighbours, including a refined region that touches the
    transmissive boundary."""
    from emma_b200 import OctTree
    t = OctTree(3, 4)
    t.refine_where(3, lambda c: c[:, 0] < 0.3)  # refined region touching x = 0
    st = (ctypes.c_longlong * 10)()
    assert lib().emma_hydro_plan_stats(t.firstoct, 3, 4, 0x3, st) == 0, lib().emma_hydro_last_error()
    assert lib().emma_hydro_plan_stats(t.firstoct, 3, 4, 0, st) == 0


def test_transmissive_corners_are_refused():
    """Transmissive boundaries on two axes meet at box edges, where a stencil needs
    a ghost of a ghost; the planner reports a tree error instead of staging one."""
    from emma_b200 import configs
    t = configs.random_uniform(level=4).build()
    st = (ctypes.c_longlong * 5)()
    assert lib().emma_hydro_plan_stats(t.firstoct, 4, 4, 0x3F, st) & 0x08
    assert lib().emma_hydro_plan_stats(t.firstoct, 4, 4, 0x0F, st) & 0x08
    lib().emma_hydro_clear_status()
    assert lib().emma_hydro_plan_stats(t.firstoct, 4, 4, 0x03, st) == 0


@pytest.mark.parametrize("part", ["halves", "quadrants", "stripes3"])
def test_multi_rank_tree_plans_this_ranks_octs(part):
    """Octs of other ranks (a multi-rank run's boundary octs) are staged as
    neighbours and never tiled: the plan of rank 0 covers exactly its own octs
    and leaf cells."""
    from helpers import PARTITIONS, assign_ranks, rank_of_octs
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    t = cfg.build()
    nrank, fn = PARTITIONS[part]
    assign_ranks(t, fn)
    rc, stats = plan_stats(cfg, t)
    assert rc == 0, lib().emma_hydro_last_error()
    for i, (octs, tiles, max_staged, staged, leaf) in enumerate(stats):
        l = cfg.lcoarse + i
        own = rank_of_octs(t, l, fn) == 0
        assert octs == own.sum()
        leaves = ~t.split_mask(l).reshape(-1, 8)
        assert leaf == leaves[own].sum()
        assert (tiles > 0) == (octs > 0)
