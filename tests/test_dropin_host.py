"""Host passes of the drop-in entries that need no GPU: clean_new_hydro
(src/hydro_utils.c:3501-3522: fieldnew := field on every cell of the level) over
the library's cached walk of the level's oct list.

A list of at least 32,768 octs that is unchanged since the previous walk is
confirmed in parallel (each oct's `next` against the cached walk) instead of
walked again; a list that changed (cells refined since, or another tree at the
same addresses) must be walked afresh.  Every case checks fieldnew == field bit
for bit on every cell of the level.  A multi-rank clean also zeroes the coarser
level's octs of other ranks (src/hydro_utils.c:3524-3544).
"""
import numpy as np

from emma_b200 import OctTree
from emma_b200.hydro import clean_new_hydro


def scramble_and_clean(t, level, rng):
    f = t.get_fields(level, 0)
    t.put_fields(level, rng.uniform(-1.0, 1.0, f.shape), which=1)
    clean_new_hydro(level, t.firstoct)
    g = t.get_fields(level, 1)
    assert np.array_equal(f.view(np.uint64), g.view(np.uint64))


def fill(t, level, rng):
    n8 = 8 * t.noct(level)
    t.set_fields(level, rng.uniform(0.5, 1.5, n8), rng.uniform(-0.5, 0.5, n8), rng.uniform(-0.5, 0.5, n8),
                 rng.uniform(-0.5, 0.5, n8), rng.uniform(0.5, 1.5, n8))


def test_clean_new_hydro_over_cached_and_changed_lists():
    rng = np.random.default_rng(7)
    t = OctTree(6, 7)
    assert t.noct(6) == 32768
    fill(t, 6, rng)
    for _ in range(3):  # the first walk, then confirmed
        scramble_and_clean(t, 6, rng)
    t.refine_where(6, lambda c: c[:, 0] < 0.25)
    n7 = t.noct(7)
    assert n7 >= 32768
    fill(t, 7, rng)
    scramble_and_clean(t, 7, rng)
    scramble_and_clean(t, 7, rng)
    # more level-7 octs: the cached walk of level 7 no longer matches the list
    t.refine_where(6, lambda c: (c[:, 0] >= 0.25) & (c[:, 0] < 0.375))
    assert t.noct(7) > n7
    fill(t, 7, rng)
    scramble_and_clean(t, 7, rng)
    scramble_and_clean(t, 6, rng)
    t.close()
    # another tree, possibly at the same addresses, with a shorter level-6 list
    # head: whatever the cached walk holds, the new list is walked
    t2 = OctTree(6, 7)
    t2.refine_where(6, lambda c: c[:, 1] < 0.5)
    fill(t2, 6, rng)
    fill(t2, 7, rng)
    for level in (6, 7, 7, 6):
        scramble_and_clean(t2, level, rng)
    t2.close()


def test_clean_new_hydro_zeroes_coarser_octs_of_other_ranks():
    """A -DWMPI rank's clean_new_hydro of level L > lcoarse also zeroes fieldnew of
    the level L-1 octs it does not own (src/hydro_utils.c:3524-3544) and leaves its
    own as they were."""
    from emma_b200 import hydro as H
    rng = np.random.default_rng(11)
    t = OctTree(6, 7)
    t.refine_where(6, lambda c: c[:, 2] < 0.5)
    fill(t, 6, rng)
    fill(t, 7, rng)
    ranks = rng.integers(0, 3, t.noct(6)).astype(np.int32)
    t.set_cpu(6, ranks)
    before = t.get_fields(6, 1)
    H.clean_new_hydro(7, t.firstoct, cpu=H.CpuInfo(rank=1, nproc=3), param=H.RunParams(lcoarse=6, lmax=7))
    after = t.get_fields(6, 1)
    other = np.repeat(ranks != 1, 8)
    assert np.all(after[:, other] == 0.0)
    assert np.array_equal(after[:, ~other], before[:, ~other])
    # level 7 itself: fieldnew := field
    assert np.array_equal(t.get_fields(7, 0), t.get_fields(7, 1))
    t.close()
