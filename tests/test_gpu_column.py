"""Column kernel of the mixed path: complete periodic levels without split cells,
16 x 16-cell columns marching through z (emma_b200/csrc/column_kernel.cuh).

Against the FP64 oracle: L1 of density, pressure and |v| <= 1e-5 after three
steps, mass and total energy conserved to 1e-12 (every face is solved once
per column and the boundary faces of two columns or z chunks get the same
bits from both).  Against the brick kernel of the same path: L1 <= 1e-6.  The
next step's dt from the maximum fused into the kernel equals the FP64
reduction's over the state it wrote, bit for bit.  The warp-shuffle x sweep
(x face states passed up a lane, the column's x boundary faces solved by the
ring threads) meets the same bars and matches the shared-memory sweep.  Balanced
runs of column-planes per CTA (segments that start and end anywhere in a column)
give the same bits as items of a fixed depth.
"""
import numpy as np
import pytest

import oracle
from emma_b200 import configs, PREC_MIXED, ResidentHydro
from helpers import l1_rel

pytestmark = pytest.mark.gpu
CFL = 0.8
GAMMA = 5.0 / 3.0


def totals(f, level):
    dv = 0.5 ** (3 * level)
    m = f[0].sum() * dv
    e = (f[4] / (GAMMA - 1.0) + 0.5 * f[0] * (f[1] ** 2 + f[2] ** 2 + f[3] ** 2)).sum() * dv
    return m, e


def l1_fields(a, b):
    va, vb = np.sqrt((a[1:4] ** 2).sum(0)), np.sqrt((b[1:4] ** 2).sum(0))
    return l1_rel(a[0], b[0]), l1_rel(a[4], b[4]), l1_rel(va, vb)


@pytest.mark.parametrize("level,nz", [(4, 2), (5, 8), (6, 16), (6, 64), (7, 32)])
def test_column_mixed_against_oracle(gpu, level, nz):
    cfg = configs.random_uniform(level=level)
    t = cfg.build()
    f0 = t.get_fields(level)[:5]
    m0, e0 = totals(f0, level)
    r = ResidentHydro(t, precision=PREC_MIXED, cfl=CFL, column=nz)
    assert r.column_tuning(level)[0] == nz
    for _ in range(3):
        r.coarse_step()
    assert r.status() == 0
    fm = r.state(level)
    m1, e1 = totals(fm, level)
    assert abs(m1 - m0) <= 1e-12 * m0
    assert abs(e1 - e0) <= 1e-12 * e0
    to = cfg.build()
    _, _, err = oracle.Restatement().run(to.firstoct, cfg.lcoarse, cfg.lmax, 3, CFL)
    assert err == 0
    for x in l1_fields(fm, to.get_fields(level)[:5]):
        assert x <= 1e-5


@pytest.mark.parametrize("config", ["turb", "random6"])
def test_column_matches_brick_kernel(gpu, config):
    cfg = configs.turb(level=6) if config == "turb" else configs.random_uniform(level=6)
    out = {}
    for col in (-1, 8):
        t = cfg.build()
        r = ResidentHydro(t, precision=PREC_MIXED, cfl=CFL, column=col)
        assert r.column_tuning(cfg.lcoarse)[0] == max(col, 0)
        for _ in range(4):
            r.coarse_step()
        assert r.status() == 0
        out[col] = (r.state(cfg.lcoarse), r.tsim)
    for x in l1_fields(out[8][0], out[-1][0]):
        assert x <= 1e-6
    assert abs(out[8][1] - out[-1][1]) <= 1e-6 * out[-1][1]


def test_column_fused_cfl_is_exact(gpu):
    """The graph's next dt comes from the maximum the column kernel fused (an FP32
    screen, exact FP64 for the candidates); it equals the reduction kernel's."""
    cfg = configs.turb(level=6)
    t = cfg.build()
    r = ResidentHydro(t, precision=PREC_MIXED, cfl=CFL, column=16)
    r.coarse_step()                 # state written by the column kernel
    dt_ref = r.comptstep(cfg.lcoarse)
    r.coarse_step()                 # its dt from the fused maximum
    assert r.adt[cfg.lcoarse - 1] == dt_ref


def test_column_host_schedule_and_graph_agree(gpu):
    """advance_level launches (host-driven schedule) and the captured graph run the
    same column kernel: identical states."""
    cfg = configs.random_uniform(level=5)
    states = []
    for graph in (False, True):
        t = cfg.build()
        r = ResidentHydro(t, precision=PREC_MIXED, cfl=CFL, column=4, use_graph=graph)
        for _ in range(3):
            r.coarse_step()
        states.append((r.state(cfg.lcoarse), r.tsim))
    assert np.array_equal(states[0][0], states[1][0])
    assert states[0][1] == states[1][1]


def test_autotuner_sweeps_the_column_kernel(gpu):
    cfg = configs.random_uniform(level=6)
    r = ResidentHydro(cfg.build(), precision=PREC_MIXED, cfl=CFL)
    planes, sweep = r.column_tuning(cfg.lcoarse)
    assert (sweep > 0).sum() >= 4  # 2, 4, 8, 16, 32, 64 planes: every divisor of 64 cells tried
    octs, ctas, brick = r.tuning(cfg.lcoarse)
    best_brick = brick[brick > 0].min()
    best_col = sweep[sweep > 0].min()
    xs, xms = r.column_xshfl(cfg.lcoarse)
    bal, bms = r.column_balanced(cfg.lcoarse)
    # the shuffle x sweep timed at the best depth against the shared-memory one,
    # then balanced runs (with the faster sweep) against the items
    assert xms[0] == best_col and xms[1] > 0
    assert bms[0] == min(xms) and bms[1] > 0
    best = min(bms)
    if planes:
        assert sweep[[2, 4, 8, 16, 32, 64].index(planes)] == best_col
        assert xs == (1 if xms[1] < xms[0] else 0)
        assert bal == (1 if bms[1] < bms[0] else 0)
        assert best <= best_brick
    else:
        assert xs == 0 and bal == 0 and best >= best_brick


@pytest.mark.parametrize("level,xs", [(5, -1), (6, 1), (7, -1), (7, 1)])
def test_column_balanced_runs_equal_items(gpu, level, xs):
    cfg = configs.random_uniform(level=level)
    out = {}
    for bal in (-1, 1):
        t = cfg.build()
        m0, e0 = totals(t.get_fields(level)[:5], level)
        r = ResidentHydro(t, precision=PREC_MIXED, cfl=CFL, column=8, xshfl=xs, balanced=bal)
        assert r.column_balanced(level)[0] == (1 if bal > 0 else 0)
        for _ in range(3):
            r.coarse_step()
        assert r.status() == 0
        fm = r.state(level)
        m1, e1 = totals(fm, level)
        assert abs(m1 - m0) <= 1e-12 * m0
        assert abs(e1 - e0) <= 1e-12 * e0
        out[bal] = (fm, r.tsim)
    assert np.array_equal(out[1][0], out[-1][0])
    assert out[1][1] == out[-1][1]


@pytest.mark.parametrize("level,nz,with_oracle", [(5, 8, True), (6, 16, True), (7, 32, False)])
def test_column_warp_shuffle_x_sweep(gpu, level, nz, with_oracle):
    cfg = configs.random_uniform(level=level)
    out = {}
    for xs in (-1, 1):
        t = cfg.build()
        m0, e0 = totals(t.get_fields(level)[:5], level)
        r = ResidentHydro(t, precision=PREC_MIXED, cfl=CFL, column=nz, xshfl=xs)
        assert r.column_tuning(level)[0] == nz
        assert r.column_xshfl(level)[0] == (1 if xs > 0 else 0)
        for _ in range(3):
            r.coarse_step()
        assert r.status() == 0
        fm = r.state(level)
        m1, e1 = totals(fm, level)
        assert abs(m1 - m0) <= 1e-12 * m0
        assert abs(e1 - e0) <= 1e-12 * e0
        out[xs] = (fm, r.tsim)
    for x in l1_fields(out[1][0], out[-1][0]):
        assert x <= 1e-6
    assert abs(out[1][1] - out[-1][1]) <= 1e-6 * out[-1][1]
    if with_oracle:
        to = cfg.build()
        _, _, err = oracle.Restatement().run(to.firstoct, cfg.lcoarse, cfg.lmax, 3, CFL)
        assert err == 0
        for x in l1_fields(out[1][0], to.get_fields(level)[:5]):
            assert x <= 1e-5
