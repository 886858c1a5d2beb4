"""Gravity-coupled hydro (the reference's -DWGRAV build) on the GPU vs the oracle.

The oracle is the gravity restatement (oracle/hydro_oracle.c built with
-DORC_WGRAV, pinned bit for bit to the reference's -DWGRAV hydro in
tests/test_oracle_pin.py) run on a copy of the same tree in the gravity cell
layout.  The GPU runs the resident path with the accelerations uploaded per
level: half-step kick of the MUSCL face velocities, forces of injected coarser
cells spread by coarse2fine_forcelin, grav_correction after each level update.
FP64: per-cell relative error <= 1e-12 after one coarse step; mixed: L1 <= 1e-5.
"""
import numpy as np
import pytest

import oracle
from emma_b200 import configs, PREC_FP64, PREC_MIXED, ResidentHydro, lib
from emma_b200._lib import ST_ARG
from helpers import per_cell_rel, l1_rel

pytestmark = pytest.mark.gpu
CFL = 0.8


def forces(tree, levels, seed=2024, amp=0.5):
    """Smooth acceleration field (a few Fourier modes) plus a small random part."""
    rng = np.random.default_rng(seed)
    out = {}
    for l in levels:
        c = tree.cell_centres(l)
        two_pi = 2 * np.pi
        fx = amp * np.sin(two_pi * c[:, 1]) + 0.1 * amp * rng.uniform(-1, 1, len(c))
        fy = amp * np.cos(two_pi * c[:, 2]) + 0.1 * amp * rng.uniform(-1, 1, len(c))
        fz = amp * np.sin(two_pi * (c[:, 0] + c[:, 1])) + 0.1 * amp * rng.uniform(-1, 1, len(c))
        out[l] = (fx, fy, fz)
    return out


def run_pair(cfg, nsteps, precision=PREC_FP64, tile_octs=0, amp=0.5):
    levels = range(cfg.lcoarse, cfg.lmax + 1)
    tg = cfg.build()
    f = forces(tg, levels, amp=amp)
    lib().emma_hydro_clear_status()
    r = ResidentHydro(tg, precision=precision, cfl=CFL, tile_octs=tile_octs, gravity=True)
    for l in levels:
        r.set_force(l, *f[l])
    for _ in range(nsteps):
        r.coarse_step(nsub=cfg.nsub)
    st = r.status()
    gpu = {l: r.state(l) for l in levels}
    gc = oracle.GravClone(cfg.build())
    for l in levels:
        gc.set_force(l, *f[l])
    tsim, adt, err = gc.run(nsteps, CFL, nsub=cfg.nsub)
    assert err == 0
    ora = {l: gc.get_fields(l)[:5] for l in levels}
    return r, st, gpu, ora, tsim


@pytest.mark.parametrize("tile_octs", [32, 8])
def test_gravity_fp64_uniform(gpu, tile_octs):
    cfg = configs.random_uniform(level=4)
    r, st, g, o, tsim = run_pair(cfg, 1, tile_octs=tile_octs)
    assert st == 0
    assert r.tsim == tsim
    e = per_cell_rel(g[4], o[4])
    assert e.max() <= 1e-12, e.max()


@pytest.mark.parametrize("tile_octs", [0, 32, 8])
def test_gravity_fp64_amr(gpu, tile_octs):
    """Refined levels: injected coarser cells carry interpolated forces."""
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    r, st, g, o, tsim = run_pair(cfg, 1, tile_octs=tile_octs)
    assert st == 0
    assert r.tsim == tsim
    for l in range(cfg.lcoarse, cfg.lmax + 1):
        e = per_cell_rel(g[l], o[l])
        assert e.max() <= 1e-12, (l, e.max())


def test_gravity_fp64_amr_several_steps(gpu):
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    r, st, g, o, tsim = run_pair(cfg, 4)
    assert st == 0
    assert abs(r.tsim - tsim) <= 1e-14 * tsim
    for l in range(cfg.lcoarse, cfg.lmax + 1):
        e = per_cell_rel(g[l], o[l])
        assert e.max() <= 1e-10, (l, e.max())


def test_gravity_mixed_l1(gpu):
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    r, st, g, o, tsim = run_pair(cfg, 3, precision=PREC_MIXED)
    assert st == 0
    for l in range(cfg.lcoarse, cfg.lmax + 1):
        assert l1_rel(g[l][0], o[l][0]) <= 1e-5, l
        assert l1_rel(g[l][4], o[l][4]) <= 1e-5, l
        vg = np.sqrt((g[l][1:4] ** 2).sum(0))
        vo = np.sqrt((o[l][1:4] ** 2).sum(0))
        assert l1_rel(vg, vo) <= 1e-5, l


def test_gravity_with_zero_force_is_plain_hydro(gpu):
    """gravity=True with zero accelerations reproduces the plain path (to the
    last bits of the fine->coarse corrections, which are atomic sums)."""
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    levels = range(cfg.lcoarse, cfg.lmax + 1)
    out = []
    for grav in (False, True):
        r = ResidentHydro(cfg.build(), precision=PREC_FP64, cfl=CFL, gravity=grav)
        for _ in range(2):
            r.coarse_step(nsub=cfg.nsub)
        assert r.status() == 0
        out.append({l: r.state(l) for l in levels})
    for l in levels:
        assert per_cell_rel(out[1][l], out[0][l]).max() <= 1e-13, l


def test_gravity_changes_the_solution(gpu):
    cfg = configs.random_uniform(level=4)
    r, st, g, o, tsim = run_pair(cfg, 1, amp=2.0)
    r0 = ResidentHydro(cfg.build(), precision=PREC_FP64, cfl=CFL)
    r0.coarse_step(nsub=cfg.nsub)
    assert np.abs(r0.state(4) - g[4]).max() > 1e-6


def test_gravity_refused_with_transmissive_boundaries(gpu):
    cfg = configs.sod(level=4)
    lib().emma_hydro_clear_status()
    with pytest.raises(RuntimeError):
        ResidentHydro(cfg.build(), precision=PREC_FP64, trans=cfg.trans, cfl=CFL, gravity=True)
    assert lib().emma_hydro_status() & ST_ARG
    lib().emma_hydro_clear_status()


def test_set_force_needs_a_gravity_upload(gpu):
    cfg = configs.random_uniform(level=3)
    r = ResidentHydro(cfg.build(), precision=PREC_FP64, cfl=CFL)
    n8 = 8 * r.noct(3)
    with pytest.raises(RuntimeError):
        r.set_force(3, np.zeros(n8), np.zeros(n8), np.zeros(n8))
    lib().emma_hydro_clear_status()


def test_dropin_gravity_matches_oracle(gpu):
    """libemmahydro_grav.so (the reference's -DWGRAV cell layout): drop-in
    HydroSolver + grav_correction level by level, as Advance_level calls them,
    on the caller's tree, against the gravity oracle on an identical tree."""
    from emma_b200 import OctTree
    from emma_b200 import hydro as H
    from test_oracle_pin import random_fields, random_forces

    def build():
        t = OctTree(4, 6, grav=True)
        for i, rad in enumerate((0.3, 0.15)):
            t.refine_where(4 + i, lambda c, rad=rad: np.linalg.norm(c - 0.5, axis=1) < rad)
        random_fields(t, range(4, 7))
        random_forces(t, range(4, 7))
        return t

    tg, to = build(), build()
    R = oracle.Restatement(grav=True)
    L = lib(True)
    L.emma_hydro_clear_status()
    dts = {4: 2e-3, 5: 1e-3, 6: 5e-4}
    for l in (4, 5, 6):
        H.clean_new_hydro(l, tg.firstoct, grav=True)
        R.clean_new(to.firstoct, l)
    for l in (6, 6, 5, 6, 6, 5, 4):
        H.HydroSolver(l, tg.firstoct, dts[l], grav=True)
        H.grav_correction(l, tg.firstoct, dts[l])
        assert R.hydro_solver(to.firstoct, l, dts[l]) == 0
        assert R.grav_correction(to.firstoct, l, dts[l]) == 0
    assert L.emma_hydro_status() == 0, L.emma_hydro_last_error()
    for l in (4, 5, 6):
        e = per_cell_rel(tg.get_fields(l)[:5], to.get_fields(l)[:5])
        assert e.max() <= 1e-12, (l, e.max())


@pytest.mark.parametrize("use_graph", [True, False])
def test_gravity_single_substep_batched_and_host_schedules(gpu, use_graph):
    """nsub = 1 (one batched launch over all levels on the graph schedule) and the
    host-driven schedule, both against the gravity oracle."""
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    levels = range(cfg.lcoarse, cfg.lmax + 1)
    tg = cfg.build()
    f = forces(tg, levels)
    r = ResidentHydro(tg, precision=PREC_FP64, cfl=CFL, gravity=True, use_graph=use_graph)
    for l in levels:
        r.set_force(l, *f[l])
    for _ in range(3):
        r.coarse_step(nsub=1)
    assert r.status() == 0
    gc = oracle.GravClone(cfg.build())
    for l in levels:
        gc.set_force(l, *f[l])
    tsim, adt, err = gc.run(3, CFL, nsub=1)
    assert err == 0 and abs(r.tsim - tsim) <= 1e-14 * tsim
    for l in levels:
        e = per_cell_rel(r.state(l), gc.get_fields(l)[:5])
        assert e.max() <= 1e-10, (l, e.max())
