"""Edge cases of the CUDA path: bounded device waits, corrupted states reported as
status bits, invalid arguments, empty levels, the smallest domain."""
import ctypes

import numpy as np
import pytest

import oracle
from emma_b200 import configs, OctTree, PREC_FP64, PREC_MIXED, ResidentHydro
from emma_b200._lib import lib, ST_ARG, ST_NAN, ST_NEG_DENSITY, ST_TIMEOUT
from emma_b200 import hydro as H
from helpers import per_cell_rel

pytestmark = pytest.mark.gpu
CFL = 0.8


def oracle_state(cfg, nsteps, tree=None):
    t = tree if tree is not None else cfg.build()
    tsim, _, err = oracle.Restatement().run(t.firstoct, cfg.lcoarse, cfg.lmax, nsteps, CFL, trans=cfg.trans,
                                           nsub=cfg.nsub)
    assert err == 0
    return t, tsim


def test_bounded_wait_reports_timeout_and_context_survives(gpu):
    """A level update waiting for a count nothing reaches gives up after the bound,
    reports EMMA_ST_TIMEOUT, and the library keeps working."""
    cfg = configs.small_amr()
    t = cfg.build()
    r = ResidentHydro(t, precision=PREC_FP64, cfl=CFL)
    bits = lib().emma_hydro_probe_wait_timeout(2000)
    assert bits & ST_TIMEOUT
    assert r.status() == 0  # the probe leaves the sticky status as it was
    r.coarse_step()
    assert r.status() == 0
    r.download()
    to, tsim = oracle_state(cfg, 1)
    assert r.tsim == tsim
    for l in range(cfg.lcoarse, cfg.lmax + 1):
        assert per_cell_rel(t.get_fields(l)[:5], to.get_fields(l)[:5]).max() <= 1e-12


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_corrupted_state_is_reported_not_fatal(gpu, precision):
    """Negative density and NaN pressure (the reference aborts) set status bits."""
    cfg = configs.random_uniform(level=4)
    r = ResidentHydro(cfg.build(), precision=precision, cfl=CFL, use_graph=False)
    st = r.state(4)
    st[0, 10] = -1.0
    st[4, 200] = np.nan
    r.set_state(4, st)
    lib().emma_hydro_clear_status()
    r.advance_level(4, 1e-3)
    bits = r.status()
    assert bits & (ST_NEG_DENSITY | ST_NAN)
    lib().emma_hydro_clear_status()
    assert r.status() == 0


def test_invalid_arguments_are_refused(gpu):
    cfg = configs.random_uniform(level=3)
    t = cfg.build()
    r = ResidentHydro(t, precision=PREC_FP64, cfl=CFL)
    L = lib()
    assert L.emma_hydro_advance_level(99, 1e-3) == ST_ARG
    assert L.emma_hydro_comptstep(3, None) == ST_ARG
    assert L.emma_hydro_get_level_state(3, None) == ST_ARG
    assert L.emma_hydro_tree_upload(t.firstoct, 1, 3, 0) == ST_ARG       # lcoarse below 2
    assert L.emma_hydro_tree_upload(t.firstoct, 3, 40, 0) == ST_ARG      # lmax beyond the level slots
    o = H.options(PREC_FP64, 0, CFL, tile_octs=16)                       # no such brick
    L.emma_hydro_set_options(ctypes.byref(o))
    assert L.emma_hydro_tree_upload(t.firstoct, 3, 3, 0) == ST_ARG
    L.emma_hydro_clear_status()


def test_empty_finer_levels(gpu):
    """lmax above the finest populated level: the empty levels are skipped as the
    reference's schedule skips them."""
    base, radii, lmax = 4, (0.3, 0.15), 8
    def build():
        t = OctTree(base, lmax)
        for i, rr in enumerate(radii):
            t.refine_where(base + i, lambda c, rr=rr: np.linalg.norm(c - 0.5, axis=1) < rr)
        rng = np.random.default_rng(7)
        for lev in range(base, base + len(radii) + 1):
            n8 = 8 * t.noct(lev)
            t.set_fields(lev, rng.uniform(0.5, 1.5, n8), rng.uniform(-.3, .3, n8), rng.uniform(-.3, .3, n8),
                         rng.uniform(-.3, .3, n8), rng.uniform(0.5, 1.5, n8))
        return t
    t = build()
    assert t.noct(lmax) == 0
    r = ResidentHydro(t, precision=PREC_FP64, cfl=CFL)
    r.coarse_step()
    assert r.status() == 0
    r.download()
    to = build()
    tsim, _, err = oracle.Restatement().run(to.firstoct, base, lmax, 1, CFL)
    assert err == 0 and r.tsim == tsim
    for l in range(base, base + len(radii) + 1):
        assert per_cell_rel(t.get_fields(l)[:5], to.get_fields(l)[:5]).max() <= 1e-12


@pytest.mark.parametrize("tile_octs", [32, 8])
def test_smallest_domain(gpu, tile_octs):
    """Level 2 (4^3 cells, 8 octs): the brick is larger than the periodic domain, so
    its ring wraps onto octs of the same brick."""
    cfg = configs.random_uniform(level=2)
    t = cfg.build()
    r = ResidentHydro(t, precision=PREC_FP64, cfl=CFL, tile_octs=tile_octs)
    for _ in range(2):
        r.coarse_step()
    assert r.status() == 0
    r.download()
    to, tsim = oracle_state(cfg, 2)
    assert r.tsim == tsim
    assert per_cell_rel(t.get_fields(2)[:5], to.get_fields(2)[:5]).max() <= 1e-12


def _interior_refined_tree():
    """Refined spheres about the centre with random fields inside 0.25 < x < 0.75 and a
    uniform state next to the x boundaries: the transmissive ghosts then see a state
    uniform along the boundary, where the device's ghost edges equal the reference's
    (the order-dependent edge fill of the reference differs only for states that vary
    along a transmissive boundary)."""
    base, lmax, radii = 5, 7, (0.22, 0.12)

    def build():
        t = OctTree(base, lmax)
        for i, rr in enumerate(radii):
            t.refine_where(base + i, lambda c, rr=rr: np.linalg.norm(c - 0.5, axis=1) < rr)
        rng = np.random.default_rng(11)
        for lev in range(base, lmax + 1):
            c = t.cell_centres(lev)
            n8 = len(c)
            inner = np.abs(c[:, 0] - 0.5) < 0.25
            f = [rng.uniform(0.5, 1.5, n8), rng.uniform(-.3, .3, n8), rng.uniform(-.3, .3, n8),
                 rng.uniform(-.3, .3, n8), rng.uniform(0.5, 1.5, n8)]
            for k, v in enumerate((1.0, 0.1, 0.0, 0.0, 1.0)):
                f[k] = np.where(inner, f[k], v)
            t.set_fields(lev, *f)
        return t
    return base, lmax, build


@pytest.mark.parametrize("nsub", [2, 1])
def test_fp64_transmissive_amr_interpolates_coarse_neighbours(gpu, nsub):
    """The transmissive build gathers coarser neighbours by limited interpolation
    (coarse2fine_hydro2); FP64 parity with the oracle, which follows the reference's
    HYDROTEST gather bit for bit."""
    base, lmax, build = _interior_refined_tree()
    t = build()
    r = ResidentHydro(t, precision=PREC_FP64, trans=0x3, cfl=CFL)
    for _ in range(2):
        r.coarse_step(nsub=nsub)
    assert r.status() == 0
    r.download()
    to = build()
    tsim, _, err = oracle.Restatement().run(to.firstoct, base, lmax, 2, CFL, trans=0x3, nsub=nsub)
    assert err == 0 and r.tsim == tsim
    for l in range(base, lmax + 1):
        assert per_cell_rel(t.get_fields(l)[:5], to.get_fields(l)[:5]).max() <= 1e-12, l


def test_mixed_transmissive_amr(gpu):
    base, lmax, build = _interior_refined_tree()
    t = build()
    r = ResidentHydro(t, precision=PREC_MIXED, trans=0x3, cfl=CFL)
    for _ in range(3):
        r.coarse_step()
    assert r.status() == 0
    r.download()
    to = build()
    _, _, err = oracle.Restatement().run(to.firstoct, base, lmax, 3, CFL, trans=0x3)
    assert err == 0
    from helpers import l1_rel
    for l in range(base, lmax + 1):
        leaf = ~to.split_mask(l)
        assert l1_rel(t.get_fields(l)[0][leaf], to.get_fields(l)[0][leaf]) <= 1e-5
        assert l1_rel(t.get_fields(l)[4][leaf], to.get_fields(l)[4][leaf]) <= 1e-5
