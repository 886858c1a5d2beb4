"""Parity of the CUDA path (libemmahydro) with the oracle.

FP64 plain path: per-cell relative error <= 1e-12 after one coarse step
(velocities relative to |v| + c_s), tree/flags/order identical by construction.
Mixed path: L1 density/pressure/velocity error vs the FP64 oracle <= 1e-5 and
mass conservation to 1e-12 on periodic boxes.
"""
import os

import numpy as np
import pytest

import oracle
from emma_b200 import configs, PREC_FP64, PREC_MIXED, ResidentHydro, OctTree
from emma_b200 import hydro as H
from helpers import per_cell_rel, l1_rel

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CFL = 0.8


def run_gpu(cfg, nsteps, precision=PREC_FP64, tile_octs=0):
    t = cfg.build()
    r = ResidentHydro(t, precision=precision, trans=cfg.trans, cfl=CFL, tile_octs=tile_octs)
    for _ in range(nsteps):
        r.coarse_step(nsub=cfg.nsub)
    st = r.status()
    r.download()
    return t, r, st


def run_oracle(cfg, nsteps):
    t = cfg.build()
    tsim, adt, err = oracle.Restatement().run(t.firstoct, cfg.lcoarse, cfg.lmax, nsteps, CFL, trans=cfg.trans,
                                              nsub=cfg.nsub)
    assert err == 0
    return t, tsim


def assert_close(tg, to, levels, tol):
    worst = 0.0
    for l in levels:
        e = per_cell_rel(tg.get_fields(l)[:5], to.get_fields(l)[:5])
        worst = max(worst, float(e.max()))
    assert worst <= tol, f"max per-cell relative error {worst:.3e} > {tol:.0e}"
    return worst


@pytest.mark.parametrize("level", [3, 4, 5])
def test_fp64_uniform_one_step(gpu, level):
    cfg = configs.random_uniform(level=level)
    tg, r, st = run_gpu(cfg, 1)
    assert st == 0
    to, tsim = run_oracle(cfg, 1)
    assert r.tsim == tsim
    assert_close(tg, to, [level], 1e-12)


def test_fp64_uniform_ten_steps(gpu):
    cfg = configs.random_uniform(level=4)
    tg, r, st = run_gpu(cfg, 10)
    assert st == 0
    to, tsim = run_oracle(cfg, 10)
    assert abs(r.tsim - tsim) <= 1e-14 * tsim
    assert_close(tg, to, [4], 1e-10)


def test_fp64_sod_tube(gpu):
    cfg = configs.sod(level=5)
    tg, r, st = run_gpu(cfg, 1)
    assert st == 0
    to, tsim = run_oracle(cfg, 1)
    assert_close(tg, to, [5], 1e-12)
    tg, r, st = run_gpu(cfg, 30)
    to, tsim = run_oracle(cfg, 30)
    assert_close(tg, to, [5], 1e-10)


@pytest.mark.parametrize("base,radii", [(4, (0.3, 0.15)), (3, (0.35, 0.2))])
def test_fp64_amr_one_step(gpu, base, radii):
    cfg = configs.small_amr(base=base, radii=radii)
    tg, r, st = run_gpu(cfg, 1)
    assert st == 0
    to, tsim = run_oracle(cfg, 1)
    assert r.tsim == tsim
    assert_close(tg, to, range(cfg.lcoarse, cfg.lmax + 1), 1e-12)


def test_fp64_sedov_one_step(gpu):
    cfg = configs.sedov()
    tg, r, st = run_gpu(cfg, 1)
    assert st == 0
    to, tsim = run_oracle(cfg, 1)
    assert_close(tg, to, range(cfg.lcoarse, cfg.lmax + 1), 1e-12)


def test_fp64_amr_mass_energy_conservation(gpu):
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    t = cfg.build()

    def totals(tree):
        m = e = 0.0
        for l in range(cfg.lcoarse, cfg.lmax + 1):
            f = tree.get_fields(l)
            leaf = ~tree.split_mask(l)
            dv = 0.5 ** (3 * l)
            m += f[0][leaf].sum() * dv
            e += f[6][leaf].sum() * dv
        return m, e

    m0, e0 = totals(t)
    r = ResidentHydro(t, precision=PREC_FP64, cfl=CFL)
    for _ in range(3):
        r.coarse_step()
    r.download()
    m1, e1 = totals(t)
    assert abs(m1 - m0) <= 1e-12 * m0
    assert abs(e1 - e0) <= 1e-12 * e0


def test_dropin_hydrosolver_matches_oracle(gpu):
    """The reference-named entries on a host tree, level by level, as Advance_level calls them."""
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    tg, to = cfg.build(), cfg.build()
    R = oracle.Restatement()
    H.lib().emma_hydro_clear_status()
    dts = {4: 2e-3, 5: 1e-3, 6: 5e-4}
    for tree_is_gpu, t in ((True, tg), (False, to)):
        for l in (4, 5, 6):
            if tree_is_gpu:
                H.clean_new_hydro(l, t.firstoct)
            else:
                R.clean_new(t.firstoct, l)
        for l in (6, 6, 5, 6, 6, 5, 4):
            if tree_is_gpu:
                H.HydroSolver(l, t.firstoct, dts[l])
            else:
                assert R.hydro_solver(t.firstoct, l, dts[l]) == 0
            if l == 6 and tree_is_gpu is False:
                pass
    assert H.lib().emma_hydro_status() == 0
    for l in (4, 5, 6):
        e = per_cell_rel(tg.get_fields(l)[:5], to.get_fields(l)[:5])
        assert e.max() <= 1e-12, (l, e.max())


def test_dropin_advancehydrogpu_writes_fieldnew_only(gpu):
    """advancehydroGPU alone (src/hydro_utils_gpu.cu:2470): fieldnew of the level's
    leaves and the coarser level's corrected cells equal the oracle's HydroSolver
    result; `field` stays as it was."""
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    tg, to = cfg.build(), cfg.build()
    R = oracle.Restatement()
    H.lib().emma_hydro_clear_status()
    for l in (4, 5, 6):
        H.clean_new_hydro(l, tg.firstoct)
        R.clean_new(to.firstoct, l)
    before = tg.get_fields(6)
    for l in (6, 5):
        assert H.advancehydroGPU(tg.firstoct, l, 1e-3) == tg.noct(l)
        assert R.hydro_solver(to.firstoct, l, 1e-3) == 0
    assert H.lib().emma_hydro_status() == 0
    assert np.array_equal(tg.get_fields(6), before)
    for l in (5, 6):
        leaf = ~tg.split_mask(l)
        e = per_cell_rel(tg.get_fields(l, which=1)[:5][:, leaf], to.get_fields(l, which=1)[:5][:, leaf])
        assert e.max() <= 1e-12, (l, e.max())
    # level 4 received level 5's fine->coarse corrections in fieldnew
    e = per_cell_rel(tg.get_fields(4, which=1)[:5], to.get_fields(4, which=1)[:5])
    assert e.max() <= 1e-12, e.max()


def test_mixed_precision_l1_and_conservation(gpu):
    cfg = configs.random_uniform(level=5)
    tm, r, st = run_gpu(cfg, 10, precision=PREC_MIXED)
    assert st == 0
    to, tsim = run_oracle(cfg, 10)
    fm, fo = tm.get_fields(5), to.get_fields(5)
    assert l1_rel(fm[0], fo[0]) <= 1e-5
    assert l1_rel(fm[4], fo[4]) <= 1e-5
    vm = np.sqrt(fm[1] ** 2 + fm[2] ** 2 + fm[3] ** 2)
    vo = np.sqrt(fo[1] ** 2 + fo[2] ** 2 + fo[3] ** 2)
    assert l1_rel(vm, vo) <= 1e-5
    t0 = cfg.build()
    m0 = t0.get_fields(5)[0].sum()
    e0 = t0.get_fields(5)[6].sum()
    assert abs(fm[0].sum() - m0) <= 1e-12 * m0
    assert abs(fm[6].sum() - e0) <= 1e-12 * e0


def _golden_cases():
    return sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz"))


@pytest.mark.parametrize("name", _golden_cases())
def test_gpu_reproduces_golden(gpu, name):
    """The reference's own outputs (tests/golden) from the resident GPU path of the
    same build variant: default, -DDUAL_E (option), -DWGRAV (the fixture's forces
    uploaded per level), -DWRADHYD (a tree of that layout, dX compared too) and
    -DWRADHYD -DHELIUM (its three tracers compared)."""
    g = np.load(os.path.join(GOLDEN, name))
    base, lmax, nsteps, trans = (int(x) for x in g["meta"][:4])
    variant = int(g["meta"][4]) if len(g["meta"]) > 4 else 0
    t = OctTree(base, lmax, rh=variant == 3, he=variant == 4)
    for i, rr in enumerate(tuple(g["radii"])):
        t.refine_where(base + i, lambda c, rr=rr: np.linalg.norm(c - 0.5, axis=1) < rr)
    for l in range(base, lmax + 1):
        t.set_fields(l, *g[f"in_{l}"][:5])
        if variant == 3:
            t.set_tracer(l, g[f"in_x_{l}"])
        if variant == 4:
            for tr in range(3):
                t.set_tracer_n(l, tr, g[f"in_x_{l}"][tr])
    r = ResidentHydro(t, precision=PREC_FP64, trans=trans, cfl=CFL, gravity=variant == 2, dual=variant == 1)
    if variant == 2:
        for l in range(base, lmax + 1):
            r.set_force(l, *g[f"in_f_{l}"])
    for _ in range(nsteps):
        r.coarse_step()
    assert r.status() == 0
    r.download()
    for l in range(base, lmax + 1):
        e = per_cell_rel(t.get_fields(l)[:5], g[f"out_{l}"][:5])
        assert e.max() <= 1e-11, (l, e.max())
        if variant in (3, 4):
            d = g[f"out_{l}"][0]
            leaf = ~t.split_mask(l)
            outs = [g[f"out_x_{l}"]] if variant == 3 else list(g[f"out_x_{l}"])
            for tr, xo in enumerate(outs):
                x = t.get_tracer_n(l, tr)
                assert (np.abs(x - xo)[leaf] / d[leaf]).max() <= 1e-11, (l, tr)


def _final_states(cfg, nsteps, nsub, use_graph, precision=PREC_FP64):
    t = cfg.build()
    r = ResidentHydro(t, precision=precision, trans=cfg.trans, cfl=CFL, use_graph=use_graph)
    for _ in range(nsteps):
        r.coarse_step(nsub=nsub)
    assert r.status() == 0
    return r.tsim, [r.state(l).copy() for l in range(cfg.lcoarse, cfg.lmax + 1)]


@pytest.mark.parametrize("nsub", [1, 2])
def test_graph_schedule_equals_host_schedule(gpu, nsub):
    """The device-side schedule in a CUDA graph reproduces the host-driven one bit for bit."""
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    t_h, s_h = _final_states(cfg, 3, nsub, use_graph=False)
    t_g, s_g = _final_states(cfg, 3, nsub, use_graph=True)
    # fine->coarse corrections are FP64 atomics: their summation order, and so
    # the last bits of coarse cells next to finer octs, may differ run to run
    assert abs(t_h - t_g) <= 1e-14 * t_h
    for a, b in zip(s_h, s_g):
        assert per_cell_rel(a, b).max() <= 1e-13
    # on a uniform level there are no atomics: bit for bit
    cfg = configs.random_uniform(level=4)
    t_h, s_h = _final_states(cfg, 3, nsub, use_graph=False)
    t_g, s_g = _final_states(cfg, 3, nsub, use_graph=True)
    assert t_h == t_g
    for a, b in zip(s_h, s_g):
        assert np.array_equal(a, b)


def test_batched_one_substep_matches_oracle(gpu):
    """nsub=1: every level advances with the same dt; all levels go through one batched launch."""
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    t = cfg.build()
    r = ResidentHydro(t, precision=PREC_FP64, cfl=CFL, use_graph=True)
    for _ in range(2):
        r.coarse_step(nsub=1)
    assert r.status() == 0
    r.download()
    to = cfg.build()
    tsim, _, err = oracle.Restatement().run(to.firstoct, cfg.lcoarse, cfg.lmax, 2, CFL, nsub=1)
    assert err == 0 and r.tsim == tsim
    assert_close(t, to, range(cfg.lcoarse, cfg.lmax + 1), 1e-12)


def test_async_steps_and_device_time(gpu):
    cfg = configs.random_uniform(level=4)
    t = cfg.build()
    r = ResidentHydro(t, precision=PREC_FP64, cfl=CFL, use_graph=True)
    for _ in range(4):
        r.step_async()
    tsim = r.time()
    to, tsim_o = run_oracle(cfg, 4)
    assert tsim == tsim_o
    r.download()
    assert_close(t, to, [4], 1e-12)


# ---------------------------------------------------------------- brick shapes
# tile_octs=32: 4x4x2-oct bricks, one per tile; 8: 2x2x2-oct bricks, four per
# tile; 0: chosen per level by the autotuner at upload.

@pytest.mark.parametrize("tile_octs", [32, 8])
@pytest.mark.parametrize("base,radii", [(4, (0.3, 0.15)), (3, (0.35, 0.2))])
def test_fp64_amr_one_step_each_shape(gpu, base, radii, tile_octs):
    cfg = configs.small_amr(base=base, radii=radii)
    tg, r, st = run_gpu(cfg, 1, tile_octs=tile_octs)
    assert st == 0
    for l in range(cfg.lcoarse, cfg.lmax + 1):
        assert r.tuning(l)[0] == tile_octs
    to, tsim = run_oracle(cfg, 1)
    assert r.tsim == tsim
    assert_close(tg, to, range(cfg.lcoarse, cfg.lmax + 1), 1e-12)


@pytest.mark.parametrize("cfg", [configs.random_uniform(level=4), configs.sod(level=5)], ids=["uniform", "sod"])
def test_fp64_small_bricks_uniform_and_transmissive(gpu, cfg):
    tg, r, st = run_gpu(cfg, 2, tile_octs=8)
    assert st == 0
    to, tsim = run_oracle(cfg, 2)
    assert r.tsim == tsim
    assert_close(tg, to, [cfg.lcoarse], 1e-12)


def test_mixed_small_bricks_l1_and_conservation(gpu):
    cfg = configs.random_uniform(level=5)
    tm, r, st = run_gpu(cfg, 5, precision=PREC_MIXED, tile_octs=8)
    assert st == 0
    to, _ = run_oracle(cfg, 5)
    fm, fo = tm.get_fields(5), to.get_fields(5)
    assert l1_rel(fm[0], fo[0]) <= 1e-5 and l1_rel(fm[4], fo[4]) <= 1e-5
    f0 = cfg.build().get_fields(5)
    assert abs(fm[0].sum() - f0[0].sum()) <= 1e-12 * f0[0].sum()
    assert abs(fm[6].sum() - f0[6].sum()) <= 1e-12 * f0[6].sum()


def test_autotuner_record_and_batched_step(gpu):
    """The autotuner times every candidate on every level, keeps the fastest, and
    the tuned plans (possibly of both shapes in one batched launch) match the oracle."""
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    t = cfg.build()
    r = ResidentHydro(t, precision=PREC_FP64, cfl=CFL, use_graph=True)
    for l in range(cfg.lcoarse, cfg.lmax + 1):
        octs, ctas, sweep = r.tuning(l)
        assert octs in (32, 8) and ctas >= 1
        tried = sweep[sweep > 0]
        assert tried.size >= 1
        k = 0 if octs == 32 else 1
        assert sweep[k, ctas - 1] == tried.min()
    # the complete base level is only tried with 4x4x2 bricks
    assert r.tuning(cfg.lcoarse)[2][1].max() == 0
    for _ in range(2):
        r.coarse_step(nsub=1)
    assert r.status() == 0
    r.download()
    to = cfg.build()
    tsim, _, err = oracle.Restatement().run(to.firstoct, cfg.lcoarse, cfg.lmax, 2, CFL, nsub=1)
    assert err == 0 and r.tsim == tsim
    assert_close(t, to, range(cfg.lcoarse, cfg.lmax + 1), 1e-12)


@pytest.mark.parametrize("lmax", [7, 8])
def test_fp64_cosmology_tree_one_step(gpu, lmax):
    """Strongly refined tree (density > 8x mean, the reference's 26-neighbour check
    rule), subcycled; the autotuner picks the bricks per level."""
    cfg = configs.cosmo(base=5, lmax=lmax)
    tg, r, st = run_gpu(cfg, 1)
    assert st == 0
    to, tsim = run_oracle(cfg, 1)
    assert r.tsim == tsim
    assert_close(tg, to, range(cfg.lcoarse, cfg.lmax + 1), 1e-12)


def test_mixed_cosmology_tree_l1(gpu):
    cfg = configs.cosmo(base=5, lmax=7)
    tm, r, st = run_gpu(cfg, 3, precision=PREC_MIXED)
    assert st == 0
    to, _ = run_oracle(cfg, 3)
    for l in range(cfg.lcoarse, cfg.lmax + 1):
        leaf = ~to.split_mask(l)
        fm, fo = tm.get_fields(l), to.get_fields(l)
        assert l1_rel(fm[0][leaf], fo[0][leaf]) <= 1e-5
        assert l1_rel(fm[4][leaf], fo[4][leaf]) <= 1e-5


def _totals(states, levels, tree):
    m = e = 0.0
    for l in levels:
        f = states[l]
        leaf = ~tree.split_mask(l)
        dv = 0.5 ** (3 * l)
        m += f[0][leaf].sum() * dv
        e += (f[4] / (5. / 3. - 1.) + 0.5 * f[0] * (f[1] ** 2 + f[2] ** 2 + f[3] ** 2))[leaf].sum() * dv
    return m, e


@pytest.mark.parametrize("config", ["turb", "roofline"])
def test_full_size_conservation_and_mixed_l1(gpu, config):
    """The benchmark workloads at full size (turbulent box 128^3, random box 256^3),
    where the oracle is too slow: size-independent properties.  Mass and total
    energy are conserved to 1e-12 on the periodic box by both paths; the mixed
    path stays within L1 1e-5 of the FP64 path."""
    cfg = configs.turb() if config == "turb" else configs.random_uniform(level=8)
    t = cfg.build()
    levels = [cfg.lcoarse]
    l = cfg.lcoarse
    init = {l: t.get_fields(l)[:5]}
    m0, e0 = _totals(init, levels, t)
    out = {}
    for prec in (PREC_FP64, PREC_MIXED):
        r = ResidentHydro(t, precision=prec, cfl=CFL)
        for _ in range(3):
            r.coarse_step(nsub=cfg.nsub)
        assert r.status() == 0
        out[prec] = {l: r.state(l)}
        m1, e1 = _totals(out[prec], levels, t)
        assert abs(m1 - m0) <= 1e-12 * m0, (prec, m1, m0)
        assert abs(e1 - e0) <= 1e-12 * e0, (prec, e1, e0)
    fm, ff = out[PREC_MIXED][l], out[PREC_FP64][l]
    assert l1_rel(fm[0], ff[0]) <= 1e-5
    assert l1_rel(fm[4], ff[4]) <= 1e-5
    assert l1_rel(np.sqrt((fm[1:4] ** 2).sum(0)), np.sqrt((ff[1:4] ** 2).sum(0))) <= 1e-5


# The benchmark configurations at their stated sizes: FP64 per-cell <= 1e-12 after one
# coarse step against the oracle (the oracle takes ~0.4 s for the Sod tube, ~5 s for
# the 128^3 box, ~40 s for the 256^3 box and ~60 s for the cosmology tree).
BENCH_CONFIGS = {
    "sod_l6": lambda: configs.sod(level=6),          # 64^3, transmissive x
    "turb_128": lambda: configs.turb(),               # 128^3 turbulent box
    "cosmo_l7_l10": lambda: configs.cosmo(),          # base 128^3, levels 7-10, subcycled
    "roofline_256": lambda: configs.random_uniform(level=8),  # 256^3 random box
}


@pytest.mark.parametrize("name", list(BENCH_CONFIGS))
def test_fp64_benchmark_config_one_step(gpu, name):
    cfg = BENCH_CONFIGS[name]()
    tg, r, st = run_gpu(cfg, 1)
    assert st == 0
    levels = [l for l in range(cfg.lcoarse, cfg.lmax + 1) if tg.noct(l) > 0]
    to, tsim = run_oracle(cfg, 1)
    assert r.tsim == tsim
    for l in levels:  # identical trees: same octs per level, same split cells
        assert tg.noct(l) == to.noct(l)
        assert np.array_equal(tg.split_mask(l), to.split_mask(l))
    assert_close(tg, to, levels, 1e-12)


def test_fp64_sod_l6_hundred_steps(gpu):
    """The Sod configuration as stated (64^3, 100 steps): per cell <= 1e-10."""
    cfg = configs.sod(level=6)
    tg, r, st = run_gpu(cfg, 100)
    assert st == 0
    to, tsim = run_oracle(cfg, 100)
    assert abs(r.tsim - tsim) <= 1e-13 * tsim
    assert_close(tg, to, [6], 1e-10)
