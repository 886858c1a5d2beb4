"""The fused coarse step (emma_b200/csrc/step_kernel.cuh): one persistent kernel
runs Advance_level's whole recursion for a subcycled resident tree.

Against the level schedule's separate launches on the same tree (the graph with
fused_step = -1, itself checked against the oracle in test_gpu_parity.py): the
same tsim and per-cell states to 1e-13 (the fine->coarse corrections are FP64
atomics, so the last bits of coarse cells next to finer octs depend on their
order), with one library kernel per captured coarse step.  Also against the
oracle directly (FP64 per cell <= 1e-12), after a state set from the host (the
CFL job), after host-driven level calls (the corrections cleared first), for
the dual-energy and tracer variants and for fewer tile groups per CTA.  The
coarse-step mode autotuner times each mode from a snapshot of the state and
restores it: a run that tuned equals one that did not.
"""
import numpy as np
import pytest

import oracle
from emma_b200 import configs, OctTree, PREC_FP64, PREC_MIXED, ResidentHydro
from helpers import per_cell_rel

pytestmark = pytest.mark.gpu
CFL = 0.8

TREES = {
    "amr_l4_6": lambda: configs.small_amr(base=4),
    "sedov_l5_7": lambda: configs.sedov(base=5),
    "cosmo_l5_7": lambda: configs.cosmo(base=5, lmax=7),
    "cosmo_l5_8": lambda: configs.cosmo(base=5, lmax=8),
}


def levels_of(t, cfg):
    return [l for l in range(cfg.lcoarse, cfg.lmax + 1) if t.noct(l) > 0]


def run(cfg, fused, precision=PREC_FP64, steps=2, **kw):
    t = cfg.build()
    r = ResidentHydro(t, precision=precision, cfl=CFL, fused=fused, **kw)
    for _ in range(steps):
        r.coarse_step(nsub=cfg.nsub)
    assert r.status() == 0
    return t, r, {l: r.state(l) for l in levels_of(t, cfg)}


def assert_states_close(a, b, tol):
    assert a.keys() == b.keys()
    worst = max(float(per_cell_rel(a[l], b[l]).max()) for l in a)
    assert worst <= tol, worst


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
@pytest.mark.parametrize("name", list(TREES))
def test_fused_step_equals_separate_launches(gpu, name, precision):
    cfg = TREES[name]()
    _, rf, sf = run(cfg, True, precision)
    fused, ctas, groups, kernels = rf.graph_info()
    assert fused == 1 and ctas > 0 and groups >= 1 and kernels == 1
    _, ru, su = run(cfg, False, precision)
    assert ru.graph_info()[0] == 0 and ru.graph_info()[3] > 10
    assert abs(rf.tsim - ru.tsim) <= 1e-13 * ru.tsim
    assert_states_close(sf, su, 1e-13)


@pytest.mark.parametrize("name", ["amr_l4_6", "cosmo_l5_8"])
def test_fused_step_matches_oracle(gpu, name):
    cfg = TREES[name]()
    tg, r, _ = run(cfg, True, steps=1)
    assert r.graph_info()[0] == 1
    r.download()
    to = cfg.build()
    tsim, _, err = oracle.Restatement().run(to.firstoct, cfg.lcoarse, cfg.lmax, 1, CFL, nsub=cfg.nsub)
    assert err == 0 and r.tsim == tsim
    worst = max(float(per_cell_rel(tg.get_fields(l)[:5], to.get_fields(l)[:5]).max()) for l in levels_of(tg, cfg))
    assert worst <= 1e-12, worst


def test_fused_step_after_host_state_and_host_levels(gpu):
    """A level state set from the host makes the fused step run a CFL reduction job
    first; host-driven level calls leave corrections that the fused step clears."""
    cfg = TREES["amr_l4_6"]()
    out = {}
    for fused in (True, False):
        t = cfg.build()
        r = ResidentHydro(t, precision=PREC_FP64, cfl=CFL, fused=fused)
        r.coarse_step(nsub=cfg.nsub)
        lf = max(levels_of(t, cfg))
        st = r.state(lf)
        st[4] *= 1.5  # a hotter finest level, set from the host
        r.set_state(lf, st)
        r.coarse_step(nsub=cfg.nsub)
        # host-driven: the finest level advanced alone (its corrections go to the coarser level)
        r.advance_level(lf, 1e-4)
        r.coarse_step(nsub=cfg.nsub)
        assert r.status() == 0
        out[fused] = ({l: r.state(l) for l in levels_of(t, cfg)}, r.tsim)
    assert abs(out[True][1] - out[False][1]) <= 1e-13 * out[False][1]
    assert_states_close(out[True][0], out[False][0], 1e-13)


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_fused_step_dual_energy(gpu, precision):
    cfg = TREES["amr_l4_6"]()
    _, rf, sf = run(cfg, True, precision, dual=True)
    assert rf.graph_info()[0] == 1
    _, ru, su = run(cfg, False, precision, dual=True)
    assert abs(rf.tsim - ru.tsim) <= 1e-13 * ru.tsim
    assert_states_close(sf, su, 1e-13)


@pytest.mark.parametrize("variant", ["rh", "he"])
def test_fused_step_tracers(gpu, variant):
    cfg = TREES["amr_l4_6"]()
    fracs = (1.0,) if variant == "rh" else (0.76, 0.24, 0.24)
    res = {}
    for fused in (True, False):
        t = cfg.build(lambda lc, lm: OctTree(lc, lm, rh=(variant == "rh"), he=(variant == "he")))
        rng = np.random.default_rng(5)
        for l in levels_of(t, cfg):
            d = t.get_fields(l, 0)[0]
            for k, frac in enumerate(fracs):
                t.set_tracer_n(l, k, d * frac * rng.uniform(0.0, 0.5, d.size))
        r = ResidentHydro(t, precision=PREC_FP64, cfl=CFL, fused=fused)
        for _ in range(2):
            r.coarse_step(nsub=cfg.nsub)
        assert r.status() == 0
        assert r.graph_info()[0] == (1 if fused else 0)
        r.download()
        st = {l: r.state(l) for l in levels_of(t, cfg)}
        tr = {l: np.stack([t.get_tracer_n(l, k) for k in range(len(fracs))]) for l in levels_of(t, cfg)}
        res[fused] = (st, tr, r.tsim)
    assert abs(res[True][2] - res[False][2]) <= 1e-13 * res[False][2]
    assert_states_close(res[True][0], res[False][0], 1e-13)
    for l in res[True][1]:
        a, b = res[True][1][l], res[False][1][l]
        d = res[False][0][l][0]
        assert (np.abs(a - b) / d).max() <= 1e-13, l


@pytest.mark.parametrize("groups", [2, 3])
def test_fused_step_fewer_tile_groups(gpu, groups):
    """The fused kernel with fewer tile groups per CTA (more registers a thread)."""
    cfg = TREES["cosmo_l5_7"]()
    _, rf, sf = run(cfg, groups, PREC_MIXED)
    assert rf.graph_info()[:3:2] == (1, groups)
    _, ru, su = run(cfg, False, PREC_MIXED)
    assert abs(rf.tsim - ru.tsim) <= 1e-13 * ru.tsim
    assert_states_close(sf, su, 1e-13)


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_step_mode_autotuned(gpu, precision):
    """The autotuner times every mode from a snapshot of the state and restores it:
    the run afterwards equals one that never tuned."""
    cfg = TREES["cosmo_l5_7"]()
    _, r, sa = run(cfg, "auto", precision)
    mode, sweep = r.step_tuning()
    timed = [x for x in sweep if x > 0]
    assert mode >= 0 and sweep[0] > 0 and len(timed) >= 2
    assert sweep[mode] == min(timed)
    assert r.graph_info()[0] == (1 if mode > 0 else 0)
    _, ru, su = run(cfg, False, precision)
    assert abs(r.tsim - ru.tsim) <= 1e-13 * ru.tsim
    assert_states_close(sa, su, 1e-13)
