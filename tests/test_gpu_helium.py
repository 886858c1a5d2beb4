"""The three tracers of the reference's -DWRADHYD -DHELIUM build on the GPU.

libemmahydro_he.so (the 184-byte CELL whose state ends with dX, dXHE, dXXHE)
runs the drop-in clean_new_hydro + HydroSolver in Advance_level's order on a
3-level tree with random ionised fractions; the oracle (oracle/hydro_oracle.c
built with -DORC_WRADHYD -DORC_HELIUM, pinned bit for bit to the reference's
-DWRADHYD -DHELIUM hydro in tests/test_oracle_pin.py) runs the same calls on an
identical tree.  FP64: per-cell relative error <= 1e-12 on d,u,v,w,p and
|T - T_ref| <= 1e-12 d for each tracer T; mixed: L1 <= 1e-5.  The resident mode
(tracers in planes 6-8 of every state buffer) runs whole coarse steps against the
oracle's Advance_level.
"""
import ctypes

import numpy as np
import pytest

import oracle
from emma_b200 import OctTree, PREC_FP64, PREC_MIXED, lib
from emma_b200 import hydro as H
from emma_b200._lib import EmmaHydroOptions
from helpers import l1_rel, per_cell_rel
from test_oracle_pin import random_fields

pytestmark = pytest.mark.gpu
LC, LMAX = 4, 6
DTS = {4: 2e-3, 5: 1e-3, 6: 5e-4}
YHE = 0.24
FRAC = (1.0 - YHE, YHE, YHE)


def build(seed=41):
    t = OctTree(LC, LMAX, he=True)
    for i, rad in enumerate((0.3, 0.15)):
        t.refine_where(LC + i, lambda c, rad=rad: np.linalg.norm(c - 0.5, axis=1) < rad)
    random_fields(t, range(LC, LMAX + 1))
    rng = np.random.default_rng(seed)
    for l in range(LC, LMAX + 1):
        d = t.get_fields(l, 0)[0]
        for tr, (frac, top) in enumerate(zip(FRAC, (1.0, 0.6, 0.4))):
            t.set_tracer_n(l, tr, d * frac * rng.uniform(0.0, top, d.size))
    return t


def advance_order(nsub=2):
    ops = []

    def adv(level):
        for _ in range(1 if level == LC else nsub):
            ops.append(("clean", level))
            if level < LMAX:
                adv(level + 1)
            ops.append(("solve", level))

    adv(LC)
    return ops


def set_precision(precision):
    L = lib("he")
    o = EmmaHydroOptions()
    L.emma_hydro_default_options(ctypes.byref(o))
    o.precision = precision
    assert L.emma_hydro_set_options(ctypes.byref(o)) == 0
    L.emma_hydro_clear_status()


def run_pair(precision, steps=1):
    set_precision(precision)
    tg, to = build(), build()
    R = oracle.Restatement(he=True)
    for _ in range(steps):
        for op, l in advance_order():
            if op == "clean":
                H.clean_new_hydro(l, tg.firstoct, grav="he")
                R.clean_new(to.firstoct, l)
            else:
                H.HydroSolver(l, tg.firstoct, DTS[l], grav="he")
                assert R.hydro_solver(to.firstoct, l, DTS[l]) == 0
    L = lib("he")
    assert L.emma_hydro_status() == 0, L.emma_hydro_last_error()
    set_precision(PREC_FP64)
    return tg, to


def test_helium_fp64_matches_oracle(gpu):
    tg, to = run_pair(PREC_FP64)
    t0 = build()
    for l in range(LC, LMAX + 1):
        e = per_cell_rel(tg.get_fields(l)[:5], to.get_fields(l)[:5])
        assert e.max() <= 1e-12, (l, e.max())
        d = to.get_fields(l)[0]
        for tr in range(3):
            x, xo = tg.get_tracer_n(l, tr), to.get_tracer_n(l, tr)
            ex = np.abs(x - xo) / d
            assert ex.max() <= 1e-12, (l, tr, ex.max())
            assert np.any(xo != t0.get_tracer_n(l, tr))  # the tracer moved
            assert np.all(x <= tg.get_fields(l)[0] * FRAC[tr])  # below its ceiling
        assert np.all(tg.get_tracer_n(l, 0) >= 0)


def test_helium_mixed_l1(gpu):
    tg, to = run_pair(PREC_MIXED, steps=2)
    for l in range(LC, LMAX + 1):
        assert l1_rel(tg.get_fields(l)[0], to.get_fields(l)[0]) <= 1e-5, l
        for tr in range(3):
            assert l1_rel(tg.get_tracer_n(l, tr), to.get_tracer_n(l, tr)) <= 1e-5, (l, tr)


@pytest.mark.parametrize("precision,nsub,use_graph", [(PREC_FP64, 2, True), (PREC_FP64, 1, False),
                                                      (PREC_MIXED, 2, True)])
def test_helium_resident_coarse_steps(gpu, precision, nsub, use_graph):
    """Resident tree of the -DWRADHYD -DHELIUM layout: whole coarse steps on the GPU,
    the three tracers in planes 6-8 of every state buffer; against the oracle's
    Advance_level on an identical tree."""
    from emma_b200 import ResidentHydro
    tg, to = build(), build()
    r = ResidentHydro(tg, precision=precision, cfl=0.8, use_graph=use_graph)
    for _ in range(2):
        r.coarse_step(nsub=nsub)
    assert r.status() == 0
    r.download()
    tsim, adt, err = oracle.Restatement(he=True).run(to.firstoct, LC, LMAX, 2, 0.8, nsub=nsub)
    assert err == 0
    for l in range(LC, LMAX + 1):
        d = to.get_fields(l)[0]
        leaf = ~to.split_mask(l)
        for tr in range(3):
            x, xo = tg.get_tracer_n(l, tr)[leaf], to.get_tracer_n(l, tr)[leaf]
            if precision == PREC_FP64:
                assert np.abs(x - xo).max() / d[leaf].min() <= 1e-11, (l, tr)
            else:
                assert l1_rel(x, xo) <= 1e-5, (l, tr)
        if precision == PREC_FP64:
            assert abs(r.tsim - tsim) <= 1e-14 * tsim
            e = per_cell_rel(tg.get_fields(l)[:5], to.get_fields(l)[:5])
            assert e.max() <= 1e-11, (l, e.max())
    set_precision(PREC_FP64)
