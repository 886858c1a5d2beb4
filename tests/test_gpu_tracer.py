"""The ionised-density tracer of the reference's -DWRADHYD build on the GPU.

libemmahydro_rh.so (the 152-byte CELL whose state ends with dX) runs the drop-in
clean_new_hydro + HydroSolver in Advance_level's order on a 3-level tree with a
random ionised fraction; the oracle (oracle/hydro_oracle.c built with
-DORC_WRADHYD, pinned bit for bit to the reference's -DWRADHYD hydro in
tests/test_oracle_pin.py) runs the same calls on an identical tree.  FP64:
per-cell relative error <= 1e-12 on d,u,v,w,p and |dX - dX_ref| <= 1e-12 d;
mixed: L1 <= 1e-5.  The resident mode of the same library (dX the sixth plane of
every state buffer) runs whole coarse steps against the oracle's Advance_level.
"""
import ctypes

import numpy as np
import pytest

import oracle
from emma_b200 import OctTree, PREC_FP64, PREC_MIXED, lib
from emma_b200 import hydro as H
from emma_b200._lib import EmmaHydroOptions, ST_ARG
from helpers import l1_rel, per_cell_rel
from test_oracle_pin import random_fields

pytestmark = pytest.mark.gpu
LC, LMAX = 4, 6
DTS = {4: 2e-3, 5: 1e-3, 6: 5e-4}


def build(seed=31):
    t = OctTree(LC, LMAX, rh=True)
    for i, rad in enumerate((0.3, 0.15)):
        t.refine_where(LC + i, lambda c, rad=rad: np.linalg.norm(c - 0.5, axis=1) < rad)
    random_fields(t, range(LC, LMAX + 1))
    rng = np.random.default_rng(seed)
    for l in range(LC, LMAX + 1):
        d = t.get_fields(l, 0)[0]
        t.set_tracer(l, d * rng.uniform(0.0, 1.0, d.size))
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
    L = lib("rh")
    o = EmmaHydroOptions()
    L.emma_hydro_default_options(ctypes.byref(o))
    o.precision = precision
    assert L.emma_hydro_set_options(ctypes.byref(o)) == 0
    L.emma_hydro_clear_status()


def run_pair(precision, steps=1):
    set_precision(precision)
    tg, to = build(), build()
    R = oracle.Restatement(rh=True)
    for _ in range(steps):
        for op, l in advance_order():
            if op == "clean":
                H.clean_new_hydro(l, tg.firstoct, grav="rh")
                R.clean_new(to.firstoct, l)
            else:
                H.HydroSolver(l, tg.firstoct, DTS[l], grav="rh")
                assert R.hydro_solver(to.firstoct, l, DTS[l]) == 0
    L = lib("rh")
    assert L.emma_hydro_status() == 0, L.emma_hydro_last_error()
    set_precision(PREC_FP64)
    return tg, to


def test_tracer_fp64_matches_oracle(gpu):
    tg, to = run_pair(PREC_FP64)
    for l in range(LC, LMAX + 1):
        e = per_cell_rel(tg.get_fields(l)[:5], to.get_fields(l)[:5])
        assert e.max() <= 1e-12, (l, e.max())
        d = to.get_fields(l)[0]
        ex = np.abs(tg.get_tracer(l) - to.get_tracer(l)) / d
        assert ex.max() <= 1e-12, (l, ex.max())
        # the tracer moved, and stays inside its ceiling
        assert np.any(to.get_tracer(l) != build().get_tracer(l))
        assert np.all(tg.get_tracer(l) >= 0) and np.all(tg.get_tracer(l) <= tg.get_fields(l)[0])


def test_tracer_mixed_l1(gpu):
    tg, to = run_pair(PREC_MIXED, steps=2)
    for l in range(LC, LMAX + 1):
        assert l1_rel(tg.get_fields(l)[0], to.get_fields(l)[0]) <= 1e-5, l
        assert l1_rel(tg.get_tracer(l), to.get_tracer(l)) <= 1e-5, l


def test_tracer_total_is_conserved(gpu):
    """On a uniform periodic level the volume sum of dX changes only by the
    ceiling, which random fractions below 1 never reach in one step."""
    set_precision(PREC_FP64)
    t = OctTree(4, 4, rh=True)
    random_fields(t, (4,))
    rng = np.random.default_rng(5)
    d = t.get_fields(4, 0)[0]
    t.set_tracer(4, d * rng.uniform(0.2, 0.8, d.size))
    m0 = t.get_tracer(4).sum()
    H.clean_new_hydro(4, t.firstoct, grav="rh")
    H.HydroSolver(4, t.firstoct, 2e-3, grav="rh")
    assert lib("rh").emma_hydro_status() == 0
    assert abs(t.get_tracer(4).sum() - m0) <= 1e-12 * m0


def test_tracer_library_refuses_dual_energy(gpu):
    L = lib("rh")
    t = build()
    o = EmmaHydroOptions()
    L.emma_hydro_default_options(ctypes.byref(o))
    o.dual_energy = 1
    assert L.emma_hydro_set_options(ctypes.byref(o)) == 0
    L.emma_hydro_clear_status()
    H.HydroSolver(LMAX, t.firstoct, 1e-4, grav="rh")
    assert L.emma_hydro_status() & ST_ARG
    set_precision(PREC_FP64)


@pytest.mark.parametrize("precision,nsub,use_graph", [(PREC_FP64, 2, True), (PREC_FP64, 1, False),
                                                      (PREC_MIXED, 2, True)])
def test_tracer_resident_coarse_steps(gpu, precision, nsub, use_graph):
    """Resident tree of the -DWRADHYD layout: whole coarse steps on the GPU (device
    schedule and graph, or host schedule), dX the sixth plane of every state buffer;
    against the oracle's Advance_level on an identical tree."""
    from emma_b200 import ResidentHydro
    tg, to = build(), build()
    r = ResidentHydro(tg, precision=precision, cfl=0.8, use_graph=use_graph)
    for _ in range(2):
        r.coarse_step(nsub=nsub)
    assert r.status() == 0
    r.download()
    tsim, adt, err = oracle.Restatement(rh=True).run(to.firstoct, LC, LMAX, 2, 0.8, nsub=nsub)
    assert err == 0
    for l in range(LC, LMAX + 1):
        d = to.get_fields(l)[0]
        leaf = ~to.split_mask(l)
        if precision == PREC_FP64:
            assert abs(r.tsim - tsim) <= 1e-14 * tsim
            e = per_cell_rel(tg.get_fields(l)[:5], to.get_fields(l)[:5])
            assert e.max() <= 1e-11, (l, e.max())
            ex = np.abs(tg.get_tracer(l) - to.get_tracer(l))[leaf] / d[leaf]
            assert ex.max() <= 1e-11, (l, ex.max())
        else:
            assert l1_rel(tg.get_tracer(l)[leaf], to.get_tracer(l)[leaf]) <= 1e-5, l
    set_precision(PREC_FP64)
