"""Checkpoints in the reference's raw-OCT restart format (src/restart.c).

emma_hydro_save_amr writes byte for byte what the reference's save_amr writes
for the same tree; emma_hydro_restore_amr rebuilds the same tree as the
reference's restore_amr from such a file (topology, fields, free-oct chain).
CPU only: the reference's src/restart.c is compiled into oracle/_ref.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle
from emma_b200 import lib

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (no reference checkout)")
UNITS = np.array([3.1e24, 2.9e7, 1.1e17, 6.0e-1, 2.0e42, 1.7e-29, 1.0e0])


def _ref_tree(rh=False):
    ref = oracle.RefTree(4, 6, ngridmax=sum(8 ** (l - 1) for l in range(1, 7)), rh=rh)
    for i, r in enumerate((0.3, 0.15)):
        ref.refine_where(4 + i, lambda c, r=r: np.linalg.norm(c - 0.5, axis=1) < r)
    rng = np.random.default_rng(7)
    for l in range(4, 7):
        n8 = 8 * ref.noct(l)
        ref.set_fields(l, rng.uniform(0.5, 1.5, n8), *(rng.uniform(-0.5, 0.5, n8) for _ in range(3)),
                       rng.uniform(0.5, 1.5, n8))
        if rh:
            ref.set_tracer(l, ref.get_fields(l, 0)[0] * rng.uniform(0.0, 1.0, n8))
    ref.run(2)
    return ref


def _snapshot(ref):
    return {l: (ref.topology(l), ref.get_fields(l, 0), ref.get_fields(l, 1)) for l in range(1, 7)}


def _same(a, b):
    for l in a:
        (ta, fa, na), (tb, fb, nb) = a[l], b[l]
        for x, y in zip(ta, tb):
            assert np.array_equal(x, y), l
        assert np.array_equal(fa, fb) and np.array_equal(na, nb), l


@needs_ref
def test_save_amr_is_byte_identical(tmp_path):
    ref = _ref_tree()
    adt = np.array([ref.L.ref_adt(l) for l in range(1, 7)])
    fa, fb = str(tmp_path / "ref.bin"), str(tmp_path / "lib.bin")
    ref.save_amr(fa, 0.0123, 0.001, 17, 3, UNITS)
    rc = lib().emma_hydro_save_amr(fb.encode(), ref.firstoct, 0.0123, 0.001, 17, 3, 4, 6,
                                   ctypes.c_void_p(adt.ctypes.data), ctypes.c_void_p(UNITS.ctypes.data), None)
    assert rc == 0
    a, b = open(fa, "rb").read(), open(fb, "rb").read()
    assert len(a) == len(b) and a == b


@pytest.mark.skipif(not oracle.ref_available(rh=True), reason="oracle/_ref -DWRADHYD build absent")
def test_save_amr_tracer_layout_is_byte_identical(tmp_path):
    """libemmahydro_rh.so writes the reference's -DWRADHYD checkpoint (1328-byte octs) byte for byte."""
    ref = _ref_tree(rh=True)
    adt = np.array([ref.L.ref_adt(l) for l in range(1, 7)])
    fa, fb = str(tmp_path / "ref.bin"), str(tmp_path / "lib.bin")
    ref.save_amr(fa, 0.0123, 0.001, 17, 3, UNITS)
    rc = lib("rh").emma_hydro_save_amr(fb.encode(), ref.firstoct, 0.0123, 0.001, 17, 3, 4, 6,
                                       ctypes.c_void_p(adt.ctypes.data), ctypes.c_void_p(UNITS.ctypes.data), None)
    assert rc == 0
    a, b = open(fa, "rb").read(), open(fb, "rb").read()
    assert len(a) == len(b) and a == b


@needs_ref
def test_restore_amr_rebuilds_the_reference_tree(tmp_path):
    ref = _ref_tree()
    before = _snapshot(ref)
    f = str(tmp_path / "ckpt.bin")
    ref.save_amr(f, 0.5, 0.0, 9, 2, UNITS)
    # the reference's restore into a fresh pool
    r2 = oracle.RefTree(4, 6, ngridmax=ref.ngridmax)
    t, ti, ns, nd = r2.restore_amr(f)
    assert (t, ti, ns, nd) == (0.5, 0.0, 9, 2)
    by_ref = _snapshot(r2)
    nfree_ref = _free_count(r2)
    # the library's restore into another fresh pool
    r3 = oracle.RefTree(4, 6, ngridmax=ref.ngridmax)
    last, root, ngrid = r3.pool()
    ts, ti2, lc, lm = ctypes.c_double(), ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    ns2, nd2 = ctypes.c_int(), ctypes.c_int()
    adt, units = np.zeros(6), np.zeros(7)
    free = ctypes.c_void_p()
    rc = lib().emma_hydro_restore_amr(f.encode(), r3.firstoct, last, 6, ngrid, root, ctypes.byref(ts),
                                      ctypes.byref(ti2), ctypes.byref(ns2), ctypes.byref(nd2), ctypes.byref(lc),
                                      ctypes.byref(lm), ctypes.c_void_p(adt.ctypes.data),
                                      ctypes.c_void_p(units.ctypes.data), ctypes.byref(free))
    assert rc == 0
    assert (ts.value, ti2.value, ns2.value, nd2.value, lc.value, lm.value) == (0.5, 0.0, 9, 2, 4, 6)
    assert np.array_equal(units, UNITS)
    r3.set_freeoct(free.value)
    _same(by_ref, _snapshot(r3))
    _same(before, by_ref)
    assert _free_count(r3) == nfree_ref


def _free_count(ref):
    """Length of the free-oct chain, walked through the OCT layout (next pointer)."""
    p, n = ref.freeoct(), 0
    off_next = 8 * 136 + 6 * 8 + 8  # cell[8], nei[6], parent, then next
    while p:
        n += 1
        p = ctypes.c_void_p.from_address(p + off_next).value
    return n


@pytest.mark.gpu
def test_resident_run_checkpoints_its_device_state(gpu, tmp_path):
    """emma_hydro_save_amr on the firstoct a resident tree was uploaded from
    writes the device state (downloaded into the tree first)."""
    from emma_b200 import configs, ResidentHydro, PREC_FP64
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    t = cfg.build()
    r = ResidentHydro(t, precision=PREC_FP64, cfl=0.8)
    for _ in range(2):
        r.coarse_step(nsub=cfg.nsub)
    assert lib().emma_hydro_is_resident(t.firstoct) == 1
    dev = {l: r.state(l) for l in range(4, 7)}
    f = str(tmp_path / "resident.bin")
    adt = np.ascontiguousarray(r.adt)
    rc = lib().emma_hydro_save_amr(f.encode(), t.firstoct, r.tsim, 0.0, 2, 0, 4, 6, ctypes.c_void_p(adt.ctypes.data),
                                   ctypes.c_void_p(UNITS.ctypes.data), None)
    assert rc == 0
    for l in range(4, 7):
        assert np.array_equal(t.get_fields(l)[:5], dev[l]), l
    raw = open(f, "rb").read()
    head = np.frombuffer(raw[:16], dtype=np.float64)
    assert head[0] == r.tsim
    nocts = sum(t.noct(l) for l in range(1, 7))
    assert len(raw) == 16 + 16 + 6 * 8 + 7 * 8 + 3 * 8 + nocts * (8 + 1200)


@pytest.mark.gpu
@needs_ref
def test_restore_into_a_resident_pool_releases_it(gpu, tmp_path):
    """Restoring a checkpoint into the pool a resident tree was uploaded from
    releases that resident tree: a following save writes the restored tree, byte
    for byte the checkpoint that was restored (same pool, same addresses), and no
    stale device state is downloaded into it."""
    from emma_b200 import ResidentHydro, PREC_FP64
    ref = _ref_tree()
    f = str(tmp_path / "ckpt.bin")
    adt = np.array([ref.L.ref_adt(l) for l in range(1, 7)])
    ref.save_amr(f, 0.5, 0.0, 9, 2, UNITS)
    # a resident run on the tree (its device state moves on), then the library's
    # restore of the checkpoint into the same pool
    r = ResidentHydro(ref, precision=PREC_FP64, cfl=0.8)
    r.coarse_step()
    assert lib().emma_hydro_is_resident(ref.firstoct) == 1
    last, root, ngrid = ref.pool()
    ts, ti2, lc, lm = ctypes.c_double(), ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    ns2, nd2 = ctypes.c_int(), ctypes.c_int()
    adt2, units = np.zeros(6), np.zeros(7)
    free = ctypes.c_void_p()
    rc = lib().emma_hydro_restore_amr(f.encode(), ref.firstoct, last, 6, ngrid, root, ctypes.byref(ts),
                                      ctypes.byref(ti2), ctypes.byref(ns2), ctypes.byref(nd2), ctypes.byref(lc),
                                      ctypes.byref(lm), ctypes.c_void_p(adt2.ctypes.data),
                                      ctypes.c_void_p(units.ctypes.data), ctypes.byref(free))
    assert rc == 0
    ref.set_freeoct(free.value)
    assert lib().emma_hydro_is_resident(ref.firstoct) == 0
    assert np.array_equal(adt2, adt)
    fout = str(tmp_path / "after.bin")
    rc = lib().emma_hydro_save_amr(fout.encode(), ref.firstoct, 0.5, 0.0, 9, 2, 4, 6,
                                   ctypes.c_void_p(adt2.ctypes.data), ctypes.c_void_p(UNITS.ctypes.data), None)
    assert rc == 0
    a, b = open(f, "rb").read(), open(fout, "rb").read()
    assert len(a) == len(b) and a == b
