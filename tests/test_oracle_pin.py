"""The C restatement (oracle/hydro_oracle.c) is pinned to the reference.

(a) bit-for-bit against the reference's own CPU hydro compiled from its
    sources (oracle/_ref), on the same tree memory, when that build exists;
(b) bit-for-bit against the committed golden fixtures the reference produced
    (tests/golden/make_golden.py), always.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle
from emma_b200 import configs
from emma_b200 import OctTree

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (no reference checkout)")


def random_fields(tree, levels, seed=12345):
    rng = np.random.default_rng(seed)
    for l in levels:
        n8 = 8 * tree.noct(l)
        d = rng.uniform(0.5, 1.5, n8)
        p = rng.uniform(0.5, 1.5, n8)
        u, v, w = (rng.uniform(-0.5, 0.5, n8) for _ in range(3))
        tree.set_fields(l, d, u, v, w, p)


def random_forces(tree, levels, seed=54321, amp=0.5):
    rng = np.random.default_rng(seed)
    for l in levels:
        n8 = 8 * tree.noct(l)
        tree.set_force(l, *(rng.uniform(-amp, amp, n8) for _ in range(3)))


def random_tracer(tree, levels, seed=777):
    """Ionised density dX = d * x with x uniform in [0, 1] (-DWRADHYD trees)."""
    rng = np.random.default_rng(seed)
    for l in levels:
        d = tree.get_fields(l, 0)[0]
        tree.set_tracer(l, d * rng.uniform(0.0, 1.0, d.size))


def random_helium(tree, levels, seed=77):
    """-DHELIUM trees: dX = d (1 - YHE) x, dXHE = d YHE y, dXXHE = d YHE z with x, y, z
    uniform in [0, 1], [0, 0.6], [0, 0.4] (YHE = 0.24)."""
    rng = np.random.default_rng(seed)
    for l in levels:
        d = tree.get_fields(l, 0)[0]
        for t, (frac, top) in enumerate(((0.76, 1.0), (0.24, 0.6), (0.24, 0.4))):
            tree.set_tracer_n(l, t, d * frac * rng.uniform(0.0, top, d.size))


def ref_vs_restatement(tx, base, lmax, radii, nsteps, seed=12345, fields=None, grav=False, dual=False, rh=False,
                       he=False):
    ref = oracle.RefTree(base, lmax, tx=tx, ngridmax=sum(8 ** (l - 1) for l in range(1, lmax + 1)), grav=grav,
                         dual=dual, rh=rh, he=he)
    for i, r in enumerate(radii):
        ref.refine_where(base + i, lambda c, r=r: np.linalg.norm(c - 0.5, axis=1) < r)
    if fields is None:
        random_fields(ref, range(base, lmax + 1), seed)
    else:
        for l in range(base, lmax + 1):
            ref.set_fields(l, *fields(ref.cell_centres(l)))
    if grav:
        random_forces(ref, range(base, lmax + 1))
        assert ref.sizeof_oct() == oracle.Restatement(grav=True).sizeof_oct() == 1648
    if rh:
        random_tracer(ref, range(base, lmax + 1))
        assert ref.sizeof_oct() == oracle.Restatement(rh=True).sizeof_oct() == 1328
    if he:
        random_helium(ref, range(base, lmax + 1))
        assert ref.sizeof_oct() == oracle.Restatement(he=True).sizeof_oct() == 1584
    ntr = 3 if he else (1 if rh else 0)
    base_ptr = ref.L.ref_grid_base()
    nbytes = ref.ngridmax * ref.sizeof_oct()
    snap = ctypes.string_at(base_ptr, nbytes)
    t1, adt1 = ref.run(nsteps)
    A = {l: (ref.get_fields(l, 0), ref.get_fields(l, 1)) for l in range(base, lmax + 1)}
    AX = {l: [(ref.get_tracer_n(l, t, 0), ref.get_tracer_n(l, t, 1)) for t in range(ntr)] for l in range(base, lmax + 1)}
    ctypes.memmove(base_ptr, snap, nbytes)
    trans = 3 if tx else 0
    t2, adt2, err = oracle.Restatement(grav=grav, rh=rh, he=he).run(ref.firstoct, base, lmax, nsteps, 0.8,
                                                                     trans=trans, dual=dual)
    assert err == 0
    assert t1 == t2 and np.array_equal(adt1, adt2)
    for l in range(base, lmax + 1):
        fA, fnA = A[l]
        assert np.array_equal(fA, ref.get_fields(l, 0)), f"field, level {l}"
        leaf = ~(ref.topology(l)[2].reshape(-1) >= 0)
        # fieldnew of split cells holds stale stencil data in the reference; not part of the state
        assert np.array_equal(fnA[:, leaf], ref.get_fields(l, 1)[:, leaf]), f"fieldnew, level {l}"
        for t in range(ntr):
            assert np.array_equal(AX[l][t][0], ref.get_tracer_n(l, t, 0)), f"tracer {t}, level {l}"
            assert np.array_equal(AX[l][t][1][leaf], ref.get_tracer_n(l, t, 1)[leaf]), f"fieldnew tracer {t}, level {l}"


@needs_ref
def test_pin_uniform_periodic():
    ref_vs_restatement(False, 4, 4, (), 3)


@needs_ref
def test_pin_amr_periodic():
    ref_vs_restatement(False, 4, 6, (0.3, 0.15), 2)


@needs_ref
def test_pin_uniform_transmissive_3d():
    ref_vs_restatement(True, 4, 4, (), 3)


@needs_ref
def test_pin_amr_transmissive():
    ref_vs_restatement(True, 4, 5, (0.3,), 2)


@needs_ref
def test_pin_sod_tube():
    sod = configs.sod()
    fields = lambda c: (np.where(c[:, 0] < 0.5, 1.0, 0.125), 0 * c[:, 0], 0 * c[:, 0], 0 * c[:, 0],
                        np.where(c[:, 0] < 0.5, 1.0, 0.1))
    assert sod.trans == 3
    ref_vs_restatement(True, 4, 4, (), 10, fields=fields)


needs_ref_grav = pytest.mark.skipif(not oracle.ref_available(grav=True), reason="oracle/_ref gravity build absent")


@needs_ref_grav
def test_pin_gravity_uniform():
    """-DWGRAV: face-state kick, grav_correction after each HydroSolver."""
    ref_vs_restatement(False, 4, 4, (), 3, grav=True)


@needs_ref_grav
def test_pin_gravity_amr():
    """-DWGRAV on two refined levels: forces of injected coarse cells interpolated
    (coarse2fine_forcelin) in the gather."""
    ref_vs_restatement(False, 4, 6, (0.3, 0.15), 2, grav=True)


needs_ref_rh = pytest.mark.skipif(not oracle.ref_available(rh=True), reason="oracle/_ref -DWRADHYD build absent")


@needs_ref_rh
def test_pin_tracer_uniform():
    """-DWRADHYD: the ionised density dX advected with the mass flux (face values
    from the centre fraction), its ceiling and fine->coarse corrections."""
    ref_vs_restatement(False, 4, 4, (), 3, rh=True)


@needs_ref_rh
def test_pin_tracer_amr():
    ref_vs_restatement(False, 4, 6, (0.3, 0.15), 2, rh=True)


needs_ref_he = pytest.mark.skipif(not oracle.ref_available(he=True), reason="oracle/_ref -DHELIUM build absent")


@needs_ref_he
def test_pin_helium_uniform():
    """-DWRADHYD -DHELIUM (NVAR 9): the hydrogen and the two helium tracers."""
    ref_vs_restatement(False, 4, 4, (), 3, he=True)


@needs_ref_he
def test_pin_helium_amr():
    ref_vs_restatement(False, 4, 6, (0.3, 0.15), 2, he=True)


needs_ref_dual = pytest.mark.skipif(not oracle.ref_available(dual=True), reason="oracle/_ref dual-energy build absent")


@needs_ref_dual
def test_pin_dual_energy_uniform():
    """-DDUAL_E: tracked internal energy with its flux, the p div(u) term and the
    E - Ekin switch (src/hydro_utils.c:3167-3180)."""
    ref_vs_restatement(False, 4, 4, (), 3, dual=True)


@needs_ref_dual
def test_pin_dual_energy_amr():
    ref_vs_restatement(False, 4, 6, (0.3, 0.15), 2, dual=True)


@needs_ref_dual
def test_pin_dual_energy_strong_shocks():
    """Pressure jumps of 1e4 make the E - Ekin switch go both ways."""
    def fields(c):
        r = np.linalg.norm(c - 0.5, axis=1)
        return (1.0 + 0 * r, 0.5 * np.sin(6.3 * c[:, 1]), 0 * r, 0 * r, np.where(r < 0.15, 1e2, 1e-2))
    ref_vs_restatement(False, 4, 5, (0.3,), 4, fields=fields, dual=True)


def _amr_tree(base, lmax, radii, seed=12345):
    t = OctTree(base, lmax)
    for i, r in enumerate(radii):
        t.refine_where(base + i, lambda c, r=r: np.linalg.norm(c - 0.5, axis=1) < r)
    random_fields(t, range(base, lmax + 1), seed)
    return t


def test_gravity_clone_without_force_is_plain_hydro():
    """The gravity restatement on a layout copy with zero force reproduces the
    plain restatement bit for bit (the copy keeps octs, links and list order)."""
    t = _amr_tree(4, 6, (0.3, 0.15))
    gc = oracle.GravClone(t)
    t1, adt1, e1 = gc.run(2, 0.8)
    t2, adt2, e2 = oracle.Restatement().run(t.firstoct, 4, 6, 2, 0.8)
    assert e1 == e2 == 0 and t1 == t2 and np.array_equal(adt1, adt2)
    for l in range(4, 7):
        assert np.array_equal(gc.get_fields(l), t.get_fields(l)), l


@needs_ref_grav
def test_gravity_clone_matches_reference_tree():
    """Gravity restatement on a copy of the library's tree == the reference's
    -DWGRAV hydro on its own tree, same configuration, forces and fields."""
    base, lmax, radii = 4, 6, (0.3, 0.15)
    t = _amr_tree(base, lmax, radii)
    ref = oracle.RefTree(base, lmax, ngridmax=sum(8 ** (l - 1) for l in range(1, lmax + 1)), grav=True)
    for i, r in enumerate(radii):
        ref.refine_where(base + i, lambda c, r=r: np.linalg.norm(c - 0.5, axis=1) < r)
    random_fields(ref, range(base, lmax + 1))
    random_forces(ref, range(base, lmax + 1))
    gc = oracle.GravClone(t)
    rng = np.random.default_rng(54321)
    for l in range(base, lmax + 1):
        n8 = 8 * t.noct(l)
        gc.set_force(l, *(rng.uniform(-0.5, 0.5, n8) for _ in range(3)))
    t1, adt1 = ref.run(2)
    t2, adt2, err = gc.run(2, 0.8)
    assert err == 0 and t1 == t2 and np.array_equal(adt1, adt2)
    for l in range(base, lmax + 1):
        assert np.array_equal(ref.get_fields(l), gc.get_fields(l)), l


def test_gravity_layout_tree_equals_layout_copy():
    """A tree built in the -DWGRAV layout (libemmahydro_grav.so) and a copy of the
    default-layout tree give the same gravity restatement results bit for bit."""
    base, lmax, radii = 4, 6, (0.3, 0.15)
    tp = _amr_tree(base, lmax, radii)
    tg = OctTree(base, lmax, grav=True)
    for i, r in enumerate(radii):
        tg.refine_where(base + i, lambda c, r=r: np.linalg.norm(c - 0.5, axis=1) < r)
    random_fields(tg, range(base, lmax + 1))
    random_forces(tg, range(base, lmax + 1))
    gc = oracle.GravClone(tp)
    random_forces(gc, range(base, lmax + 1))
    t1, adt1, e1 = oracle.Restatement(grav=True).run(tg.firstoct, base, lmax, 2, 0.8)
    t2, adt2, e2 = gc.run(2, 0.8)
    assert e1 == e2 == 0 and t1 == t2 and np.array_equal(adt1, adt2)
    for l in range(base, lmax + 1):
        assert np.array_equal(tg.get_fields(l), gc.get_fields(l)), l


def test_dropin_grav_correction_matches_oracle():
    """libemmahydro_grav.so's grav_correction (host loop, no GPU) == the oracle's."""
    from emma_b200 import hydro as H
    trees = []
    for _ in range(2):
        t = OctTree(4, 5, grav=True)
        t.refine_where(4, lambda c: np.linalg.norm(c - 0.5, axis=1) < 0.3)
        random_fields(t, (4, 5))
        random_forces(t, (4, 5))
        trees.append(t)
    for l in (5, 4):
        H.grav_correction(l, trees[0].firstoct, 3e-3)
        assert oracle.Restatement(grav=True).grav_correction(trees[1].firstoct, l, 3e-3) == 0
    for l in (4, 5):
        assert np.array_equal(trees[0].get_fields(l), trees[1].get_fields(l)), l
    assert not np.array_equal(trees[0].get_fields(5), _amr_fields_only(4, 5))


def _amr_fields_only(base, level):
    t = OctTree(base, level, grav=True)
    t.refine_where(base, lambda c: np.linalg.norm(c - 0.5, axis=1) < 0.3)
    random_fields(t, (base, level))
    return t.get_fields(level)


def _golden_cases():
    return sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz")) if os.path.isdir(GOLDEN) else []


@pytest.mark.parametrize("name", _golden_cases())
def test_restatement_reproduces_golden(name):
    """The reference's outputs committed as fixtures, reproduced bit for bit by the
    restatement of the same build variant (default, -DDUAL_E, -DWGRAV, -DWRADHYD,
    -DWRADHYD -DHELIUM)."""
    g = np.load(os.path.join(GOLDEN, name))
    base, lmax, nsteps, trans = (int(x) for x in g["meta"][:4])
    variant = int(g["meta"][4]) if len(g["meta"]) > 4 else 0
    radii = tuple(g["radii"])
    t = OctTree(base, lmax, grav=variant == 2, rh=variant == 3, he=variant == 4)
    for i, r in enumerate(radii):
        t.refine_where(base + i, lambda c, r=r: np.linalg.norm(c - 0.5, axis=1) < r)
    for l in range(base, lmax + 1):
        t.set_fields(l, *g[f"in_{l}"][:5])
        if variant == 2:
            t.set_force(l, *g[f"in_f_{l}"])
        if variant == 3:
            t.set_tracer(l, g[f"in_x_{l}"])
        if variant == 4:
            for tr in range(3):
                t.set_tracer_n(l, tr, g[f"in_x_{l}"][tr])
    R = oracle.Restatement(grav=variant == 2, rh=variant == 3, he=variant == 4)
    tsim, adt, err = R.run(t.firstoct, base, lmax, nsteps, 0.8, trans=trans, dual=variant == 1)
    assert err == 0
    assert tsim == float(g["tsim"])
    for l in range(base, lmax + 1):
        assert np.array_equal(t.get_fields(l, 0), g[f"out_{l}"]), f"level {l}"
        if variant == 3:
            assert np.array_equal(t.get_tracer(l, 0), g[f"out_x_{l}"]), f"dX, level {l}"
        if variant == 4:
            for tr in range(3):
                assert np.array_equal(t.get_tracer_n(l, tr, 0), g[f"out_x_{l}"][tr]), f"tracer {tr}, level {l}"


@needs_ref
def test_reference_library_runs_its_own_hydro():
    """With libemmahydro loaded first (it exports HydroSolver too), the reference
    library must still call its own HydroSolver: its CPU time per cell-update
    stays in the reference's range and its result equals the restatement's."""
    from emma_b200 import lib
    lib()  # load the product library (exports the same drop-in names)
    ref_vs_restatement(False, 3, 3, (), 1)
    ref = oracle.RefTree(4, 4, ngridmax=1000)
    random_fields(ref, [4])
    ref.reset_counters()
    ref.run(1)
    assert ref.cell_updates() == 4096
    assert ref.cell_updates() / ref.hydro_seconds() < 5e6  # a CPU, not a GPU
