"""Device-side refinement of a resident tree against the reference's own marking,
2:1 check rule and refinement (L_clean_marks + L_mark_cells, L_check_rule,
L_refine_cells, src/amr.c:1480, 883, 746, 286), built with its density criterion
(oracle/ref_amr_sntest.c: field.d > 1.1).

Both runs start from the same tree built the same way in a fresh pool, so the
free-oct chain, and with it every new oct's place in the pool, is the same:
after each mark and check the marks must be equal, and after the refinements
the level lists (order, positions, neighbour, parent and child links), the
marks, the fields of every cell and the head of the free chain (as an offset
into the pool) must be identical.  The next hydro step on the refined
tree (device, FP64) must match the oracle's restatement per cell to 1e-12.
"""
import ctypes

import numpy as np
import pytest

import oracle
from emma_b200 import lib, PREC_FP64, ResidentHydro
from emma_b200.hydro import RunParams
from helpers import per_cell_rel

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(mark=True), reason="oracle/_ref mark build absent")]
CFL = 0.8
UNITS = np.ones(7)


def blob_tree(lcoarse, lmax, radii, centre, width, seed=3):
    """The reference's tree refined in spheres about the box centre, with a
    density blob off the centre (1 + 0.6 exp(-r^2/w^2)) and small random velocities."""
    ngrid = sum(8 ** (l - 1) for l in range(1, lmax + 1)) + 1024
    ref = oracle.RefTree(lcoarse, lmax, ngridmax=ngrid, mark=True)
    for i, r in enumerate(radii):
        ref.refine_where(lcoarse + i, lambda c, r=r: np.linalg.norm(c - 0.5, axis=1) < r)
    rng = np.random.default_rng(seed)
    for l in range(lcoarse, lmax + 1):
        n8 = 8 * ref.noct(l)
        if n8 == 0:
            continue
        c = ref.cell_centres(l)
        d = 1.0 + 0.6 * np.exp(-((c - np.asarray(centre)) ** 2).sum(1) / width ** 2)
        ref.set_fields(l, d, *(0.05 * rng.standard_normal(n8) for _ in range(3)), np.ones(n8))
    return ref


def snapshot(ref, lmax):
    out = {}
    for l in range(1, lmax + 1):
        out[l] = (ref.oct_xyz(l), ref.topology(l), ref.marks(l), ref.get_fields(l, 0)[:5])
    return out


def assert_same(a, b):
    assert a.keys() == b.keys()
    for l in a:
        (xa, ta, ma, fa), (xb, tb, mb, fb) = a[l], b[l]
        assert np.array_equal(xa, xb), f"oct positions of level {l}"
        for k, (p, q) in enumerate(zip(ta, tb)):
            assert np.array_equal(p, q), f"topology array {k} of level {l}"
        assert np.array_equal(ma, mb), f"marks of level {l}"
        assert np.array_equal(fa, fb), f"fields of level {l}"


CASES = {
    # three levels, the blob across the edge of the refined spheres: octs are
    # created and destroyed on levels 5 and 6, marks cancelled by the 2:1 rule
    "spheres": dict(lcoarse=4, lmax=6, radii=(0.3, 0.15), centre=(0.64, 0.5, 0.45), width=0.1,
                    seq=[("mark", 5), ("mark", 4), ("check", 4), ("refine", 4), ("check", 5), ("refine", 5)]),
    # level 5 refined without re-refining level 4 first: the 2:1 rule cancels the
    # marks of octs on the edge of level 5
    "edge": dict(lcoarse=4, lmax=6, radii=(0.3, 0.15), centre=(0.72, 0.5, 0.5), width=0.12,
                 seq=[("mark", 5), ("check", 5), ("refine", 5)]),
    # a uniform base level with an empty finer level: refinement creates it
    "uniform": dict(lcoarse=5, lmax=6, radii=(), centre=(0.3, 0.6, 0.5), width=0.12,
                    seq=[("mark", 5), ("check", 5), ("refine", 5)]),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("nsmooth", [1, 2])
def test_device_refinement_matches_reference(gpu, tmp_path, case, nsmooth):
    p = CASES[case]
    lc, lm = p["lcoarse"], p["lmax"]
    # the reference
    ref = blob_tree(lc, lm, p["radii"], p["centre"], p["width"])
    marks_ref = {}
    for op, l in p["seq"]:
        if op == "mark":
            ref.clean_marks(l)
            ref.mark_cells(l, nsmooth, 1.1)
        elif op == "check":
            ref.check_rule(l)
            marks_ref[l] = ref.marks(l)
        else:
            ref.refine_cells(l)
    expected = snapshot(ref, lm)
    free_expected = ref.freeoct() - ref.L.ref_grid_base()
    refined = str(tmp_path / "refined.bin")
    ref.save_amr(refined, 0.0, 0.0, 0, 0, UNITS)

    # the device, on the same tree built again in a fresh pool
    ref = blob_tree(lc, lm, p["radii"], p["centre"], p["width"])
    L = lib()
    r = ResidentHydro(ref, precision=PREC_FP64, cfl=CFL)
    rp = RunParams()
    rp.lcoarse, rp.lmax = lc, lm
    last, _, ngrid = ref.pool()
    base = ref.L.ref_grid_base()
    limit = base + ngrid * ref.sizeof_oct()
    fo = ref.firstoct
    created = cancelled = 0
    for op, l in p["seq"]:
        if op == "mark":
            assert L.emma_hydro_mark_cells(l, ctypes.byref(rp), fo, nsmooth, 1.1, None) == 0
        elif op == "check":
            assert L.emma_hydro_check_rule(l, ctypes.byref(rp), fo, None) == 0
            assert L.emma_hydro_marks_to_host(fo, l) == 0
            assert np.array_equal(ref.marks(l), marks_ref[l]), f"marks of level {l} after the check rule"
            cancelled += int((marks_ref[l] == 10).sum())
        else:
            n0 = ref.noct(l + 1)
            f = L.emma_hydro_refine_cells(l, ctypes.byref(rp), fo, last, ref.freeoct(), None, limit, 1.0)
            assert f, L.emma_hydro_last_error()
            ref.set_freeoct(f)
            created += abs(ref.noct(l + 1) - n0)
    assert L.emma_hydro_status() == 0
    assert created > 0
    assert (cancelled > 0) == (case == "edge")
    for l in range(lc, lm + 1):  # the marks the device holds, into the host cells
        if ref.noct(l):
            assert L.emma_hydro_marks_to_host(fo, l) == 0
    r.download()
    assert_same(expected, snapshot(ref, lm))
    assert ref.freeoct() - base == free_expected

    # the next hydro step on the refined tree
    r.coarse_step()
    assert r.status() == 0
    dev = {l: r.state(l) for l in range(lc, lm + 1) if ref.noct(l)}
    tsim_dev = r.tsim
    # the reference's restore overwrites the pool: the resident tree goes first
    assert L.emma_hydro_tree_release(fo) == 0
    ref.restore_amr(refined)
    tsim, _, err = oracle.Restatement().run(ref.firstoct, lc, lm, 1, CFL)
    assert err == 0 and tsim == tsim_dev
    worst = 0.0
    for l, st in dev.items():
        worst = max(worst, float(per_cell_rel(st, ref.get_fields(l)[:5]).max()))
    assert worst <= 1e-12, worst
