"""Drop-in entries on the trees of a multi-rank run (the reference's -DWMPI build).

Each rank's level lists hold its own octs and the octs of other ranks (its
boundary octs).  HydroSolver advances cpu->rank's octs only and reads the others
as neighbours (src/hydro_utils.c:2997,3124,3417); fine->coarse corrections of
coarser octs of other ranks accumulate in their fieldnew, zeroed by
clean_new_hydro (src/hydro_utils.c:3524-3544).  The reference's MPI exchanges
run between the calls; here they are restated on the host, on one tree per
rank:
  mpi_exchange_hydro (src/communication.c:2054): before each solve, every oct of
      another rank takes its owner's `field`;
  mpi_hydro_correct (src/communication.c:2959, scatter_mpi_hydro_ext :1968):
      after each solve of a level above lcoarse, each rank's coarser octs of
      other ranks send their fieldnew, and the owner sets
      fieldnew = U2W(W2U(fieldnew) + W2U(received)).
The ranks run one after another on one GPU (no kernel waits for another).  The
result must equal the single-rank oracle on the same tree (FP64 per-cell
relative error <= 1e-12; only the order of the correction sums differs).
"""
import ctypes

import numpy as np
import pytest

import oracle
from emma_b200 import OctTree, lib
from emma_b200 import hydro as H
from emma_b200._lib import EmmaHydroOptions, ST_ARG
from helpers import GAMMA, PARTITIONS, assign_ranks, per_cell_rel, rank_of_octs
from test_oracle_pin import random_fields, random_forces

pytestmark = pytest.mark.gpu
LC, LMAX = 4, 6
DTS = {4: 2e-3, 5: 1e-3, 6: 5e-4}
DEFDENS = 10.0  # U2W's stand-in density for an empty cell (src/hydro_utils.c:38)


def build(grav=False):
    """grav: True (-DWGRAV layout with forces) or "rh" (-DWRADHYD layout with an ionised fraction)."""
    rh = grav == "rh"
    t = OctTree(LC, LMAX, grav=(grav is True), rh=rh)
    for i, rad in enumerate((0.3, 0.15)):
        t.refine_where(LC + i, lambda c, rad=rad: np.linalg.norm(c - 0.5, axis=1) < rad)
    random_fields(t, range(LC, LMAX + 1))
    if grav is True:
        random_forces(t, range(LC, LMAX + 1))
    if rh:
        rng = np.random.default_rng(99)
        for l in range(LC, LMAX + 1):
            d = t.get_fields(l, 0)[0]
            t.set_tracer(l, d * rng.uniform(0.0, 1.0, d.size))
    return t


def advance_order(nsub=2):
    """Advance_level's order of cleans and solves for one coarse step
    (src/advanceamr.c:321-1290: clean at :423, finer level at :852, solve at :989)."""
    ops = []

    def adv(level):
        for _ in range(1 if level == LC else nsub):
            ops.append(("clean", level))
            if level < LMAX:
                adv(level + 1)
            ops.append(("solve", level))

    adv(LC)
    return ops


def w2u(w, dual):
    """W2U (src/hydro_utils.c:66): d, du, dv, dw, E, eint."""
    d, u, v, wz, p, a, E = w
    return np.stack([d, d * u, d * v, d * wz, E, p / (GAMMA - 1.0)])


def u2w(U, dual):
    """U2W (src/hydro_utils.c:35), with or without -DDUAL_E."""
    d, du, dv, dw, E, eint = U
    dl = np.where(d == 0.0, DEFDENS, d)
    if dual:
        p = eint * (GAMMA - 1.0)
    else:
        p = (GAMMA - 1.0) * (E - (du * du + dv * dv + dw * dw) / dl * 0.5)
    return np.stack([d, du / dl, dv / dl, dw / dl, p, np.sqrt(GAMMA * p / dl), E])


def exchange_fields(trees, owner):
    """mpi_exchange_hydro: the octs of other ranks take their owner's field."""
    for l in range(1, LMAX + 1):
        if trees[0].noct(l) == 0:
            continue
        src = [t.get_fields(l) for t in trees]
        cell_owner = np.repeat(owner[l], 8)
        for r, t in enumerate(trees):
            w = src[r].copy()
            for q in range(len(trees)):
                if q != r:
                    m = cell_owner == q
                    w[:, m] = src[q][:, m]
            t.put_fields(l, w)
        if trees[0].rh:
            xs = [t.get_tracer(l, 0) for t in trees]
            for r, t in enumerate(trees):
                x = xs[r].copy()
                for q in range(len(trees)):
                    if q != r:
                        x[cell_owner == q] = xs[q][cell_owner == q]
                t.put_tracer(l, x, which=0)


def hydro_correct(trees, owner, level, dual):
    """mpi_hydro_correct for `level`: level-1 octs of other ranks send their
    fieldnew (the corrections this rank's solve added), owners add them."""
    lc = level - 1
    cell_owner = np.repeat(owner[lc], 8)
    fnew = [t.get_fields(lc, 1) for t in trees]
    rh = trees[0].rh
    xnew = [t.get_tracer(lc, 1) if rh else np.zeros(fnew[0].shape[1]) for t in trees]  # U.dX = W.dX
    out = [f.copy() for f in fnew]
    xout = [x.copy() for x in xnew]
    sent = 0
    for r in range(len(trees)):
        for q in range(len(trees)):
            if q == r:
                continue
            m = (cell_owner == q) & (np.any(fnew[r] != 0.0, axis=0) | (xnew[r] != 0.0))
            if m.any():
                U = w2u(out[q][:, m], dual) + w2u(fnew[r][:, m], dual)
                out[q][:, m] = u2w(U, dual)
                xout[q][m] = xout[q][m] + xnew[r][m]
                sent += int(m.sum())
    for q, t in enumerate(trees):
        t.put_fields(lc, out[q], which=1)
        if rh:
            t.put_tracer(lc, xout[q], which=1)
    return sent


def run_ranks(part, grav=False, dual=False, fn=None):
    nrank, fn = PARTITIONS[part] if fn is None else fn
    trees = [build(grav) for _ in range(nrank)]
    for t in trees:
        assign_ranks(t, fn)
    owner = {l: rank_of_octs(trees[0], l, fn) for l in range(1, LMAX + 1) if trees[0].noct(l)}
    params = H.RunParams(lcoarse=LC, lmax=LMAX)
    cpus = [H.CpuInfo(rank=r, nproc=nrank) for r in range(nrank)]
    L = lib(grav)
    L.emma_hydro_clear_status()
    sent = 0
    for op, l in advance_order():
        if op == "clean":
            for r, t in enumerate(trees):
                H.clean_new_hydro(l, t.firstoct, grav=grav, cpu=cpus[r], param=params)
            continue
        exchange_fields(trees, owner)
        for r, t in enumerate(trees):
            H.HydroSolver(l, t.firstoct, DTS[l], cpu=cpus[r], grav=grav)
            if grav is True:
                H.grav_correction(l, t.firstoct, DTS[l], cpu=cpus[r])
        assert L.emma_hydro_status() == 0, L.emma_hydro_last_error()
        if l > LC:
            sent += hydro_correct(trees, owner, l, dual)
    assert sent > 0  # the partition cuts coarse-fine boundaries: corrections cross ranks
    return trees, owner


def run_single(grav=False, dual=False):
    t = build(grav)
    R = oracle.Restatement(grav=(grav is True), rh=(grav == "rh"))
    for op, l in advance_order():
        if op == "clean":
            R.clean_new(t.firstoct, l)
        else:
            assert R.hydro_solver(t.firstoct, l, DTS[l], dual=dual) == 0
            if grav is True:
                assert R.grav_correction(t.firstoct, l, DTS[l]) == 0
    return t


def check_owned(trees, owner, ref, tol=1e-12):
    for l in range(LC, LMAX + 1):
        o = ref.get_fields(l)[:5]
        cell_owner = np.repeat(owner[l], 8)
        for r, t in enumerate(trees):
            m = cell_owner == r
            if m.any():
                e = per_cell_rel(t.get_fields(l)[:5][:, m], o[:, m])
                assert e.max() <= tol, (l, r, e.max())
                if getattr(ref, "rh", False):
                    ex = np.abs(t.get_tracer(l)[m] - ref.get_tracer(l)[m]) / o[0][m]
                    assert ex.max() <= tol, (l, r, "dX", ex.max())


@pytest.mark.parametrize("part", ["slabs", "quadrants", "stripes3"])
def test_multi_rank_dropin_matches_single_rank_oracle(gpu, part):
    trees, owner = run_ranks(part)
    check_owned(trees, owner, run_single())


def test_multi_rank_dropin_gravity(gpu):
    """-DWGRAV layout: grav_correction of each rank's own leaves after its solve."""
    trees, owner = run_ranks("quadrants", grav=True)
    check_owned(trees, owner, run_single(grav=True))


def test_multi_rank_dropin_tracer(gpu):
    """-DWRADHYD layout: dX exchanged with the fields, its corrections sent like theirs."""
    trees, owner = run_ranks("quadrants", grav="rh")
    check_owned(trees, owner, run_single(grav="rh"))


def test_multi_rank_dropin_dual_energy(gpu):
    L = lib()
    o = EmmaHydroOptions()
    L.emma_hydro_default_options(ctypes.byref(o))
    o.dual_energy = 1
    assert L.emma_hydro_set_options(ctypes.byref(o)) == 0
    trees, owner = run_ranks("slabs", dual=True)
    check_owned(trees, owner, run_single(dual=True))


def test_multi_rank_dropin_mixed_precision(gpu):
    """The mixed path on the ranks' trees: L1 <= 1e-5 against the single-rank FP64 oracle."""
    from emma_b200 import PREC_MIXED
    from helpers import l1_rel
    L = lib()
    o = EmmaHydroOptions()
    L.emma_hydro_default_options(ctypes.byref(o))
    o.precision = PREC_MIXED
    assert L.emma_hydro_set_options(ctypes.byref(o)) == 0
    trees, owner = run_ranks("stripes3")
    ref = run_single()
    for l in range(LC, LMAX + 1):
        cell_owner = np.repeat(owner[l], 8)
        g = np.zeros_like(ref.get_fields(l)[:5])
        for r, t in enumerate(trees):
            m = cell_owner == r
            g[:, m] = t.get_fields(l)[:5][:, m]
        o_ = ref.get_fields(l)[:5]
        assert l1_rel(g[0], o_[0]) <= 1e-5 and l1_rel(g[4], o_[4]) <= 1e-5, l


def test_other_ranks_octs_are_left_alone(gpu):
    """advancehydroGPU returns this rank's oct count and writes no fieldnew of
    another rank's oct at the level; HydroSolver leaves their field as it was."""
    nrank, fn = PARTITIONS["stripes3"]
    t = build()
    assign_ranks(t, fn)
    for l in range(LC, LMAX + 1):
        H.clean_new_hydro(l, t.firstoct, cpu=H.CpuInfo(rank=1, nproc=3), param=H.RunParams(lcoarse=LC, lmax=LMAX))
    own = {l: rank_of_octs(t, l, fn) == 1 for l in range(LC, LMAX + 1)}
    before = {l: (t.get_fields(l, 0), t.get_fields(l, 1)) for l in range(LC, LMAX + 1)}
    n = H.advancehydroGPU(t.firstoct, LMAX, DTS[LMAX], cpu=H.CpuInfo(rank=1, nproc=3))
    assert n == own[LMAX].sum()
    other = ~np.repeat(own[LMAX], 8)
    assert np.array_equal(t.get_fields(LMAX, 1)[:, other], before[LMAX][1][:, other])
    H.HydroSolver(LMAX - 1, t.firstoct, DTS[LMAX - 1], cpu=H.CpuInfo(rank=1, nproc=3))
    other = ~np.repeat(own[LMAX - 1], 8)
    assert np.array_equal(t.get_fields(LMAX - 1, 0)[:, other], before[LMAX - 1][0][:, other])
    assert lib().emma_hydro_status() == 0, lib().emma_hydro_last_error()


def test_clean_new_zeroes_coarser_octs_of_other_ranks(gpu):
    """clean_new_hydro(level) of a multi-rank run: fieldnew := field at `level`;
    one level coarser, the octs of other ranks start from zero when level > lcoarse."""
    nrank, fn = PARTITIONS["halves"]
    t = build()
    assign_ranks(t, fn)
    params = H.RunParams(lcoarse=LC, lmax=LMAX)
    cpu = H.CpuInfo(rank=0, nproc=2)
    below = t.get_fields(LC - 1, 1)
    H.clean_new_hydro(LC, t.firstoct, cpu=cpu, param=params)  # level == lcoarse: nothing zeroed
    assert np.array_equal(t.get_fields(LC - 1, 1), below)
    H.clean_new_hydro(LC + 1, t.firstoct, cpu=cpu, param=params)
    f, fn_ = t.get_fields(LC, 0), t.get_fields(LC, 1)
    other = np.repeat(rank_of_octs(t, LC, fn) != 0, 8)
    assert np.all(fn_[:, other] == 0.0) and np.array_equal(fn_[:, ~other], f[:, ~other])
    assert np.array_equal(t.get_fields(LC + 1, 1), t.get_fields(LC + 1, 0))


def test_resident_mode_refuses_octs_of_other_ranks(gpu):
    from emma_b200 import ResidentHydro, PREC_FP64
    nrank, fn = PARTITIONS["halves"]
    t = build()
    assign_ranks(t, fn)
    lib().emma_hydro_clear_status()
    with pytest.raises(RuntimeError):
        ResidentHydro(t, precision=PREC_FP64, rank=0)
    assert lib().emma_hydro_status() & ST_ARG
    lib().emma_hydro_clear_status()
