"""Field dumps in the reference's ALLOCT format (dumpalloct_serial, src/io.c:1233).

The library's files are compared byte for byte with the oracle's restatement of
dumpalloct_serial (oracle/hydro_oracle.c, orc_dump_alloct) on the same tree:
host trees on the CPU (single rank, one rank of a multi-rank tree, the -DWGRAV
layout), and on the GPU a resident tree whose hydro fields are gathered from the
device state, against the oracle on the downloaded tree.  For trees of the plain
cell layout both are also compared with the reference's own dumpalloct_serial
(src/io.c compiled into oracle/_ref/libemmaref_io.so), which pins the restatement.
"""
import os
import struct

import numpy as np
import pytest

import oracle
from emma_b200 import OctTree, configs, hydro as H
from emma_b200._lib import ST_ARG as EMMA_ST_ARG
from helpers import PARTITIONS, assign_ranks
from test_oracle_pin import random_fields, random_forces

FIELDS = [(0, "x"), (1, "y"), (2, "z"), (3, "l"), (4, "cpu"), (12, "marked"), (13, "field.d"), (14, "field.u"),
          (15, "field.v"), (16, "field.w"), (17, "field.p")]
GRAV_FIELDS = [(5, "gdata.d"), (7, "gdata.p"), (8, "res"), (9, "f0"), (10, "f1"), (11, "f2")]


def dump_pair(tmp_path, tree, fields, rank=0, ndumps=3, tsim=0.123456789, grav=False, lcoarse=None, lmax=None):
    lc = tree.lcoarse if lcoarse is None else lcoarse
    lm = tree.lmax if lmax is None else lmax
    ids, names = [f[0] for f in fields], [f[1] for f in fields]
    a, b = str(tmp_path / "lib") + "/", str(tmp_path / "orc") + "/"
    os.makedirs(a)
    os.makedirs(b)
    assert H.dump_alloct(a, tree.firstoct, lc, lm, ids, names, rank=rank, ndumps=ndumps, tsim=tsim, grav=grav) == 0
    assert oracle.Restatement(grav=grav).dump_alloct(b, tree.firstoct, lc, lm, ids, names, rank=rank,
                                                     ndumps=ndumps, tsim=tsim) == 0
    ref = None
    if not grav and oracle.ref_dump_available():
        ref = str(tmp_path / "ref") + "/"
        os.makedirs(ref)
        assert oracle.ref_dump_alloct(ref, tree.firstoct, lc, lm, ids, names, rank=rank, ndumps=ndumps,
                                      tsim=tsim) == 0
    out = {}
    for name in names:
        rel = f"grid_{name}/{name}.{ndumps:05d}.p{rank:05d}"
        with open(a + rel, "rb") as fa, open(b + rel, "rb") as fb:
            da, db = fa.read(), fb.read()
        assert da == db, name
        if ref is not None:
            with open(ref + rel, "rb") as fr:
                assert fr.read() == da, f"{name}: the reference's dumpalloct_serial"
        out[name] = da
    return out


@pytest.mark.skipif(not oracle.ref_dump_available(), reason="oracle/_ref io build absent")
def test_dump_matches_reference_dumpalloct_serial(tmp_path):
    """The library's dump and the restatement equal the reference's own function's
    bytes on trees of several depths and on the cosmology-like tree."""
    for cfg in (configs.small_amr(base=4, radii=(0.3, 0.15)), configs.small_amr(base=3, radii=(0.3,)),
                configs.cosmo(base=5, lmax=7)):
        t = cfg.build()
        d = tmp_path / cfg.name
        d.mkdir()
        dump_pair(d, t, FIELDS, ndumps=7, tsim=0.5 ** 7)


def parse(data):
    n = struct.unpack("<i", data[:4])[0]
    head = struct.unpack("<7f", data[4:32])
    vals = np.frombuffer(data[32:], dtype="<f4")
    assert len(vals) == n
    return n, data[4:8], head[1:], vals


def test_dump_matches_oracle_amr_tree(tmp_path):
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    t = cfg.build()
    out = dump_pair(tmp_path, t, FIELDS)
    n, tword, bounds, d = parse(out["field.d"])
    # leaves of levels 4..5 and every cell of lmax = 6
    expect = sum(int((~t.split_mask(l)).sum()) for l in (4, 5)) + 8 * t.noct(6)
    assert n == expect
    assert tword == struct.pack("<d", 0.123456789)[:4]
    assert bounds == (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    n2, _, _, lev = parse(out["l"])
    assert set(np.unique(lev)) == {4.0, 5.0, 6.0}


def test_dump_one_rank_of_a_multi_rank_tree(tmp_path):
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    t = cfg.build()
    assign_ranks(t, PARTITIONS["slabs"][1])
    out = dump_pair(tmp_path, t, FIELDS[:5] + FIELDS[6:7], rank=1, ndumps=12)
    n, _, bounds, cpu = parse(out["cpu"])
    assert n > 0 and np.all(cpu == 1.0)
    assert bounds[0] == 0.625 and bounds[1] == 1.0  # rank 1 owns x >= 5/8 of the coarse grid


def test_dump_gravity_layout(tmp_path):
    t = OctTree(4, 5, grav=True)
    t.refine_where(4, lambda c: np.linalg.norm(c - 0.5, axis=1) < 0.3)
    random_fields(t, (4, 5))
    random_forces(t, (4, 5))
    out = dump_pair(tmp_path, t, GRAV_FIELDS + FIELDS[6:8], grav=True)
    _, _, _, f0 = parse(out["f0"])
    assert np.any(f0 != 0.0)


def test_dump_tracer_layout(tmp_path):
    """libemmahydro_rh.so reads the 152-byte cells of the -DWRADHYD layout."""
    t = OctTree(4, 5, rh=True)
    t.refine_where(4, lambda c: np.linalg.norm(c - 0.5, axis=1) < 0.3)
    random_fields(t, (4, 5))
    ids, names = [f[0] for f in FIELDS], [f[1] for f in FIELDS]
    a, b = str(tmp_path / "lib") + "/", str(tmp_path / "orc") + "/"
    os.makedirs(a)
    os.makedirs(b)
    assert H.dump_alloct(a, t.firstoct, 4, 5, ids, names, grav="rh") == 0
    assert oracle.Restatement(rh=True).dump_alloct(b, t.firstoct, 4, 5, ids, names) == 0
    for name in names:
        rel = f"grid_{name}/{name}.00000.p00000"
        assert open(a + rel, "rb").read() == open(b + rel, "rb").read(), name


def test_dump_refuses_unknown_ids(tmp_path):
    t = configs.small_amr(base=3, radii=(0.3,)).build()
    d = str(tmp_path) + "/"
    assert H.dump_alloct(d, t.firstoct, 3, 4, [13, 18], ["d", "rad"]) == EMMA_ST_ARG
    assert H.dump_alloct(d, t.firstoct, 3, 4, [5], ["gdata.d"]) == EMMA_ST_ARG  # no gdata in this layout
    assert not os.path.exists(d + "grid_d")


@pytest.mark.gpu
def test_dump_from_resident_device_state(gpu, tmp_path):
    """Hydro fields of a resident tree are gathered on the GPU; the bytes equal the
    oracle's dump of the tree downloaded after the same steps."""
    from emma_b200 import ResidentHydro, PREC_FP64
    cfg = configs.small_amr(base=4, radii=(0.3, 0.15))
    t = cfg.build()
    r = ResidentHydro(t, precision=PREC_FP64, cfl=0.8)
    for _ in range(2):
        r.coarse_step(nsub=cfg.nsub)
    assert r.status() == 0
    ids, names = [f[0] for f in FIELDS], [f[1] for f in FIELDS]
    a = str(tmp_path / "dev") + "/"
    os.makedirs(a)
    assert H.dump_alloct(a, t.firstoct, cfg.lcoarse, cfg.lmax, ids, names, ndumps=1, tsim=r.tsim) == 0
    r.download()
    b = str(tmp_path / "orc") + "/"
    os.makedirs(b)
    assert oracle.Restatement().dump_alloct(b, t.firstoct, cfg.lcoarse, cfg.lmax, ids, names, ndumps=1,
                                            tsim=r.tsim) == 0
    c = None
    if oracle.ref_dump_available():
        c = str(tmp_path / "ref") + "/"
        os.makedirs(c)
        assert oracle.ref_dump_alloct(c, t.firstoct, cfg.lcoarse, cfg.lmax, ids, names, ndumps=1, tsim=r.tsim) == 0
    for name in names:
        rel = f"grid_{name}/{name}.00001.p00000"
        with open(a + rel, "rb") as fa, open(b + rel, "rb") as fb:
            da = fa.read()
            assert da == fb.read(), name
        if c is not None:
            assert open(c + rel, "rb").read() == da, name
