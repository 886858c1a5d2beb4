"""Analytic check of the Sod tube against the reference's exact Riemann solver.

oracle/_ref/riemann is the reference's utils/Riemann.c (exact solution of the
1-D Riemann problem, gamma = 5/3) compiled by oracle/Makefile.  The 64^3 tube
with transmissive x boundaries is advanced on the GPU (FP64 and mixed) to
t ~ 0.15; the density and pressure profiles along x must lie within 4 per cent
(L1, relative) of the exact solution at that time and the velocity within 4 per
cent of its peak (mean deviation): the oracle's own run sits near 2 per cent on
these 64 cells.
"""
import os
import subprocess

import numpy as np
import pytest

from emma_b200 import configs, ResidentHydro, PREC_FP64, PREC_MIXED
from conftest import ROOT

pytestmark = pytest.mark.gpu
RIEMANN = os.path.join(ROOT, "oracle", "_ref", "riemann")


def exact(tmp_path, t):
    with open(tmp_path / "Input.riemann", "w") as f:
        f.write(f"1. 0. 1.\n0.125 0. 0.1\n0.5 {t:.8f}\n")
    subprocess.run([RIEMANN], cwd=tmp_path, check=True, stdout=subprocess.DEVNULL)
    return np.loadtxt(tmp_path / "test1.dat")  # x, d, u, p on 1024 points


@pytest.mark.skipif(not os.path.exists(RIEMANN), reason="oracle/_ref/riemann not built")
@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_sod_tube_against_exact_riemann_solution(gpu, tmp_path, precision):
    cfg = configs.sod(level=6)
    tree = cfg.build()
    r = ResidentHydro(tree, precision=precision, trans=cfg.trans, cfl=0.8)
    for _ in range(200):
        r.coarse_step(nsub=cfg.nsub)
        if r.tsim >= 0.15:
            break
    assert r.status() == 0 and 0.15 <= r.tsim < 0.2
    st = r.state(6)
    x = tree.cell_centres(6)[:, 0]
    ex = exact(tmp_path, r.tsim)
    order = np.argsort(ex[:, 0], kind="stable")
    xe = ex[order, 0]
    for k, q in ((1, st[0]), (2, st[1]), (3, st[4])):
        want = np.interp(x, xe, ex[order, k])
        err = np.abs(q - want).sum() / np.abs(want).sum() if k != 2 else np.abs(q - want).mean() / np.abs(want).max()
        assert err <= 0.04, (k, err)
