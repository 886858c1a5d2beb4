"""Synthetic initial conditions of the hydro benchmark configurations.

There is no public dataset for this path: each configuration is a seeded
function of cell-centre position (so it does not depend on oct order), with the
shapes, sizes and value distributions of the reference's own test setups.
Seed 12345 is the reference's SEED (src/param.h:9); gamma = 5/3 (src/param.h:4).

  sod        uniform level 6 (64^3), x<0.5: rho=1,p=1 else rho=0.125,p=0.1, v=0;
             transmissive x (HYDROTEST + TRANSXM/TRANSXP), periodic y,z
  turb       uniform level 7 (128^3), periodic; ln rho and the three velocity
             components are Gaussian fields with P(k) ~ k^-4, 1<=|k|<=32, times a
             Gaussian filter exp(-k^2/(2*32^2)), unit variance; velocity scaled to
             rms |v| = 2 c_s with c_s = sqrt(gamma/<rho>); p = 1
  sedov      base level 6 refined to 7 where the cell centre is within r<0.25 of
             the box centre and to 8 within r<0.125; rho=1, p=1e-5, energy 1
             deposited as pressure in the 8 finest cells touching the centre
  cosmo      base level 7 refined to 8,9,10 where the density (trilinear from the
             base field) exceeds 8x the mean, 2:1 balanced; delta Gaussian with
             P(k) ~ k^-2 (k<=64), rho = exp(sigma delta)/<.>, v = grad(phi) scaled
             to rms 0.3 c_s, p = 1e-2 rho^(5/3)
  roofline   uniform level 8 (256^3), periodic; rho,p ~ U(0.5,1.5), u,v,w ~ U(-0.5,0.5)
             drawn in that order as (256,256,256) arrays indexed [ix,iy,iz]
"""
import numpy as np

from .tree import OctTree
from ._lib import TRANS_XM, TRANS_XP

GAMMA = 5.0 / 3.0
SEED = 12345


def _cell_index(centres, n):
    """Integer cell coordinates (n per dim) of cell centres in [0,1)."""
    return np.floor(centres * n).astype(np.int64).clip(0, n - 1)


def _gauss_field(n, rng, slope, kmin, kmax, kfilter=None):
    """Unit-variance periodic Gaussian random field with P(k) ~ k^slope."""
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    kx, ky, kz = np.meshgrid(k1, k1, k1[: n // 2 + 1], indexing="ij")
    k = np.sqrt(kx * kx + ky * ky + kz * kz)
    amp = np.zeros_like(k)
    sel = (k >= kmin) & (k <= kmax)
    amp[sel] = k[sel] ** (slope / 2.0)
    if kfilter is not None:
        amp *= np.exp(-k * k / (4.0 * kfilter * kfilter))  # sqrt of exp(-k^2/(2 kf^2))
    noise = rng.standard_normal((n, n, n))
    f = np.fft.irfftn(np.fft.rfftn(noise) * amp, s=(n, n, n), axes=(0, 1, 2))
    f -= f.mean()
    return f / f.std()


class Config:
    """A named configuration: tree, initial fields and run parameters."""

    def __init__(self, name, lcoarse, lmax, steps, trans=0, cfl=0.8, nsub=2):
        self.name, self.lcoarse, self.lmax = name, lcoarse, lmax
        self.steps, self.trans, self.cfl, self.nsub = steps, trans, cfl, nsub
        self.dt_param = 1e9
        self.time_max = 1e9
        self.builder = None

    def build(self, tree_factory=OctTree):
        return self.builder(tree_factory)


def _uniform(tree_factory, level, fields_fn):
    t = tree_factory(level, level)
    c = t.cell_centres(level)
    t.set_fields(level, *fields_fn(c))
    return t


def sod(level=6):
    cfg = Config("sod", level, level, 100, trans=TRANS_XM | TRANS_XP)

    def fields(c):
        left = c[:, 0] < 0.5
        d = np.where(left, 1.0, 0.125)
        p = np.where(left, 1.0, 0.1)
        z = np.zeros(len(c))
        return d, z, z.copy(), z.copy(), p

    cfg.builder = lambda tf: _uniform(tf, level, fields)
    return cfg


def random_uniform(level=8, seed=SEED, steps=20):
    """The roofline configuration (and its smaller parity variants)."""
    cfg = Config("roofline" if level == 8 else f"random_l{level}", level, level, steps)
    n = 2 ** level

    def fields(c):
        rng = np.random.default_rng(seed)
        rho = rng.uniform(0.5, 1.5, (n, n, n))
        p = rng.uniform(0.5, 1.5, (n, n, n))
        u = rng.uniform(-0.5, 0.5, (n, n, n))
        v = rng.uniform(-0.5, 0.5, (n, n, n))
        w = rng.uniform(-0.5, 0.5, (n, n, n))
        ix, iy, iz = _cell_index(c, n).T
        return rho[ix, iy, iz], u[ix, iy, iz], v[ix, iy, iz], w[ix, iy, iz], p[ix, iy, iz]

    cfg.builder = lambda tf: _uniform(tf, level, fields)
    return cfg


def turb(level=7, seed=SEED, steps=50):
    cfg = Config("turb", level, level, steps)
    n = 2 ** level

    def fields(c):
        rng = np.random.default_rng(seed)
        g = _gauss_field(n, rng, -4.0, 1.0, 32.0, kfilter=32.0)
        rho = np.exp(g)
        vel = [_gauss_field(n, rng, -4.0, 1.0, 32.0, kfilter=32.0) for _ in range(3)]
        cs = np.sqrt(GAMMA * 1.0 / rho.mean())
        vrms = np.sqrt(np.mean(vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2))
        vel = [v * (2.0 * cs / vrms) for v in vel]
        ix, iy, iz = _cell_index(c, n).T
        p = np.ones(len(c))
        return rho[ix, iy, iz], vel[0][ix, iy, iz], vel[1][ix, iy, iz], vel[2][ix, iy, iz], p

    cfg.builder = lambda tf: _uniform(tf, level, fields)
    return cfg


def sedov(base=6, radii=(0.25, 0.125), steps=100, e0=1.0):
    lmax = base + len(radii)
    cfg = Config("sedov", base, lmax, steps)

    def build(tf):
        t = tf(base, lmax)
        for i, r in enumerate(radii):
            lev = base + i
            t.refine_where(lev, lambda c, r=r: np.linalg.norm(c - 0.5, axis=1) < r)
        for lev in range(base, lmax + 1):
            c = t.cell_centres(lev)
            d = np.ones(len(c))
            p = np.full(len(c), 1e-5)
            z = np.zeros(len(c))
            if lev == lmax:
                dx = 0.5 ** lev
                hot = np.all(np.abs(c - 0.5) < dx, axis=1)  # the 8 cells touching the centre
                p[hot] = (GAMMA - 1.0) * (e0 / 8.0) / dx ** 3
            t.set_fields(lev, d, z, z.copy(), z.copy(), p)
        return t

    cfg.builder = build
    return cfg


def small_amr(base=4, radii=(0.3, 0.15), seed=SEED):
    """Small 3-level random tree for parity tests (spheres about the centre)."""
    lmax = base + len(radii)
    cfg = Config(f"amr_l{base}_{lmax}", base, lmax, 2)

    def build(tf):
        t = tf(base, lmax)
        for i, r in enumerate(radii):
            t.refine_where(base + i, lambda c, r=r: np.linalg.norm(c - 0.5, axis=1) < r)
        rng = np.random.default_rng(seed)
        for lev in range(base, lmax + 1):
            n8 = 8 * t.noct(lev)
            d = rng.uniform(0.5, 1.5, n8)
            p = rng.uniform(0.5, 1.5, n8)
            u, v, w = (rng.uniform(-0.5, 0.5, n8) for _ in range(3))
            t.set_fields(lev, d, u, v, w, p)
        return t

    cfg.builder = build
    return cfg


def _balance_marks(t, lev, mark):
    """Extend marks so every refined cell's face neighbours at this level exist
    refined-compatible (2:1 across faces, edges and corners), like the
    reference's neighbour smoothing before refinement (src/amr.c:746)."""
    n = 2 ** lev
    c = t.cell_centres(lev)
    ijk = _cell_index(c, n)
    grid = np.zeros((n, n, n), bool)
    grid[tuple(ijk.T)] = mark
    # dilate by one parent cell in every direction (26 neighbours, periodic)
    g = grid.copy()
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                g |= np.roll(grid, (dx, dy, dz), axis=(0, 1, 2))
    return g[tuple(ijk.T)]


def _check_rule(t, lev, mark):
    """Cancel the marks of cells whose oct lacks one of its 26 neighbour octs at
    this level, as the reference's L_check_rule does (src/amr.c:746-868: the
    face, edge and corner neighbours of the oct must all exist)."""
    n = 2 ** (lev - 1)
    ijk = np.rint(t.oct_xyz(lev) * n).astype(np.int64) % n
    occ = np.zeros((n, n, n), bool)
    occ[tuple(ijk.T)] = True
    ok = occ.copy()
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                if dx or dy or dz:
                    ok &= np.roll(occ, (dx, dy, dz), axis=(0, 1, 2))
    return mark & np.repeat(ok[tuple(ijk.T)], 8)


def cosmo(base=7, lmax=10, seed=SEED, sigma=None, steps=20, target_cells=(5e6, 1e7)):
    cfg = Config("cosmo", base, lmax, steps)
    n = 2 ** base

    def density_field():
        rng = np.random.default_rng(seed)
        delta = _gauss_field(n, rng, -2.0, 1.0, 64.0)
        return delta, rng

    def build(tf, sig=sigma):
        delta, rng = density_field()
        s = 1.6 if sig is None else sig
        rho = np.exp(s * delta)
        rho /= rho.mean()
        t = tf(base, lmax)

        def rho_at(c):
            # trilinear interpolation of the base-level field at points c (periodic)
            x = c * n - 0.5
            i0 = np.floor(x).astype(np.int64)
            f = x - i0
            out = np.zeros(len(c))
            for dx in (0, 1):
                for dy in (0, 1):
                    for dz in (0, 1):
                        wgt = (np.where(dx, f[:, 0], 1 - f[:, 0]) * np.where(dy, f[:, 1], 1 - f[:, 1])
                               * np.where(dz, f[:, 2], 1 - f[:, 2]))
                        out += wgt * rho[(i0[:, 0] + dx) % n, (i0[:, 1] + dy) % n, (i0[:, 2] + dz) % n]
            return out

        for lev in range(base, lmax):
            c = t.cell_centres(lev)
            mark = rho_at(c) > 8.0
            mark = _check_rule(t, lev, _balance_marks(t, lev, mark))
            t.refine(lev, mark)
        # velocities from the potential of the same field, phi_k = -delta_k / k^2
        k1 = np.fft.fftfreq(n, d=1.0 / n) * 2 * np.pi
        kx, ky, kz = np.meshgrid(k1, k1, k1[: n // 2 + 1], indexing="ij")
        k2 = kx * kx + ky * ky + kz * kz
        k2[0, 0, 0] = 1.0
        dk = np.fft.rfftn(delta)
        phik = -dk / k2
        vel = [np.fft.irfftn(1j * kk * phik, s=(n, n, n), axes=(0, 1, 2)) for kk in (kx, ky, kz)]
        cs = np.sqrt(GAMMA * 1e-2 * np.mean(rho ** (GAMMA - 1.0)))
        vr = np.sqrt(np.mean(vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2))
        vel = [v * (0.3 * cs / vr) for v in vel]
        for lev in range(base, lmax + 1):
            c = t.cell_centres(lev)
            ijk = _cell_index(c, n)
            d = rho_at(c) if lev > base else rho[tuple(ijk.T)]
            u, v, w = (vv[tuple(ijk.T)] for vv in vel)
            p = 1e-2 * d ** GAMMA
            t.set_fields(lev, d, u, v, w, p)
        return t

    cfg.builder = build
    return cfg


CONFIGS = {"sod": sod, "turb": turb, "sedov": sedov, "cosmo": cosmo, "roofline": random_uniform}
