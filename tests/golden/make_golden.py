"""Generate the golden fixtures from the reference's own CPU hydro (oracle/_ref).

Run from the repository root where the reference checkout is available:
    make -C oracle && python tests/golden/make_golden.py
Each fixture: a seeded small tree (uniform or refined spheres about the box
centre), the input primitive fields per level, and the reference's `field`
(d,u,v,w,p,a,E) per level after `nsteps` coarse steps at CFL 0.8.  Build
variants (meta[4]): 0 the default, 1 -DDUAL_E, 2 -DWGRAV (input forces per
level), 3 -DWRADHYD (input and output ionised density dX per level), 4 -DWRADHYD
-DHELIUM (input and output dX, dXHE, dXXHE per level).
Existing fixture files are kept; only missing ones are written.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

CASES = [
    # name, base, lmax, radii, nsteps, transmissive(x), field kind, build variant
    ("uniform_l3_periodic", 3, 3, (), 3, 0, "random", 0),
    ("sod_l4_transmissive", 4, 4, (), 8, 3, "sod", 0),
    ("amr_l3_5_periodic", 3, 5, (0.35, 0.2), 2, 0, "random", 0),
    ("amr_l3_4_dual", 3, 4, (0.35,), 2, 0, "random", 1),
    ("amr_l3_4_gravity", 3, 4, (0.35,), 2, 0, "random", 2),
    ("amr_l3_4_tracer", 3, 4, (0.35,), 2, 0, "random", 3),
    ("amr_l3_4_helium", 3, 4, (0.35,), 2, 0, "random", 4),
]
HELIUM = ((0.76, 1.0), (0.24, 0.6), (0.24, 0.4))  # (mass fraction, top of the ionised share) per tracer


def fields(kind, c, rng):
    n = len(c)
    if kind == "sod":
        left = c[:, 0] < 0.5
        z = np.zeros(n)
        return np.where(left, 1.0, 0.125), z, z.copy(), z.copy(), np.where(left, 1.0, 0.1)
    d = rng.uniform(0.5, 1.5, n)
    p = rng.uniform(0.5, 1.5, n)
    u, v, w = (rng.uniform(-0.5, 0.5, n) for _ in range(3))
    return d, u, v, w, p


def main():
    for name, base, lmax, radii, nsteps, trans, kind, variant in CASES:
        path = os.path.join(HERE, name + ".npz")
        if os.path.exists(path):
            continue
        ref = oracle.RefTree(base, lmax, tx=bool(trans), ngridmax=sum(8 ** (l - 1) for l in range(1, lmax + 1)),
                             dual=variant == 1, grav=variant == 2, rh=variant == 3, he=variant == 4)
        for i, r in enumerate(radii):
            ref.refine_where(base + i, lambda c, r=r: np.linalg.norm(c - 0.5, axis=1) < r)
        rng = np.random.default_rng(12345)
        out = {"meta": np.array([base, lmax, nsteps, trans, variant]), "radii": np.array(radii, dtype=np.float64)}
        for l in range(base, lmax + 1):
            f = fields(kind, ref.cell_centres(l), rng)
            ref.set_fields(l, *f)
            out[f"in_{l}"] = np.array(f)
            if variant == 2:
                fo = np.array([rng.uniform(-0.5, 0.5, len(f[0])) for _ in range(3)])
                ref.set_force(l, *fo)
                out[f"in_f_{l}"] = fo
            if variant == 3:
                x = f[0] * rng.uniform(0.0, 1.0, len(f[0]))
                ref.set_tracer(l, x)
                out[f"in_x_{l}"] = x
            if variant == 4:
                xs = np.array([f[0] * frac * rng.uniform(0.0, top, len(f[0])) for frac, top in HELIUM])
                for t in range(3):
                    ref.set_tracer_n(l, t, xs[t])
                out[f"in_x_{l}"] = xs
        tsim, adt = ref.run(nsteps)
        out["tsim"] = np.array(tsim)
        out["adt"] = adt
        for l in range(base, lmax + 1):
            out[f"out_{l}"] = ref.get_fields(l, 0)
            if variant == 3:
                out[f"out_x_{l}"] = ref.get_tracer(l, 0)
            if variant == 4:
                out[f"out_x_{l}"] = np.array([ref.get_tracer_n(l, t, 0) for t in range(3)])
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
