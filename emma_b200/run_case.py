"""Run a configuration for a few coarse steps and print the level-kernel timing.

    python -m emma_b200.run_case --config random --level 6 --precision mixed --steps 3

Used to profile one configuration in isolation (for example under ncu).
"""
import argparse
import ctypes
import json

from . import configs, ResidentHydro, PREC_FP64, PREC_MIXED, lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="random", choices=["random", "turb", "sod", "sedov", "cosmo", "amr"])
    ap.add_argument("--level", type=int, default=6)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--steps", type=int, default=3)
    a = ap.parse_args()
    cfg = {"random": lambda: configs.random_uniform(level=a.level), "turb": lambda: configs.turb(level=a.level),
           "sod": lambda: configs.sod(level=a.level), "sedov": configs.sedov, "cosmo": configs.cosmo,
           "amr": configs.small_amr}[a.config]()
    tree = cfg.build()
    r = ResidentHydro(tree, precision=PREC_MIXED if a.precision == "mixed" else PREC_FP64, trans=cfg.trans,
                      cfl=cfg.cfl)
    L = lib()
    L.emma_hydro_reset_counters()
    for _ in range(a.steps):
        r.coarse_step(nsub=cfg.nsub)
    avg, n, cells = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
    L.emma_hydro_kernel_timing(ctypes.byref(avg), ctypes.byref(n), ctypes.byref(cells))
    print(json.dumps({"config": cfg.name, "precision": a.precision, "status": r.status(), "launches": n.value,
                      "avg_launch_ms": avg.value, "cells_per_launch": cells.value / max(n.value, 1),
                      "cell_updates_per_s_kernel": cells.value / (avg.value * n.value * 1e-3) if n.value else None}))


if __name__ == "__main__":
    main()
