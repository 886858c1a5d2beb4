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
    # host-driven schedule: every level-kernel launch is timed with CUDA events
    r = ResidentHydro(tree, precision=PREC_MIXED if a.precision == "mixed" else PREC_FP64, trans=cfg.trans,
                      cfl=cfg.cfl, use_graph=False)
    L = lib()
    per_step = []
    tot_ms, tot_n, tot_cells = 0.0, 0, 0
    for _ in range(a.steps):
        L.emma_hydro_reset_counters()
        r.coarse_step(nsub=cfg.nsub)
        avg, n, cells = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
        L.emma_hydro_kernel_timing(ctypes.byref(avg), ctypes.byref(n), ctypes.byref(cells))
        per_step.append(round(avg.value * n.value, 4))
        tot_ms += avg.value * n.value
        tot_n += n.value
        tot_cells += cells.value
    print(json.dumps({"config": cfg.name, "precision": a.precision, "status": r.status(), "launches": tot_n,
                      "avg_launch_ms": tot_ms / max(tot_n, 1), "cells_per_launch": tot_cells / max(tot_n, 1),
                      "kernel_ms_per_step": per_step,
                      "cell_updates_per_s_kernel": tot_cells / (tot_ms * 1e-3) if tot_ms else None}))


if __name__ == "__main__":
    main()
