"""Run a configuration for a few coarse steps and print the level-kernel timing.

    python -m emma_b200.run_case --config random --level 6 --precision mixed --steps 3
    python -m emma_b200.run_case --config turb --level 7 --precision fp64 --steps 2 --dropin rh
    python -m emma_b200.run_case --config turb --level 7 --precision mixed --steps 4 --tracer
    python -m emma_b200.run_case --config random --level 8 --precision mixed --steps 3 --column 32
    python -m emma_b200.run_case --config cosmo --precision mixed --steps 3 --graph

Used to profile one configuration in isolation (for example under ncu).  --dropin
runs the drop-in clean_new_hydro + HydroSolver on the finest level of the host tree
instead of the resident schedule, through libemmahydro.so (plain) or the -DWRADHYD
library (rh, with an ionised fraction of 1/2).  --graph adds coarse steps on the CUDA
graph (device time per step; for a subcycled tree on the fused coarse-step kernel,
the device time of its jobs summed per level).
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
    ap.add_argument("--dropin", default=None, choices=["plain", "rh"])
    ap.add_argument("--tracer", action="store_true", help="resident run of the -DWRADHYD library (dX = d/2)")
    ap.add_argument("--column", type=int, default=0,
                    help="column kernel of complete periodic levels (mixed): 0 autotuned, -1 off, n planes per item")
    ap.add_argument("--graph", action="store_true", help="also time coarse steps on the CUDA graph")
    ap.add_argument("--fused", default="auto", choices=["auto", "on", "off", "2", "3", "4"],
                    help="subcycled graph steps: autotuned, fused kernel (as many tile groups as fit, or k), "
                         "or the level schedule's separate launches")
    a = ap.parse_args()
    cfg = {"random": lambda: configs.random_uniform(level=a.level), "turb": lambda: configs.turb(level=a.level),
           "sod": lambda: configs.sod(level=a.level), "sedov": configs.sedov, "cosmo": configs.cosmo,
           "amr": configs.small_amr}[a.config]()
    if a.dropin is not None:
        return dropin(a, cfg)
    if a.tracer:
        from .tree import OctTree
        tree = cfg.build(lambda lc, lm: OctTree(lc, lm, rh=True))
        for lev in range(cfg.lcoarse, cfg.lmax + 1):
            if tree.noct(lev):
                tree.set_tracer(lev, 0.5 * tree.get_fields(lev, 0)[0])
    else:
        tree = cfg.build()
    # host-driven schedule: every level-kernel launch is timed with CUDA events
    r = ResidentHydro(tree, precision=PREC_MIXED if a.precision == "mixed" else PREC_FP64, trans=cfg.trans,
                      cfl=cfg.cfl, use_graph=False, column=a.column)
    L = lib("rh" if a.tracer else False)
    per_step = []
    tot_ms, tot_n, tot_cells = 0.0, 0, 0
    levels = {}
    for _ in range(a.steps):
        L.emma_hydro_reset_counters()
        r.coarse_step(nsub=cfg.nsub)
        avg, n, cells = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
        L.emma_hydro_kernel_timing(ctypes.byref(avg), ctypes.byref(n), ctypes.byref(cells))
        per_step.append(round(avg.value * n.value, 4))
        tot_ms += avg.value * n.value
        tot_n += n.value
        tot_cells += cells.value
        for lev in range(cfg.lcoarse, cfg.lmax + 1):
            ms, n, cells = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
            L.emma_hydro_kernel_timing_level(lev, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(cells))
            if n.value:
                acc = levels.setdefault(lev, [0.0, 0, 0])
                acc[0] += ms.value
                acc[1] += n.value
                acc[2] += cells.value
    per_level = {lev: {"ms_per_launch": round(v[0] / v[1], 4), "launches": v[1],
                       "cell_updates_per_s": v[2] / (v[0] * 1e-3) if v[0] else None}
                 for lev, v in sorted(levels.items())}
    print(json.dumps({"config": cfg.name, "level": cfg.lcoarse, "precision": a.precision, "status": r.status(),
                      "column_planes": r.column_tuning(cfg.lcoarse)[0], "launches": tot_n,
                      "avg_launch_ms": tot_ms / max(tot_n, 1), "cells_per_launch": tot_cells / max(tot_n, 1),
                      "kernel_ms_per_step": per_step, "per_level": per_level,
                      "cell_updates_per_s_kernel": tot_cells / (tot_ms * 1e-3) if tot_ms else None}))
    if a.graph:
        graph_steps(a, cfg, r, L)


def graph_steps(a, cfg, r, L):
    """Coarse steps on the CUDA graph, timed with CUDA events on the library's stream."""
    modes = {"auto": "auto", "on": True, "off": False}
    r.set_fused(modes[a.fused] if a.fused in modes else int(a.fused))
    r.set_use_graph(True)
    r.coarse_step(nsub=cfg.nsub)  # captures the graph
    ms = []
    jobs = {}
    for _ in range(a.steps):
        t = ctypes.c_double()
        if L.emma_hydro_timed_coarse_steps(1e9, 1e9, cfg.nsub, 1, ctypes.byref(t)) != 0:
            raise RuntimeError(L.emma_hydro_last_error().decode())
        ms.append(round(t.value, 4))
        info = r.graph_info()
        if info[0]:
            for kind, lev, us, sched in r.fused_jobs():
                k = f"{'level' if kind == 1 else 'cfl'}_{lev}"
                acc = jobs.setdefault(k, [0.0, 0, 0.0])
                acc[0] += us
                acc[1] += 1
                acc[2] += sched
    f, ctas, groups, kernels = r.graph_info()
    mode, sweep = r.step_tuning()
    print(json.dumps({"graph": True, "fused": f, "ctas": ctas, "tile_groups_per_cta": groups,
                      "step_mode": mode, "step_sweep_ms": [round(x, 4) for x in sweep],
                      "kernels_per_step": kernels, "ms_per_step": ms, "status": r.status(),
                      "jobs_us_per_step": {k: round(v[0] / a.steps, 1) for k, v in sorted(jobs.items())},
                      "jobs_per_step": {k: v[1] // a.steps for k, v in sorted(jobs.items())},
                      "schedule_us_per_step": {k: round(v[2] / a.steps, 1) for k, v in sorted(jobs.items())}}))


def dropin(a, cfg):
    from .tree import OctTree
    from . import hydro as H
    from ._lib import EmmaHydroOptions
    key = "rh" if a.dropin == "rh" else False
    tree = cfg.build(lambda lc, lm: OctTree(lc, lm, rh=(key == "rh")))
    level = cfg.lmax
    if key == "rh":
        tree.set_tracer(level, 0.5 * tree.get_fields(level, 0)[0])
    L = lib(key)
    o = EmmaHydroOptions()
    L.emma_hydro_default_options(ctypes.byref(o))
    o.precision = PREC_MIXED if a.precision == "mixed" else PREC_FP64
    L.emma_hydro_set_options(ctypes.byref(o))
    L.emma_hydro_reset_counters()
    for _ in range(a.steps):
        H.clean_new_hydro(level, tree.firstoct, grav=key)
        H.HydroSolver(level, tree.firstoct, 1e-4, grav=key)
    avg, n, cells = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
    L.emma_hydro_kernel_timing(ctypes.byref(avg), ctypes.byref(n), ctypes.byref(cells))
    print(json.dumps({"config": cfg.name, "dropin": a.dropin, "precision": a.precision, "status": L.emma_hydro_status(),
                      "launches": n.value, "avg_launch_ms": avg.value,
                      "cells_per_launch": cells.value / max(n.value, 1)}))


if __name__ == "__main__":
    main()
