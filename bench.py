"""Benchmark of the hydro level advance on B200: cell-updates/s, mixed vs FP64.

python bench.py [--gpus N] [--steps K] [--warmup W] [--config turb] [--impl mine|reference]

A step is one coarse step of the hydro-only level schedule over the whole tree
(all levels, subcycled), i.e. one pass of the hot path over one batch of
synthetic input.  `value` = cell-updates/s of the mixed-precision path with the
state resident in HBM (one cell-update = one leaf cell advanced by one level
substep).  `e2e` = the same metric through the reference-facing entries on the
host OCT tree: every step calls clean_new_hydro + HydroSolver on each level, which
pack the level's cells, copy them to the device and back and unpack them.
`e2e_resident` = the resident C ABI with host buffers: every step uploads the
level states from pinned host memory and downloads them.
The FP64 plain path is timed on the same workload and reported beside it.

Multi-GPU: the path is run as independent replicas (one per rank), value =
cell-updates of all ranks / max time over ranks.

--impl reference times the reference's own CPU hydro (oracle/_ref, compiled from
its sources; single-threaded, as the reference is) on a bounded sample of the
same configuration.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 1024 * 1024
METRIC = "hydro cell-updates/s, mixed vs FP64 on 1 B200 at L1<=1e-5; % HBM roofline"
ALG_BYTES_PER_CELL = 80  # 5 FP64 primitives read + 5 written per cell-update


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return out
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except Exception:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if sm:
            out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(smax), reasons=sorted(reasons), samples=len(sm))
        return out


def build_config(name):
    from emma_b200 import configs
    if name == "turb":
        return configs.turb()
    if name == "roofline":
        return configs.random_uniform(level=8)
    if name == "sod":
        return configs.sod()
    if name == "sedov":
        return configs.sedov()
    if name == "cosmo":
        return configs.cosmo()
    raise SystemExit(f"unknown config {name}")


def traffic_per_cell(config, precision):
    """DRAM bytes per cell-update of the level kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        f = line.split()
        if f and not f[0].startswith("#") and f[0] == f"{config}/{precision}":
            return float(f[1])
    return None


def run_mine(args, rank, world):
    import torch
    from emma_b200 import ResidentHydro, PREC_FP64, PREC_MIXED, lib
    from emma_b200._lib import ptr

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    # a dedicated stream: the library launches on it and the CUDA events below are recorded on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    L = lib()
    cfg = build_config(args.config)
    t0 = time.time()
    tree = cfg.build()
    build_s = time.time() - t0
    levels = list(range(cfg.lcoarse, cfg.lmax + 1))
    L.emma_hydro_set_stream(ctypes.c_void_p(stream.cuda_stream))
    state_bytes = sum(5 * 8 * 8 * tree.noct(l) for l in levels)
    flush = state_bytes < 2 * L2_BYTES
    flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda") if flush else None

    results = {}
    for prec_name, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        # whole coarse steps: CUDA graph with the device-side level schedule
        r = ResidentHydro(tree, precision=prec, trans=cfg.trans, cfl=cfg.cfl, use_graph=True, gravity=args.gravity,
                          dual=args.dual)
        if args.gravity:
            for l in levels:
                r.set_force(l, *synthetic_force(tree, l))
        tuning = {}
        kernels = set()
        for l in levels:
            rec = r.tuning(l)
            if rec is not None:
                planes, csweep = r.column_tuning(l)
                xs, xms = r.column_xshfl(l)
                bal, bms = r.column_balanced(l)
                sweep = ("warp-shuffle" if xs else "shared-memory") + " x sweep, " + \
                    ("balanced runs per CTA" if bal else "items")
                tuning[str(l)] = {"tile_octs": rec[0], "ctas_per_sm": rec[1],
                                  "sweep_ms": {"4x4x2": [round(x, 4) for x in rec[2][0][:3]],
                                               "2x2x2": [round(x, 4) for x in rec[2][1][:3]],
                                               "column_planes_2_4_8_16_32_64": [round(x, 4) for x in csweep],
                                               "column_x_sweep_shared_memory_warp_shuffle": [round(x, 4) for x in xms],
                                               "column_items_balanced": [round(x, 4) for x in bms]},
                                  "kernel": f"column ({planes} planes per item, {sweep})" if planes else "brick"}
                kernels.add(f"column_kernel<2, {'true' if xs else 'false'}>" if planes else
                            ("level_batch_kernel<MathF32>" if prec == PREC_MIXED else "level_batch_kernel<MathF64>"))
        init_states = {l: r.state(l) for l in levels}
        r.coarse_step(nsub=cfg.nsub)  # builds and instantiates the graph
        for _ in range(max(args.warmup - 1, 0)):
            r.step_async(nsub=cfg.nsub)
        torch.cuda.synchronize()
        r.time()
        if world > 1:
            torch.distributed.barrier()
        L.emma_hydro_reset_counters()
        evs = []
        with ClockSampler(dev) as clk:
            torch.cuda.synchronize()
            for _ in range(args.steps):
                if flush:
                    flush_buf.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                r.step_async(nsub=cfg.nsub)
                b.record(stream)
                evs.append((a, b))
            torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        updates = L.emma_hydro_cell_updates()
        status = r.status()
        fused, fused_ctas, fused_groups, launches_per_step = r.graph_info()
        step_mode, step_sweep = r.step_tuning()
        if step_mode >= 0 and any(step_sweep):
            tuning["coarse_step"] = {"mode": "fused, %d tile groups per CTA" % step_mode if step_mode else
                                     "separate launches",
                                     "ms_per_step": {("separate launches" if k == 0 else f"fused, {k} groups"): round(x, 4)
                                                     for k, x in enumerate(step_sweep) if x > 0}}
        if fused:
            kernels.add("step_kernel<MathF32>" if prec == PREC_MIXED else "step_kernel<MathF64>")
        res = {"ms": ms, "updates": updates, "launches": launches_per_step * args.steps, "status": status,
               "clocks": clk.summary(), "autotune": tuning, "kernels": sorted(kernels),
               "fused_step": {"ctas": fused_ctas, "tile_groups_per_cta": fused_groups} if fused else None}
        # level-kernel time per launch: the same steps on the host-driven schedule,
        # each level-kernel launch timed with CUDA events on the library stream
        r2 = r
        r2.set_use_graph(False)
        for _ in range(2):
            r2.coarse_step(nsub=cfg.nsub)
        L.emma_hydro_reset_counters()
        for _ in range(min(args.steps, 5)):
            if flush:
                flush_buf.zero_()
                torch.cuda.synchronize()
            r2.coarse_step(nsub=cfg.nsub)
        kavg, kcnt, kcells = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
        L.emma_hydro_kernel_timing(ctypes.byref(kavg), ctypes.byref(kcnt), ctypes.byref(kcells))
        res.update(kernel_avg_ms=kavg.value, kernel_launches=kcnt.value, kernel_cells=kcells.value)
        # e2e through the C ABI with host buffers: H2D states, coarse step, D2H states
        r.set_use_graph(True)
        pinned = {l: torch.from_numpy(init_states[l]).pin_memory() for l in levels}
        outs = {l: torch.empty_like(pinned[l]).pin_memory() for l in levels}
        r.coarse_step(nsub=cfg.nsub)
        torch.cuda.synchronize()
        h2d = d2h = 0
        e2e_ms = 0.0
        for _ in range(args.steps):
            if flush:
                flush_buf.zero_()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for l in levels:
                L.emma_hydro_set_level_state(l, ctypes.c_void_p(pinned[l].data_ptr()))
                h2d += pinned[l].numel() * 8
            r.step_async(nsub=cfg.nsub)
            for l in levels:
                L.emma_hydro_get_level_state(l, ctypes.c_void_p(outs[l].data_ptr()))
                d2h += outs[l].numel() * 8
            b.record(stream)
            torch.cuda.synchronize()
            e2e_ms += a.elapsed_time(b)
        res["e2e_ms"] = e2e_ms
        res["h2d"] = h2d // max(args.steps, 1)
        res["d2h"] = d2h // max(args.steps, 1)
        # state after a few coarse steps from the initial condition, for the L1 comparison
        for l in levels:
            r.set_state(l, init_states[l])
        r.tsim = 0.0
        r.adt[:] = 0.0
        for _ in range(min(args.steps, 10)):
            r.coarse_step(nsub=cfg.nsub)
        res["final"] = {l: r.state(l) for l in levels}
        res["dt"] = {l: float(r.adt[l - 1]) for l in levels}
        results[prec_name] = res
    # e2e through the reference-facing entries on the host tree: every step calls
    # clean_new_hydro + HydroSolver once per level (finest first) at the level's
    # CFL step; each call packs the level from the OCT structs, copies it to the
    # device, runs the level kernel, copies it back and unpacks it
    # (the drop-in entries carry no gravity: a gravity run reports the resident e2e)
    results["dropin"] = None if args.gravity else run_dropin(args, L, cfg, tree, levels, results["mixed"]["dt"], world)
    # L1 of the mixed path against the FP64 path (the FP64 path equals the oracle to 1e-12)
    fm, ff = results["mixed"]["final"], results["fp64"]["final"]
    num = {k: 0.0 for k in ("rho", "p", "v")}
    den = {k: 0.0 for k in ("rho", "p", "v")}
    for l in levels:
        dv = 0.5 ** (3 * l)
        leaf = ~tree.split_mask(l)
        a, b = fm[l][:, leaf], ff[l][:, leaf]
        va, vb = np.sqrt((a[1:4] ** 2).sum(0)), np.sqrt((b[1:4] ** 2).sum(0))
        for k, (x, y) in {"rho": (a[0], b[0]), "p": (a[4], b[4]), "v": (va, vb)}.items():
            num[k] += np.abs(x - y).sum() * dv
            den[k] += np.abs(y).sum() * dv
    l1 = {k: float(num[k] / den[k]) for k in num}
    return cfg, tree, results, l1, build_s, flush


def max_over_ranks(values, world, device):
    """Each timing as the maximum over the ranks of the job (replicas: every rank
    advanced its own copy; the job took as long as the slowest rank)."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def synthetic_force(tree, level, amp=0.5):
    """Smooth periodic acceleration field (gravity workloads): a few Fourier modes."""
    c = tree.cell_centres(level)
    w = 2 * np.pi
    return (amp * np.sin(w * c[:, 1]), amp * np.cos(w * c[:, 2]), amp * np.sin(w * (c[:, 0] + c[:, 1])))


def run_dropin(args, L, cfg, tree, levels, dts, world):
    """Times the drop-in HydroSolver (mixed precision) on the host tree, wall
    clock around synchronous calls; returns ms, cell-updates and bytes copied."""
    import torch
    from emma_b200 import PREC_MIXED
    from emma_b200.hydro import options, clean_new_hydro, HydroSolver
    o = options(PREC_MIXED, cfg.trans, cfg.cfl, dual=args.dual)
    L.emma_hydro_set_options(ctypes.byref(o))
    order = sorted(levels, reverse=True)
    leaf = sum(int((~tree.split_mask(l)).sum()) for l in order)
    for _ in range(max(args.warmup, 1)):  # the first call of a level builds its mirror
        for l in order:
            clean_new_hydro(l, tree.firstoct)
            HydroSolver(l, tree.firstoct, dts[l])
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    L.emma_hydro_reset_counters()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for l in order:
            clean_new_hydro(l, tree.firstoct)
            HydroSolver(l, tree.firstoct, dts[l])
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3
    h2d, d2h = ctypes.c_longlong(), ctypes.c_longlong()
    L.emma_hydro_transfer_bytes(ctypes.byref(h2d), ctypes.byref(d2h))
    return {"ms": ms, "updates": L.emma_hydro_cell_updates(), "leaf_per_step": leaf,
            "h2d": h2d.value // max(args.steps, 1), "d2h": d2h.value // max(args.steps, 1),
            "status": L.emma_hydro_status()}


# Reference samples: the reference's own CPU hydro on the configuration's own tree at
# its full size.  A uniform level is sampled as a prefix of its oct list (stock
# clean_new_hydro + HydroSolver on the first REF_SAMPLE_OCTS octs, the rest of the
# tree in place as their neighbours); an AMR tree runs whole coarse steps.
REF_SAMPLE_OCTS = 65536


def _quiet(fn):
    """Run fn with the reference's stdout prints silenced."""
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        return fn()
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)


def reference_tree(config):
    """The configuration's tree built and filled by the reference (oracle/_ref), or None."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cfg = build_config(config)
    tx = bool(cfg.trans)
    if not oracle.ref_available(tx=tx):
        return cfg, None
    # room for every oct plus the reference's free-oct chain head (src/emma.c:765)
    ngrid = sum(8 ** (l - 1) for l in range(1, cfg.lmax + 1)) + 1024
    if cfg.lmax > cfg.lcoarse:
        ngrid = sum(8 ** (l - 1) for l in range(1, cfg.lcoarse + 1)) + 2 * 10 ** 6
    ref = _quiet(lambda: oracle.RefTree(cfg.lcoarse, cfg.lmax, tx=tx, ngridmax=ngrid))
    _quiet(lambda: cfg.build(lambda lc, lm: ref))  # the configuration's own generator, on the reference's tree
    return cfg, ref


def reference_steps(cfg, ref, nsteps):
    """nsteps samples; returns (seconds inside HydroSolver, cell-updates, sample text)."""
    ref.reset_counters()
    if cfg.lmax == cfg.lcoarse:
        n = min(REF_SAMPLE_OCTS, ref.noct(cfg.lcoarse))
        for _ in range(nsteps):
            _quiet(lambda: ref.hydro_solver_prefix(cfg.lcoarse, n))
        sample = (f"clean_new_hydro + HydroSolver on the first {n:,} octs ({8 * n:,} cells) of the "
                  f"{8 * ref.noct(cfg.lcoarse):,}-cell level-{cfg.lcoarse} list of the full-size tree, per step")
    else:
        _quiet(lambda: ref.run(nsteps, nsub=cfg.nsub))
        sample = "whole coarse steps (all levels, subcycled) of the full-size tree"
    return ref.hydro_seconds(), ref.cell_updates(), sample


def cpu_baseline_sample(config, nsteps=3):
    """The reference's own CPU hydro on a bounded sample of the same workload."""
    cfg, ref = reference_tree(config)
    if ref is None:
        return None
    secs, cells, sample = reference_steps(cfg, ref, 1 if cfg.lmax > cfg.lcoarse else nsteps)
    return {"value": cells / secs, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
            "sample": f"{cfg.name}: {sample}, {1 if cfg.lmax > cfg.lcoarse else nsteps} step(s)", "seconds": secs}


def run_reference(args):
    """--impl reference: the reference's CPU hydro on the same configuration at its
    full size, each step a bounded sample (see reference_steps)."""
    line = {"impl": "reference", "metric": METRIC, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True}
    t0 = time.time()
    cfg, ref = reference_tree(args.config)
    if ref is None:
        line["unavailable"] = "oracle/_ref (the reference CPU hydro compiled from its sources) is not built"
        print(json.dumps(line))
        return
    build_s = time.time() - t0
    if args.warmup:
        reference_steps(cfg, ref, args.warmup)
    t0 = time.time()
    secs, cells, sample = reference_steps(cfg, ref, args.steps)
    wall = time.time() - t0
    v = cells / secs
    leaf = sum(int(8 * ref.noct(l)) for l in range(cfg.lcoarse, cfg.lmax + 1))
    line.update({"value": v, "ms_per_step": 1000 * secs / max(args.steps, 1), "scaling": "weak",
                 "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                 "config": {"workload": cfg.name, "levels": [cfg.lcoarse, cfg.lmax], "tree_cells": leaf,
                            "sample": sample, "cells_per_step": cells // max(args.steps, 1)},
                 "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                                  "sample": f"{sample}; single-threaded like the reference's hydro"},
                 "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                 "wall_s": wall, "tree_build_s": build_s})
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="roofline", choices=["turb", "roofline", "sod", "sedov", "cosmo"])
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--gravity", action="store_true",
                    help="gravity-coupled hydro (-DWGRAV) with a smooth synthetic acceleration field")
    ap.add_argument("--dual", action="store_true", help="dual-energy hydro (-DDUAL_E)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    import torch
    import datetime
    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    cfg, tree, res, l1, build_s, flushed = run_mine(args, rank, world)
    mixed, fp64 = res["mixed"], res["fp64"]
    # max over ranks of the timed device time
    dropin = res["dropin"]
    ms_m, ms_f, ms_e = mixed["ms"], fp64["ms"], mixed["e2e_ms"]
    ms_d = dropin["ms"] if dropin is not None else ms_e
    ms_m, ms_f, ms_e, ms_d = max_over_ranks([ms_m, ms_f, ms_e, ms_d], world, "cuda")
    upd_m = mixed["updates"] * world
    value = upd_m / (ms_m * 1e-3)
    value_fp64 = fp64["updates"] * world / (ms_f * 1e-3)
    e2e_resident = mixed["updates"] * world / (ms_e * 1e-3)
    e2e = (dropin["updates"] if dropin is not None else mixed["updates"]) * world / (ms_d * 1e-3)
    peak, peak_kind = peaks()
    cells_per_launch = mixed["kernel_cells"] / max(mixed["kernel_launches"], 1)
    achieved = ALG_BYTES_PER_CELL * cells_per_launch / (mixed["kernel_avg_ms"] * 1e-3) / 1e9
    achieved_f = ALG_BYTES_PER_CELL * cells_per_launch / (fp64["kernel_avg_ms"] * 1e-3) / 1e9
    tpc = traffic_per_cell(args.config, "mixed")
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    cpu = None if args.no_cpu_baseline or world > 1 else cpu_baseline_sample(args.config)
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_m / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 flux / f64 state", "data": "synthetic",
        "config": {"workload": cfg.name, "levels": [cfg.lcoarse, cfg.lmax],
                   "leaf_cells_per_step": mixed["updates"] // args.steps,
                   "precision": "mixed (FP32 reconstruction/HLLC, FP64 compensated update)",
                   "l2": "flushed between steps (256 MiB write)" if flushed else "state larger than L2",
                   "parallelism": f"replicas x{world}", "cfl": cfg.cfl, "nsub": cfg.nsub,
                   "gravity": bool(args.gravity), "dual_energy": bool(args.dual)},
        "fp64": {"value": value_fp64, "unit": "cell-updates/s", "ms_per_step": ms_f / args.steps,
                 "roofline_frac": achieved_f / peak, "status": fp64["status"]},
        "mixed_over_fp64": value / value_fp64,
        "l1_vs_fp64": l1,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": (tpc * cells_per_launch) if tpc else None,
                     "kernel": " + ".join(mixed["kernels"]), "alg_bytes_per_cell": ALG_BYTES_PER_CELL,
                     "cells_per_launch": cells_per_launch, "avg_launch_ms": mixed["kernel_avg_ms"]},
        "e2e": ({"value": e2e, "unit": "cell-updates/s", "h2d_bytes_per_step": dropin["h2d"],
                 "d2h_bytes_per_step": dropin["d2h"], "ms_per_step": ms_d / args.steps,
                 "api": "clean_new_hydro + HydroSolver per level on the host OCT tree (mixed), wall clock",
                 "leaf_cells_per_step": dropin["leaf_per_step"], "status": dropin["status"]}
                if dropin is not None else
                {"value": e2e, "unit": "cell-updates/s", "h2d_bytes_per_step": mixed["h2d"],
                 "d2h_bytes_per_step": mixed["d2h"], "ms_per_step": ms_d / args.steps,
                 "api": "resident C ABI with pinned host states (the drop-in entries have no gravity coupling)"}),
        "e2e_resident": {"value": e2e_resident, "unit": "cell-updates/s", "h2d_bytes_per_step": mixed["h2d"],
                         "d2h_bytes_per_step": mixed["d2h"],
                         "api": "emma_hydro_set_level_state + coarse step + emma_hydro_get_level_state, pinned host"},
        "autotune": {"mixed": mixed["autotune"], "fp64": fp64["autotune"],
                     "candidates": "brick 4x4x2 octs x1 or 2x2x2 octs x4 per 256-thread tile, 1..occupancy CTAs "
                                   "per SM; mixed path on complete periodic levels without split cells: the column "
                                   "kernel (16x16-cell columns) with 2..64 cell planes per work item"},
        "gpu_launches": mixed["launches"],
        "gpu_launches_per_step": mixed["launches"] // max(args.steps, 1),
        "fused_step": mixed["fused_step"],
        "clocks": mixed["clocks"],
        "status": mixed["status"],
        "host_tree_build_s": build_s,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
