"""Host-side interface of the hydro level advance (mirrors the reference's entry points).

ResidentHydro drives the resident path: upload a tree once, advance levels or
coarse steps on the GPU, read states back.  The reference-named drop-in entries
(HydroSolver, advancehydroGPU, clean_new_hydro) are exposed as functions with
the reference's arguments; they operate on the caller's host tree in place.
"""
import ctypes

import numpy as np

from ._lib import EmmaHydroOptions, PREC_FP64, PREC_MIXED, check, lib, ptr


def options(precision=PREC_FP64, trans=0, cfl=0.85, device=0, use_graph=True, tile_octs=0, gravity=False,
            dual=False, column=0, fused="auto", xshfl=0, balanced=0):
    """tile_octs: 0 = brick shape autotuned per level at upload, 32 = 4x4x2-oct
    bricks, 8 = 2x2x2-oct bricks (four per tile).  gravity: the -DWGRAV coupling
    (forces from ResidentHydro.set_force).  dual: the -DDUAL_E tracked internal energy.
    column (mixed path, complete periodic levels without split cells): 0 = the
    autotuner picks the column kernel or the brick kernel, -1 = brick kernel only,
    n > 0 = column kernel with n cell planes per work item.  fused (subcycled
    coarse steps on the graph): "auto" = the autotuner picks the fused kernel (one
    persistent kernel per coarse step) or the level schedule's separate launches,
    True = fused with as many tile groups per CTA as fit, an int k = fused with k
    groups, False = separate launches.  xshfl (column kernel's x sweep): 0 = the
    autotuner's pick, 1 = warp shuffles, -1 = shared memory.  balanced (column
    kernel's work split): 0 = the autotuner's pick, 1 = an equal run of the level's
    column-planes per CTA, -1 = items of the chosen depth."""
    o = EmmaHydroOptions()
    lib().emma_hydro_default_options(ctypes.byref(o))
    o.precision, o.trans_flags, o.cfl, o.device = precision, trans, cfl, device
    o.use_graph = 1 if use_graph else 0
    o.tile_octs = tile_octs
    o.gravity = 1 if gravity else 0
    o.dual_energy = 1 if dual else 0
    o.column = column
    o.column_xshfl = xshfl
    o.column_balanced = balanced
    if fused == "auto":
        o.fused_step = 0
    elif fused is True:
        o.fused_step = 99
    elif fused is False:
        o.fused_step = -1
    else:
        o.fused_step = int(fused)
    return o


class ResidentHydro:
    """Levels lcoarse..lmax of an oct tree resident on the GPU."""

    def __init__(self, tree, precision=PREC_FP64, trans=0, cfl=0.85, rank=0, use_graph=True, tile_octs=0,
                 gravity=False, dual=False, column=0, fused="auto", xshfl=0, balanced=0):
        self.tree = tree
        self.column = column
        self.xshfl = xshfl
        self.balanced = balanced
        self.fused = fused
        self.gravity, self.dual = gravity, dual
        self.lcoarse, self.lmax = tree.lcoarse, tree.lmax
        self.trans, self.cfl, self.use_graph, self.tile_octs = trans, cfl, use_graph, tile_octs
        self.precision = precision
        # a tree of the -DWRADHYD layout runs on libemmahydro_rh.so (its tracer advanced too)
        self._L = L = lib("he" if getattr(tree, "he", False) else ("rh" if getattr(tree, "rh", False) else False))
        o = self._options()
        check(L.emma_hydro_init(ctypes.byref(o)), "init")
        check(L.emma_hydro_set_options(ctypes.byref(o)), "set_options")
        L.emma_hydro_clear_status()
        check(L.emma_hydro_tree_upload(tree.firstoct, self.lcoarse, self.lmax, rank), "tree_upload")
        self.adt = np.zeros(self.lmax)
        self.tsim = 0.0

    def _options(self):
        return options(self.precision, self.trans, self.cfl, use_graph=self.use_graph, tile_octs=self.tile_octs,
                       gravity=self.gravity, dual=self.dual, column=self.column, fused=self.fused,
                       xshfl=self.xshfl, balanced=self.balanced)

    def _apply(self):
        o = self._options()
        check(self._L.emma_hydro_set_options(ctypes.byref(o)), "set_options")

    def set_use_graph(self, use_graph):
        """Switch between CUDA-graph coarse steps and the host-driven schedule
        (the resident tree and its tuned plans stay)."""
        self.use_graph = use_graph
        self._apply()

    def set_precision(self, precision):
        self.precision = precision
        self._apply()

    def set_fused(self, fused):
        """Mode of subcycled graph steps (see options: "auto", True, k, False)."""
        self.fused = fused
        self._apply()

    def graph_info(self):
        """The captured coarse step: (1 if it is one fused kernel, its CTAs, tile groups
        per CTA, kernel launches of one coarse step)."""
        f, ctas, groups, kn = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._L.emma_hydro_graph_info(ctypes.byref(f), ctypes.byref(ctas), ctypes.byref(groups),
                                            ctypes.byref(kn)), "graph_info")
        return f.value, ctas.value, groups.value, kn.value

    def step_tuning(self):
        """(coarse-step mode: 0 separate launches, k fused with k tile groups; ms per
        coarse step the autotuner measured, [0] separate launches, [k] k groups)."""
        groups = ctypes.c_int()
        sweep = np.zeros(5)
        check(self._L.emma_hydro_step_tuning(ctypes.byref(groups), ptr(sweep)), "step_tuning")
        return groups.value, sweep

    def fused_jobs(self):
        """The jobs of the last fused coarse step: list of (kind, level, duration in us,
        schedule in us), kind 1 a level iteration, 2 a CFL reduction; the duration runs
        from its release to the next job's release and includes the schedule that ran
        before that release (the last item)."""
        kinds, levels, t, sch = np.zeros(256, np.int32), np.zeros(256, np.int32), np.zeros(256), np.zeros(256)
        n = self._L.emma_hydro_fused_job_log(256, ptr(kinds), ptr(levels), ptr(t), ptr(sch))
        if n < 0:
            check(-n, "fused_job_log")
        return [(int(kinds[i]), int(levels[i]), float(t[i + 1] - t[i]), float(sch[i + 1])) for i in range(n - 1)]

    def step_async(self, dt_param=1e9, time_max=1e9, nsub=2):
        """Queue one coarse step on the device schedule without waiting."""
        check(self._L.emma_hydro_advance_coarse_step_async(dt_param, time_max, nsub), "advance_coarse_step_async")

    def time(self):
        t = ctypes.c_double()
        check(self._L.emma_hydro_get_time(ctypes.byref(t), ptr(self.adt)), "get_time")
        self.tsim = t.value
        return self.tsim

    def noct(self, level):
        return self._L.emma_hydro_level_noct(level)

    def state(self, level):
        n8 = 8 * self.noct(level)
        out = np.zeros((5, n8))
        if n8:
            check(self._L.emma_hydro_get_level_state(level, ptr(out)), "get_level_state")
        return out

    def set_state(self, level, st):
        st = np.ascontiguousarray(st, dtype=np.float64)
        check(self._L.emma_hydro_set_level_state(level, ptr(st)), "set_level_state")

    def set_force(self, level, fx, fy, fz):
        """Gravitational acceleration of the level's cells (gravity=True uploads)."""
        f = np.ascontiguousarray(np.stack([fx, fy, fz]), dtype=np.float64)
        check(self._L.emma_hydro_set_level_force(level, ptr(f)), "set_level_force")

    def comptstep(self, level):
        dt = ctypes.c_double()
        check(self._L.emma_hydro_comptstep(level, ctypes.byref(dt)), "comptstep")
        return dt.value

    def clean_new(self, level):
        check(self._L.emma_hydro_clean_new(level), "clean_new")

    def advance_level(self, level, dt):
        check(self._L.emma_hydro_advance_level(level, dt), "advance_level")

    def coarse_step(self, dt_param=1e9, time_max=1e9, nsub=2):
        t = ctypes.c_double(self.tsim)
        check(self._L.emma_hydro_advance_coarse_step(dt_param, time_max, nsub, ctypes.byref(t), ptr(self.adt)),
              "advance_coarse_step")
        self.tsim = t.value
        return self.tsim

    def status(self):
        return self._L.emma_hydro_status()

    def tuning(self, level):
        """Autotuner record of a level: (octs per brick, CTAs per SM, sweep) with
        sweep[shape][ctas-1] the measured ms per launch (0 = not tried)."""
        octs, ctas = ctypes.c_int(), ctypes.c_int()
        sweep = np.zeros(8)
        rc = self._L.emma_hydro_tuning(level, ctypes.byref(octs), ctypes.byref(ctas), ptr(sweep))
        return (octs.value, ctas.value, sweep.reshape(2, 4)) if rc == 0 else None

    def column_tuning(self, level):
        """(cell planes per work item of the level's column-kernel launches, 0 = brick
        kernel; ms per launch the autotuner measured with 2, 4, 8, 16, 32, 64 planes)."""
        planes = ctypes.c_int()
        sweep = np.zeros(6)
        check(self._L.emma_hydro_column_tuning(level, ctypes.byref(planes), ptr(sweep)), "column_tuning")
        return planes.value, sweep

    def column_xshfl(self, level):
        """(1 if the level's column-kernel launches pass x face states by warp shuffle,
        0 if through shared memory; the autotuner's ms per launch of the shared-memory
        and the shuffle sweep at the chosen depth, 0 = not timed)."""
        on = ctypes.c_int()
        ms = np.zeros(2)
        check(self._L.emma_hydro_column_xshfl(level, ctypes.byref(on), ptr(ms)), "column_xshfl")
        return on.value, ms

    def column_balanced(self, level):
        """(1 if the level's column-kernel launches give each CTA an equal run of the
        level's column-planes, 0 for items of the chosen depth; the autotuner's ms per
        launch of the items and the balanced runs, 0 = not timed)."""
        on = ctypes.c_int()
        ms = np.zeros(2)
        check(self._L.emma_hydro_column_balanced(level, ctypes.byref(on), ptr(ms)), "column_balanced")
        return on.value, ms

    def set_column(self, column, xshfl=None):
        """Column-kernel options (see options); the resident tree and its plans stay."""
        self.column = column
        if xshfl is not None:
            self.xshfl = xshfl
        self._apply()

    def download(self):
        check(self._L.emma_hydro_tree_download(self.tree.firstoct), "tree_download")


class CpuInfo(ctypes.Structure):
    """The part of the reference's struct CPUINFO (src/prototypes.h) the drop-in
    entries read: `rank`, its first member."""
    _fields_ = [("rank", ctypes.c_int), ("nproc", ctypes.c_int)]


class RunParams(ctypes.Structure):
    """The leading members of the reference's struct RUNPARAMS (src/prototypes.h,
    REAL = double) up to lmax; clean_new_hydro reads lcoarse."""
    _fields_ = [("npartmax", ctypes.c_int), ("ngridmax", ctypes.c_int), ("nbuff", ctypes.c_int),
                ("ndumps", ctypes.c_int), ("dt_dump", ctypes.c_double), ("nsteps", ctypes.c_int),
                ("lcoarse", ctypes.c_int), ("lmax", ctypes.c_int)]


def _ref(x):
    return None if x is None else ctypes.byref(x)


def HydroSolver(level, firstoct, dtnew, cpu=None, grav=False):
    """Drop-in HydroSolver (src/hydro_utils.c:3378) on a host tree; grav: a tree of
    the -DWGRAV layout through libemmahydro_grav.so (gravity-coupled advance), or
    "rh": a tree of the -DWRADHYD layout through libemmahydro_rh.so (the ionised
    density advected too).  cpu: a CpuInfo (advance the octs of cpu.rank only), or
    None for rank 0."""
    lib(grav).HydroSolver(level, None, firstoct, _ref(cpu), None, 0, dtnew)


def advancehydroGPU(firstoct, level, dtnew, cpu=None, grav=False):
    """Drop-in advancehydroGPU (src/hydro_utils_gpu.cu:2470); returns octs advanced."""
    return lib(grav).advancehydroGPU(firstoct, level, _ref(cpu), None, 0, 0.5 ** level, dtnew)


def clean_new_hydro(level, firstoct, grav=False, cpu=None, param=None):
    """Drop-in clean_new_hydro (src/hydro_utils.c:3501); param: a RunParams
    (its lcoarse decides whether the coarser level's octs of other ranks start
    from zero, as in a -DWMPI run)."""
    lib(grav).clean_new_hydro(level, _ref(param), firstoct, _ref(cpu))


def dump_alloct(folder, firstoct, lcoarse, lmax, ids, names, rank=0, ndumps=0, tsim=0.0, grav=False):
    """Field dump in the reference's ALLOCT format (dumpalloct_serial, src/io.c:1233):
    one file per (id, name) under folder (ending in '/').  A tree resident on the
    GPU dumps its hydro fields (ids 13-17) from the device state."""
    idv = (ctypes.c_int * len(ids))(*ids)
    nv = (ctypes.c_char_p * len(names))(*[n.encode() for n in names])
    return lib(grav).emma_hydro_dump_alloct(folder.encode(), firstoct, lcoarse, lmax, rank, ndumps, tsim, len(ids),
                                            ctypes.cast(idv, ctypes.c_void_p), ctypes.cast(nv, ctypes.c_void_p))


def grav_correction(level, firstoct, dt, cpu=None):
    """Drop-in grav_correction (src/hydro_utils.c:2388) of libemmahydro_grav.so."""
    lib(True).grav_correction(level, None, firstoct, _ref(cpu), dt)
