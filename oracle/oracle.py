"""ctypes bindings of the oracle libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm, always as the checker or the timed CPU
baseline, never on the product path.

  Restatement  -- oracle/_build/liboracle[_grav].so, the C restatement of the hydro
                  level advance (hydro_oracle.c); runs in place on any struct OCT tree
                  (_grav: the -DWGRAV cell layout, gravity-coupled hydro).
  RefTree      -- oracle/_ref/libemmaref[_tx|_grav].so, the reference's own CPU hydro
                  compiled from its sources with ref_driver.c (tree built by the
                  reference's build_initial_grid / L_refine_cells).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
ORACLE_LIB_GRAV = os.path.join(HERE, "_build", "liboracle_grav.so")
ORACLE_LIB_RH = os.path.join(HERE, "_build", "liboracle_rh.so")
ORACLE_LIB_HE = os.path.join(HERE, "_build", "liboracle_he.so")
REF_LIB = os.path.join(HERE, "_ref", "libemmaref.so")
REF_LIB_TX = os.path.join(HERE, "_ref", "libemmaref_tx.so")
REF_LIB_GRAV = os.path.join(HERE, "_ref", "libemmaref_grav.so")
REF_LIB_DUAL = os.path.join(HERE, "_ref", "libemmaref_dual.so")
REF_LIB_RH = os.path.join(HERE, "_ref", "libemmaref_rh.so")
REF_LIB_SP = os.path.join(HERE, "_ref", "libemmaref_sp.so")
REF_LIB_MARK = os.path.join(HERE, "_ref", "libemmaref_mark.so")
REF_LIB_HE = os.path.join(HERE, "_ref", "libemmaref_he.so")
REF_LIB_IO = os.path.join(HERE, "_ref", "libemmaref_io.so")

HYDROTEST = 0x40
DUAL_E = 0x80
c_int, c_double, c_void_p, c_ll = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def flags_for(trans, dual=False):
    """Oracle flags for the library's transmissive flags (which follow HYDROTEST
    semantics) and dual-energy option."""
    return ((trans | HYDROTEST) if trans else 0) | (DUAL_E if dual else 0)


class Restatement:
    """grav=True: the -DWGRAV layout and gravity coupling (liboracle_grav.so);
    rh=True: the -DWRADHYD layout with the advected ionised density (liboracle_rh.so);
    he=True: its -DHELIUM variant, three tracers (liboracle_he.so)."""
    _libs = {}

    def __init__(self, grav=False, rh=False, he=False):
        assert (grav + rh + he) <= 1, "one layout at a time"
        path = ORACLE_LIB_GRAV if grav else (ORACLE_LIB_RH if rh else (ORACLE_LIB_HE if he else ORACLE_LIB))
        if path not in Restatement._libs:
            if not os.path.exists(path):
                raise RuntimeError(f"oracle restatement not built: {path}")
            L = ctypes.CDLL(path)
            L.orc_hydro_solver.argtypes = [c_void_p, c_int, c_double, c_int]
            L.orc_hydro_solver.restype = c_int
            L.orc_clean_new_hydro.argtypes = [c_void_p, c_int]
            L.orc_comptstep_hydro.argtypes = [c_void_p, c_int, c_double]
            L.orc_comptstep_hydro.restype = c_double
            L.orc_run.argtypes = [c_void_p, c_int, c_int, c_int, c_double, c_double, c_int, c_double, c_int,
                                  c_double, c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]
            L.orc_run.restype = c_double
            L.orc_cell_updates.restype = c_ll
            if grav:
                L.orc_grav_correction.argtypes = [c_void_p, c_int, c_double]
                L.orc_grav_correction.restype = c_int
            L.orc_dump_alloct.argtypes = [ctypes.c_char_p, c_void_p, c_int, c_int, c_int, c_int, c_double, c_int,
                                          c_void_p, c_void_p]
            L.orc_dump_alloct.restype = c_int
            Restatement._libs[path] = L
        self.L = Restatement._libs[path]
        self.grav = grav

    def run(self, firstoct, lcoarse, lmax, nsteps, cfl, trans=0, nsub=2, dt_param=1e9, time_max=1e9, tsim0=0.0,
            dual=False):
        adt = np.zeros(lmax)
        nd, err = c_int(), c_int()
        t = self.L.orc_run(firstoct, lcoarse, lmax, nsteps, dt_param, time_max, nsub, cfl, flags_for(trans, dual),
                           tsim0, _p(adt), ctypes.byref(nd), ctypes.byref(err))
        return t, adt, err.value

    def hydro_solver(self, firstoct, level, dt, trans=0, dual=False):
        return self.L.orc_hydro_solver(firstoct, level, dt, flags_for(trans, dual))

    def clean_new(self, firstoct, level):
        self.L.orc_clean_new_hydro(firstoct, level)

    def comptstep(self, firstoct, level, cfl):
        return self.L.orc_comptstep_hydro(firstoct, level, cfl)

    def grav_correction(self, firstoct, level, dt):
        return self.L.orc_grav_correction(firstoct, level, dt)

    def dump_alloct(self, folder, firstoct, lcoarse, lmax, ids, names, rank=0, ndumps=0, tsim=0.0):
        """dumpalloct_serial (src/io.c:1233) restated: one file per field under folder."""
        idv = (c_int * len(ids))(*ids)
        nv = (ctypes.c_char_p * len(names))(*[n.encode() for n in names])
        return self.L.orc_dump_alloct(folder.encode(), firstoct, lcoarse, lmax, rank, ndumps, tsim, len(ids),
                                      ctypes.cast(idv, c_void_p), ctypes.cast(nv, c_void_p))

    def sizeof_oct(self):
        return self.L.orc_sizeof_oct()

    def cell_updates(self):
        return self.L.orc_cell_updates()

    def reset(self):
        self.L.orc_reset_counters()


class GravClone:
    """Copy of a default-layout tree in the -DWGRAV layout (liboracle_grav.so), for
    running the gravity restatement on the same octs and list order."""

    def __init__(self, tree):
        R = Restatement(grav=True)
        L = R.L
        L.orc_grav_clone.restype = c_void_p
        L.orc_grav_clone.argtypes = [c_void_p, c_int]
        L.orc_grav_first.restype = c_void_p
        L.orc_grav_first.argtypes = [c_void_p]
        L.orc_grav_set_force.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p]
        L.orc_grav_get_field.argtypes = [c_void_p, c_int, c_int, c_void_p]
        L.orc_grav_free.argtypes = [c_void_p]
        self.R, self.L, self.src = R, L, tree
        self.lcoarse, self.lmax = tree.lcoarse, tree.lmax
        self.h = L.orc_grav_clone(tree.firstoct, tree.lmax)
        if not self.h:
            raise RuntimeError("tree copy into the gravity layout failed")

    @property
    def firstoct(self):
        return self.L.orc_grav_first(self.h)

    def noct(self, level):
        return self.src.noct(level)

    def set_force(self, level, fx, fy, fz):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (fx, fy, fz)]
        self.L.orc_grav_set_force(self.h, level, *[_p(a) for a in arrs])

    def get_fields(self, level, which=0):
        n = self.src.noct(level)
        out = np.zeros((7, 8 * n))
        if n:
            self.L.orc_grav_get_field(self.h, level, which, _p(out))
        return out

    def run(self, nsteps, cfl, nsub=2, dt_param=1e9, time_max=1e9, tsim0=0.0):
        return self.R.run(self.firstoct, self.lcoarse, self.lmax, nsteps, cfl, nsub=nsub, dt_param=dt_param,
                          time_max=time_max, tsim0=tsim0)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_grav_free(self.h)
            self.h = None


def _ref_path(tx=False, grav=False, dual=False, rh=False, sp=False, mark=False, he=False):
    if he:
        return REF_LIB_HE
    if mark:
        return REF_LIB_MARK
    if sp:
        return REF_LIB_SP
    if rh:
        return REF_LIB_RH
    return REF_LIB_DUAL if dual else (REF_LIB_GRAV if grav else (REF_LIB_TX if tx else REF_LIB))


def ref_available(tx=False, grav=False, dual=False, rh=False, sp=False, mark=False, he=False):
    return os.path.exists(_ref_path(tx, grav, dual, rh, sp, mark, he))


def ref_dump_available():
    return os.path.exists(REF_LIB_IO)


_io_lib = []


def ref_dump_alloct(folder, firstoct, lcoarse, lmax, ids, names, rank=0, ndumps=0, tsim=0.0):
    """The reference's own dumpalloct_serial (src/io.c:1233, oracle/ref_io_driver.c) on a
    tree of the plain cell layout (any builder: struct OCT and CELL are the reference's):
    one file per field under folder (which ends with '/')."""
    if not _io_lib:
        L = ctypes.CDLL(REF_LIB_IO, mode=os.RTLD_NOW | os.RTLD_LOCAL)
        L.ref_dump_alloct.argtypes = [ctypes.c_char_p, c_void_p, c_int, c_int, c_int, c_int, c_double, c_int,
                                      ctypes.POINTER(c_int), ctypes.POINTER(ctypes.c_char_p)]
        L.ref_dump_alloct.restype = c_int
        _io_lib.append(L)
    n = len(ids)
    id_arr = (c_int * n)(*ids)
    name_arr = (ctypes.c_char_p * n)(*[x.encode() for x in names])
    return _io_lib[0].ref_dump_alloct(folder.encode(), firstoct, lcoarse, lmax, rank, ndumps, tsim, n, id_arr,
                                      name_arr)


class RefTree:
    """A tree built and advanced by the reference's own CPU hydro (one live tree per library)."""

    _libs = {}

    def __init__(self, lcoarse, lmax, tx=False, ngridmax=None, hstride=1024, grav=False, dual=False, rh=False,
                 sp=False, mark=False, he=False):
        """sp: the reference built with -DSINGLEPRECISION (REAL = float); mark: its
        src/amr.c built with the density refinement criterion (ref_amr_sntest.c);
        he: built with -DWRADHYD -DHELIUM (three tracers)."""
        assert (tx + grav + dual + rh + sp + mark + he) <= 1, "one build variant at a time"
        path = _ref_path(tx, grav, dual, rh, sp, mark, he)
        if path not in RefTree._libs:
            if not os.path.exists(path):
                raise RuntimeError(f"reference oracle not built: {path}")
            L = ctypes.CDLL(path, mode=os.RTLD_NOW | os.RTLD_LOCAL)
            L.ref_run.restype = c_double
            L.ref_run.argtypes = [c_int, c_double, c_double, c_int, c_double, ctypes.POINTER(c_int)]
            L.ref_comptstep_hydro.restype = c_double
            L.ref_hydro_solver.argtypes = [c_int, c_double]
            L.ref_grid_base.restype = c_void_p
            L.ref_firstoct_array.restype = c_void_p
            L.ref_hydro_seconds.restype = c_double
            L.ref_cell_updates.restype = c_ll
            L.ref_adt.restype = c_double
            L.ref_init.argtypes = [c_int, c_int, c_int, c_int]
            RefTree._libs[path] = L
        self.grav = grav
        self.L = RefTree._libs[path]
        self.lcoarse, self.lmax = lcoarse, lmax
        if ngridmax is None:
            ngridmax = sum(8 ** (l - 1) for l in range(1, lcoarse + 1)) * (2 if lmax > lcoarse else 1) + 8 ** min(lmax, 7) // 2 + 1024
        self.ngridmax = int(ngridmax)
        if self.L.ref_init(lcoarse, lmax, self.ngridmax, hstride) != 0:
            raise RuntimeError("ref_init failed")

    @property
    def firstoct(self):
        return self.L.ref_firstoct_array()

    def noct(self, level):
        return self.L.ref_noct(level)

    def set_tracer(self, level, dX):
        """-DWRADHYD build: the ionised density dX of field and fieldnew (list order)."""
        a = np.ascontiguousarray(dX, dtype=np.float64)
        self.L.ref_set_tracer.argtypes = [c_int, c_void_p]
        self.L.ref_set_tracer(level, _p(a))

    def set_tracer_n(self, level, t, x):
        """Tracer t (0: dX; -DHELIUM 1: dXHE, 2: dXXHE) of field and fieldnew."""
        a = np.ascontiguousarray(x, dtype=np.float64)
        self.L.ref_set_tracer_n.argtypes = [c_int, c_int, c_void_p]
        self.L.ref_set_tracer_n(level, t, _p(a))

    def get_tracer_n(self, level, t, which=0):
        out = np.zeros(8 * self.noct(level))
        self.L.ref_get_tracer_n.argtypes = [c_int, c_int, c_int, c_void_p]
        self.L.ref_get_tracer_n(level, t, which, _p(out))
        return out

    def get_tracer(self, level, which=0):
        out = np.zeros(8 * self.noct(level))
        self.L.ref_get_tracer.argtypes = [c_int, c_int, c_void_p]
        self.L.ref_get_tracer(level, which, _p(out))
        return out

    def oct_xyz(self, level):
        n = self.noct(level)
        out = np.zeros((n, 3))
        if n:
            self.L.ref_oct_xyz(level, _p(out))
        return out

    def cell_centres(self, level):
        dx = 0.5 ** level
        off = np.array([[c % 2, (c // 2) % 2, c // 4] for c in range(8)], dtype=np.float64)
        return (self.oct_xyz(level)[:, None, :] + (off[None] + 0.5) * dx).reshape(-1, 3)

    def refine(self, level, mark):
        mark = np.ascontiguousarray(mark, dtype=np.int8)
        return self.L.ref_refine(level, _p(mark))

    def refine_where(self, level, pred):
        return self.refine(level, pred(self.cell_centres(level)))

    def set_fields(self, level, d, u, v, w, p):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (d, u, v, w, p)]
        self.L.ref_set_field(level, *[_p(a) for a in arrs])

    def get_fields(self, level, which=0):
        n = self.noct(level)
        out = np.zeros((7, 8 * n))
        if n:
            self.L.ref_get_field(level, which, _p(out))
        return out

    def set_force(self, level, fx, fy, fz):
        """Gravitational acceleration of every cell of a level (gravity build only)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (fx, fy, fz)]
        self.L.ref_set_force(level, *[_p(a) for a in arrs])

    def sizeof_oct(self):
        return self.L.ref_sizeof_oct()

    def save_amr(self, filename, tsim, tinit, nsteps, ndumps, units7):
        """The reference's save_amr (src/restart.c:12) of this tree."""
        u = np.ascontiguousarray(units7, dtype=np.float64)
        self.L.ref_save_amr.argtypes = [ctypes.c_char_p, c_double, c_double, c_int, c_int, c_void_p]
        self.L.ref_save_amr(filename.encode(), tsim, tinit, nsteps, ndumps, _p(u))

    def restore_amr(self, filename):
        """The reference's restore_amr (src/restart.c:108) into this tree's pool."""
        t, ti, ns, nd = c_double(), c_double(), c_int(), c_int()
        self.L.ref_restore_amr.argtypes = [ctypes.c_char_p] + [ctypes.c_void_p] * 4
        self.L.ref_restore_amr(filename.encode(), ctypes.byref(t), ctypes.byref(ti), ctypes.byref(ns),
                               ctypes.byref(nd))
        return t.value, ti.value, ns.value, nd.value

    def pool(self):
        """(lastoct array, root cell, pool size in octs) of the reference's tree."""
        for n in ("ref_lastoct_array", "ref_root_cell", "ref_freeoct"):
            getattr(self.L, n).restype = c_void_p
        return self.L.ref_lastoct_array(), self.L.ref_root_cell(), self.L.ref_ngridmax()

    def set_freeoct(self, f):
        self.L.ref_set_freeoct.argtypes = [c_void_p]
        self.L.ref_set_freeoct(f)

    def freeoct(self):
        self.L.ref_freeoct.restype = c_void_p
        return self.L.ref_freeoct()

    def topology(self, level):
        n = self.noct(level)
        nei = np.zeros(6 * n, np.int32)
        par = np.zeros(n, np.int32)
        ch = np.zeros(8 * n, np.int32)
        lev = np.zeros(n, np.int32)
        if n:
            self.L.ref_topology(level, _p(nei), _p(par), _p(ch), _p(lev))
        return nei.reshape(n, 6), par, ch.reshape(n, 8), lev

    def run(self, nsteps, nsub=2, dt_param=1e9, time_max=1e9, tsim0=0.0):
        nd = c_int()
        t = self.L.ref_run(nsteps, dt_param, time_max, nsub, tsim0, ctypes.byref(nd))
        return t, np.array([self.L.ref_adt(l) for l in range(1, self.lmax + 1)])

    def hydro_solver_prefix(self, level, nsample):
        """clean_new_hydro + HydroSolver of the reference on the first `nsample`
        octs of the level list (a bounded sample of one level step); returns dt."""
        self.L.ref_hydro_solver_prefix.argtypes = [c_int, c_int]
        self.L.ref_hydro_solver_prefix.restype = c_double
        return self.L.ref_hydro_solver_prefix(level, nsample)

    # refinement of one level (mark-criterion build): L_clean_marks, L_mark_cells,
    # L_check_rule, L_refine_cells (src/amr.c:1480, 883, 746, 286)
    def clean_marks(self, level):
        self.L.ref_clean_marks(level)

    def mark_cells(self, level, nsmooth, threshold):
        self.L.ref_mark_cells.argtypes = [c_int, c_int, c_double]
        self.L.ref_mark_cells(level, nsmooth, threshold)

    def check_rule(self, level):
        self.L.ref_check_rule(level)

    def refine_cells(self, level):
        self.L.ref_refine_cells(level)

    def marks(self, level):
        out = np.zeros(8 * self.noct(level))
        if out.size:
            self.L.ref_get_marks.argtypes = [c_int, c_void_p]
            self.L.ref_get_marks(level, _p(out))
        return out

    def hydro_seconds(self):
        return self.L.ref_hydro_seconds()

    def cell_updates(self):
        return self.L.ref_cell_updates()

    def reset_counters(self):
        self.L.ref_reset_counters()
