"""ctypes bindings of libemmahydro.so (include/emma_hydro.h).

The library is built in-tree (emma_b200/libemmahydro.so, see emma_b200/build.py).
There is no fallback: if the shared library is missing or fails to load, every
entry point raises, so a CUDA path that did not run can never look like one
that did.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libemmahydro.so")
LIB_PATH_GRAV = os.path.join(_HERE, "libemmahydro_grav.so")
LIB_PATH_RH = os.path.join(_HERE, "libemmahydro_rh.so")
LIB_PATH_HE = os.path.join(_HERE, "libemmahydro_he.so")

_libs = {}

c_int, c_double, c_ll, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_longlong, ctypes.c_void_p
P = ctypes.POINTER


class EmmaHydroOptions(ctypes.Structure):
    _fields_ = [("precision", c_int), ("trans_flags", c_int), ("cfl", c_double),
                ("tile_octs", c_int), ("device", c_int), ("use_graph", c_int), ("gravity", c_int),
                ("dual_energy", c_int), ("column", c_int), ("fused_step", c_int),
                ("column_xshfl", c_int), ("column_balanced", c_int)]


PREC_FP64, PREC_MIXED = 0, 1
TRANS_XM, TRANS_XP, TRANS_YM, TRANS_YP, TRANS_ZM, TRANS_ZP = 1, 2, 4, 8, 16, 32
ST_NEG_DENSITY, ST_NEG_PSTAR, ST_NAN, ST_TREE, ST_CUDA, ST_ARG, ST_TIMEOUT = 1, 2, 4, 8, 16, 32, 64

# (name, restype, argtypes) for every entry declared in include/emma_hydro.h
SIGNATURES = [
    ("emma_hydro_status", c_int, []),
    ("emma_hydro_clear_status", None, []),
    ("emma_hydro_last_error", ctypes.c_char_p, []),
    ("emma_hydro_default_options", None, [P(EmmaHydroOptions)]),
    ("HydroSolver", None, [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_double]),
    ("advancehydroGPU", c_int, [c_void_p, c_int, c_void_p, c_void_p, c_int, c_double, c_double]),
    ("clean_new_hydro", None, [c_int, c_void_p, c_void_p, c_void_p]),
    ("create_hydstencil_GPU", None, [c_void_p, c_int]),
    ("destroy_hydstencil_GPU", None, [c_void_p, c_int]),
    ("create_pinned_stencil", None, [P(c_void_p), c_int]),
    ("destroy_pinned_stencil", None, [P(c_void_p), c_int]),
    ("emma_hydro_init", c_int, [P(EmmaHydroOptions)]),
    ("emma_hydro_set_options", c_int, [P(EmmaHydroOptions)]),
    ("emma_hydro_shutdown", None, []),
    ("emma_hydro_set_stream", c_int, [c_void_p]),
    ("emma_hydro_kernel_launches", c_ll, []),
    ("emma_hydro_transfer_bytes", c_int, [P(c_ll), P(c_ll)]),
    ("emma_hydro_dropin_profile", c_int, [P(ctypes.c_double)]),
    ("emma_hydro_tree_upload", c_int, [c_void_p, c_int, c_int, c_int]),
    ("emma_hydro_tree_download", c_int, [c_void_p]),
    ("emma_hydro_fields_upload", c_int, [c_void_p]),
    ("emma_hydro_clean_new", c_int, [c_int]),
    ("emma_hydro_comptstep", c_int, [c_int, P(c_double)]),
    ("emma_hydro_advance_level", c_int, [c_int, c_double]),
    ("emma_hydro_advance_coarse_step", c_int, [c_double, c_double, c_int, P(c_double), c_void_p]),
    ("emma_hydro_advance_coarse_step_async", c_int, [c_double, c_double, c_int]),
    ("emma_hydro_get_time", c_int, [P(c_double), c_void_p]),
    ("emma_hydro_set_time", c_int, [c_double, c_void_p]),
    ("emma_hydro_level_noct", c_int, [c_int]),
    ("emma_hydro_get_level_state", c_int, [c_int, c_void_p]),
    ("emma_hydro_set_level_state", c_int, [c_int, c_void_p]),
    ("emma_hydro_set_level_force", c_int, [c_int, c_void_p]),
    ("emma_hydro_is_resident", c_int, [c_void_p]),
    ("emma_hydro_tree_release", c_int, [c_void_p]),
    ("emma_hydro_mark_cells", c_int, [c_int, c_void_p, c_void_p, c_int, c_double, c_void_p]),
    ("emma_hydro_check_rule", c_int, [c_int, c_void_p, c_void_p, c_void_p]),
    ("emma_hydro_marks_to_host", c_int, [c_void_p, c_int]),
    ("emma_hydro_refine_cells", c_void_p, [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                           c_double]),
    ("emma_hydro_dump_alloct", c_int, [ctypes.c_char_p, c_void_p, c_int, c_int, c_int, c_int, c_double, c_int,
                                       c_void_p, c_void_p]),
    ("emma_hydro_save_amr", c_int, [ctypes.c_char_p, c_void_p, c_double, c_double, c_int, c_int, c_int, c_int,
                                    c_void_p, c_void_p, c_void_p]),
    ("emma_hydro_restore_amr", c_int, [ctypes.c_char_p, c_void_p, c_void_p, c_int, c_ll, c_void_p, P(c_double),
                                       P(c_double), P(c_int), P(c_int), P(c_int), P(c_int), c_void_p, c_void_p,
                                       P(c_void_p)]),
    ("emma_hydro_set_level_force_device", c_int, [c_int, c_void_p]),
    ("emma_hydro_level_leaf_cells", c_ll, [c_int]),
    ("emma_hydro_cell_updates", c_ll, []),
    ("emma_hydro_reset_counters", None, []),
    ("emma_hydro_kernel_timing", c_int, [P(c_double), P(c_ll), P(c_ll)]),
    ("emma_hydro_kernel_timing_level", c_int, [c_int, P(c_double), P(c_ll), P(c_ll)]),
    ("emma_hydro_graph_info", c_int, [P(c_int), P(c_int), P(c_int), P(c_int)]),
    ("emma_hydro_fused_job_log", c_int, [c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("emma_hydro_timed_coarse_steps", c_int, [c_double, c_double, c_int, c_int, P(c_double)]),
    ("emma_hydro_step_tuning", c_int, [P(c_int), c_void_p]),
    ("emma_hydro_tuning", c_int, [c_int, P(c_int), P(c_int), c_void_p]),
    ("emma_hydro_column_tuning", c_int, [c_int, P(c_int), c_void_p]),
    ("emma_hydro_column_xshfl", c_int, [c_int, P(c_int), c_void_p]),
    ("emma_hydro_column_balanced", c_int, [c_int, P(c_int), c_void_p]),
    ("emma_hydro_probe_wait_timeout", c_int, [c_ll]),
    ("emma_hydro_plan_stats", c_int, [c_void_p, c_int, c_int, c_int, c_void_p]),
    ("emma_hydro_level_dt_noalloc", c_int, [c_void_p, c_ll, c_int, c_double, c_void_p, P(c_double)]),
    ("emma_hydro_noalloc_forget", None, []),
    ("emma_tree_create", c_void_p, [c_int, c_int, c_ll]),
    ("emma_tree_destroy", None, [c_void_p]),
    ("emma_tree_refine", c_int, [c_void_p, c_int, c_void_p]),
    ("emma_tree_firstoct", c_void_p, [c_void_p]),
    ("emma_tree_noct", c_int, [c_void_p, c_int]),
    ("emma_tree_oct_xyz", None, [c_void_p, c_int, c_void_p]),
    ("emma_tree_set_field", None, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("emma_tree_get_field", None, [c_void_p, c_int, c_int, c_void_p]),
    ("emma_tree_put_field", None, [c_void_p, c_int, c_int, c_void_p]),
    ("emma_tree_set_cpu", None, [c_void_p, c_int, c_void_p]),
    ("emma_tree_topology", None, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
]


GRAV_SIGNATURES = [
    ("grav_correction", None, [c_int, c_void_p, c_void_p, c_void_p, c_double]),
    ("emma_tree_set_force", None, [c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
]


RH_SIGNATURES = [
    ("emma_tree_set_tracer", None, [c_void_p, c_int, c_void_p]),
    ("emma_tree_get_tracer", None, [c_void_p, c_int, c_int, c_void_p]),
    ("emma_tree_put_tracer", None, [c_void_p, c_int, c_int, c_void_p]),
]


HE_SIGNATURES = [
    ("emma_tree_set_tracer_n", None, [c_void_p, c_int, c_int, c_void_p]),
    ("emma_tree_get_tracer_n", None, [c_void_p, c_int, c_int, c_int, c_void_p]),
    ("emma_tree_put_tracer_n", None, [c_void_p, c_int, c_int, c_int, c_void_p]),
]


def lib(grav=False):
    """Load libemmahydro.so once; grav=True: libemmahydro_grav.so (the -DWGRAV cell
    layout), grav="rh": libemmahydro_rh.so (the -DWRADHYD layout), grav="he":
    libemmahydro_he.so (the -DWRADHYD -DHELIUM layout).  Raises if the library is
    not built."""
    key = grav if grav in ("rh", "he") else ("grav" if grav else "plain")
    if key in _libs:
        return _libs[key]
    path = {"plain": LIB_PATH, "grav": LIB_PATH_GRAV, "rh": LIB_PATH_RH, "he": LIB_PATH_HE}[key]
    if not os.path.exists(path):
        raise RuntimeError(f"{os.path.basename(path)} is not built ({path}); run emma_b200.build.build()")
    # RTLD_LOCAL: the drop-in entries carry the reference's names (HydroSolver, ...);
    # they must not interpose on another library that defines the same symbols
    L = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    extra = {"plain": [], "grav": GRAV_SIGNATURES, "rh": RH_SIGNATURES, "he": RH_SIGNATURES + HE_SIGNATURES}[key]
    for name, res, args in SIGNATURES + extra:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _libs[key] = L
    return L


def ptr(a):
    """Data pointer of a C-contiguous numpy array."""
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)


def check(rc, what="", grav=False):
    """Raise on a non-zero status bitmask returned by the library."""
    if rc != 0:
        msg = lib(grav).emma_hydro_last_error().decode(errors="replace")
        raise RuntimeError(f"libemmahydro {what} failed: status=0x{rc & 0xffffffff:x} {msg}")
