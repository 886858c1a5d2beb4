"""The C-ABI library loads and exports every entry declared in include/*.h (no GPU needed)."""
import ctypes
import os
import re

from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include"))) if f.endswith(".h")]


GRAV_HEADER = os.path.join(ROOT, "include", "emma_hydro_grav.h")
RH_HEADER = os.path.join(ROOT, "include", "emma_hydro_rh.h")
HE_HEADER = os.path.join(ROOT, "include", "emma_hydro_he.h")


def declared_functions(headers=None):
    """Functions declared in the headers (default: all but the layout libraries' own)."""
    names = set()
    for h in (headers if headers is not None else [h for h in HEADERS if h not in (GRAV_HEADER, RH_HEADER, HE_HEADER)]):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src, flags=re.M):
            name = m.group(1)
            if name not in ("static_assert", "_Static_assert", "sizeof"):
                names.add(name)
    return names


def test_headers_declare_the_reference_entries():
    names = declared_functions()
    for ref_name in ("HydroSolver", "advancehydroGPU", "clean_new_hydro", "create_hydstencil_GPU",
                     "destroy_hydstencil_GPU", "create_pinned_stencil", "destroy_pinned_stencil"):
        assert ref_name in names


def test_library_exports_every_declared_symbol():
    from emma_b200._lib import LIB_PATH, SIGNATURES
    L = ctypes.CDLL(LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    bound = {n for n, _, _ in SIGNATURES}
    assert declared_functions() <= bound, declared_functions() - bound


def test_gravity_library_exports_everything():
    """libemmahydro_grav.so (the -DWGRAV cell layout) exports the default entries
    and its own (grav_correction, the force setter of test trees)."""
    from emma_b200._lib import LIB_PATH_GRAV, SIGNATURES, GRAV_SIGNATURES
    L = ctypes.CDLL(LIB_PATH_GRAV)
    names = declared_functions([h for h in HEADERS if h not in (RH_HEADER, HE_HEADER)])
    assert {"grav_correction", "emma_tree_set_force"} <= names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert names <= {n for n, _, _ in SIGNATURES + GRAV_SIGNATURES}


def test_tracer_library_exports_everything():
    """libemmahydro_rh.so (the -DWRADHYD cell layout) exports the default entries and
    the tracer accessors of test trees."""
    from emma_b200._lib import LIB_PATH_RH, SIGNATURES, RH_SIGNATURES
    L = ctypes.CDLL(LIB_PATH_RH)
    names = declared_functions([h for h in HEADERS if h not in (GRAV_HEADER, HE_HEADER)])
    assert {"emma_tree_set_tracer", "emma_tree_get_tracer"} <= names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert names <= {n for n, _, _ in SIGNATURES + RH_SIGNATURES}


def test_helium_library_exports_everything():
    """libemmahydro_he.so (the -DWRADHYD -DHELIUM cell layout) exports the default
    entries, the single-tracer accessors and the three-tracer ones of test trees."""
    from emma_b200._lib import LIB_PATH_HE, SIGNATURES, RH_SIGNATURES, HE_SIGNATURES
    L = ctypes.CDLL(LIB_PATH_HE)
    names = declared_functions([h for h in HEADERS if h != GRAV_HEADER])
    assert {"emma_tree_set_tracer_n", "emma_tree_get_tracer_n", "emma_tree_put_tracer_n"} <= names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert names <= {n for n, _, _ in SIGNATURES + RH_SIGNATURES + HE_SIGNATURES}


def test_struct_layout_matches_reference():
    # struct OCT must be 1200 bytes (src/prototypes.h:1028 with -DWHYDRO2, REAL=double)
    from oracle import Restatement
    assert Restatement().L.orc_sizeof_oct() == 1200


def test_hgrid_size_matches_reference_builds():
    """create_pinned_stencil allocates EMMA_SIZEOF_HGRID bytes per stencil entry:
    the reference's sizeof(struct HGRID) in the default and the -DWGRAV build."""
    import re
    import oracle
    src = open(os.path.join(ROOT, "include", "emma_oct.h")).read()
    grav, he, rh, plain = (int(x) for x in re.findall(r"#define EMMA_SIZEOF_HGRID (\d+)", src))
    for name, want in (("libemmaref.so", plain), ("libemmaref_grav.so", grav), ("libemmaref_rh.so", rh),
                       ("libemmaref_he.so", he)):
        path = os.path.join(ROOT, "oracle", "_ref", name)
        if not os.path.exists(path):
            continue
        assert ctypes.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW).ref_sizeof_hgrid() == want, name
