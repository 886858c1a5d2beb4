"""Host oct tree (EMMA's struct OCT layout) built by libemmahydro.

Thin wrapper over the emma_tree_* entries of include/emma_hydro.h: build the
complete levels 1..lcoarse, refine cells selected by a predicate on their
centres (reference construction order), set and read fields per level in list
order (oct*8 + cell, cell = ix + 2 iy + 4 iz).
"""
import numpy as np

from ._lib import lib, ptr

# cell offsets inside an oct, in units of the cell size, cell = ix + 2 iy + 4 iz
CELL_OFF = np.array([[c % 2, (c // 2) % 2, c // 4] for c in range(8)], dtype=np.float64)


class OctTree:
    """An EMMA oct tree in host memory (levels lcoarse..lmax are hydro levels)."""

    def __init__(self, lcoarse, lmax, ngridmax=0, grav=False, rh=False, he=False):
        """grav: the reference's -DWGRAV cell layout (built by libemmahydro_grav.so),
        for the gravity-coupled drop-in entries; rh: its -DWRADHYD layout (the cells
        carry the ionised density dX; libemmahydro_rh.so); he: its -DWRADHYD -DHELIUM
        layout (dX and the helium densities dXHE, dXXHE; libemmahydro_he.so)."""
        assert (bool(grav) + bool(rh) + bool(he)) <= 1, "one cell layout at a time"
        self.lcoarse, self.lmax = lcoarse, lmax
        self.grav, self.rh, self.he = grav, rh or he, he
        self.ntracers = 3 if he else (1 if rh else 0)
        self._L = lib("he" if he else ("rh" if rh else grav))
        self._t = self._L.emma_tree_create(lcoarse, lmax, ngridmax)
        if not self._t:
            raise RuntimeError("emma_tree_create failed")

    def close(self):
        if self._t:
            self._L.emma_tree_destroy(self._t)
            self._t = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def firstoct(self):
        return self._L.emma_tree_firstoct(self._t)

    def noct(self, level):
        return self._L.emma_tree_noct(self._t, level)

    def oct_xyz(self, level):
        n = self.noct(level)
        out = np.zeros((n, 3))
        if n:
            self._L.emma_tree_oct_xyz(self._t, level, ptr(out))
        return out

    def cell_centres(self, level):
        dx = 0.5 ** level
        xyz = self.oct_xyz(level)
        return (xyz[:, None, :] + (CELL_OFF[None] + 0.5) * dx).reshape(-1, 3)

    def refine(self, level, mark):
        mark = np.ascontiguousarray(mark, dtype=np.int8)
        assert mark.size == 8 * self.noct(level)
        rc = self._L.emma_tree_refine(self._t, level, ptr(mark))
        if rc < 0:
            raise RuntimeError(f"refinement of level {level} refused for {-rc} cells (2:1 rule)")
        return rc

    def refine_where(self, level, pred):
        return self.refine(level, pred(self.cell_centres(level)))

    def set_fields(self, level, d, u, v, w, p):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (d, u, v, w, p)]
        self._L.emma_tree_set_field(self._t, level, *[ptr(a) for a in arrs])

    def set_force(self, level, fx, fy, fz):
        """Gravitational acceleration f[3] of every cell of a level (grav trees only)."""
        assert self.grav, "the default cell layout has no force"
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (fx, fy, fz)]
        self._L.emma_tree_set_force(self._t, level, *[ptr(a) for a in arrs])

    def set_tracer(self, level, dX):
        """Ionised density dX of field and fieldnew of every cell of a level (rh trees)."""
        assert self.rh, "only the -DWRADHYD layout has dX"
        a = np.ascontiguousarray(dX, dtype=np.float64)
        assert a.size == 8 * self.noct(level)
        self._L.emma_tree_set_tracer(self._t, level, ptr(a))

    def put_tracer(self, level, dX, which=0):
        """dX of `field` (which=0) or `fieldnew` (which=1) only (rh trees)."""
        assert self.rh, "only the -DWRADHYD layout has dX"
        a = np.ascontiguousarray(dX, dtype=np.float64)
        assert a.size == 8 * self.noct(level)
        self._L.emma_tree_put_tracer(self._t, level, which, ptr(a))

    def set_tracer_n(self, level, t, x):
        """Tracer t (0: dX; he trees 1: dXHE, 2: dXXHE) of field and fieldnew."""
        assert t < self.ntracers, "the cell layout has no such tracer"
        if not self.he:
            return self.set_tracer(level, x)
        a = np.ascontiguousarray(x, dtype=np.float64)
        assert a.size == 8 * self.noct(level)
        self._L.emma_tree_set_tracer_n(self._t, level, t, ptr(a))

    def get_tracer_n(self, level, t, which=0):
        assert t < self.ntracers, "the cell layout has no such tracer"
        if not self.he:
            return self.get_tracer(level, which)
        out = np.zeros(8 * self.noct(level))
        if out.size:
            self._L.emma_tree_get_tracer_n(self._t, level, t, which, ptr(out))
        return out

    def get_tracer(self, level, which=0):
        assert self.rh, "only the -DWRADHYD layout has dX"
        out = np.zeros(8 * self.noct(level))
        if out.size:
            self._L.emma_tree_get_tracer(self._t, level, which, ptr(out))
        return out

    def get_fields(self, level, which=0):
        """(7, 8*noct): d,u,v,w,p,a,E of `field` (which=0) or `fieldnew` (which=1)."""
        n = self.noct(level)
        out = np.zeros((7, 8 * n))
        if n:
            self._L.emma_tree_get_field(self._t, level, which, ptr(out))
        return out

    def put_fields(self, level, w7, which=0):
        """Write (7, 8*noct) d,u,v,w,p,a,E as they are into `field` (which=0) or
        `fieldnew` (which=1): the inverse of get_fields."""
        n = self.noct(level)
        w7 = np.ascontiguousarray(w7, dtype=np.float64)
        assert w7.shape == (7, 8 * n)
        if n:
            self._L.emma_tree_put_field(self._t, level, which, ptr(w7))

    def set_cpu(self, level, ranks):
        """Owner rank (struct OCT cpu) of every oct of a level, in list order."""
        r = np.ascontiguousarray(ranks, dtype=np.int32)
        assert r.size == self.noct(level)
        if r.size:
            self._L.emma_tree_set_cpu(self._t, level, ptr(r))

    def topology(self, level):
        n = self.noct(level)
        nei = np.zeros(6 * n, np.int32)
        par = np.zeros(n, np.int32)
        ch = np.zeros(8 * n, np.int32)
        lev = np.zeros(n, np.int32)
        if n:
            self._L.emma_tree_topology(self._t, level, ptr(nei), ptr(par), ptr(ch), ptr(lev))
        return nei.reshape(n, 6), par, ch.reshape(n, 8), lev

    def split_mask(self, level):
        return self.topology(level)[2].reshape(-1) >= 0
