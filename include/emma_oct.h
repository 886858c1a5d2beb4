/*
 * emma_oct.h -- the oct-tree memory layout that EMMA's hydro entry points pass
 * around, declared for a build with -DWHYDRO2 (and neither -DWRAD, -DPIC nor
 * -DWRADHYD), REAL = double, NVAR = 6; with EMMA_WGRAV defined, for the
 * reference's -DWGRAV build (libemmahydro_grav.so); with EMMA_WRADHYD defined,
 * for its -DWRADHYD build without -DHELIUM (NVAR = 7: the ionised density dX
 * follows E in Wtype; libemmahydro_rh.so); with EMMA_HELIUM defined too, for its
 * -DWRADHYD -DHELIUM build (NVAR = 9: dX, then the singly and doubly ionised
 * helium densities dXHE, dXXHE; libemmahydro_he.so).
 *
 * This is an interface, not an implementation: libemmahydro reads and writes the
 * caller's tree in place, so the field order, types and padding must be exactly
 * those of the reference (src/prototypes.h:611 Wtype, :653 Utype, :825 CELL,
 * :1028 OCT).  Sizes are checked at compile time: CELL 136 B, OCT 1200 B
 * (EMMA_WGRAV: CELL 192 B, OCT 1648 B; EMMA_WRADHYD: CELL 152 B, OCT 1328 B;
 * EMMA_WRADHYD + EMMA_HELIUM: CELL 184 B, OCT 1584 B).
 * Only the members the hydro path uses are named; nothing else is assumed.
 */
#ifndef EMMA_OCT_H
#define EMMA_OCT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double REAL;

struct Wtype {           /* primitive state of a cell, src/prototypes.h:611 */
  REAL d, u, v, w, p;    /* density, velocity, pressure */
  REAL a;                /* sound speed */
  REAL E;                /* total energy density */
#ifdef EMMA_WRADHYD
  REAL dX;               /* ionised density, advected with the gas */
#ifdef EMMA_HELIUM
  REAL dXHE, dXXHE;      /* singly and doubly ionised helium densities */
#endif
#endif
};

#if defined(EMMA_HELIUM) && !defined(EMMA_WRADHYD)
#error "EMMA_HELIUM extends the -DWRADHYD layout: define EMMA_WRADHYD too"
#endif

#if defined(EMMA_WGRAV) && defined(EMMA_WRADHYD)
#error "libemmahydro is built for one of the -DWGRAV and -DWRADHYD layouts at a time"
#endif

struct OCT;

#ifdef EMMA_WGRAV
struct Gtype {           /* src/prototypes.h:818 */
  REAL d, p;             /* density contrast, potential */
};
#endif

struct CELL {            /* src/prototypes.h:825 (WHYDRO2 [+ WGRAV] members only) */
  struct OCT *child;     /* finer oct, NULL for a leaf */
  REAL marked;           /* refinement mark */
  int idx;               /* index of the cell within its oct: ix + 2 iy + 4 iz */
#ifdef EMMA_WGRAV
  struct Gtype gdata;
  REAL pnew;             /* new potential */
  REAL res;              /* residual */
  REAL f[3];             /* gravitational acceleration of the cell */
#endif
  struct Wtype field;    /* state at the start of the level step */
  struct Wtype fieldnew; /* state being built during the level step */
};

struct OCT {             /* src/prototypes.h:1028 */
  struct CELL cell[8];
  struct CELL *nei[6];   /* face neighbours at level-1: -x,+x,-y,+y,-z,+z */
  struct CELL *parent;   /* parent cell at level-1 */
  struct OCT *next;      /* next oct of the same level (list order) */
  struct OCT *prev;
  struct OCT *nexthash;
  REAL x, y, z;          /* lower-left corner */
  int cpu;               /* owning rank */
  int level;             /* level of the cells of this oct */
};

/* Opaque in this library: the drop-in entries read only CPUINFO's `rank` (the
 * first member, offset 0 under every compile-time flag set of the reference) and,
 * in clean_new_hydro, RUNPARAMS's `lcoarse` (offset 28 with REAL = double). */
struct CPUINFO;
struct RUNPARAMS;
struct HGRID;

/* sizeof(struct HGRID) with the flags above (-DWHYDRO2, NVAR 6; the stencil cells
 * also carry f[3] with -DWGRAV; NVAR 7 with -DWRADHYD) */
#if defined(EMMA_WGRAV)
#define EMMA_SIZEOF_HGRID 21760
#elif defined(EMMA_HELIUM)
#define EMMA_SIZEOF_HGRID 23104
#elif defined(EMMA_WRADHYD)
#define EMMA_SIZEOF_HGRID 18752
#else
#define EMMA_SIZEOF_HGRID 16576
#endif

#ifdef __cplusplus
}
#endif

#if defined(EMMA_WGRAV)
#define EMMA_SIZEOF_CELL 192
#define EMMA_SIZEOF_OCT 1648
#elif defined(EMMA_HELIUM)
#define EMMA_SIZEOF_CELL 184
#define EMMA_SIZEOF_OCT 1584
#elif defined(EMMA_WRADHYD)
#define EMMA_SIZEOF_CELL 152
#define EMMA_SIZEOF_OCT 1328
#else
#define EMMA_SIZEOF_CELL 136
#define EMMA_SIZEOF_OCT 1200
#endif
#ifdef __cplusplus
static_assert(sizeof(struct CELL) == EMMA_SIZEOF_CELL, "struct CELL must match the reference layout");
static_assert(sizeof(struct OCT) == EMMA_SIZEOF_OCT, "struct OCT must match the reference layout");
#else
_Static_assert(sizeof(struct CELL) == EMMA_SIZEOF_CELL, "struct CELL must match the reference layout");
_Static_assert(sizeof(struct OCT) == EMMA_SIZEOF_OCT, "struct OCT must match the reference layout");
#endif

#endif
