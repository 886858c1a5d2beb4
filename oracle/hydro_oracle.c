/*
 * hydro_oracle.c -- CPU restatement of EMMA's hydro level advance (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against; it is never linked into, or called by, the product library.
 *
 * It restates, on the reference's own oct-tree memory layout, what
 * HydroSolver() (src/hydro_utils.c:3378) does for one AMR level:
 *   gather of the 27-oct neighbourhood      src/hydro_utils.c:2852-3028 (default)
 *                                           src/hydro_utils.c:2465-2845 (HYDROTEST)
 *   MUSCL-Hancock predictor                 src/hydro_utils.c:976-1259
 *   hybrid PVRS/TRRS/TSRS + Newton p*       src/hydro_utils.c:580-777
 *   HLLC wave speeds and fluxes             src/hydro_utils.c:1264-1399, 1407-2238
 *   flux-divergence update                  src/hydro_utils.c:3036-3088
 *   scatter + fine->coarse correction       src/hydro_utils.c:3096-3303
 *   field := fieldnew, split-cell averaging src/hydro_utils.c:3408-3483
 * plus clean_new_hydro (:3501), L_comptstep_hydro (src/advanceamr.c:92) and the
 * hydro-only subset of Advance_level (src/advanceamr.c:243-1299), and the
 * ALLOCT field dump dumpalloct_serial (src/io.c:1233) -- the dump alone is
 * parity unpinned: io.c does not build without MPI and the reference holds no
 * dump fixtures, so it follows the source as read.
 *
 * Every floating-point expression keeps the reference's operation order so the
 * results are bit-identical when both are built with gcc -O2 -ffp-contract=off
 * (checked in tests/test_oracle_pin.py).  Differences in organisation, all
 * value-preserving: MUSCL face states of a stencil cell are computed once per
 * target oct and reused (the reference recomputes identical values up to 9
 * times); the reference's abort() calls become error bits.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "hydro_oracle.h"

#define GAM (5. / 3.)     /* GAMMA, src/param.h:4 */
#define P_MIN (1e-10)     /* PMIN,  src/param.h:20 */
#define DEF_DENS 10.      /* DEFDENS, src/hydro_utils.c:19 */
#define N_ITER_MAX 10     /* NITERMAX, src/hydro_utils.c:17 */
#define ERR_TOL 1e-10     /* ERRTOL, src/hydro_utils.c:18 */

/* ---- memory layout of the reference tree (src/prototypes.h:611,825,1028) */
#if defined(ORC_HELIUM) && !defined(ORC_WRADHYD)
#error "ORC_HELIUM extends the -DWRADHYD layout (build with ORC_WRADHYD too)"
#endif
#ifdef ORC_HELIUM
/* -DWRADHYD -DHELIUM: the ionised hydrogen density dX and the singly and doubly
 * ionised helium densities dXHE, dXXHE, advected with the gas (NVAR 9,
 * src/prototypes.h:62-66); YHE = 0.24 (src/param.h:47-48) */
#define YHE_ (0.24)
#define NTR 3
typedef struct { double d, u, v, w, p, a, E, dX, dXHE, dXXHE; } oW;      /* struct Wtype */
typedef struct { double d, du, dv, dw, E, eint, dX, dXHE, dXXHE; } oU;  /* struct Utype */
#elif defined(ORC_WRADHYD)
/* -DWRADHYD: the ionised density dX, advected with the gas (NVAR 7; YHE = 0
 * without -DHELIUM / -DHESIMPLE, src/param.h:47-54) */
#define YHE_ (0.)
#define NTR 1
typedef struct { double d, u, v, w, p, a, E, dX; } oW;      /* struct Wtype */
typedef struct { double d, du, dv, dw, E, eint, dX; } oU;  /* struct Utype */
#else
typedef struct { double d, u, v, w, p, a, E; } oW;      /* struct Wtype */
typedef struct { double d, du, dv, dw, E, eint; } oU;  /* struct Utype */
#endif
struct oOct;
typedef struct oCell {
  struct oOct *child;
  double marked;
  int idx;
#ifdef ORC_WGRAV
  double gd, gp;   /* struct Gtype gdata (src/prototypes.h:818) */
  double pnew, res;
  double f[3];     /* gravitational acceleration of the cell */
#endif
  oW field;
  oW fieldnew;
} oCell;
typedef struct oOct {
  oCell cell[8];
  oCell *nei[6];
  oCell *parent;
  struct oOct *next, *prev, *nexthash;
  double x, y, z;
  int cpu;
  int level;
} oOct;
#if defined(ORC_WGRAV) && defined(ORC_WRADHYD)
#error "the gravity and tracer layouts are built separately"
#elif defined(ORC_WGRAV)
_Static_assert(sizeof(oCell) == 192, "CELL layout (-DWGRAV)");
_Static_assert(sizeof(oOct) == 1648, "OCT layout (-DWGRAV)");
#elif defined(ORC_HELIUM)
_Static_assert(sizeof(oCell) == 184, "CELL layout (-DWRADHYD -DHELIUM)");
_Static_assert(sizeof(oOct) == 1584, "OCT layout (-DWRADHYD -DHELIUM)");
#elif defined(ORC_WRADHYD)
_Static_assert(sizeof(oCell) == 152, "CELL layout (-DWRADHYD)");
_Static_assert(sizeof(oOct) == 1328, "OCT layout (-DWRADHYD)");
#else
_Static_assert(sizeof(oCell) == 136, "CELL layout");
_Static_assert(sizeof(oOct) == 1200, "OCT layout");
#endif

#ifdef ORC_WRADHYD
/* tracer t of a state: dX, then (HELIUM) dXHE, dXXHE, consecutive in both types */
#define TRW(W, t) ((&(W)->dX)[t])
/* the mass fraction each tracer is a part of (src/hydro_utils.c:1244-1252):
 * hydrogen 1 - YHE, helium YHE */
static const double TRFRAC[3] = {1. - YHE_, YHE_, YHE_};
#endif

static int g_err = 0;
static long long g_updates = 0;

long long orc_cell_updates(void) { return g_updates; }
void orc_reset_counters(void) { g_updates = 0; }
int orc_sizeof_oct(void) { return (int)sizeof(oOct); }

static oOct *oct_of(oCell *c) { return (oOct *)((char *)c - (size_t)c->idx * sizeof(oCell)); }

/* Face neighbour of cell `ic` (icell = ix + 2 iy + 4 iz) in direction k
 * (0:-x 1:+x 2:-y 3:+y 4:-z 5:+z), the mapping of getcellnei (src/oct.c:116):
 * *same = 1 if inside the oct, else the neighbour is in the oct across face k. */
static void cell_nei(int ic, int k, int *same, int *nc) {
  int axis = k >> 1, bit = 1 << axis, plus = k & 1;
  int inside = plus ? !(ic & bit) : (ic & bit);
  *same = inside ? 1 : 0;
  *nc = ic ^ bit;
}

/* ---------------------------------------------- primitives (src/hydro_utils.c:29-89) */
static void get_E(oW *W) {
  W->E = W->p / (GAM - 1.) + 0.5 * W->d * (W->u * W->u + W->v * W->v + W->w * W->w);
}
static void to_cons(const oW *W, oU *U) {
  U->d = W->d;
  U->du = W->d * W->u;
  U->dv = W->d * W->v;
  U->dw = W->d * W->w;
  U->eint = W->p / (GAM - 1.);
  U->E = W->E;
#ifdef ORC_WRADHYD
  for (int t = 0; t < NTR; t++) TRW(U, t) = TRW(W, t);
#endif
}
/* dual: -DDUAL_E, the pressure from the tracked internal energy (src/hydro_utils.c:45-49) */
static void to_prim(const oU *U, oW *W, int dual) {
  double dl = (U->d == 0. ? DEF_DENS : U->d);
  W->d = U->d;
  W->u = U->du / dl;
  W->v = U->dv / dl;
  W->w = U->dw / dl;
  if (dual) W->p = U->eint * (GAM - 1.);
  else W->p = (GAM - 1.) * (U->E - ((U->du) * (U->du) + (U->dv) * (U->dv) + (U->dw) * (U->dw)) / (dl)*0.5);
  W->E = U->E;
#ifdef ORC_WRADHYD
  for (int t = 0; t < NTR; t++) TRW(W, t) = TRW(U, t);
#endif
  W->a = sqrt(GAM * W->p / dl);
}

/* ---------------------------------------------- MUSCL-Hancock (src/hydro_utils.c:201-269, 976-1259) */
static double limit1(double m, double p) {
  /* minmod_W with beta = 1 */
  if (p > 0) return fmax(fmax(0., fmin(m, p)), fmin(m, p));
  return fmin(fmin(0., fmax(m, p)), fmax(m, p));
}

/* primitive 5-vectors: 0:d 1:u 2:v 3:w 4:p */
static void as5(const oW *W, double q[5]) { q[0] = W->d; q[1] = W->u; q[2] = W->v; q[3] = W->w; q[4] = W->p; }

/* Half-step predictor -dt/(2dx) (A Dx + B Dy + C Dz) in primitive variables,
 * matrix_jacobian (src/hydro_utils.c:976).  The non-zero entries are added in
 * the reference's column order; skipped zero entries only ever add +-0. */
static void predictor(const oW *W0, double dt, double dx, double D[3][5], double Wt[5]) {
  double acc[5] = {0., 0., 0., 0., 0.};
  double vel[3] = {W0->u, W0->v, W0->w};
  double daa = W0->d * W0->a * W0->a;
  double id = 1. / W0->d;
  int dir, i;
  for (dir = 0; dir < 3; dir++) {
    double s = vel[dir];
    /* column 0 */
    acc[0] += s * D[dir][0];
    /* column 1 */
    if (dir == 0) acc[0] += W0->d * D[dir][1];
    acc[1] += s * D[dir][1];
    if (dir == 0) acc[4] += daa * D[dir][1];
    /* column 2 */
    if (dir == 1) acc[0] += W0->d * D[dir][2];
    acc[2] += s * D[dir][2];
    if (dir == 1) acc[4] += daa * D[dir][2];
    /* column 3 */
    if (dir == 2) acc[0] += W0->d * D[dir][3];
    acc[3] += s * D[dir][3];
    if (dir == 2) acc[4] += daa * D[dir][3];
    /* column 4 */
    acc[1 + dir] += id * D[dir][4];
    acc[4] += s * D[dir][4];
  }
  for (i = 0; i < 5; i++) Wt[i] = acc[i] * (-dt / dx * 0.5);
}

/* ---------------------------------------------- per-oct stencil */
typedef struct {
  oW w[27][8];
  char split[27][8];
#ifdef ORC_WGRAV
  double f[27][8][3]; /* force of each stencil cell */
#endif
  /* memoised MUSCL face states, 6 per stencil cell */
  oW face[27][8][6];
  char done[27][8];
} Stencil;

static const int SLOT_OFF[6] = {-1, 1, -3, 3, -9, 9};
static const int FACE_SLOT[7] = {12, 14, 10, 16, 4, 22, 13};

/* MUSCL_BOUND2 on stencil cell (slot, ic): fills st->face[slot][ic][0..5]. */
static void muscl_cell(Stencil *st, int slot, int ic, double dt, double dx) {
  const oW *W0 = &st->w[slot][ic];
  double q0[5], D[3][5], Wt[5];
  static const double fx[6] = {-0.5, 0.5, 0.0, 0.0, 0.0, 0.0};
  static const double fy[6] = {0.0, 0.0, -0.5, 0.5, 0.0, 0.0};
  static const double fz[6] = {0.0, 0.0, 0.0, 0.0, -0.5, 0.5};
  int dir, k, f;
  as5(W0, q0);
  for (dir = 0; dir < 3; dir++) {
    int same, nc;
    double qm[5], qp[5];
    cell_nei(ic, 2 * dir, &same, &nc);
    as5(&st->w[same ? slot : slot + SLOT_OFF[2 * dir]][nc], qm);
    cell_nei(ic, 2 * dir + 1, &same, &nc);
    as5(&st->w[same ? slot : slot + SLOT_OFF[2 * dir + 1]][nc], qp);
    for (k = 0; k < 5; k++) D[dir][k] = limit1(q0[k] - qm[k], qp[k] - q0[k]);
  }
  predictor(W0, dt, dx, D, Wt);
  for (f = 0; f < 6; f++) {
    oW *Wi = &st->face[slot][ic][f];
    double r[5];
    for (k = 0; k < 5; k++) r[k] = q0[k] + fx[f] * D[0][k] + fy[f] * D[1][k] + fz[f] * D[2][k] + Wt[k];
    Wi->d = r[0]; Wi->u = r[1]; Wi->v = r[2]; Wi->w = r[3];
    Wi->p = fmax(r[4], P_MIN);
    if (Wi->d < 0) g_err |= ORC_ERR_NEG_DENSITY;
#ifdef ORC_WGRAV
    /* half-step gravity kick of the face velocities (src/hydro_utils.c:1219-1226) */
    Wi->u += -st->f[slot][ic][0] * 0.5 * dt;
    Wi->v += -st->f[slot][ic][1] * 0.5 * dt;
    Wi->w += -st->f[slot][ic][2] * 0.5 * dt;
#endif
    get_E(Wi);
    Wi->a = sqrt(GAM * Wi->p / Wi->d);
#ifdef ORC_WRADHYD
    /* the face value is the face density times the centre's ionised fraction; the
     * reconstructed dX is overwritten (src/hydro_utils.c:1244-1246) */
    for (int t = 0; t < NTR; t++) {
      double X0 = TRW(W0, t) / (W0->d * (TRFRAC[t]));
      TRW(Wi, t) = Wi->d * (TRFRAC[t]) * X0;
    }
#endif
  }
  st->done[slot][ic] = 1;
}

static const oW *face_state(Stencil *st, int slot, int ic, int f, double dt, double dx) {
  if (!st->done[slot][ic]) muscl_cell(st, slot, ic, dt, dx);
  return &st->face[slot][ic][f];
}

/* ---------------------------------------------- Riemann solvers (src/hydro_utils.c:580-777) */
typedef struct { double d, u, p, a; } oW1;

static double f_root_prime(double p, const oW1 *L, const oW1 *R) {
  double AL = 2. / ((GAM + 1.) * L->d), AR = 2. / ((GAM + 1.) * R->d);
  double BL = (GAM - 1.) / (GAM + 1.) * L->p, BR = (GAM - 1.) / (GAM + 1.) * R->p;
  double fL = (p > L->p ? sqrt(AL / (BL + p)) * (1. - (p - L->p) / (2. * (BL + p)))
                        : pow(p / L->p, -(GAM + 1) / (2. * GAM)) / (L->d * L->a));
  double fR = (p > R->p ? sqrt(AR / (BR + p)) * (1. - (p - R->p) / (2. * (BR + p)))
                        : pow(p / R->p, -(GAM + 1) / (2. * GAM)) / (R->d * R->a));
  return fL + fR;
}

static double f_root(double p, const oW1 *L, const oW1 *R, double *u) {
  double AL = 2. / ((GAM + 1.) * L->d), AR = 2. / ((GAM + 1.) * R->d);
  double BL = (GAM - 1.) / (GAM + 1.) * L->p, BR = (GAM - 1.) / (GAM + 1.) * R->p;
  double fL = (p > L->p ? (p - L->p) * sqrt(AL / (BL + p))
                        : 2. * L->a / (GAM - 1.) * (pow(p / L->p, (GAM - 1) / (2. * GAM)) - 1.));
  double fR = (p > R->p ? (p - R->p) * sqrt(AR / (BR + p))
                        : 2. * R->a / (GAM - 1.) * (pow(p / R->p, (GAM - 1) / (2. * GAM)) - 1.));
  double du = R->u - L->u;
  *u = 0.5 * (L->u + R->u) + 0.5 * (fR - fL);
  return fL + fR + du;
}

/* findPressure_Hybrid (src/hydro_utils.c:625) */
static double p_star_hybrid(const oW1 *L, const oW1 *R, double *ustar) {
  double dbar = 0.5 * (L->d + R->d), abar = 0.5 * (L->a + R->a);
  double ppvrs = 0.5 * ((L->p + R->p) + (L->u - R->u) * dbar * abar);
  double pmax = fmax(L->p, R->p), pmin = fmin(L->p, R->p);
  double pstar = ppvrs;
  if (((pmax / pmin) < 2.) && ((pmin < pstar) && (pstar < pmax))) {
    *ustar = 0.5 * ((L->u + R->u) + (L->p - R->p) / (dbar * abar));
  } else if (pstar < pmin) {
    double z = (GAM - 1.) / (2. * GAM);
    double iz = (2. * GAM) / (GAM - 1.);
    pstar = pow((L->a + R->a - (GAM - 1.) / 2. * (R->u - L->u)) / (L->a / pow(L->p, z) + R->a / pow(R->p, z)), iz);
    *ustar = L->u - 2. * L->a / (GAM - 1.) * (pow(pstar / L->p, z) - 1.);
  } else {
    double p0 = fmax(0., ppvrs);
    double AL = 2. / ((GAM + 1.) * L->d), AR = 2. / ((GAM + 1.) * R->d);
    double BL = (GAM - 1.) / (GAM + 1.) * L->p, BR = (GAM - 1.) / (GAM + 1.) * R->p;
    double GL = sqrt(AL / (p0 + BL)), GR = sqrt(AR / (p0 + BR));
    pstar = (GL * L->p + GR * R->p - (R->u - L->u)) / (GL + GR);
    *ustar = 0.5 * ((L->u + R->u) + (pstar - R->p) * GR - (pstar - L->p) * GL);
  }
  return pstar;
}

/* findPressure (src/hydro_utils.c:680): Newton iteration on the exact solver */
static double p_star_exact(const oW1 *L, const oW1 *R, double *u) {
  double unsurz = (2.0 * GAM) / (GAM - 1.0);
  double pmin = fmin(L->p, R->p), pmax = fmax(L->p, R->p);
  double AL = 2. / ((GAM + 1.) * L->d), AR = 2. / ((GAM + 1.) * R->d);
  double BL = (GAM - 1.) / (GAM + 1.) * L->p, BR = (GAM - 1.) / (GAM + 1.) * R->p;
  double ppv0 = 0.5 * (L->p + R->p) - 0.125 * (R->u - L->u) * (R->d + L->d) * (R->a + L->a);
  double ptr0 = pow((L->a + R->a - 0.5 * (GAM - 1) * (R->u - L->u)) /
                        (L->a / pow(L->p, 1. / unsurz) + R->a / pow(R->p, 1. / unsurz)),
                    unsurz);
  double ppv = fmax(ERR_TOL, ppv0), ptr = fmax(ERR_TOL, ptr0);
  double GL = sqrt(AL / (ppv + BL)), GR = sqrt(AR / (ppv + BR));
  double pts0 = (GL * L->p + GR * R->p - (R->u - L->u)) / (GL + GR);
  double pts = fmax(ERR_TOL, pts0);
  double p, dp, porg, err, u2;
  int i;
  if (((pmax / pmin) < 2.0) && ((pmin <= ppv) && (ppv <= pmax))) p = ppv;
  else if (ppv < pmin) p = ptr;
  else p = pts;
  for (i = 0; i < N_ITER_MAX; i++) {
    dp = f_root(p, L, R, &u2) / f_root_prime(p, L, R);
    if (isnan(dp)) { g_err |= ORC_ERR_NAN; break; }
    if (fabs(dp) < ERR_TOL) break;
    while ((p - dp) < 0) dp = dp * 0.5;
    porg = p;
    p = p - dp;
    err = 2. * fabs(p - porg) / (fabs(p + porg));
    if (err < ERR_TOL) break;
    if (f_root(p, L, R, &u2) < ERR_TOL) break;
  }
  f_root(p, L, R, &u2);
  *u = u2;
  return p;
}

/* speedestimate{X,Y,Z}_HLLC (src/hydro_utils.c:1264): normal velocity index n */
static void wave_speeds(const oW *WL, const oW *WR, int n, double *SL, double *SR, double *ustar) {
  oW1 L, R;
  double pstar, qL, qR;
  double vl[3] = {WL->u, WL->v, WL->w}, vr[3] = {WR->u, WR->v, WR->w};
  L.d = WL->d; L.u = vl[n]; L.p = WL->p; L.a = sqrt(GAM * L.p / L.d);
  R.d = WR->d; R.u = vr[n]; R.p = WR->p; R.a = sqrt(GAM * R.p / R.d);
  pstar = p_star_hybrid(&L, &R, ustar);
  if (pstar < 0) pstar = p_star_exact(&L, &R, ustar);
  if (pstar < 0) g_err |= ORC_ERR_NEG_PSTAR;
  qL = (pstar <= WL->p ? 1. : sqrt(1. + (GAM + 1.) / (2. * GAM) * ((pstar) / WL->p - 1.)));
  qR = (pstar <= WR->p ? 1. : sqrt(1. + (GAM + 1.) / (2. * GAM) * ((pstar) / WR->p - 1.)));
  *SL = L.u - L.a * qL;
  *SR = R.u + R.a * qR;
  if ((*SL) > (*SR)) {
    *SL = fmin(L.u - L.a, R.u - R.a);
    *SR = fmax(L.u + L.a, R.u + R.a);
  }
  if ((*SL) > (*SR)) g_err |= ORC_ERR_SLSR;
  if (isnan(*ustar)) g_err |= ORC_ERR_NAN;
}

/* Euler flux along axis n of a conserved state, getflux_{X,Y,Z} (src/hydro_utils.c:916-968).
 * m[] are the momenta, t1/t2 the transverse momentum indices in the order the
 * reference sums them. */
static void euler_flux(const oU *U, int n, double f[5]) {
  double m[3] = {U->du, U->dv, U->dw};
  double mn = m[n];
  int t1 = (n == 0) ? 1 : 0, t2 = (n == 2) ? 1 : 2;
  double all = U->du * U->du + U->dv * U->dv + U->dw * U->dw;
  f[0] = mn;
  f[1 + n] = 0.5 * (3. - GAM) * mn * mn / U->d + (GAM - 1.) * U->E - 0.5 * (GAM - 1.) * (m[t1] * m[t1] + m[t2] * m[t2]) / U->d;
  f[1 + t1] = mn * m[t1] / U->d;
  f[1 + t2] = mn * m[t2] / U->d;
  f[4] = GAM * mn / U->d * U->E - 0.5 * (GAM - 1.) * mn / (U->d * U->d) * all;
}
#ifdef ORC_WRADHYD
/* tracer fluxes f[6..8] of getflux_{X,Y,Z} (src/hydro_utils.c:925-929,943-947,961-965) */
static double tracer_flux(const oU *U, int n, int t) {
  double m[3] = {U->du, U->dv, U->dw};
  return m[n] * TRW(U, t) / U->d;
}
#endif

/* HLLC flux across a face normal to axis n from left/right MUSCL states
 * (src/hydro_utils.c:2055-2138, same branches for y :1783, z :1508).
 * us (optional, -DDUAL_E): the state Us of the branch taken (the upwind state or
 * the star state), from which the sweeps take the internal-energy flux and the
 * face velocity of divu (src/hydro_utils.c:2126-2129). */
static void hllc_flux(const oW *WL, const oW *WR, int n, double F[5], oU *us, double *fx) {
  double SL, SR, ustar;
  oU UL, UR;
  int k;
  for (k = 0; k < 5; k++) F[k] = 0.;
#ifdef ORC_WRADHYD
  if (fx) for (int t = 0; t < NTR; t++) fx[t] = 0.;
#endif
  wave_speeds(WL, WR, n, &SL, &SR, &ustar);
  to_cons(WL, &UL);
  to_cons(WR, &UR);
  if (SL >= 0.) {
    euler_flux(&UL, n, F);
    if (us) *us = UL;
#ifdef ORC_WRADHYD
    if (fx) for (int t = 0; t < NTR; t++) fx[t] = tracer_flux(&UL, n, t);
#endif
  } else if (SR <= 0.) {
    euler_flux(&UR, n, F);
    if (us) *us = UR;
#ifdef ORC_WRADHYD
    if (fx) for (int t = 0; t < NTR; t++) fx[t] = tracer_flux(&UR, n, t);
#endif
  } else if ((SL < 0.) && (ustar >= 0.)) {
    const oW *W = WL;
    const oU *U = &UL;
    double vel[3] = {W->u, W->v, W->w}, mom[3] = {U->du, U->dv, U->dw};
    double un = vel[n], fact;
    euler_flux(U, n, F);
    fact = W->d * (SL - un) / (SL - ustar);
    F[0] += (fact * 1. - U->d) * SL;
    for (k = 0; k < 3; k++) F[1 + k] += (fact * (k == n ? ustar : vel[k]) - mom[k]) * SL;
    F[4] += (fact * (U->E / U->d + (ustar - un) * (ustar + W->p / (W->d * (SL - un)))) - U->E) * SL;
#ifdef ORC_WRADHYD
    /* src/hydro_utils.c:1534-1535 (and :1809, :2115 for y, x) */
    if (fx)
      for (int t = 0; t < NTR; t++) fx[t] = tracer_flux(U, n, t) + (fact * TRW(W, t) / W->d - TRW(U, t)) * SL;
#endif
    if (us) {
      double m[3];
      for (k = 0; k < 3; k++) m[k] = fact * (k == n ? ustar : vel[k]);
      us->d = fact * 1.;
      us->du = m[0]; us->dv = m[1]; us->dw = m[2];
      us->E = fact * (U->E / U->d + (ustar - un) * (ustar + W->p / (W->d * (SL - un))));
    }
  } else if ((ustar <= 0.) && (SR > 0.)) {
    const oW *W = WR;
    const oU *U = &UR;
    double vel[3] = {W->u, W->v, W->w}, mom[3] = {U->du, U->dv, U->dw};
    double un = vel[n], fact;
    euler_flux(U, n, F);
    fact = W->d * (SR - un) / (SR - ustar);
    F[0] += (fact * 1. - U->d) * SR;
    for (k = 0; k < 3; k++) F[1 + k] += (fact * (k == n ? ustar : vel[k]) - mom[k]) * SR;
    F[4] += (fact * (U->E / U->d + (ustar - un) * (ustar + W->p / (W->d * (SR - un)))) - U->E) * SR;
#ifdef ORC_WRADHYD
    if (fx)
      for (int t = 0; t < NTR; t++) fx[t] = tracer_flux(U, n, t) + (fact * TRW(W, t) / W->d - TRW(U, t)) * SR;
#endif
    if (us) {
      double m[3];
      for (k = 0; k < 3; k++) m[k] = fact * (k == n ? ustar : vel[k]);
      us->d = fact * 1.;
      us->du = m[0]; us->dv = m[1]; us->dw = m[2];
      us->E = fact * (U->E / U->d + (ustar - un) * (ustar + W->p / (W->d * (SR - un))));
    }
  }
}

/* ---------------------------------------------- gather (src/hydro_utils.c:2852-3028 / 2465-2845) */
static int flag_on(int flags, int f) { return (flags & f) != 0; }

/* coarse2fine_hydro2 (src/hydro_utils.c:311): limited-slope interpolation of a
 * coarse leaf cell into 8 sub-cell states (HYDROTEST gather only). */
static void interp_coarse(oCell *cell, oW Wi[8], int flags) {
  oOct *oct = oct_of(cell);
  double dxcur = pow(0.5, oct->level);
  double q0[5], D[3][5];
  const oW *W0 = &cell->field;
  const oW *Wm = NULL, *Wp = NULL;
  int dir, k, ix, iy, iz;
  as5(W0, q0);
  for (dir = 0; dir < 3; dir++) {
    int same, nc;
    double qm[5], qp[5];
    cell_nei(cell->idx, 2 * dir, &same, &nc);
    if (same) Wm = &oct->cell[nc].field;
    else if (oct->nei[2 * dir] != NULL && oct->nei[2 * dir]->child != NULL) Wm = &oct->nei[2 * dir]->child->cell[nc].field;
    if (flag_on(flags, ORC_TRANSXM) && oct->x == 0. && dir == 0) Wm = &cell->field;
    if (flag_on(flags, ORC_TRANSYM) && oct->y == 0. && dir == 1) Wm = &cell->field;
    if (flag_on(flags, ORC_TRANSZM) && oct->z == 0. && dir == 2) Wm = &cell->field;
    cell_nei(cell->idx, 2 * dir + 1, &same, &nc);
    if (same) Wp = &oct->cell[nc].field;
    else if (oct->nei[2 * dir + 1] != NULL && oct->nei[2 * dir + 1]->child != NULL) Wp = &oct->nei[2 * dir + 1]->child->cell[nc].field;
    if (flag_on(flags, ORC_TRANSXP) && (oct->x + 2. * dxcur) == 1. && dir == 0) Wp = &cell->field;
    if (flag_on(flags, ORC_TRANSYP) && (oct->y + 2. * dxcur) == 1. && dir == 1) Wp = &cell->field;
    if (flag_on(flags, ORC_TRANSZP) && (oct->z + 2. * dxcur) == 1. && dir == 2) Wp = &cell->field;
    if (Wm == NULL || Wp == NULL) { g_err |= ORC_ERR_TREE; Wm = Wp = W0; }
    as5(Wm, qm);
    as5(Wp, qp);
    for (k = 0; k < 5; k++) D[dir][k] = limit1(q0[k] - qm[k], qp[k] - q0[k]);
  }
  for (iz = 0; iz < 2; iz++)
    for (iy = 0; iy < 2; iy++)
      for (ix = 0; ix < 2; ix++) {
        double ox = -0.25 + ix * 0.5, oy = -0.25 + iy * 0.5, oz = -0.25 + iz * 0.5;
        double r[5];
        oW *W = &Wi[ix + 2 * iy + 4 * iz];
        for (k = 0; k < 5; k++) r[k] = q0[k] + ox * D[0][k] + oy * D[1][k] + oz * D[2][k];
        W->d = r[0]; W->u = r[1]; W->v = r[2]; W->w = r[3]; W->p = r[4];
        get_E(W);
        W->a = sqrt(GAM * W->p / W->d);
      }
}


/* mirror maps of the transmissive ghost octs (src/hydro_utils.c:2504-2610) */
static const int MIRROR[6][8] = {
    {0, 0, 2, 2, 4, 4, 6, 6}, /* -x */
    {1, 1, 3, 3, 5, 5, 7, 7}, /* +x */
    {0, 1, 0, 1, 4, 5, 4, 5}, /* -y */
    {2, 3, 2, 3, 7, 6, 6, 7}, /* +y (as in the reference, cells 4/5 swapped) */
    {0, 1, 2, 3, 0, 1, 2, 3}, /* -z */
    {4, 5, 6, 7, 4, 5, 6, 7}, /* +z */
};
static const int TFLAG[6] = {ORC_TRANSXM, ORC_TRANSXP, ORC_TRANSYM, ORC_TRANSYP, ORC_TRANSZM, ORC_TRANSZP};

static int at_boundary(const oOct *o, int k) {
  double dx = pow(0.5, o->level);
  switch (k) {
    case 0: return o->x == 0.;
    case 1: return (o->x + 2. * dx) == 1.;
    case 2: return o->y == 0.;
    case 3: return (o->y + 2. * dx) == 1.;
    case 4: return o->z == 0.;
    default: return (o->z + 2. * dx) == 1.;
  }
}

#ifdef ORC_WGRAV
/* coarse2fine_forcelin (src/poisson_utils.c:315-425): the force of a coarse leaf
 * cell spread over its 8 sub-cells by unlimited one-sided differences: a
 * sub-cell on the - side of an axis uses f0 - f(-neighbour), on the + side
 * f(+neighbour) - f0, times an offset of -/+1/4; transmissive faces use the
 * cell itself as the neighbour. */
static void force_lin(oCell *cell, double floc[24], int flags) {
  oOct *oct = oct_of(cell);
  const double *U0 = cell->f;
  double D[6][3];
  int dir, i, ix, iy, iz;
  for (dir = 0; dir < 3; dir++) {
    const double *Um = NULL, *Up = NULL;
    int same, nc;
    cell_nei(cell->idx, 2 * dir, &same, &nc);
    if (same) Um = oct->cell[nc].f;
    else if (oct->nei[2 * dir] != NULL && oct->nei[2 * dir]->child != NULL) Um = oct->nei[2 * dir]->child->cell[nc].f;
    if (!same && flag_on(flags, TFLAG[2 * dir]) && at_boundary(oct, 2 * dir)) Um = U0;
    cell_nei(cell->idx, 2 * dir + 1, &same, &nc);
    if (same) Up = oct->cell[nc].f;
    else if (oct->nei[2 * dir + 1] != NULL && oct->nei[2 * dir + 1]->child != NULL)
      Up = oct->nei[2 * dir + 1]->child->cell[nc].f;
    if (!same && flag_on(flags, TFLAG[2 * dir + 1]) && at_boundary(oct, 2 * dir + 1)) Up = U0;
    if (Um == NULL || Up == NULL) { g_err |= ORC_ERR_TREE; Um = Up = U0; }
    for (i = 0; i < 3; i++) D[2 * dir][i] = U0[i] - Um[i];
    for (i = 0; i < 3; i++) D[2 * dir + 1][i] = Up[i] - U0[i];
  }
  for (iz = 0; iz < 2; iz++)
    for (iy = 0; iy < 2; iy++)
      for (ix = 0; ix < 2; ix++) {
        double *fp = floc + 3 * (ix + 2 * iy + 4 * iz);
        for (i = 0; i < 3; i++)
          fp[i] = U0[i] + D[ix][i] * (-0.25 + ix * 0.5) + D[2 + iy][i] * (-0.25 + iy * 0.5) +
                  D[4 + iz][i] * (-0.25 + iz * 0.5);
      }
}
#endif

/* One step of the recursive neighbour walk: from the level-(L-1) cell `cell`,
 * find the level-(L-1) cell across direction k, fill stencil slot `slot`, and
 * return that cell (the start of the next order of the walk). */
static oCell *fill_slot(Stencil *st, int slot, oCell *cell, int k, int flags) {
  oCell *nc = NULL;
  const int *map = NULL;
  oW Wi[8];
  char ch[8];
  int c;
  int hydrotest = flag_on(flags, ORC_HYDROTEST);
  if (cell->child != NULL) {
    nc = cell->child->nei[k];
    if (hydrotest && flag_on(flags, TFLAG[k]) && at_boundary(cell->child, k)) {
      nc = cell;
      map = MIRROR[k];
    }
  } else {
    int same, vc;
    oOct *oct = oct_of(cell);
    cell_nei(cell->idx, k, &same, &vc);
    if (same) {
      nc = &oct->cell[vc];
    } else {
      if (oct->nei[k] != NULL && oct->nei[k]->child != NULL) nc = &oct->nei[k]->child->cell[vc];
      if (hydrotest && flag_on(flags, TFLAG[k]) && at_boundary(oct, k)) {
        nc = cell;
        map = MIRROR[k];
      }
    }
  }
  if (nc == NULL) { g_err |= ORC_ERR_TREE; return NULL; }
#ifdef ORC_WGRAV
  double floc[24];
#endif
  if (nc->child != NULL) {
    for (c = 0; c < 8; c++) { Wi[c] = nc->child->cell[c].field; ch[c] = (nc->child->cell[c].child != NULL); }
#ifdef ORC_WGRAV
    for (c = 0; c < 8; c++) memcpy(floc + 3 * c, nc->child->cell[c].f, sizeof(double) * 3);
#endif
  } else {
    if (hydrotest) interp_coarse(nc, Wi, flags);
    else for (c = 0; c < 8; c++) Wi[c] = nc->field;
    for (c = 0; c < 8; c++) ch[c] = 0;
#ifdef ORC_WGRAV
    force_lin(nc, floc, flags);
#endif
  }
  for (c = 0; c < 8; c++) {
    int s = map ? map[c] : c;
    st->w[slot][c] = Wi[s];
    st->split[slot][c] = ch[s];
#ifdef ORC_WGRAV
    memcpy(st->f[slot][c], floc + 3 * s, sizeof(double) * 3);
#endif
  }
  return nc;
}

/* recursive_neighbor_gather_oct (src/hydro_utils.c:2852): fill `slot` from the
 * level-(L-1) cell across direction `k` of `cell`; order 1 (faces) recurses to
 * order 2 (edges) in the directions off the first axis, order 2 to order 3
 * (corners) off both axes.  Slots already visited are skipped, so the walk
 * order decides which path fills an edge/corner slot, as in the reference. */
static void walk(Stencil *st, char *visit, int slot, int i1, int i2, int order, int k, oCell *cell, int flags) {
  int i;
  oCell *nc = fill_slot(st, slot, cell, k, flags);
  if (nc == NULL || order == 3) return;
  for (i = 0; i < 6; i++) {
    int s2;
    if ((i >> 1) == (i1 >> 1)) continue;
    if (order == 2 && (i >> 1) == (i2 >> 1)) continue;
    s2 = slot + SLOT_OFF[i];
    if (visit[s2]) continue;
    visit[s2] = 1;
    walk(st, visit, s2, i1, order == 1 ? i : i2, order + 1, i, nc, flags);
  }
}

static void gather(Stencil *st, oOct *o, int flags) {
  char visit[27];
  int c, k;
  memset(visit, 0, sizeof(visit));
  memset(st->done, 0, sizeof(st->done));
  for (c = 0; c < 8; c++) {
    st->w[13][c] = o->cell[c].field;
    st->split[13][c] = (o->cell[c].child != NULL);
#ifdef ORC_WGRAV
    memcpy(st->f[13][c], o->cell[c].f, sizeof(double) * 3);
#endif
  }
  visit[13] = 1;
  for (k = 0; k < 6; k++) {
    int slot = 13 + SLOT_OFF[k];
    visit[slot] = 1;
    walk(st, visit, slot, k, -1, 1, k, o->parent, flags);
  }
}

/* ---------------------------------------------- level advance */
static Stencil g_st;

int orc_hydro_solver(void **firstoct_v, int level, double dt, int flags) {
  oOct **firstoct = (oOct **)firstoct_v;
  double dx = pow(0.5, level);
  double dtsurdx = dt / dx;
  oOct *o;
  int c, k, n = 0;
  g_err = 0;
  const int dual = flag_on(flags, ORC_DUAL_E);
  for (o = firstoct[level - 1]; o != NULL; o = o->next) {
    double flux[8][6][9];  /* [5]: internal-energy flux (-DDUAL_E), [6..8]: tracer fluxes (-DWRADHYD) */
    double divu[8];
    if (o->cpu != 0) continue;
    n++;
    gather(&g_st, o, flags);
    /* sweeps x, y, z: two faces per cell per direction, split neighbours cancelled */
    for (c = 0; c < 8; c++) {
      int dir;
      /* -DDUAL_E: eint of the cell's old state (W2U of its field) */
      const double eold = g_st.w[13][c].p / (GAM - 1.);
      divu[c] = 0.;
      for (dir = 0; dir < 3; dir++) {
        int s;
        for (s = 0; s < 2; s++) {
          int kf = 2 * dir + s, same, vc, nslot;
          const oW *Wc, *Wn;
          double F[9];
          oU us;
          cell_nei(c, kf, &same, &vc);
          nslot = same ? 13 : FACE_SLOT[kf];
          Wc = face_state(&g_st, 13, c, kf, dt, dx);
          Wn = face_state(&g_st, nslot, vc, kf ^ 1, dt, dx);
          F[6] = F[7] = F[8] = 0.;
#ifdef ORC_WRADHYD
          if (s == 0) hllc_flux(Wn, Wc, dir, F, dual ? &us : NULL, &F[6]);
          else hllc_flux(Wc, Wn, dir, F, dual ? &us : NULL, &F[6]);
#else
          if (s == 0) hllc_flux(Wn, Wc, dir, F, dual ? &us : NULL, NULL);
          else hllc_flux(Wc, Wn, dir, F, dual ? &us : NULL, NULL);
#endif
          F[5] = 0.;
          if (dual) {
            /* src/hydro_utils.c:2126-2129: ebar, the internal-energy flux and the
             * p div(u) term of the face (summed whether or not the neighbour is split) */
            double mom[3] = {us.du, us.dv, us.dw};
            double ebar = (us.E - 0.5 * (us.du * us.du + us.dv * us.dv + us.dw * us.dw) / us.d);
            double divuloc = (GAM - 1.) * (mom[dir] / us.d) * eold;
            F[5] = (mom[dir] / us.d * ebar);
            divu[c] += (s == 0) ? -divuloc : divuloc;
          }
          for (k = 0; k < 9; k++) flux[c][kf][k] = F[k] * (double)(!g_st.split[nslot][vc]);
        }
      }
    }
    /* updatefield + scatterstencil, cell by cell in order */
    for (c = 0; c < 8; c++) {
      oCell *cell = &o->cell[c];
      if (!g_st.split[13][c]) {
        oU dU, U;
        double one = 1., ekin;
        int f;
        memset(&dU, 0, sizeof(dU));
        for (f = 0; f < 6; f++) {
          dU.d += flux[c][f][0] * dtsurdx * one;
          dU.du += flux[c][f][1] * dtsurdx * one;
          dU.dv += flux[c][f][2] * dtsurdx * one;
          dU.dw += flux[c][f][3] * dtsurdx * one;
          dU.E += flux[c][f][4] * dtsurdx * one;
          dU.eint += flux[c][f][5] * dtsurdx * one;
#ifdef ORC_WRADHYD
          for (int t = 0; t < NTR; t++) TRW(&dU, t) += flux[c][f][6 + t] * dtsurdx * one;  /* src/hydro_utils.c:3068-3072 */
#endif
          one *= -1.;
        }
        if (isnan(cell->fieldnew.u)) g_err |= ORC_ERR_NAN;
        to_cons(&cell->fieldnew, &U);
        U.d += dU.d;
        U.du += dU.du;
        U.dv += dU.dv;
        U.dw += dU.dw;
        U.E += dU.E;
#ifdef ORC_WRADHYD
        for (int t = 0; t < NTR; t++) TRW(&U, t) += TRW(&dU, t);  /* src/hydro_utils.c:3158-3162 */
#endif
        ekin = 0.5 * (U.du * U.du + U.dv * U.dv + U.dw * U.dw) / U.d;
        if (dual) {
          /* src/hydro_utils.c:3167-3177: tracked eint, unless E - Ekin is well resolved */
          U.eint += dU.eint;
          U.eint += (-divu[c] * dtsurdx);
          if ((U.E - ekin) > 0.5 * pow(divu[c], 2)) U.eint = U.E - ekin;
        } else {
          U.eint = U.E - ekin;
        }
        U.eint = fmax(U.eint * (GAM - 1.), P_MIN) / (GAM - 1.);
        to_prim(&U, &cell->fieldnew, dual);
        cell->fieldnew.p = fmax(cell->fieldnew.p, P_MIN);
        cell->fieldnew.a = sqrt(GAM * cell->fieldnew.p / cell->fieldnew.d);
        get_E(&cell->fieldnew);
        if (isnan(cell->fieldnew.u)) g_err |= ORC_ERR_NAN;
#ifdef ORC_WRADHYD
        /* ceiling of the ionised fraction (src/hydro_utils.c:3197-3198) */
        if (cell->fieldnew.dX < 0) cell->fieldnew.dX = 0.;
        if (cell->fieldnew.dX > (cell->fieldnew.d * (1. - YHE_))) cell->fieldnew.dX = cell->fieldnew.d * (1. - YHE_);
#ifdef ORC_HELIUM
        /* the helium densities have a ceiling only (src/hydro_utils.c:3199-3202) */
        if (cell->fieldnew.dXHE > (cell->fieldnew.d * (YHE_))) cell->fieldnew.dXHE = cell->fieldnew.d * (YHE_);
        if (cell->fieldnew.dXXHE > (cell->fieldnew.d * (YHE_))) cell->fieldnew.dXXHE = cell->fieldnew.d * (YHE_);
#endif
#endif
      }
      /* fine -> coarse flux correction into unsplit coarse neighbours */
      for (k = 0; k < 6; k++) {
        int same, vc;
        oCell *cc;
        if (flag_on(flags, TFLAG[k]) && at_boundary(o, k)) continue;
        cell_nei(c, k, &same, &vc);
        if (same) continue;
        cc = o->nei[k];
        if (cc != NULL && cc->child == NULL) {
          oW W = cc->fieldnew;
          oU U;
          int one = (k & 1) ? 1 : -1; /* (int)POW(-1., k+1) */
          to_cons(&W, &U);
          U.d += flux[c][k][0] * dtsurdx * one * 0.125;
          U.du += flux[c][k][1] * dtsurdx * one * 0.125;
          U.dv += flux[c][k][2] * dtsurdx * one * 0.125;
          U.dw += flux[c][k][3] * dtsurdx * one * 0.125;
          U.E += flux[c][k][4] * dtsurdx * one * 0.125;
          if (dual) U.eint += flux[c][k][5] * dtsurdx * one * 0.125;
#ifdef ORC_WRADHYD
          for (int t = 0; t < NTR; t++) TRW(&U, t) += flux[c][k][6 + t] * dtsurdx * one * 0.125;
#endif
          to_prim(&U, &W, dual);
          cc->fieldnew = W;
        }
      }
    }
  }
  /* field := fieldnew (leaves); split cells := mean of children's primitives */
  if (n > 0) {
    for (o = firstoct[level - 1]; o != NULL; o = o->next) {
      for (c = 0; c < 8; c++) {
        oCell *cell = &o->cell[c];
        if (cell->child == NULL) {
          cell->field = cell->fieldnew;
          g_updates++;
        } else {
          oW W;
          int i;
          memset(&W, 0, sizeof(W));
          for (i = 0; i < 8; i++) {
            const oW *Wc = &cell->child->cell[i].field;
            W.d += Wc->d * 0.125;
            W.u += Wc->u * 0.125;
            W.v += Wc->v * 0.125;
            W.w += Wc->w * 0.125;
            W.p += Wc->p * 0.125;
#ifdef ORC_WRADHYD
            for (int t = 0; t < NTR; t++) TRW(&W, t) += TRW(Wc, t) * 0.125;  /* src/hydro_utils.c:3446-3460 */
#endif
          }
          get_E(&W);
          cell->field = W;
        }
      }
    }
  }
  return g_err;
}

#ifdef ORC_WGRAV
/* grav_correction (src/hydro_utils.c:2388-2444, PRIMITIVE): the full-step
 * gravity kick of the leaf velocities after HydroSolver, then E. */
int orc_grav_correction(void **firstoct_v, int level, double dt) {
  oOct **firstoct = (oOct **)firstoct_v;
  oOct *o;
  int c, err = 0;
  for (o = firstoct[level - 1]; o != NULL; o = o->next) {
    if (o->cpu != 0) continue;
    for (c = 0; c < 8; c++) {
      oCell *cell = &o->cell[c];
      oW W;
      if (cell->child != NULL) continue;
      W = cell->field;
      W.u += (-cell->f[0] * dt);
      W.v += (-cell->f[1] * dt);
      W.w += (-cell->f[2] * dt);
      get_E(&W);
      if (W.p < 0) err |= ORC_ERR_NAN;
      cell->field = W;
    }
  }
  return err;
}
#endif

void orc_clean_new_hydro(void **firstoct_v, int level) {
  oOct **firstoct = (oOct **)firstoct_v;
  oOct *o;
  int c;
  for (o = firstoct[level - 1]; o != NULL; o = o->next)
    for (c = 0; c < 8; c++) o->cell[c].fieldnew = o->cell[c].field;
}

/* L_comptstep_hydro (src/advanceamr.c:92), over every cell of the level */
double orc_comptstep_hydro(void **firstoct_v, int level, double cfl) {
  oOct **firstoct = (oOct **)firstoct_v;
  double dt = 1e9, smax = 0., dxcur = pow(0.5, level);
  oOct *o;
  int c;
  for (o = firstoct[level - 1]; o != NULL; o = o->next) {
    if (o->cpu != 0) continue;
    for (c = 0; c < 8; c++) {
      const oW *W = &o->cell[c].field;
      double va = sqrt(W->u * W->u + W->v * W->v + W->w * W->w);
      double aa = sqrt(GAM * W->p / W->d);
      smax = fmax(smax, va + aa);
    }
  }
  if (smax > 0.) dt = fmin(dxcur * cfl / (smax * 3.), dt);
  return dt;
}

/* ---------------------------------------------- level schedule (src/advanceamr.c:243-1299) */
typedef struct {
  oOct **first;
  int lcoarse, lmax, nsub, flags;
  double dt_param, time_max, cfl;
  double *adt;
  int err;
} Sched;

static int level_noct(oOct **first, int level) {
  int n = 0;
  oOct *o;
  for (o = first[level - 1]; o != NULL; o = o->next) n++;
  return n;
}

static double advance_level(Sched *S, int level, double tloc) {
  double dt = 0., dtnew, dthydro, dtfine;
  double *adt = S->adt;
  int is = 0;
  do {
    orc_clean_new_hydro((void **)S->first, level);
    dtnew = S->dt_param;
    dtnew = ((S->time_max - tloc) < dtnew ? (S->time_max - tloc) : dtnew);
    dthydro = orc_comptstep_hydro((void **)S->first, level, S->cfl);
    dtnew = (dthydro < dtnew ? dthydro : dtnew);
    adt[level - 1] = dtnew;
    if (level == S->lcoarse) adt[level - 2] = adt[level - 1];
    if (adt[level - 2] < adt[level - 1]) adt[level - 1] = adt[level - 2];
    else adt[level - 1] = fmin(adt[level - 1], adt[level - 2] - dt);
    if (level < S->lmax && level_noct(S->first, level + 1) > 0) {
      dtfine = advance_level(S, level + 1, tloc);
      adt[level - 1] = dtfine;
      if (level == S->lcoarse) adt[level - 2] = adt[level - 1];
    }
    S->err |= orc_hydro_solver((void **)S->first, level, adt[level - 1], S->flags);
#ifdef ORC_WGRAV
    S->err |= orc_grav_correction((void **)S->first, level, adt[level - 1]); /* src/advanceamr.c:999 */
#endif
    dt += adt[level - 1];
    tloc += adt[level - 1];
    is++;
  } while ((dt < adt[level - 2]) && (is < S->nsub));
  return dt;
}

double orc_run(void **firstoct, int lcoarse, int lmax, int nsteps, double dt_param,
               double time_max, int nsub, double cfl, int flags, double tsim0,
               double *adt, int *steps_done, int *err) {
  Sched S;
  int n, l;
  double tsim = tsim0;
  S.first = (oOct **)firstoct;
  S.lcoarse = lcoarse; S.lmax = lmax; S.nsub = nsub; S.flags = flags;
  S.dt_param = dt_param; S.time_max = time_max; S.cfl = cfl; S.adt = adt; S.err = 0;
  for (l = 1; l <= lmax; l++) adt[l - 1] = dt_param;
  for (n = 0; n < nsteps && tsim < time_max; n++) {
    advance_level(&S, lcoarse, tsim);
    tsim += adt[lcoarse - 1];
  }
  if (steps_done) *steps_done = n;
  if (err) *err = S.err;
  return tsim;
}

#ifdef ORC_WGRAV
/* ---------------------------------------------- plain-layout tree -> -DWGRAV copy
 * Test helper: the product library's trees use the default (no WGRAV) layout;
 * this copies one, pointers remapped, into the gravity layout so the gravity
 * restatement can run on the same octs in the same list order.  Forces start
 * at zero. */
typedef struct pCell {
  struct pOct *child;
  double marked;
  int idx;
  oW field;
  oW fieldnew;
} pCell;
typedef struct pOct {
  pCell cell[8];
  pCell *nei[6];
  pCell *parent;
  struct pOct *next, *prev, *nexthash;
  double x, y, z;
  int cpu;
  int level;
} pOct;
_Static_assert(sizeof(pOct) == 1200, "plain OCT layout");

typedef struct {
  oOct *octs;
  const pOct **src;  /* sorted by address, with the copy index in idx */
  long *idx;
  long n;
  oCell root;
  oOct **first;
  int lmax;
} GravClone;

static GravClone *g_sort_ctx;
static int cmp_src(const void *a, const void *b) {
  const pOct *x = g_sort_ctx->src[*(const long *)a], *y = g_sort_ctx->src[*(const long *)b];
  return (x > y) - (x < y);
}

static oOct *clone_oct(GravClone *C, const pOct *o) {
  long lo = 0, hi = C->n - 1;
  if (o == NULL) return NULL;
  while (lo <= hi) {
    long m = (lo + hi) / 2;
    const pOct *x = C->src[C->idx[m]];
    if (x == o) return &C->octs[C->idx[m]];
    if (x < o) lo = m + 1;
    else hi = m - 1;
  }
  return NULL;
}

/* A cell pointer of the source tree: a cell of a copied oct, or the stand-in
 * root cell (the parent-level cell whose child is the level-1 oct). */
static oCell *clone_cell(GravClone *C, const pCell *c, const pOct *top, int *err) {
  oOct *o;
  if (c == NULL) return NULL;
  if (c->child == top && top != NULL) return &C->root;
  o = clone_oct(C, (const pOct *)((const char *)c - (size_t)c->idx * sizeof(pCell)));
  if (o == NULL) { *err = 1; return NULL; }
  return &o->cell[c->idx];
}

void *orc_grav_clone(void **src_first_v, int lmax) {
  const pOct **src_first = (const pOct **)src_first_v;
  GravClone *C = (GravClone *)calloc(1, sizeof(GravClone));
  const pOct *o, *top = src_first[0];
  long n = 0, i;
  int l, c, k, err = 0;
  C->lmax = lmax;
  for (l = 1; l <= lmax; l++)
    for (o = src_first[l - 1]; o != NULL; o = o->next) n++;
  C->n = n;
  C->octs = (oOct *)calloc((size_t)(n > 0 ? n : 1), sizeof(oOct));
  C->src = (const pOct **)malloc(sizeof(pOct *) * (size_t)(n > 0 ? n : 1));
  C->idx = (long *)malloc(sizeof(long) * (size_t)(n > 0 ? n : 1));
  C->first = (oOct **)calloc((size_t)lmax, sizeof(oOct *));
  n = 0;
  for (l = 1; l <= lmax; l++)
    for (o = src_first[l - 1]; o != NULL; o = o->next) { C->src[n] = o; C->idx[n] = n; n++; }
  g_sort_ctx = C;
  qsort(C->idx, (size_t)n, sizeof(long), cmp_src);
  C->root.child = clone_oct(C, top);
  for (i = 0; i < n; i++) {
    const pOct *s = C->src[i];
    oOct *d = &C->octs[i];
    for (c = 0; c < 8; c++) {
      d->cell[c].child = clone_oct(C, s->cell[c].child);
      d->cell[c].marked = s->cell[c].marked;
      d->cell[c].idx = s->cell[c].idx;
      d->cell[c].field = s->cell[c].field;
      d->cell[c].fieldnew = s->cell[c].fieldnew;
    }
    for (k = 0; k < 6; k++) d->nei[k] = clone_cell(C, s->nei[k], top, &err);
    d->parent = clone_cell(C, s->parent, top, &err);
    d->next = clone_oct(C, s->next);
    d->prev = clone_oct(C, s->prev);
    d->x = s->x; d->y = s->y; d->z = s->z;
    d->cpu = s->cpu;
    d->level = s->level;
  }
  for (l = 1; l <= lmax; l++) C->first[l - 1] = clone_oct(C, src_first[l - 1]);
  if (err) {
    orc_grav_free(C);
    return NULL;
  }
  return C;
}

void **orc_grav_first(void *h) { return (void **)((GravClone *)h)->first; }

void orc_grav_set_force(void *h, int level, const double *fx, const double *fy, const double *fz) {
  GravClone *C = (GravClone *)h;
  oOct *o;
  long i = 0;
  int c;
  for (o = C->first[level - 1]; o != NULL; o = o->next, i++)
    for (c = 0; c < 8; c++) {
      o->cell[c].f[0] = fx[8 * i + c];
      o->cell[c].f[1] = fy[8 * i + c];
      o->cell[c].f[2] = fz[8 * i + c];
    }
}

/* d,u,v,w,p,a,E of field (which=0) or fieldnew (which=1) as 7 planes, list order */
void orc_grav_get_field(void *h, int level, int which, double *out) {
  GravClone *C = (GravClone *)h;
  oOct *o;
  long i = 0, n = 0;
  int c;
  for (o = C->first[level - 1]; o != NULL; o = o->next) n++;
  for (o = C->first[level - 1]; o != NULL; o = o->next, i++)
    for (c = 0; c < 8; c++) {
      const oW *W = which ? &o->cell[c].fieldnew : &o->cell[c].field;
      long k = 8 * i + c;
      out[k] = W->d; out[8 * n + k] = W->u; out[16 * n + k] = W->v; out[24 * n + k] = W->w;
      out[32 * n + k] = W->p; out[40 * n + k] = W->a; out[48 * n + k] = W->E;
    }
}

void orc_grav_free(void *h) {
  GravClone *C = (GravClone *)h;
  if (C == NULL) return;
  free(C->octs);
  free(C->src);
  free(C->idx);
  free(C->first);
  free(C);
}
#endif

/* ---- ALLOCT field dump: dumpalloct_serial (src/io.c:1233-1358) -------------
 * For each selected field: directory <folder>grid_<name>/ (mkdir 0755) and file
 * <name>.<ndumps %05d>.p<rank %05d> in it (:1274-1283).  Header (:1291-1298,
 * rewritten with the final values at :1349-1356): int n_cell, then tsim, xmin,
 * xmax, ymin, ymax, zmin, zmax as 4-byte words; tsim is the caller's double, of
 * which fwrite(&tsim, sizeof(float)) writes the first 4 bytes.  Body
 * (:1304-1340): levels lcoarse..lmax, the octs of `rank` in list order
 * (cpu->octList, src/oct.c:250-270), and in each oct the cells without a child
 * (every cell when the oct is at lmax), one float per field and cell, the value of
 * assign_grid_field (src/io.c:32-104): 0-2 cell corner x,y,z, 3 level, 4 cpu,
 * 12 marked, 13-17 field d,u,v,w,p; with ORC_WGRAV 5 gdata.d, 7 gdata.p, 8 res,
 * 9-11 f[0..2].  The bounds are the min of the oct corners and the max of corner
 * + oct size 0.5^(level-1) over the dumped cells, kept as floats.
 * Returns 0, or -1 for an id this layout has no member for or an I/O error. */
#include <stdio.h>
#include <sys/stat.h>

static int orc_grid_field(int id, const oOct *o, const oCell *c, float *v) {
  const double dxc = pow(0.5, o->level);
  switch (id) {
    case 0: *v = (float)(o->x + (double)(c->idx & 1) * dxc); return 0;
    case 1: *v = (float)(o->y + (double)((c->idx >> 1) & 1) * dxc); return 0;
    case 2: *v = (float)(o->z + (double)(c->idx >> 2) * dxc); return 0;
    case 3: *v = (float)o->level; return 0;
    case 4: *v = (float)o->cpu; return 0;
#ifdef ORC_WGRAV
    case 5: *v = (float)c->gd; return 0;
    case 7: *v = (float)c->gp; return 0;
    case 8: *v = (float)c->res; return 0;
    case 9: case 10: case 11: *v = (float)c->f[id - 9]; return 0;
#endif
    case 12: *v = (float)c->marked; return 0;
    case 13: *v = (float)c->field.d; return 0;
    case 14: *v = (float)c->field.u; return 0;
    case 15: *v = (float)c->field.v; return 0;
    case 16: *v = (float)c->field.w; return 0;
    case 17: *v = (float)c->field.p; return 0;
    default: return -1;
  }
}

static void orc_alloct_header(FILE *f, int n, double tsim, const float b[6]) {
  fwrite(&n, sizeof(int), 1, f);
  fwrite(&tsim, 4, 1, f);
  fwrite(b, sizeof(float), 6, f);
}

int orc_dump_alloct(const char *folder, void **firstoct, int lcoarse, int lmax, int rank, int ndumps, double tsim,
                    int nfields, const int *ids, const char *const *names) {
  FILE *fp[32];
  float b[6] = {2.f, -1.f, 2.f, -1.f, 2.f, -1.f};  /* xmin, xmax, ymin, ymax, zmin, zmax */
  int n = 0, i, level, c, rc = 0;
  char dir[512], path[1024];
  if (nfields < 1 || nfields > 32) return -1;
  for (i = 0; i < nfields; i++) {
    float probe;
    oCell dummy_cell;
    oOct dummy_oct;
    memset(&dummy_oct, 0, sizeof(dummy_oct));
    memset(&dummy_cell, 0, sizeof(dummy_cell));
    if (orc_grid_field(ids[i], &dummy_oct, &dummy_cell, &probe) != 0) return -1;
  }
  for (i = 0; i < nfields; i++) {
    snprintf(dir, sizeof(dir), "%sgrid_%s/", folder, names[i]);
    mkdir(dir, 0755);
    snprintf(path, sizeof(path), "%s%s.%05d.p%05d", dir, names[i], ndumps, rank);
    fp[i] = fopen(path, "wb");
    if (fp[i] == NULL) {
      while (i-- > 0) fclose(fp[i]);
      return -1;
    }
    orc_alloct_header(fp[i], 0, tsim, b);
  }
  for (level = lcoarse; level <= lmax; level++) {
    const double dx = pow(0.5, level - 1);
    const oOct *o;
    for (o = (const oOct *)firstoct[level - 1]; o != NULL; o = o->next) {
      if (o->cpu != rank) continue;
      for (c = 0; c < 8; c++) {
        if (o->cell[c].child != NULL && o->level != lmax) continue;
        n++;
        for (i = 0; i < nfields; i++) {
          float v;
          orc_grid_field(ids[i], o, &o->cell[c], &v);
          fwrite(&v, sizeof(float), 1, fp[i]);
        }
        if (o->x < b[0]) b[0] = (float)o->x;
        if (o->y < b[2]) b[2] = (float)o->y;
        if (o->z < b[4]) b[4] = (float)o->z;
        if (o->x + dx > b[1]) b[1] = (float)(o->x + dx);
        if (o->y + dx > b[3]) b[3] = (float)(o->y + dx);
        if (o->z + dx > b[5]) b[5] = (float)(o->z + dx);
      }
    }
  }
  for (i = 0; i < nfields; i++) {
    rewind(fp[i]);
    orc_alloct_header(fp[i], n, tsim, b);
    if (ferror(fp[i])) rc = -1;
    if (fclose(fp[i]) != 0) rc = -1;
  }
  return rc;
}
