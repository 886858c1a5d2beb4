// hydro_math.cuh -- per-cell and per-face hydro arithmetic for the level kernels.
//
// Two instantiations:
//   MathF64 -- the plain path.  Every expression keeps the operation order of
//              the reference CPU hydro (src/hydro_utils.c) so that, compiled with
//              -fmad=false and IEEE division/square root, results match the
//              reference to the last bit except where libm pow() differs from
//              CUDA's pow() (TRRS branch and exact-solver fallback).
//   MathF32 -- the mixed path's reconstruction, wave speeds and fluxes in FP32:
//              the same algorithm with one reciprocal per density, approximate
//              (single-instruction) division, reciprocal and square root
//              (level_f32.cu is built with -use_fast_math) and algebraic
//              simplifications (d a^2 = gamma p).
//
// Primitive vectors are 5-wide: 0:d 1:u 2:v 3:w 4:p.  Face index k:
// 0:-x 1:+x 2:-y 3:+y 4:-z 5:+z.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace emma {

constexpr double kGam = 5. / 3.;   // GAMMA, src/param.h:4
constexpr double kPmin = 1e-10;    // PMIN, src/param.h:20
constexpr double kErrTol = 1e-10;  // ERRTOL, src/hydro_utils.c:18
constexpr int kNiterMax = 10;      // NITERMAX, src/hydro_utils.c:17

// Tracers advected with the gas by the -DWRADHYD builds: NT = 1, the ionised
// density dX, with the helium mass fraction YHE = 0 (no -DHELIUM, src/param.h:53);
// NT = 3, dX and the singly and doubly ionised helium densities dXHE, dXXHE, with
// YHE = 0.24 (-DHELIUM, src/param.h:48).  Tracer t is a part of the mass fraction
// frac(t): hydrogen 1 - YHE, helium YHE (src/hydro_utils.c:1244-1252).
template <int NT>
struct Tracers {
  static constexpr double kYhe = (NT == 3) ? 0.24 : 0.;
  __host__ __device__ static constexpr double frac(int t) { return t == 0 ? 1. - kYhe : kYhe; }
};

// status bits (mirrors EMMA_ST_* of emma_hydro.h)
constexpr unsigned kStNegDensity = 0x01, kStNegPstar = 0x02, kStNan = 0x04, kStTree = 0x08, kStTimeout = 0x40;

// ============================================================== FP64 (plain)
struct MathF64 {
  using R = double;

  // minmod_W, beta = 1 (src/hydro_utils.c:201)
  static __device__ __forceinline__ double limit(double m, double p) {
    if (p > 0) return fmax(fmax(0., fmin(m, p)), fmin(m, p));
    return fmin(fmin(0., fmax(m, p)), fmax(m, p));
  }

  // MUSCL_BOUND2 slopes + matrix_jacobian predictor (src/hydro_utils.c:976-1189).
  // q0: cell, qm/qp: neighbours per axis.  Out: D[3][5] slopes, Wt[5] predictor.
  // azero: the cell's stored sound speed is 0 (an averaged split cell)
  static __device__ __forceinline__ void muscl(const double q0[5], const double qm[3][5], const double qp[3][5],
                                               double dt, double dx, double D[3][5], double Wt[5],
                                               bool azero = false) {
#pragma unroll
    for (int dir = 0; dir < 3; dir++)
#pragma unroll
      for (int k = 0; k < 5; k++) D[dir][k] = limit(q0[k] - qm[dir][k], qp[dir][k] - q0[k]);
    // stored sound speed of the cell, as U2W/scatter computes it (src/hydro_utils.c:64,3186)
    const double a0 = azero ? 0. : sqrt(kGam * q0[4] / q0[0]);
    const double daa = q0[0] * a0 * a0;
    const double id = 1. / q0[0];
    double acc[5] = {0., 0., 0., 0., 0.};
#pragma unroll
    for (int dir = 0; dir < 3; dir++) {
      const double s = q0[1 + dir];
      acc[0] += s * D[dir][0];
      if (dir == 0) { acc[0] += q0[0] * D[0][1]; }
      acc[1] += s * D[dir][1];
      if (dir == 0) { acc[4] += daa * D[0][1]; }
      if (dir == 1) { acc[0] += q0[0] * D[1][2]; }
      acc[2] += s * D[dir][2];
      if (dir == 1) { acc[4] += daa * D[1][2]; }
      if (dir == 2) { acc[0] += q0[0] * D[2][3]; }
      acc[3] += s * D[dir][3];
      if (dir == 2) { acc[4] += daa * D[2][3]; }
      acc[1 + dir] += id * D[dir][4];
      acc[4] += s * D[dir][4];
    }
    const double fac = -dt / dx * 0.5;
#pragma unroll
    for (int i = 0; i < 5; i++) Wt[i] = acc[i] * fac;
  }

  // E and a of a face state from its (d,u,v,w,p)
  static __device__ __forceinline__ void face_finish(double W[7]) {
    W[6] = W[4] / (kGam - 1.) + 0.5 * W[0] * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]);
    W[5] = sqrt(kGam * W[4] / W[0]);
  }

  struct S1 { double d, u, p, a; };

  static __device__ double froot_prime(double p, const S1 &L, const S1 &R) {
    double AL = 2. / ((kGam + 1.) * L.d), AR = 2. / ((kGam + 1.) * R.d);
    double BL = (kGam - 1.) / (kGam + 1.) * L.p, BR = (kGam - 1.) / (kGam + 1.) * R.p;
    double fL = (p > L.p ? sqrt(AL / (BL + p)) * (1. - (p - L.p) / (2. * (BL + p)))
                         : pow(p / L.p, -(kGam + 1) / (2. * kGam)) / (L.d * L.a));
    double fR = (p > R.p ? sqrt(AR / (BR + p)) * (1. - (p - R.p) / (2. * (BR + p)))
                         : pow(p / R.p, -(kGam + 1) / (2. * kGam)) / (R.d * R.a));
    return fL + fR;
  }
  static __device__ double froot(double p, const S1 &L, const S1 &R, double *u) {
    double AL = 2. / ((kGam + 1.) * L.d), AR = 2. / ((kGam + 1.) * R.d);
    double BL = (kGam - 1.) / (kGam + 1.) * L.p, BR = (kGam - 1.) / (kGam + 1.) * R.p;
    double fL = (p > L.p ? (p - L.p) * sqrt(AL / (BL + p))
                         : 2. * L.a / (kGam - 1.) * (pow(p / L.p, (kGam - 1) / (2. * kGam)) - 1.));
    double fR = (p > R.p ? (p - R.p) * sqrt(AR / (BR + p))
                         : 2. * R.a / (kGam - 1.) * (pow(p / R.p, (kGam - 1) / (2. * kGam)) - 1.));
    *u = 0.5 * (L.u + R.u) + 0.5 * (fR - fL);
    return fL + fR + (R.u - L.u);
  }
  // findPressure (src/hydro_utils.c:680): rare fallback when the hybrid estimate is negative
  static __device__ __noinline__ double pstar_exact(const S1 &L, const S1 &R, double *u, unsigned &st) {
    const double unsurz = (2.0 * kGam) / (kGam - 1.0);
    double pmin = fmin(L.p, R.p), pmax = fmax(L.p, R.p);
    double AL = 2. / ((kGam + 1.) * L.d), AR = 2. / ((kGam + 1.) * R.d);
    double BL = (kGam - 1.) / (kGam + 1.) * L.p, BR = (kGam - 1.) / (kGam + 1.) * R.p;
    double ppv0 = 0.5 * (L.p + R.p) - 0.125 * (R.u - L.u) * (R.d + L.d) * (R.a + L.a);
    double ptr0 = pow((L.a + R.a - 0.5 * (kGam - 1) * (R.u - L.u)) /
                          (L.a / pow(L.p, 1. / unsurz) + R.a / pow(R.p, 1. / unsurz)),
                      unsurz);
    double ppv = fmax(kErrTol, ppv0), ptr = fmax(kErrTol, ptr0);
    double GL = sqrt(AL / (ppv + BL)), GR = sqrt(AR / (ppv + BR));
    double pts = fmax(kErrTol, (GL * L.p + GR * R.p - (R.u - L.u)) / (GL + GR));
    double p, u2;
    if (((pmax / pmin) < 2.0) && ((pmin <= ppv) && (ppv <= pmax))) p = ppv;
    else if (ppv < pmin) p = ptr;
    else p = pts;
    for (int i = 0; i < kNiterMax; i++) {
      double dp = froot(p, L, R, &u2) / froot_prime(p, L, R);
      if (isnan(dp)) { st |= kStNan; break; }
      if (fabs(dp) < kErrTol) break;
      for (int h = 0; h < 1100 && (p - dp) < 0; h++) dp = dp * 0.5;  // bounded halving
      double porg = p;
      p = p - dp;
      double err = 2. * fabs(p - porg) / (fabs(p + porg));
      if (err < kErrTol) break;
      if (froot(p, L, R, &u2) < kErrTol) break;
    }
    froot(p, L, R, &u2);
    *u = u2;
    return p;
  }

  // Two-rarefaction star state of findPressure_Hybrid (src/hydro_utils.c:645-650),
  // {p*, u*}.  Not inlined: its pow() expansions would otherwise be repeated in
  // every copy of the Riemann solver and crowd the instruction cache.
  static __device__ __noinline__ double2 trrs(double aL, double aR, double uL, double uR, double pL, double pR) {
    const double z = (kGam - 1.) / (2. * kGam);
    const double iz = (2. * kGam) / (kGam - 1.);
    const double pstar = pow((aL + aR - (kGam - 1.) / 2. * (uR - uL)) / (aL / pow(pL, z) + aR / pow(pR, z)), iz);
    const double ustar = uL - 2. * aL / (kGam - 1.) * (pow(pstar / pL, z) - 1.);
    return make_double2(pstar, ustar);
  }

  // findPressure_Hybrid + speedestimate*_HLLC (src/hydro_utils.c:625,1264)
  static __device__ __forceinline__ void speeds(const double WL[7], const double WR[7], int n, double &SL, double &SR,
                                                double &ustar, unsigned &st) {
    const double uLn = (n == 0) ? WL[1] : ((n == 1) ? WL[2] : WL[3]);
    const double uRn = (n == 0) ? WR[1] : ((n == 1) ? WR[2] : WR[3]);
    S1 L{WL[0], uLn, WL[4], sqrt(kGam * WL[4] / WL[0])};
    S1 R{WR[0], uRn, WR[4], sqrt(kGam * WR[4] / WR[0])};
    double dbar = 0.5 * (L.d + R.d), abar = 0.5 * (L.a + R.a);
    double ppvrs = 0.5 * ((L.p + R.p) + (L.u - R.u) * dbar * abar);
    double pmax = fmax(L.p, R.p), pmin = fmin(L.p, R.p);
    double pstar = ppvrs;
    if (((pmax / pmin) < 2.) && ((pmin < pstar) && (pstar < pmax))) {
      ustar = 0.5 * ((L.u + R.u) + (L.p - R.p) / (dbar * abar));
    } else if (pstar < pmin) {
      const double2 r = trrs(L.a, R.a, L.u, R.u, L.p, R.p);
      pstar = r.x;
      ustar = r.y;
    } else {
      double p0 = fmax(0., ppvrs);
      double AL = 2. / ((kGam + 1.) * L.d), AR = 2. / ((kGam + 1.) * R.d);
      double BL = (kGam - 1.) / (kGam + 1.) * L.p, BR = (kGam - 1.) / (kGam + 1.) * R.p;
      double GL = sqrt(AL / (p0 + BL)), GR = sqrt(AR / (p0 + BR));
      pstar = (GL * L.p + GR * R.p - (R.u - L.u)) / (GL + GR);
      ustar = 0.5 * ((L.u + R.u) + (pstar - R.p) * GR - (pstar - L.p) * GL);
    }
    if (pstar < 0) pstar = pstar_exact(L, R, &ustar, st);
    if (pstar < 0) st |= kStNegPstar;
    double qL = (pstar <= WL[4] ? 1. : sqrt(1. + (kGam + 1.) / (2. * kGam) * ((pstar) / WL[4] - 1.)));
    double qR = (pstar <= WR[4] ? 1. : sqrt(1. + (kGam + 1.) / (2. * kGam) * ((pstar) / WR[4] - 1.)));
    SL = L.u - L.a * qL;
    SR = R.u + R.a * qR;
    if (SL > SR) {
      SL = fmin(L.u - L.a, R.u - R.a);
      SR = fmax(L.u + L.a, R.u + R.a);
    }
    if (isnan(ustar)) st |= kStNan;
  }

  // Face state toward face k from the slope along k's axis only (the other
  // axes enter the reference's sum with coefficient 0).
  // g (optional): the gravity kick -f dt/2 of the face velocities, added after
  // the pressure floor and before E and a (src/hydro_utils.c:1219-1226)
  static __device__ __forceinline__ void face_ax(const double q0[5], const double Dax[5], const double Wt[5], int k,
                                                 double W[7], unsigned &st, const double *g = nullptr) {
    const double f = (k & 1) ? 0.5 : -0.5;
#pragma unroll
    for (int i = 0; i < 5; i++) W[i] = q0[i] + f * Dax[i] + Wt[i];
    W[4] = fmax(W[4], kPmin);
    if (W[0] < 0) st |= kStNegDensity;
    if (g != nullptr) {
      W[1] += g[0];
      W[2] += g[1];
      W[3] += g[2];
    }
    face_finish(W);
  }

  // State rotated to the face frame: r = {d, u_n, u_t1, u_t2, p, E, |m|^2},
  // t1 < t2 the transverse axes in x,y,z order, |m|^2 summed in x,y,z order.
  static __device__ __forceinline__ void rotate(const double W[7], int n, double r[7]) {
    r[0] = W[0];
    r[1] = (n == 0) ? W[1] : ((n == 1) ? W[2] : W[3]);
    r[2] = (n == 0) ? W[2] : W[1];
    r[3] = (n == 2) ? W[2] : W[3];
    r[4] = W[4];
    r[5] = W[6];
    const double m0 = W[0] * W[1], m1 = W[0] * W[2], m2 = W[0] * W[3];
    r[6] = m0 * m0 + m1 * m1 + m2 * m2;
  }

  // getflux_{X,Y,Z} of W2U(W) (src/hydro_utils.c:66,916-968) in the face frame
  static __device__ __forceinline__ void euler_rot(const double r[7], double f[5]) {
    const double d = r[0], E = r[5];
    const double mn = d * r[1], mt1 = d * r[2], mt2 = d * r[3];
    f[0] = mn;
    f[1] = 0.5 * (3. - kGam) * mn * mn / d + (kGam - 1.) * E - 0.5 * (kGam - 1.) * (mt1 * mt1 + mt2 * mt2) / d;
    f[2] = mn * mt1 / d;
    f[3] = mn * mt2 / d;
    f[4] = kGam * mn / d * E - 0.5 * (kGam - 1.) * mn / (d * d) * r[6];
  }

  // HLLC flux across a face normal to axis n (src/hydro_utils.c:2055-2138),
  // returned in x,y,z order: F = {mass, mom_x, mom_y, mom_z, energy}.
  // du (dual-energy builds, optional): from the state Us of the branch taken (the
  // upwind or the star state), du[0] = Us.m_n / Us.d and du[1] = ebar =
  // Us.E - |Us.m|^2 / (2 Us.d) (src/hydro_utils.c:2126-2128).
  // xs, fx (tracer builds, optional): the centre fractions of the NT tracers,
  // xs[2 t] left and xs[2 t + 1] right, and their fluxes fx[t].
  template <int NT = 1>
  static __device__ __forceinline__ void hllc(const double WL[7], const double WR[7], int n, double F[5],
                                              unsigned &st, double *du = nullptr, const double *xs = nullptr,
                                              double *fx = nullptr) {
    double SL, SR, ustar;
    speeds(WL, WR, n, SL, SR, ustar, st);
    double rL[7], rR[7], G[5] = {0., 0., 0., 0., 0.};
    rotate(WL, n, rL);
    rotate(WR, n, rR);
    if (du != nullptr) du[0] = du[1] = 0.;
    if (fx != nullptr)
      for (int t = 0; t < NT; t++) fx[t] = 0.;
    if (SL >= 0. || SR <= 0.) {
      const double *r = (SL >= 0.) ? rL : rR;
      euler_rot(r, G);
      if (du != nullptr) {  // Us = W2U of the upwind face state
        const double mn = r[0] * r[1];
        du[0] = mn / r[0];
        du[1] = (r[5] - 0.5 * r[6] / r[0]);
      }
      if (fx != nullptr)  // tracers: face values from the centre fractions, flux du dT / d
        for (int t = 0; t < NT; t++) {
          const double dT = (r[0] * Tracers<NT>::frac(t)) * xs[2 * t + ((SL >= 0.) ? 0 : 1)];
          fx[t] = (r[0] * r[1]) * dT / r[0];
        }
    } else {
      const bool left = (SL < 0.) && (ustar >= 0.);
      const bool right = (ustar <= 0.) && (SR > 0.);
      if (left || right) {
        const double *r = left ? rL : rR;
        const double S = left ? SL : SR;
        euler_rot(r, G);
        const double d = r[0], un = r[1], E = r[5];
        const double fact = d * (S - un) / (S - ustar);
        const double Es = (E / d + (ustar - un) * (ustar + r[4] / (d * (S - un))));
        G[0] += (fact * 1. - d) * S;
        G[1] += (fact * ustar - d * un) * S;
        G[2] += (fact * r[2] - d * r[2]) * S;
        G[3] += (fact * r[3] - d * r[3]) * S;
        G[4] += (fact * Es - E) * S;
        if (fx != nullptr)  // tracer fluxes with the star correction (src/hydro_utils.c:1534-1539)
          for (int t = 0; t < NT; t++) {
            const double dT = (d * Tracers<NT>::frac(t)) * xs[2 * t + (left ? 0 : 1)];
            fx[t] = (d * un) * dT / d + (fact * dT / d - dT) * S;
          }
        if (du != nullptr) {  // the star state: momenta in x,y,z order for the sum of squares
          const double ds = fact * 1., mn = fact * ustar, m1 = fact * r[2], m2 = fact * r[3];
          const double mm = (n == 2) ? ((m1 * m1 + m2 * m2) + mn * mn) : ((mn * mn + m1 * m1) + m2 * m2);
          du[0] = mn / ds;
          du[1] = (fact * Es - 0.5 * mm / ds);
        }
      }
    }
    F[0] = G[0];
    F[1] = (n == 0) ? G[1] : G[2];
    F[2] = (n == 0) ? G[2] : ((n == 1) ? G[1] : G[3]);
    F[3] = (n == 2) ? G[1] : G[3];
    F[4] = G[4];
  }
};

// ============================================================== FP32 (mixed)
struct MathF32 {
  using R = float;
  static constexpr float G = 5.f / 3.f;

  // approximate reciprocal / division (built with -use_fast_math: single MUFU ops)
  static __device__ __forceinline__ float rcp(float x) { return __fdividef(1.f, x); }
  static __device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

  static __device__ __forceinline__ float limit(float m, float p) {
    // minmod with beta = 1: 0 if signs differ, else the smaller magnitude, as the
    // median of (0, m, p): four min/max operations, no compare
    return fmaxf(fminf(m, p), fminf(fmaxf(m, p), 0.f));
  }

  static __device__ __forceinline__ void muscl(const float q0[5], const float qm[3][5], const float qp[3][5],
                                               float dtdx_half, float D[3][5], float Wt[5], bool azero = false) {
#pragma unroll
    for (int dir = 0; dir < 3; dir++)
#pragma unroll
      for (int k = 0; k < 5; k++) D[dir][k] = limit(q0[k] - qm[dir][k], qp[dir][k] - q0[k]);
    const float id = rcp(q0[0]);
    const float gp = azero ? 0.f : G * q0[4];  // d a^2
    float acc0 = q0[1] * D[0][0] + q0[0] * D[0][1] + q0[2] * D[1][0] + q0[0] * D[1][2] + q0[3] * D[2][0] + q0[0] * D[2][3];
    float acc1 = q0[1] * D[0][1] + id * D[0][4] + q0[2] * D[1][1] + q0[3] * D[2][1];
    float acc2 = q0[1] * D[0][2] + q0[2] * D[1][2] + id * D[1][4] + q0[3] * D[2][2];
    float acc3 = q0[1] * D[0][3] + q0[2] * D[1][3] + q0[3] * D[2][3] + id * D[2][4];
    float acc4 = gp * (D[0][1] + D[1][2] + D[2][3]) + q0[1] * D[0][4] + q0[2] * D[1][4] + q0[3] * D[2][4];
    Wt[0] = -dtdx_half * acc0;
    Wt[1] = -dtdx_half * acc1;
    Wt[2] = -dtdx_half * acc2;
    Wt[3] = -dtdx_half * acc3;
    Wt[4] = -dtdx_half * acc4;
  }

  // Face state toward face k from the predicted centre state X = W0 + Wt.
  static __device__ __forceinline__ void face_px(const float X[5], const float Dax[5], int k, float W[7],
                                                 unsigned &st) {
    const float s = (k & 1) ? 0.5f : -0.5f;
#pragma unroll
    for (int i = 0; i < 5; i++) W[i] = __fmaf_rn(s, Dax[i], X[i]);  // explicit: same rounding at every call site
    W[4] = fmaxf(W[4], (float)kPmin);
    if (W[0] < 0.f) st |= kStNegDensity;
    W[5] = rcp(W[0]);
    W[6] = sqrtf(G * W[4] * W[5]);
  }

  static __device__ __forceinline__ float pstar_exact(float dL, float uL, float pL, float aL, float dR, float uR,
                                                   float pR, float aR, float *u) {
    // Newton iteration on the exact two-rarefaction/shock function (Toro sec. 4.3)
    const float g1 = (G - 1.f) / (2.f * G), g2 = (G + 1.f) / (2.f * G);
    const float AL = 2.f / ((G + 1.f) * dL), AR = 2.f / ((G + 1.f) * dR);
    const float BL = (G - 1.f) / (G + 1.f) * pL, BR = (G - 1.f) / (G + 1.f) * pR;
    float p = fmaxf(1e-10f, 0.5f * (pL + pR) - 0.125f * (uR - uL) * (dL + dR) * (aL + aR));
    float fL = 0.f, fR = 0.f;
    for (int i = 0; i < kNiterMax; i++) {
      float dfL, dfR;
      if (p > pL) { float q = sqrtf(AL / (BL + p)); fL = (p - pL) * q; dfL = q * (1.f - (p - pL) / (2.f * (BL + p))); }
      else { float r = __powf(p / pL, g1); fL = 2.f * aL / (G - 1.f) * (r - 1.f); dfL = __powf(p / pL, -g2) / (dL * aL); }
      if (p > pR) { float q = sqrtf(AR / (BR + p)); fR = (p - pR) * q; dfR = q * (1.f - (p - pR) / (2.f * (BR + p))); }
      else { float r = __powf(p / pR, g1); fR = 2.f * aR / (G - 1.f) * (r - 1.f); dfR = __powf(p / pR, -g2) / (dR * aR); }
      float dp = (fL + fR + (uR - uL)) / (dfL + dfR);
      if (!(fabsf(dp) >= 1e-10f)) break;
      for (int h = 0; h < 200 && (p - dp) < 0.f; h++) dp *= 0.5f;
      float porg = p;
      p -= dp;
      if (2.f * fabsf(p - porg) / fabsf(p + porg) < 1e-7f) break;
    }
    *u = 0.5f * (uL + uR) + 0.5f * (fR - fL);
    return p;
  }

  // HLLC flux across a face normal to axis n; states W = {d,u,v,w,p,1/d,a}.
  // du (dual-energy builds, optional): the upwind or star state's normal velocity
  // and ebar = Us.E - |Us.m|^2 / (2 Us.d), the latter in a form free of the
  // E - Ekin cancellation: p/(g-1) upwind, fact (p/((g-1) d) + (u*-u)((u*-u)/2 +
  // p/(d (S-u)))) in the star region (algebraically the reference's expression).
  template <int NT = 1>
  static __device__ __forceinline__ void hllc(const float WL[7], const float WR[7], int n, float F[5], unsigned &st,
                                              float *du = nullptr, const float *xs = nullptr, float *fx = nullptr) {
    const float dL = WL[0], pL = WL[4], aL = WL[6];
    const float dR = WR[0], pR = WR[4], aR = WR[6];
    const float uL = (n == 0) ? WL[1] : ((n == 1) ? WL[2] : WL[3]);
    const float uR = (n == 0) ? WR[1] : ((n == 1) ? WR[2] : WR[3]);
    // hybrid PVRS / TRRS / TSRS star pressure (Toro sec. 9.5.2), as the reference.
    // The three estimates are evaluated without branches and one is selected: a
    // warp whose faces need different ones pays for each of them either way (and
    // for the divergence), here without the branch bookkeeping.
    const float dbar = 0.5f * (dL + dR), abar = 0.5f * (aL + aR);
    const float ppvrs = 0.5f * ((pL + pR) + (uL - uR) * dbar * abar);
    const float pmax = fmaxf(pL, pR), pmin = fminf(pL, pR);
    const bool use_pvrs = (pmax < 2.f * pmin) && (pmin < ppvrs) && (ppvrs < pmax);
    const bool use_trrs = !use_pvrs && (ppvrs < pmin);
    const float u_pv = 0.5f * ((uL + uR) + fdiv(pL - pR, dbar * abar));
    // two rarefactions: p* = (num/den)^(1/z), and (p*/pL)^z = (num/den) pL^-z;
    // 1/z = 2G/(G-1) = 5 for G = 5/3: the fifth power by three multiplications
    // (a negative ratio, a vacuum-generating pair, then gives a negative p* and the
    // exact solver, as the reference's pow() with its integer exponent does)
    constexpr float z = (G - 1.f) / (2.f * G);
    static_assert(2.f * G / (G - 1.f) == 5.f, "p* = ratio^5 needs G = 5/3");
    const float num = aL + aR - (G - 1.f) * 0.5f * (uR - uL);
    const float pLz = __powf(pL, -z), pRz = __powf(pR, -z);
    const float ratio = fdiv(num, aL * pLz + aR * pRz);
    const float r2 = ratio * ratio;
    const float p_tr = r2 * r2 * ratio;
    const float u_tr = uL - 2.f * aL / (G - 1.f) * (ratio * pLz - 1.f);
    // two shocks: g = sqrt(A / (p0 + B)) with A = 2 / ((G + 1) d), one rsqrt a side
    const float p0 = fmaxf(0.f, ppvrs);
    const float BL = (G - 1.f) / (G + 1.f) * pL, BR = (G - 1.f) / (G + 1.f) * pR;
    const float c2 = 0.8660254037844386f;  // sqrt(2 / (G + 1)) for G = 5/3
    static_assert(G == 5.f / 3.f, "c2 is sqrt(2 / (G + 1))");
    const float GL = c2 * rsqrtf(dL * (p0 + BL)), GR = c2 * rsqrtf(dR * (p0 + BR));
    const float p_ts = fdiv(GL * pL + GR * pR - (uR - uL), GL + GR);
    const float u_ts = 0.5f * ((uL + uR) + (p_ts - pR) * GR - (p_ts - pL) * GL);
    float pstar = use_pvrs ? ppvrs : (use_trrs ? p_tr : p_ts);
    float ustar = use_pvrs ? u_pv : (use_trrs ? u_tr : u_ts);
    if (pstar < 0.f) pstar = pstar_exact(dL, uL, pL, aL, dR, uR, pR, aR, &ustar);
    if (pstar < 0.f) st |= kStNegPstar;
    const float g2 = (G + 1.f) / (2.f * G);
    // shock factors sqrt(1 + g2 (p*/p - 1)) = sqrt(x / p) = x rsqrt(x p), x = p + g2 (p* - p)
    const float xL = pL + g2 * (pstar - pL), xR = pR + g2 * (pstar - pR);
    const float qL = (pstar <= pL) ? 1.f : xL * rsqrtf(xL * pL);
    const float qR = (pstar <= pR) ? 1.f : xR * rsqrtf(xR * pR);
    float SL = uL - aL * qL, SR = uR + aR * qR;
    if (SL > SR) {
      SL = fminf(uL - aL, uR - aR);
      SR = fmaxf(uL + aL, uR + aR);
    }
    if (isnan(ustar)) st |= kStNan;
    // upwind side and its rotated state
    const bool useL = (SL >= 0.f) || (!(SR <= 0.f) && (ustar >= 0.f));
    const float *W = useL ? WL : WR;
    const float d = W[0], p = W[4], id = W[5];
    const float un = useL ? uL : uR;
    const float t1 = (n == 0) ? W[2] : W[1];
    const float t2 = (n == 2) ? W[2] : W[3];
    const float E = p * (1.f / (G - 1.f)) + 0.5f * d * (un * un + t1 * t1 + t2 * t2);
    const float mn = d * un;
    float G0 = mn, GN = mn * un + p, G1 = mn * t1, G2 = mn * t2, G4 = un * (E + p);
    // star-region correction, evaluated without branches and selected: inside the
    // star region (SL < 0 < SR) the side condition holds for every non-NaN u*
    const bool star = !(SL >= 0.f || SR <= 0.f);
    const bool side = (SL < 0.f && ustar >= 0.f) || (ustar <= 0.f && SR > 0.f);
    const float S = useL ? SL : SR;
    const float Smu = S - un;
    const float fact = fdiv(d * Smu, S - ustar);
    const float H0 = G0 + (fact - d) * S;
    const float HN = GN + (fact * ustar - mn) * S;
    const float H1 = G1 + (fact - d) * t1 * S;
    const float H2 = G2 + (fact - d) * t2 * S;
    const float H4 = G4 + (fact * (E * id + (ustar - un) * (ustar + fdiv(p, d * Smu))) - E) * S;
    if (star) {
      G0 = side ? H0 : 0.f;
      GN = side ? HN : 0.f;
      G1 = side ? H1 : 0.f;
      G2 = side ? H2 : 0.f;
      G4 = side ? H4 : 0.f;
    }
    if (fx != nullptr)  // tracers: face values from the centre fractions, flux du dT / d (+ star correction)
      for (int t = 0; t < NT; t++) {
        const float dT = d * (float)Tracers<NT>::frac(t) * xs[2 * t + (useL ? 0 : 1)];
        const float f6 = mn * dT * id;
        const float h6 = f6 + (fact * dT * id - dT) * S;
        fx[t] = star ? (side ? h6 : 0.f) : f6;
      }
    if (du != nullptr) {
      const float ig = 1.f / (G - 1.f), dd = ustar - un;
      const float es = fact * (p * ig * id + dd * (0.5f * dd + fdiv(p, d * Smu)));
      du[0] = star ? (side ? ustar : 0.f) : un;
      du[1] = star ? (side ? es : 0.f) : p * ig;
    }
    F[0] = G0;
    F[1] = (n == 0) ? GN : G1;
    F[2] = (n == 0) ? G1 : ((n == 1) ? GN : G2);
    F[3] = (n == 2) ? GN : G2;
    F[4] = G4;
  }
};

}  // namespace emma
