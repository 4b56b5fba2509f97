// Pointwise physics of the nodal-DG right-hand side, shared by host and device:
// the equation plugins' flux, Lax-Friedrichs numerical flux and Riemann wave
// speeds, and the boundary-condition plugins.  Each function states the
// Apollo plugin hook it computes; the arithmetic follows that hook operation
// by operation so that float64 results agree to round-off.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define APOLLO_HD __host__ __device__ __forceinline__
#else
#define APOLLO_HD inline
#endif

namespace apollo {

enum EqKind : int {
  EQ_ADVECTION = 0,  // advectionEqn, 1 field
  EQ_EULER = 1,      // eulerEqn, 5 fields
  EQ_MAXWELL = 2,    // phMaxwellEqn, 8 fields
  EQ_EULER2D = 3,    // eulerEqn restricted to rho w = 0, 4 fields
  EQ_MAXWELL_TM = 4  // phMaxwellEqn restricted to (Ez, Bx, By) with chi = gamma = 0, 3 fields
};

enum BcKind : int {
  BC_FIXED = 0, BC_VORTEX = 1, BC_TM = 2, BC_PEC = 3,
  BC_EULER_WALL = 4,      // eulerWallBC
  BC_EULER_ZEROGRAD = 5,  // eulerZeroGradientBC
  BC_EULER_STATE = 6      // eulerInflowBC / eulerDirichletBC: a constant ghost state, p = (rho, rhou, rhov, rhow, E)
};

// Euler numerical fluxes by Apollo's Numerical_Flux codes (wxeulereqn.cc:10-15);
// stored in EqParams::p[3] of the Euler kinds
// Numerical fluxes: Apollo's Euler Numerical_Flux codes (wxeulereqn.cc:10-15);
// NF_UPWIND is an extension for advection (dissipation |n.u| instead of
// Apollo's max(|ux|, |uy|)) and for the planar Maxwell TM form (no
// dissipation on the normal magnetic field, whose wave speed is 0), held in
// the equation parameters' slot 3
enum NumFlux : int { NF_LF = 0, NF_HLL = 1, NF_ROE = 2, NF_WAVE = 4, NF_UPWIND = 8 };

enum ErrBits : int { ERRB_NONPHYS = 1, ERRB_NAN = 2, ERRB_TIMEOUT = 4 };

constexpr int kMaxBc = 8;

struct EqParams {
  double p[4];  // advection: ux uy uz; Euler: gamma minP minD; Maxwell: c0 gamma chi
};

struct BcTable {
  int n;
  int kind[kMaxBc];
  double p[kMaxBc][8];
};

template <int EQ> struct Eq;

APOLLO_HD double dmax2(double a, double b) { return a > b ? a : b; }
// |x| after conversion to int (truncation toward zero).  Apollo's HLL flux
// calls abs() on a double where only int abs(int) is declared
// (wxeulereqn.cc:1170), so its wave-speed bound |S_R| enters truncated;
// reproduced for |x| < 2^31.
APOLLO_HD double abs_int(double x) { return (double)abs((int)x); }
APOLLO_HD float abs_int(float x) { return (float)abs((int)x); }
APOLLO_HD double dmax3(double a, double b, double c) {
  double m1 = a > b ? a : b;
  return m1 > c ? m1 : c;
}

// ------------------------------------------------------------ advection ----
// WxAdvectionEqn: flux wxadvectioneqn.cc:176-185, DGnumericalFlux :189-208,
// rp wave speeds :35-66.
template <> struct Eq<EQ_ADVECTION> {
  static constexpr int M = 1;
  template <class T>
  APOLLO_HD static void flux2(const EqParams& P, const T* q, T* F, T* G, int* err) {
    F[0] = T(P.p[0]) * q[0];
    G[0] = T(P.p[1]) * q[0];
  }
  template <class T>
  APOLLO_HD static T numflux(const EqParams& P, T nx, T ny, T* qM, T* qP, T* nf, int* err) {
    T fM[1], fP[1], gM[1], gP[1];
    flux2(P, qM, fM, gM, err);
    flux2(P, qP, fP, gP, err);
    T lambda = T(dmax2(fabs(P.p[0]), fabs(P.p[1])));
    // the upwind extension dissipates with the normal speed; the returned
    // speed (the dt policy's) stays Apollo's
    const T diss = (int)P.p[3] == NF_UPWIND ? fabs(nx * T(P.p[0]) + ny * T(P.p[1])) : lambda;
    nf[0] = T(0.5) * (nx * (fM[0] + fP[0]) + ny * (gM[0] + gP[0]) + diss * (qM[0] - qP[0]));
    return lambda;
  }
  APOLLO_HD static double speed2(const EqParams& P, const double* q) {
    return dmax3(0.0, P.p[0] * P.p[0], P.p[1] * P.p[1]);
  }
  // the Lax-Friedrichs speed of numflux, in float64
  APOLLO_HD static double lf_lambda(const EqParams& P, const double* qM, const double* qP) {
    return dmax2(fabs(P.p[0]), fabs(P.p[1]));
  }
};

// ---------------------------------------------------------------- Euler ----
// WxEulerEqn: flux wxeulereqn.cc:809-871, primitiveVariables :1326-1341,
// Lax-Friedrichs :1097-1117, Roe-averaged speeds of rp :145-235.
template <int MF>
struct EulerBase {
  static constexpr int M = MF;
  static constexpr int IE = MF - 1;  // energy index (4 for 5 fields, 3 for 4 fields)
  template <class T>
  APOLLO_HD static void flux_dir(const EqParams& P, int d, const T* q, T* f, int* err) {
    T gamma1 = T(P.p[0]) - T(1.0);
    T minP = T(P.p[1]), minD = T(P.p[2]);
    T rho = q[0];
    if (minD == T(0) && rho <= T(0)) *err |= ERRB_NONPHYS;
    if (rho < minD) rho = minD;
    T qu = d == 0 ? q[1] : q[2];
    T qv = d == 0 ? q[2] : (MF == 5 ? q[3] : T(0));
    T qw = d == 0 ? (MF == 5 ? q[3] : T(0)) : q[1];
    T u = qu / rho, v = qv / rho, w = qw / rho, E = q[IE];
    T p = gamma1 * (E - T(0.5) * rho * (u * u + v * v + w * w));
    if (p <= T(0)) {
      if (minP == T(0)) *err |= ERRB_NONPHYS;
      else p = minP;
    }
    f[0] = rho * u;
    T fu = rho * u * u + p, fv = rho * u * v, fw = rho * u * w;
    if (d == 0) {
      f[1] = fu; f[2] = fv;
      if (MF == 5) f[3] = fw;
    } else {
      f[2] = fu; f[1] = fw;
      if (MF == 5) f[3] = fv;
    }
    f[IE] = (E + p) * u;
  }
  template <class T>
  APOLLO_HD static void flux2(const EqParams& P, const T* q, T* F, T* G, int* err) {
    flux_dir(P, 0, q, F, err);
    flux_dir(P, 1, q, G, err);
  }
  template <class T>
  APOLLO_HD static void prim(const EqParams& P, T* qc, T* qp) {
    T gamma = T(P.p[0]), minP = T(P.p[1]), minD = T(P.p[2]);
    qp[0] = qc[0];
    if (qp[0] <= T(0)) { qc[0] = minD; qp[0] = minD; }
    T q3 = MF == 5 ? qc[3] : T(0);
    qp[1] = qc[1] / qc[0];
    qp[2] = qc[2] / qc[0];
    qp[3] = q3 / qc[0];
    qp[4] = (gamma - T(1.)) * (qc[IE] - T(0.5) * (qc[1] * qc[1] + qc[2] * qc[2] + q3 * q3) / qc[0]);
    if (qp[4] <= T(0.)) {
      qp[4] = minP;
      qc[IE] = minP / (gamma - T(1.)) + T(0.5) * qp[0] * (qp[1] * qp[1] + qp[2] * qp[2] + qp[3] * qp[3]);
    }
  }
  // DGnumericalFlux by the Numerical_Flux code in P.p[3] (wxeulereqn.cc:876-893).
  // qM and qP are modified as the reference modifies them (primitive-variable
  // floors, the rotation of HLL, Roe and Wave).
  template <class T>
  APOLLO_HD static T numflux(const EqParams& P, T nx, T ny, T* qM, T* qP, T* nf, int* err) {
    const int kind = (int)P.p[3];
    if (kind == NF_HLL) return hll(P, nx, ny, qM, qP, nf, err);
    if (kind == NF_ROE) return roe(P, nx, ny, qM, qP, nf, err);
    // case 4 (Wave) falls through to the Lax-Friedrichs flux (:888-892): what
    // remains of the wave-propagation flux is its effect on the traces
    if (kind == NF_WAVE) wave_prelude(P, nx, ny, qM, qP, err);
    return lf(P, nx, ny, qM, qP, nf, err);
  }
  // Lax-Friedrichs (:1097-1117)
  template <class T>
  APOLLO_HD static T lf(const EqParams& P, T nx, T ny, T* qM, T* qP, T* nf, int* err) {
    T fM[MF], fP[MF], gM[MF], gP[MF], pM[5], pP[5];
    flux2(P, qM, fM, gM, err);
    flux2(P, qP, fP, gP, err);
    prim(P, qM, pM);
    prim(P, qP, pP);
    T gamma = T(P.p[0]);
    T c0M = sqrt(pM[1] * pM[1] + pM[2] * pM[2] + pM[3] * pM[3]) + sqrt(gamma * pM[4] / pM[0]);
    T c0P = sqrt(pP[1] * pP[1] + pP[2] * pP[2] + pP[3] * pP[3]) + sqrt(gamma * pP[4] / pP[0]);
    T lambda = c0M > c0P ? c0M : c0P;
#pragma unroll
    for (int c = 0; c < MF; ++c)
      nf[c] = T(0.5) * (nx * (fM[c] + fP[c]) + ny * (gM[c] + gP[c]) + lambda * (qM[c] - qP[c]));
    return lambda;
  }
  // momentum into the face's normal-tangent frame, in place
  template <class T>
  APOLLO_HD static void rotate_in(T nx, T ny, T* q) {
    T ru = q[1], rv = q[2];
    q[1] = nx * ru + ny * rv;
    q[2] = -ny * ru + nx * rv;
  }
  template <class T>
  APOLLO_HD static T max_speed(const EqParams& P, const T* pM, const T* pP) {
    T gamma = T(P.p[0]);
    T c0M = sqrt(pM[1] * pM[1] + pM[2] * pM[2] + pM[3] * pM[3]) + sqrt(gamma * pM[4] / pM[0]);
    T c0P = sqrt(pP[1] * pP[1] + pP[2] * pP[2] + pP[3] * pP[3]) + sqrt(gamma * pP[4] / pP[0]);
    return c0M > c0P ? c0M : c0P;
  }
  // Roe-averaged velocity and enthalpy of the rotated, floored traces
  template <class T>
  APOLLO_HD static void roe_avg(const EqParams& P, const T* qM, const T* qP, const T* pM, const T* pP, T& rMs,
                                T& rPs, T& u, T& v, T& w, T& H) {
    T HM = (qM[IE] + pM[4]) / pM[0];
    T HP = (qP[IE] + pP[4]) / pP[0];
    rMs = sqrt(pM[0]);
    rPs = sqrt(pP[0]);
    u = (rMs * pM[1] + rPs * pP[1]) / (rMs + rPs);
    v = (rMs * pM[2] + rPs * pP[2]) / (rMs + rPs);
    w = (rMs * pM[3] + rPs * pP[3]) / (rMs + rPs);
    H = (rMs * HM + rPs * HP) / (rMs + rPs);
  }
  // HLL (:1121-1202), with the reference's truncated |S_R| (abs_int)
  template <class T>
  APOLLO_HD static T hll(const EqParams& P, T nx, T ny, T* qM, T* qP, T* nf, int* err) {
    T fM[MF], fP[MF], gM[MF], gP[MF], pM[5], pP[5], fx[MF];
    rotate_in(nx, ny, qM);
    rotate_in(nx, ny, qP);
    flux2(P, qM, fM, gM, err);  // the y fluxes are evaluated (and checked), not used
    flux2(P, qP, fP, gP, err);
    prim(P, qM, pM);
    prim(P, qP, pP);
    const T gamma = T(P.p[0]);
    const T cM = sqrt(gamma * pM[4] / pM[0]), cP = sqrt(gamma * pP[4] / pP[0]);
    T rMs, rPs, u, v, w, H;
    roe_avg(P, qM, qP, pM, pP, rMs, rPs, u, v, w, H);
    const T c2 = (gamma - T(1.)) * (H - T(0.5) * (u * u + v * v + w * w)), c = sqrt(c2);
    T a = pM[1] - cM, b = u - c;
    const T SL = a < b ? a : b;
    a = pP[1] + cP;
    b = u + c;
    const T SR = a > b ? a : b;
    const T zero = T(0.0);
    const T t1 = ((SR < zero ? SR : zero) - (zero < SL ? zero : SL)) / (SR - SL);
    const T t2 = T(1.) - t1;
    const T t3 = (SR * fabs(SL) - SL * abs_int(SR)) / (T(2.) * (SR - SL));
#pragma unroll
    for (int n = 0; n < MF; ++n) fx[n] = t1 * fP[n] + t2 * fM[n] - t3 * (qP[n] - qM[n]);
    nf[0] = fx[0];
    nf[1] = nx * fx[1] - ny * fx[2];
    nf[2] = ny * fx[1] + nx * fx[2];
    if (MF == 5) nf[3] = T(0.0);
    nf[IE] = fx[IE];
    return max_speed(P, pM, pP);
  }
  // Roe (:1206-1275).  The reference assigns nflux[1] twice (:1267-1268), the
  // second time with the y-momentum flux, and never sets nflux[2]: its
  // zero-initialised flux buffer (wxnodaldg2dmethod.cc:98) keeps 0 there.
  template <class T>
  APOLLO_HD static T roe(const EqParams& P, T nx, T ny, T* qM, T* qP, T* nf, int* err) {
    T fM[MF], fP[MF], pM[5], pP[5], fx[MF];
    rotate_in(nx, ny, qM);
    rotate_in(nx, ny, qP);
    prim(P, qM, pM);
    prim(P, qP, pP);
    const T gamma = T(P.p[0]);
    T rMs, rPs, u, v, w, H;
    roe_avg(P, qM, qP, pM, pP, rMs, rPs, u, v, w, H);
    const T rho = rMs * rPs;
    const T c2 = (gamma - T(1.)) * (H - T(0.5) * (u * u + v * v + w * w)), c = sqrt(c2);
    T dw1 = T(-0.5) * rho * (pP[1] - pM[1]) / c + T(0.5) * (pP[4] - pM[4]) / c2;
    T dw2 = (pP[0] - pM[0]) - (pP[4] - pM[4]) / c2;
    T dw3 = rho * (pP[2] - pM[2]);
    T dw4 = T(0.5) * rho * (pP[1] - pM[1]) / c + T(0.5) * (pP[4] - pM[4]) / c2;
    dw1 = fabs(u - c) * dw1;
    dw2 = fabs(u) * dw2;
    dw3 = fabs(u) * dw3;
    dw4 = fabs(u + c) * dw4;
    flux_dir(P, 0, qM, fM, err);
    flux_dir(P, 0, qP, fP, err);
#pragma unroll
    for (int n = 0; n < MF; ++n) fx[n] = T(0.5) * (fM[n] + fP[n]);
    fx[0] = fx[0] - T(0.5) * (dw1 * T(1.) + dw2 * T(1.) + dw3 * T(0.) + dw4 * T(1.));
    fx[1] = fx[1] - T(0.5) * (dw1 * (u - c) + dw2 * u + dw3 * T(0.) + dw4 * (u + c));
    fx[2] = fx[2] - T(0.5) * (dw1 * v + dw2 * v + dw3 * T(1.) + dw4 * v);
    fx[IE] = fx[IE] - T(0.5) * (dw1 * (H - u * c) + dw2 * (u * u + v * v) / T(2.) + dw3 * v + dw4 * (H + u * c));
    nf[0] = fx[0];
    nf[1] = ny * fx[1] + nx * fx[2];
    nf[2] = T(0.0);
    if (MF == 5) nf[3] = T(0.0);
    nf[IE] = fx[IE];
    return max_speed(P, pM, pP);
  }
  // The part of the wave-propagation flux (:1279-1322) that outlives the
  // fall-through: the traces rotated in place, the x fluxes' checks, and the
  // Riemann solver rp(0, ql = qP, qr = qM) (:94-235) with its checks and
  // pressure floor on the traces' energies.
  template <class T>
  APOLLO_HD static void wave_prelude(const EqParams& P, T nx, T ny, T* qM, T* qP, int* err) {
    T fM[MF], fP[MF];
    rotate_in(nx, ny, qM);
    rotate_in(nx, ny, qP);
    flux_dir(P, 0, qM, fM, err);
    flux_dir(P, 0, qP, fP, err);
    T* ql = qP;
    T* qr = qM;
    if (ql[0] < T(0) || qr[0] < T(0)) {
      *err |= ERRB_NONPHYS;
      return;
    }
    const T g1 = T(P.p[0]) - T(1), minP = T(P.p[1]);
    const T l3 = MF == 5 ? ql[3] : T(0), r3 = MF == 5 ? qr[3] : T(0);
    const T rl = sqrt(ql[0]), rr = sqrt(qr[0]);
    T pl = g1 * (ql[IE] - T(0.5) * (ql[1] * ql[1] + ql[2] * ql[2] + l3 * l3) / ql[0]);
    T pr = g1 * (qr[IE] - T(0.5) * (qr[1] * qr[1] + qr[2] * qr[2] + r3 * r3) / qr[0]);
    if (minP == T(0) && (pl < T(0) || pr < T(0))) *err |= ERRB_NONPHYS;
    if (pl < minP) {
      ql[IE] = minP / (T(P.p[0]) - T(1)) + T(0.5) * (ql[1] * ql[1] + ql[2] * ql[2] + l3 * l3) / ql[0];
      pl = minP;
    }
    if (pr < minP) {
      qr[IE] = minP / (T(P.p[0]) - T(1)) + T(0.5) * (qr[1] * qr[1] + qr[2] * qr[2] + r3 * r3) / qr[0];
      pr = minP;
    }
    const T rsq2 = rl + rr;
    const T u = (ql[1] / rl + qr[1] / rr) / rsq2;
    const T v = (ql[2] / rl + qr[2] / rr) / rsq2;
    const T w = (l3 / rl + r3 / rr) / rsq2;
    const T enth = ((ql[IE] + pl) / rl + (qr[IE] + pr) / rr) / rsq2;
    if (g1 * (enth - T(0.5) * (u * u + v * v + w * w)) < T(0)) *err |= ERRB_NONPHYS;
  }
  APOLLO_HD static double lf_lambda(const EqParams& P, const double* qM, const double* qP) {
    double a[MF], b[MF], pM[5], pP[5];
    for (int c = 0; c < MF; ++c) { a[c] = qM[c]; b[c] = qP[c]; }
    prim(P, a, pM);
    prim(P, b, pP);
    const double gamma = P.p[0];
    const double c0M = sqrt(pM[1] * pM[1] + pM[2] * pM[2] + pM[3] * pM[3]) + sqrt(gamma * pM[4] / pM[0]);
    const double c0P = sqrt(pP[1] * pP[1] + pP[2] * pP[2] + pP[3] * pP[3]) + sqrt(gamma * pP[4] / pP[0]);
    return c0M > c0P ? c0M : c0P;
  }
  // max over the Roe solver's waves (ql = qr = q) of max(sx^2, sy^2)
  APOLLO_HD static double speed2(const EqParams& P, const double* q) {
    double g1 = P.p[0] - 1.0, lam = 0.0;
    double q3 = MF == 5 ? q[3] : 0.0, E = q[IE];
    double s[2][3];
    for (int d = 0; d < 2; ++d) {
      double qmu = d == 0 ? q[1] : q[2];
      double qmv = d == 0 ? q[2] : q3;
      double qmw = d == 0 ? q3 : q[1];
      double rs = sqrt(q[0]);
      double p = g1 * (E - 0.5 * (qmu * qmu + qmv * qmv + qmw * qmw) / q[0]);
      double rsq2 = rs + rs;
      double u = (qmu / rs + qmu / rs) / rsq2;
      double v = (qmv / rs + qmv / rs) / rsq2;
      double w = (qmw / rs + qmw / rs) / rsq2;
      double u2 = u * u + v * v + w * w;
      double enth = ((E + p) / rs + (E + p) / rs) / rsq2;
      double a = sqrt(g1 * (enth - 0.5 * u2));
      s[d][0] = u - a; s[d][1] = u; s[d][2] = u + a;
    }
    for (int mw = 0; mw < 3; ++mw) lam = dmax3(lam, s[0][mw] * s[0][mw], s[1][mw] * s[1][mw]);
    return lam;
  }
};
template <> struct Eq<EQ_EULER> : EulerBase<5> {};
template <> struct Eq<EQ_EULER2D> : EulerBase<4> {};

// -------------------------------------------------------------- Maxwell ----
// WxPHMaxwellEqn: flux wxphmaxwelleqn.cc:450-498, DGnumericalFlux :503-522,
// wave speeds of rp (+-c0, +-c0 gamma, +-c0 chi).
template <> struct Eq<EQ_MAXWELL> {
  static constexpr int M = 8;
  template <class T>
  APOLLO_HD static void flux_dir(const EqParams& P, int d, const T* q, T* f) {
    T c0 = T(P.p[0]), gm = T(P.p[1]), chi = T(P.p[2]);
    int iex = 0, iey = 1, iez = 2, ibx = 3, iby = 4, ibz = 5;
    if (d == 1) { iex = 1; iey = 2; iez = 0; ibx = 4; iby = 5; ibz = 3; }
    f[iex] = chi * c0 * c0 * q[6];
    f[iey] = c0 * c0 * q[ibz];
    f[iez] = -c0 * c0 * q[iby];
    f[ibx] = gm * q[7];
    f[iby] = -q[iez];
    f[ibz] = q[iey];
    f[6] = chi * q[iex];
    f[7] = gm * c0 * c0 * q[ibx];
  }
  template <class T>
  APOLLO_HD static void flux2(const EqParams& P, const T* q, T* F, T* G, int* err) {
    flux_dir(P, 0, q, F);
    flux_dir(P, 1, q, G);
  }
  template <class T>
  APOLLO_HD static T numflux(const EqParams& P, T nx, T ny, T* qM, T* qP, T* nf, int* err) {
    T fM[8], fP[8], gM[8], gP[8];
    flux2(P, qM, fM, gM, err);
    flux2(P, qP, fP, gP, err);
    T lambda = T(dmax3(P.p[2] * P.p[0], P.p[1] * P.p[0], P.p[0]));
#pragma unroll
    for (int c = 0; c < 8; ++c)
      nf[c] = T(0.5) * (nx * (fM[c] + fP[c]) + ny * (gM[c] + gP[c]) + lambda * (qM[c] - qP[c]));
    return lambda;
  }
  APOLLO_HD static double lf_lambda(const EqParams& P, const double* qM, const double* qP) {
    return dmax3(P.p[2] * P.p[0], P.p[1] * P.p[0], P.p[0]);
  }
  APOLLO_HD static double speed2(const EqParams& P, const double* q) {
    double c0 = P.p[0], g = P.p[1], k = P.p[2];
    double s[6] = {c0, -c0, c0 * g, -c0 * g, c0 * k, -c0 * k};
    double lam = 0.0;
    for (int mw = 0; mw < 6; ++mw) lam = dmax3(lam, s[mw] * s[mw], s[mw] * s[mw]);
    return lam;
  }
};

// Transverse-magnetic triple (Ez, Bx, By) of phMaxwellEqn with chi = gamma = 0:
// the same flux entries as the 8-field system, the others being zero.
template <> struct Eq<EQ_MAXWELL_TM> {
  static constexpr int M = 3;
  template <class T>
  APOLLO_HD static void flux2(const EqParams& P, const T* q, T* F, T* G, int* err) {
    T c0 = T(P.p[0]);
    F[0] = -c0 * c0 * q[2];
    F[1] = T(0) * T(0);
    F[2] = -q[0];
    G[0] = c0 * c0 * q[1];
    G[1] = q[0];
    G[2] = T(0) * T(0);
  }
  template <class T>
  APOLLO_HD static T numflux(const EqParams& P, T nx, T ny, T* qM, T* qP, T* nf, int* err) {
    T fM[3], fP[3], gM[3], gP[3];
    flux2(P, qM, fM, gM, err);
    flux2(P, qP, fP, gP, err);
    T lambda = T(dmax3(0.0 * P.p[0], 0.0 * P.p[0], P.p[0]));
#pragma unroll
    for (int c = 0; c < 3; ++c)
      nf[c] = T(0.5) * (nx * (fM[c] + fP[c]) + ny * (gM[c] + gP[c]) + lambda * (qM[c] - qP[c]));
    if ((int)P.p[3] == NF_UPWIND) {
      // the upwind extension: n.B travels at speed 0 (the flux along n maps
      // (Ez, B) to c^2 (n x B)_z and Ez (n_y, -n_x), with eigenvalues +-c on
      // (Ez, tangential B) and 0 on n.B), so its jump is not dissipated
      const T dBn = nx * (qM[1] - qP[1]) + ny * (qM[2] - qP[2]);
      nf[1] = nf[1] - T(0.5) * lambda * dBn * nx;
      nf[2] = nf[2] - T(0.5) * lambda * dBn * ny;
    }
    return lambda;
  }
  APOLLO_HD static double lf_lambda(const EqParams& P, const double* qM, const double* qP) {
    return dmax3(0.0 * P.p[0], 0.0 * P.p[0], P.p[0]);
  }
  APOLLO_HD static double speed2(const EqParams& P, const double* q) {
    double c0 = P.p[0];
    return dmax3(0.0, c0 * c0, c0 * c0);
  }
};

// Whether the face flux is evaluated from each side of an interior face.
// Apollo computes every element's faces from that element's side; the
// kernels compute a face once and negate it for the partner where
// f*(n, a, b) = -f*(-n, b, a), which holds for Lax-Friedrichs and for
// Apollo's Roe flux but not for its HLL (the truncated bound |S_R| differs
// between the sides) nor for Wave (traces rotated against an unrotated normal).
template <int EQ>
APOLLO_HD bool flux_two_sided(const EqParams& P) {
  if (EQ != EQ_EULER && EQ != EQ_EULER2D) return false;
  const int kind = (int)P.p[3];
  return kind == NF_HLL || kind == NF_WAVE;
}

// ---------------------------------------------------- boundary conditions ----
// WxGridFixedBC::applyBC (wxgridfixedbc.cc:17-20): field 0 set to `value`; the
// other fields (for systems) are copied from the interior trace.
// WxIsentropicVortexBC::applyBC (wxisentropicvortexbc.cc:20-43): exact vortex
// at time t.  WxMaxwellTransverseMagnetic::applyBC (:13-23): Ez -> -Ez.
// WxPHMaxwellConductingWallBC::applyBC (:12-41): perfect conductor mirror.
template <int EQ, class T>
APOLLO_HD void apply_bc(const BcTable& B, int tag, double t, double x, double y, T nx, T ny, const T* q, T* qb) {
  constexpr int M = Eq<EQ>::M;
  int idx = tag - 1;
  if (idx < 0 || idx >= B.n) idx = 0;
  int kind = B.kind[idx];
  const double* p = B.p[idx];
#pragma unroll
  for (int c = 0; c < M; ++c) qb[c] = q[c];
  if (kind == BC_FIXED) {
    qb[0] = T(p[0]);
  } else if (kind == BC_VORTEX) {
    if (EQ == EQ_EULER || EQ == EQ_EULER2D) {
      double u0 = p[0], v0 = p[1], x0 = p[2], y0 = p[3], gamma = p[4], beta = p[5];
      const double pi = 3.141592653589793;
      double xmut = x - u0 * t, ymvt = y - v0 * t;
      double rr = sqrt((xmut - x0) * (xmut - x0) + (ymvt - y0) * (ymvt - y0));
      double u = u0 - beta * exp(1. - rr * rr) * (ymvt - y0) / (2. * pi);
      double v = v0 + beta * exp(1. - rr * rr) * (xmut - x0) / (2. * pi);
      double base = 1. - ((gamma - 1.) * beta * beta * exp(2. * (1. - rr * rr)) / (16. * gamma * pi * pi));
      double rho1 = pow(base, 1. / (gamma - 1));
      double p1 = pow(rho1, gamma);
      qb[0] = T(rho1);
      qb[1] = T(rho1 * u);
      qb[2] = T(rho1 * v);
      if (M == 5) qb[3] = T(0.0);
      qb[M - 1] = T(p1 / (gamma - 1) + 0.5 * rho1 * (u * u + v * v));
    }
  } else if (kind == BC_EULER_WALL) {
    // WxEulerWallBC::applyBC (wxeulerwallbc.cc:13-22): normal momentum reflected
    if (EQ == EQ_EULER || EQ == EQ_EULER2D) {
      qb[1] = q[1] - T(2.) * (nx * q[1] + ny * q[2]) * nx;
      qb[2] = q[2] - T(2.) * (nx * q[1] + ny * q[2]) * ny;
      if (M == 5) qb[3] = T(0.0);
    }
  } else if (kind == BC_EULER_ZEROGRAD) {
    // WxEulerZeroGradientBC::applyBC: the interior trace (copied above)
  } else if (kind == BC_EULER_STATE) {
    // WxEulerInflowBC / WxEulerDirichletBC::applyBC: a state fixed at setup
    if (EQ == EQ_EULER || EQ == EQ_EULER2D) {
      qb[0] = T(p[0]);
      qb[1] = T(p[1]);
      qb[2] = T(p[2]);
      if (M == 5) qb[3] = T(p[3]);
      qb[M - 1] = T(p[4]);
    }
  } else if (kind == BC_TM) {
    if (EQ == EQ_MAXWELL) qb[2] = -q[2];
    else if (EQ == EQ_MAXWELL_TM) qb[0] = -q[0];
  } else if (kind == BC_PEC) {
    if (EQ == EQ_MAXWELL) {
      T ex = q[0], ey = q[1], ez = q[2], bx = q[3], by = q[4], bz = q[5], phi = q[6], psi = q[7];
      T en = ex * nx + ey * ny, et = ex * ny - ey * nx;
      qb[0] = en * nx - et * ny;
      qb[1] = en * ny + et * nx;
      qb[2] = -ez;
      T bn = -bx * nx - by * ny, bt = -bx * ny + by * nx;
      qb[3] = bn * nx - bt * ny;
      qb[4] = bn * ny + bt * nx;
      qb[5] = bz;
      qb[6] = -phi;
      qb[7] = psi;
    } else if (EQ == EQ_MAXWELL_TM) {
      T ez = q[0], bx = q[1], by = q[2];
      qb[0] = -ez;
      T bn = -bx * nx - by * ny, bt = -bx * ny + by * nx;
      qb[1] = bn * nx - bt * ny;
      qb[2] = bn * ny + bt * nx;
    }
  }
}

}  // namespace apollo
