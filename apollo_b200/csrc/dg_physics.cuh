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

enum BcKind : int { BC_FIXED = 0, BC_VORTEX = 1, BC_TM = 2, BC_PEC = 3 };

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
    nf[0] = T(0.5) * (nx * (fM[0] + fP[0]) + ny * (gM[0] + gP[0]) + lambda * (qM[0] - qP[0]));
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
  template <class T>
  APOLLO_HD static T numflux(const EqParams& P, T nx, T ny, T* qM, T* qP, T* nf, int* err) {
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
