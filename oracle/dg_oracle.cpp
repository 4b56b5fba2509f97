// ORACLE — test infrastructure only.  This is a plain-C++ restatement of
// Apollo's nodal-DG right-hand side (src/subsolvers/wxnodaldg2dmethod.cc), its
// operator and geometry setup (src/lib/wxcubature2d.cc, wxnodaldggeometry2d.cc,
// wxNodalDGMatrices.h, wxmath.h), its equation plugins (advection, Euler,
// perfectly-hyperbolic Maxwell) and boundary conditions, and PETSc TSSSP's
// default SSPRK(5,2) stepper with Apollo's dt policy (src/solvers/apsolver.cc).
// It is the checker for the CUDA path and the CPU baseline of the benchmark;
// nothing in the shipped library links or calls it.
//
// Loop order, operator definitions and the reversed partner Gauss order follow
// the reference so that FP64 results agree with the reference algorithm to
// round-off.  Per-point physics hooks can be swapped for the reference's own
// compiled plugin code (see ref_adapter.cpp) through orc_set_ref_plugins().
//
// Differences from the reference, all deliberate:
//  * PETSc dense LU is replaced by LU with partial pivoting (same result to
//    round-off); PETSc is not available here.
//  * Periodic face pairing is added (the reference pairs faces only by shared
//    vertices, wxnodaldggeometry2d.cc:235-367): vertices carry a canonical id and
//    faces pair when their canonical vertex pairs match.
//  * Boundary tags are per face.  The reference writes one tag into all six
//    connectivity slots of an element (wxnodaldggeometry2d.cc:348-356), so an
//    element touching two differently tagged boundaries uses the last tag on
//    both; with one tag per mesh (every config here) the two agree.
//  * exit(1) on non-physical states becomes an error flag.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <limits>
#include <map>
#include <utility>
#include <vector>

#include "../apollo_b200/csrc/dg_tables.inc"

#include <thread>

namespace {

// ---------------------------------------------------------------- basis ----
// wxmath.h:306-351 (JacobiP, orthonormal), :353-370 (GradJacobiP)
double jacobi_p(double x, double alpha, double beta, int N) {
  double ab = alpha + beta, ab1 = alpha + beta + 1.0, a1 = alpha + 1.0, b1 = beta + 1.0;
  double gamma0 = std::pow(2.0, ab1) / ab1 * std::tgamma(a1) * std::tgamma(b1) / std::tgamma(ab1);
  double PL0 = 1.0 / std::sqrt(gamma0);
  if (N == 0) return PL0;
  double gamma1 = a1 * b1 / (ab + 3.0) * gamma0;
  double PL1 = ((ab + 2.0) * x / 2.0 + (alpha - beta) / 2.0) / std::sqrt(gamma1);
  if (N == 1) return PL1;
  double aold = 2.0 / (2.0 + ab) * std::sqrt(a1 * b1 / (ab + 3.0));
  double PL2 = 0.0;
  for (int i = 1; i <= N - 1; ++i) {
    double h1 = 2.0 * i + ab;
    double anew = 2.0 / (h1 + 2.0) * std::sqrt((i + 1) * (i + ab1) * (i + a1) * (i + b1) / (h1 + 1.0) / (h1 + 3.0));
    double bnew = -(alpha * alpha - beta * beta) / h1 / (h1 + 2.0);
    PL2 = 1.0 / anew * (-aold * PL0 + (x - bnew) * PL1);
    aold = anew; PL0 = PL1; PL1 = PL2;
  }
  return PL2;
}

double grad_jacobi_p(double z, double alpha, double beta, int N) {
  if (N == 0) return 0.0;
  return std::sqrt(N * (N + alpha + beta + 1)) * jacobi_p(z, alpha + 1, beta + 1, N - 1);
}

// wxNodalDGMatrices.h:7-20
double simplex2d_p(double a, double b, int i, int j) {
  double h1 = jacobi_p(a, 0.0, 0.0, i), h2 = jacobi_p(b, 2.0 * i + 1.0, 0.0, j);
  return std::sqrt(2.0) * h1 * h2 * std::pow(1.0 - b, (double)i);
}

// wxNodalDGMatrices.h:68-105
void grad_simplex2d_p(double a, double b, int id, int jd, double* dr, double* ds) {
  double fa = jacobi_p(a, 0.0, 0.0, id), dfa = grad_jacobi_p(a, 0.0, 0.0, id);
  double gb = jacobi_p(b, 2.0 * id + 1, 0.0, jd), dgb = grad_jacobi_p(b, 2.0 * id + 1, 0.0, jd);
  double dmr = dfa * gb;
  if (id > 0) dmr *= std::pow(0.5 * (1.0 - b), id - 1.0);
  double dms = dfa * gb * 0.5 * (1.0 + a);
  if (id > 0) dms *= std::pow(0.5 * (1.0 - b), id - 1.0);
  double tmp = dgb * std::pow(0.5 * (1.0 - b), (double)id);
  if (id > 0) tmp -= (0.5 * id) * gb * std::pow(0.5 * (1.0 - b), id - 1.0);
  dms += fa * tmp;
  dmr *= std::pow(2.0, id + 0.5);
  dms *= std::pow(2.0, id + 0.5);
  *dr = dmr; *ds = dms;
}

void rs_to_ab(double r, double s, double* a, double* b) {
  *b = s;
  *a = (s == 1.0) ? -1.0 : 2.0 * (1.0 + r) / (1.0 - s) - 1.0;
}

// Row-major dense matrices.  vand: [npts][Np], V_ij = phi_j(r_i, s_i)
// (wxNodalDGMatrices.h:36-65), mode order (i outer, j inner).
std::vector<double> vandermonde(int N, const std::vector<double>& r, const std::vector<double>& s) {
  int Np = (N + 1) * (N + 2) / 2, n = (int)r.size();
  std::vector<double> V((size_t)n * Np);
  int sk = 0;
  for (int i = 0; i <= N; ++i)
    for (int j = 0; j <= N - i; ++j, ++sk)
      for (int k = 0; k < n; ++k) {
        double a, b; rs_to_ab(r[k], s[k], &a, &b);
        V[(size_t)k * Np + sk] = simplex2d_p(a, b, i, j);
      }
  return V;
}

void grad_vandermonde(int N, const std::vector<double>& r, const std::vector<double>& s,
                      std::vector<double>& Vr, std::vector<double>& Vs) {
  int Np = (N + 1) * (N + 2) / 2, n = (int)r.size();
  Vr.assign((size_t)n * Np, 0.0); Vs.assign((size_t)n * Np, 0.0);
  int sk = 0;
  for (int i = 0; i <= N; ++i)
    for (int j = 0; j <= N - i; ++j, ++sk)
      for (int k = 0; k < n; ++k) {
        double a, b, dr, ds; rs_to_ab(r[k], s[k], &a, &b);
        grad_simplex2d_p(a, b, i, j, &dr, &ds);
        Vr[(size_t)k * Np + sk] = dr; Vs[(size_t)k * Np + sk] = ds;
      }
}

std::vector<double> matmul(const std::vector<double>& A, const std::vector<double>& B, int m, int k, int n) {
  std::vector<double> C((size_t)m * n, 0.0);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) {
      double acc = 0.0;
      for (int l = 0; l < k; ++l) acc += A[(size_t)i * k + l] * B[(size_t)l * n + j];
      C[(size_t)i * n + j] = acc;
    }
  return C;
}

std::vector<double> transpose(const std::vector<double>& A, int m, int n) {
  std::vector<double> T((size_t)n * m);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) T[(size_t)j * m + i] = A[(size_t)i * n + j];
  return T;
}

// Dense inverse by LU with partial pivoting (stands in for PETSc MatLUFactor +
// MatMatSolve, wxnodaldggeometry2d.cc:147-177).
std::vector<double> invert(std::vector<double> A, int n) {
  std::vector<double> inv((size_t)n * n, 0.0);
  std::vector<int> piv(n);
  for (int i = 0; i < n; ++i) piv[i] = i;
  for (int c = 0; c < n; ++c) {
    int p = c; double best = std::fabs(A[(size_t)c * n + c]);
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(A[(size_t)r * n + c]) > best) { best = std::fabs(A[(size_t)r * n + c]); p = r; }
    if (p != c) {
      for (int j = 0; j < n; ++j) std::swap(A[(size_t)c * n + j], A[(size_t)p * n + j]);
      std::swap(piv[c], piv[p]);
    }
    for (int r = c + 1; r < n; ++r) {
      double f = A[(size_t)r * n + c] / A[(size_t)c * n + c];
      A[(size_t)r * n + c] = f;
      for (int j = c + 1; j < n; ++j) A[(size_t)r * n + j] -= f * A[(size_t)c * n + j];
    }
  }
  for (int col = 0; col < n; ++col) {
    std::vector<double> y(n);
    for (int i = 0; i < n; ++i) {
      double v = (piv[i] == col) ? 1.0 : 0.0;
      for (int j = 0; j < i; ++j) v -= A[(size_t)i * n + j] * y[j];
      y[i] = v;
    }
    for (int i = n - 1; i >= 0; --i) {
      double v = y[i];
      for (int j = i + 1; j < n; ++j) v -= A[(size_t)i * n + j] * inv[(size_t)j * n + col];
      inv[(size_t)i * n + col] = v / A[(size_t)i * n + i];
    }
  }
  return inv;
}

// wxmath.h:173-209 (Gauss-Legendre on [x1,x2], ascending points)
void gauleg(double x1, double x2, std::vector<double>& x, std::vector<double>& w, int n) {
  x.assign(n, 0.0); w.assign(n, 0.0);
  const double EPS = 3.0e-13, PI = 3.14159265358979323846;
  int m = (n + 1) / 2;
  double xm = 0.5 * (x2 + x1), xl = 0.5 * (x2 - x1);
  for (int i = 1; i <= m; ++i) {
    double z = std::cos(PI * (i - 0.25) / (n + 0.5)), z1, pp;
    do {
      double p1 = 1.0, p2 = 0.0, p3;
      for (int j = 1; j <= n; ++j) {
        p3 = p2; p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
    } while (std::fabs(z - z1) > EPS);
    x[i - 1] = xm - xl * z;
    x[n - i] = xm + xl * z;
    w[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
    w[n - i] = w[i - 1];
  }
}

// wxcubature2d.cc:433-442: y[rows][meqn] = A[rows][cols] x[cols][meqn]
inline void mat_vec(int rows, int cols, int meqn, const double* A, const double* x, double* y) {
  for (int i = 0; i < rows * meqn; ++i) y[i] = 0.0;
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c)
      for (int z = 0; z < meqn; ++z) y[r * meqn + z] += A[r * cols + c] * x[c * meqn + z];
}

inline double dmax2(double a, double b) { return a > b ? a : b; }
inline double dmax3(double a, double b, double c) { double m1 = a > b ? a : b; return m1 > c ? m1 : c; }

enum { EQ_ADVECTION = 0, EQ_EULER = 1, EQ_MAXWELL = 2 };
enum { BC_FIXED = 0, BC_VORTEX = 1, BC_TM = 2, BC_PEC = 3, BC_EULER_WALL = 4, BC_EULER_INFLOW = 5,
       BC_EULER_ZEROGRAD = 6, BC_EULER_DIRICHLET = 7 };
// Euler Numerical_Flux codes (wxeulereqn.cc:10-15), held in eqp[3]
// (NF_UPWIND: an extension, not in Apollo: advection with dissipation |n.u|;
// the Maxwell TM fields without dissipation of the normal magnetic field)
enum { NF_LF = 0, NF_HLL = 1, NF_ROE = 2, NF_WAVE = 4, NF_UPWIND = 8 };
enum { ERR_NONPHYS = 1, ERR_NAN = 2, ERR_JAC = 4 };

typedef void (*flux_fn)(void* ctx, int d, const double* q, double* f);
typedef void (*numflux_fn)(void* ctx, const double* n, double* qM, double* qP, double* f, double* lam);

struct Oracle {
  int N, Np, Nc, Ng, Nfp3, K, meqn, eq;
  double eqp[4];
  std::vector<double> r, s, V, Vc, Drc, Dsc, VT, DrT, DsT, interp, interpT, VVT, cw, gw;
  std::vector<int> fmask;
  std::vector<double> x, y;      // [K][Np]
  std::vector<int> conn;         // [K][6] element, face (or -tag, -tag)
  std::vector<int> bc_kind;      // [nbc]
  std::vector<double> bc_par;    // [nbc][8]
  double dtscale, rmin, cfl;
  int err;
  // optional reference plugin hooks
  flux_fn ref_flux = nullptr; numflux_fn ref_numflux = nullptr; void* ref_ctx = nullptr;
  int nthreads = 1;
  std::vector<double> area_total; // per-field area integrals of the last RHS
  // Euler limiter eulerLimiterHW (orc_set_limiter)
  bool lim_on = false;
  int lim_kind = 0;  // 0: eulerLimiterHW, 1: tuAliabadiLimiter
  double lim_gamma = 1.4, lim_minP = 0.0, lim_minD = 0.0;
  std::vector<double> lim_ave;
  // source plugins (orc_add_source): kind, output field (Apollo's index), params
  std::vector<int> src_kind, src_out;
  std::vector<double> src_par;  // [nsrc][9]
};

// Source plugins, WxHyperbolicSrc::compSource (src/hyper/wxhyperbolicsrc.cc:64-80)
// adding src() into the output field.  kind 1: tranverseMagneticSrc
// (src/hyperapps/maxwell/wxtransversemagneticsrc.h:37-44); kind 2:
// pointCurrentSrc (src/hyperapps/maxwell/wxpointcurrent.h: setup keys xLocation,
// yLocation, radius, currentDensity, frequency, phase, charge, mass, epsilon0).
// tx = [t, x, y].
void add_sources(const Oracle& o, const double* tx, double* s) {
  for (size_t i = 0; i < o.src_kind.size(); ++i) {
    const double* p = &o.src_par[i * 9];
    const double t = tx[0], x = tx[1], y = tx[2];
    double v = 0.0;
    if (o.src_kind[i] == 1) {
      v = std::exp(t) * (x * (1 - x) * y * (1 - y) + 2. * x * (1 - x) + 2 * y * (1 - y));
    } else if (o.src_kind[i] == 2) {
      const double qbyme = p[6] / (p[7] * p[8]);
      if (std::sqrt((x - p[0]) * (x - p[0]) + (y - p[1]) * (y - p[1])) < p[2]) v = p[3] * qbyme * std::sin(p[4] * t + p[5]);
    }
    s[o.src_out[i]] += v;
  }
}

// ----------------------------------------------------------- plugins ----
// Advection: wxadvectioneqn.cc:176-208
void adv_flux(const Oracle& o, int d, const double* q, double* f) {
  f[0] = (d == 0 ? o.eqp[0] : (d == 1 ? o.eqp[1] : o.eqp[2])) * q[0];
}
// Euler: wxeulereqn.cc:809-871 (flux), :1326-1341 (primitiveVariables),
// :1097-1117 (Lax-Friedrichs)
void euler_flux(Oracle& o, int d, const double* q, double* f) {
  double gamma = o.eqp[0], minP = o.eqp[1], minD = o.eqp[2];
  double g1 = gamma - 1.0;
  int mu = 1, mv = 2, mw = 3;
  if (d == 1) { mu = 2; mv = 3; mw = 1; }
  else if (d == 2) { mu = 3; mv = 1; mw = 2; }
  double rho = q[0];
  if (minD == 0.0 && rho <= 0) o.err |= ERR_NONPHYS;
  if (rho < minD) rho = minD;
  double u = q[mu] / rho, v = q[mv] / rho, w = q[mw] / rho, E = q[4];
  double p = g1 * (E - 0.5 * rho * (u * u + v * v + w * w));
  if (p <= 0) {
    if (minP == 0.0) o.err |= ERR_NONPHYS; else p = minP;
  }
  f[0] = rho * u;
  f[mu] = rho * u * u + p;
  f[mv] = rho * u * v;
  f[mw] = rho * u * w;
  f[4] = (E + p) * u;
}
void euler_prim(const Oracle& o, double* qc, double* qp) {
  double gamma = o.eqp[0], minP = o.eqp[1], minD = o.eqp[2];
  qp[0] = qc[0];
  if (qp[0] <= 0.) { qc[0] = minD; qp[0] = minD; }
  qp[1] = qc[1] / qc[0]; qp[2] = qc[2] / qc[0]; qp[3] = qc[3] / qc[0];
  qp[4] = (gamma - 1.) * (qc[4] - 0.5 * (qc[1] * qc[1] + qc[2] * qc[2] + qc[3] * qc[3]) / qc[0]);
  if (qp[4] <= 0.) {
    qp[4] = minP;
    qc[4] = minP / (gamma - 1.) + 0.5 * qp[0] * (qp[1] * qp[1] + qp[2] * qp[2] + qp[3] * qp[3]);
  }
}
// Maxwell: wxphmaxwelleqn.cc:450-522
void maxwell_flux(const Oracle& o, int d, const double* q, double* f) {
  double c0 = o.eqp[0], gm = o.eqp[1], chi = o.eqp[2];
  int iex = 0, iey = 1, iez = 2, ibx = 3, iby = 4, ibz = 5;
  if (d == 1) { iex = 1; iey = 2; iez = 0; ibx = 4; iby = 5; ibz = 3; }
  else if (d == 2) { iex = 2; iey = 0; iez = 1; ibx = 5; iby = 3; ibz = 4; }
  f[iex] = chi * c0 * c0 * q[6];
  f[iey] = c0 * c0 * q[ibz];
  f[iez] = -c0 * c0 * q[iby];
  f[ibx] = gm * q[7];
  f[iby] = -q[iez];
  f[ibz] = q[iey];
  f[6] = chi * q[iex];
  f[7] = gm * c0 * c0 * q[ibx];
}

void eq_flux(Oracle& o, int d, const double* q, double* f) {
  if (o.ref_flux) { o.ref_flux(o.ref_ctx, d, q, f); return; }
  if (o.eq == EQ_ADVECTION) adv_flux(o, d, q, f);
  else if (o.eq == EQ_EULER) euler_flux(o, d, q, f);
  else maxwell_flux(o, d, q, f);
}

// Euler fluxes other than LF, following wxeulereqn.cc:1121-1322 step by step.
// Momentum to the face's normal-tangent frame, in place.
void euler_rotate(const double* n, double* q) {
  double ru = q[1], rv = q[2];
  q[1] = n[0] * ru + n[1] * rv;
  q[2] = -n[1] * ru + n[0] * rv;
}
double euler_speed(const Oracle& o, const double* pM, const double* pP) {
  double gamma = o.eqp[0];
  double c0M = std::sqrt(pM[1] * pM[1] + pM[2] * pM[2] + pM[3] * pM[3]) + std::sqrt(gamma * pM[4] / pM[0]);
  double c0P = std::sqrt(pP[1] * pP[1] + pP[2] * pP[2] + pP[3] * pP[3]) + std::sqrt(gamma * pP[4] / pP[0]);
  return dmax2(c0M, c0P);
}
// HLL, :1121-1202.  abs(SR) there is int abs(int) (only <cmath> and the C
// library's int abs are in scope), so SR enters truncated toward zero.
double euler_hll(Oracle& o, const double* n, double* qM, double* qP, double* nf) {
  double fM[5], fP[5], gM[5], gP[5], pM[5], pP[5], fx[5];
  double gamma = o.eqp[0];
  euler_rotate(n, qM);
  euler_rotate(n, qP);
  euler_flux(o, 0, qM, fM); euler_flux(o, 0, qP, fP); euler_flux(o, 1, qM, gM); euler_flux(o, 1, qP, gP);
  euler_prim(o, qM, pM); euler_prim(o, qP, pP);
  double HM = (qM[4] + pM[4]) / pM[0], cM = std::sqrt(gamma * pM[4] / pM[0]);
  double HP = (qP[4] + pP[4]) / pP[0], cP = std::sqrt(gamma * pP[4] / pP[0]);
  double rMs = std::sqrt(pM[0]), rPs = std::sqrt(pP[0]);
  double u = (rMs * pM[1] + rPs * pP[1]) / (rMs + rPs);
  double v = (rMs * pM[2] + rPs * pP[2]) / (rMs + rPs);
  double w = (rMs * pM[3] + rPs * pP[3]) / (rMs + rPs);
  double H = (rMs * HM + rPs * HP) / (rMs + rPs);
  double c2 = (gamma - 1.) * (H - 0.5 * (u * u + v * v + w * w)), c = std::sqrt(c2);
  double a = pM[1] - cM, b = u - c;
  double SL = a < b ? a : b;
  a = pP[1] + cP;
  b = u + c;
  double SR = a > b ? a : b;
  double zero = 0.0;
  double t1 = ((SR < zero ? SR : zero) - (zero < SL ? zero : SL)) / (SR - SL);
  double t2 = 1. - t1;
  double t3 = (SR * std::fabs(SL) - SL * (double)std::abs((int)SR)) / (2. * (SR - SL));
  for (int i = 0; i < 5; ++i) fx[i] = t1 * fP[i] + t2 * fM[i] - t3 * (qP[i] - qM[i]);
  nf[0] = fx[0];
  nf[1] = n[0] * fx[1] - n[1] * fx[2];
  nf[2] = n[1] * fx[1] + n[0] * fx[2];
  nf[3] = 0.0;
  nf[4] = fx[4];
  return euler_speed(o, pM, pP);
}
// Roe, :1206-1275: nflux[1] is assigned twice (the second, y-momentum, value
// stays) and nflux[2] is never set, so it keeps the caller's buffer, which is
// Apollo's zero-initialised flux array (wxnodaldg2dmethod.cc:98).
double euler_roe(Oracle& o, const double* n, double* qM, double* qP, double* nf) {
  double fM[5], fP[5], pM[5], pP[5], fx[5];
  double gamma = o.eqp[0];
  euler_rotate(n, qM);
  euler_rotate(n, qP);
  euler_prim(o, qM, pM); euler_prim(o, qP, pP);
  double HM = (qM[4] + pM[4]) / pM[0];
  double HP = (qP[4] + pP[4]) / pP[0];
  double rMs = std::sqrt(pM[0]), rPs = std::sqrt(pP[0]);
  double rho = rMs * rPs;
  double u = (rMs * pM[1] + rPs * pP[1]) / (rMs + rPs);
  double v = (rMs * pM[2] + rPs * pP[2]) / (rMs + rPs);
  double w = (rMs * pM[3] + rPs * pP[3]) / (rMs + rPs);
  double H = (rMs * HM + rPs * HP) / (rMs + rPs);
  double c2 = (gamma - 1.) * (H - 0.5 * (u * u + v * v + w * w)), c = std::sqrt(c2);
  double dw1 = -0.5 * rho * (pP[1] - pM[1]) / c + 0.5 * (pP[4] - pM[4]) / c2;
  double dw2 = (pP[0] - pM[0]) - (pP[4] - pM[4]) / c2;
  double dw3 = rho * (pP[2] - pM[2]);
  double dw4 = 0.5 * rho * (pP[1] - pM[1]) / c + 0.5 * (pP[4] - pM[4]) / c2;
  dw1 = std::fabs(u - c) * dw1;
  dw2 = std::fabs(u) * dw2;
  dw3 = std::fabs(u) * dw3;
  dw4 = std::fabs(u + c) * dw4;
  euler_flux(o, 0, qM, fM);
  euler_flux(o, 0, qP, fP);
  for (int i = 0; i < 5; ++i) fx[i] = 0.5 * (fM[i] + fP[i]);
  fx[0] -= 0.5 * (dw1 * 1. + dw2 * 1. + dw3 * 0. + dw4 * 1.);
  fx[1] -= 0.5 * (dw1 * (u - c) + dw2 * u + dw3 * 0. + dw4 * (u + c));
  fx[2] -= 0.5 * (dw1 * v + dw2 * v + dw3 * 1. + dw4 * v);
  fx[3] = 0.0;
  fx[4] -= 0.5 * (dw1 * (H - u * c) + dw2 * (u * u + v * v) / 2. + dw3 * v + dw4 * (H + u * c));
  nf[0] = fx[0];
  nf[1] = n[1] * fx[1] + n[0] * fx[2];
  nf[2] = 0.0;
  nf[3] = 0.0;
  nf[4] = fx[4];
  return euler_speed(o, pM, pP);
}
// Wave, :1279-1322 then the switch's fall-through into LF (:888-892): the
// traces are rotated in place and pass the Riemann solver rp(0, qP, qM)
// (:94-199), whose checks may fail and whose pressure floor may rewrite the
// energies; the wave flux itself is overwritten by the LF flux that follows.
void euler_wave_prelude(Oracle& o, const double* n, double* qM, double* qP) {
  double fM[5], fP[5];
  euler_rotate(n, qM);
  euler_rotate(n, qP);
  euler_flux(o, 0, qM, fM);
  euler_flux(o, 0, qP, fP);
  double* ql = qP;
  double* qr = qM;
  double g1 = o.eqp[0] - 1, minP = o.eqp[1];
  if (ql[0] < 0 || qr[0] < 0) { o.err |= ERR_NONPHYS; return; }
  double rl = std::sqrt(ql[0]), rr = std::sqrt(qr[0]);
  double pl = g1 * (ql[4] - 0.5 * (ql[1] * ql[1] + ql[2] * ql[2] + ql[3] * ql[3]) / ql[0]);
  double pr = g1 * (qr[4] - 0.5 * (qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]) / qr[0]);
  if (minP == 0.0 && (pl < 0 || pr < 0)) o.err |= ERR_NONPHYS;
  if (pl < minP) { ql[4] = minP / (o.eqp[0] - 1) + 0.5 * (ql[1] * ql[1] + ql[2] * ql[2] + ql[3] * ql[3]) / ql[0]; pl = minP; }
  if (pr < minP) { qr[4] = minP / (o.eqp[0] - 1) + 0.5 * (qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]) / qr[0]; pr = minP; }
  double rsq2 = rl + rr;
  double u = (ql[1] / rl + qr[1] / rr) / rsq2, v = (ql[2] / rl + qr[2] / rr) / rsq2, w = (ql[3] / rl + qr[3] / rr) / rsq2;
  double enth = ((ql[4] + pl) / rl + (qr[4] + pr) / rr) / rsq2;
  if (g1 * (enth - 0.5 * (u * u + v * v + w * w)) < 0) o.err |= ERR_NONPHYS;
}

// DGnumericalFlux (qM/qP may be modified by the Euler primitive clamp, as in
// the reference).
void eq_numflux(Oracle& o, const double* n, double* qM, double* qP, double* nf, double* lam) {
  if (o.eq == EQ_ADVECTION && (int)o.eqp[3] == NF_UPWIND) {
    // the upwind extension: 1/2 [n.u (qM + qP) + |n.u| (qM - qP)] written as
    // the Lax-Friedrichs form with the normal speed as its dissipation; the
    // returned speed (the dt policy's) is Apollo's
    double fM[1], fP[1], gM[1], gP[1];
    adv_flux(o, 0, qM, fM); adv_flux(o, 0, qP, fP); adv_flux(o, 1, qM, gM); adv_flux(o, 1, qP, gP);
    const double diss = std::fabs(n[0] * o.eqp[0] + n[1] * o.eqp[1]);
    nf[0] = 0.5 * (n[0] * (fM[0] + fP[0]) + n[1] * (gM[0] + gP[0]) + diss * (qM[0] - qP[0]));
    *lam = dmax2(std::fabs(o.eqp[0]), std::fabs(o.eqp[1]));
    return;
  }
  if (o.eq == EQ_MAXWELL && (int)o.eqp[3] == NF_UPWIND) {
    // the upwind extension for the TM fields (Ez, Bx, By = 2, 3, 4) with
    // chi = gamma = 0: Apollo's Lax-Friedrichs flux without the dissipation
    // of the normal magnetic field, whose wave speed is 0
    double fM[8], fP[8], gM[8], gP[8];
    maxwell_flux(o, 0, qM, fM); maxwell_flux(o, 0, qP, fP); maxwell_flux(o, 1, qM, gM); maxwell_flux(o, 1, qP, gP);
    const double lambda = dmax3(o.eqp[2] * o.eqp[0], o.eqp[1] * o.eqp[0], o.eqp[0]);
    for (int c = 0; c < o.meqn; ++c)
      nf[c] = 0.5 * (n[0] * (fM[c] + fP[c]) + n[1] * (gM[c] + gP[c]) + lambda * (qM[c] - qP[c]));
    const double dBn = n[0] * (qM[3] - qP[3]) + n[1] * (qM[4] - qP[4]);
    nf[3] -= 0.5 * lambda * dBn * n[0];
    nf[4] -= 0.5 * lambda * dBn * n[1];
    *lam = lambda;
    return;
  }
  if (o.ref_numflux) { o.ref_numflux(o.ref_ctx, n, qM, qP, nf, lam); return; }
  double fM[8], fP[8], gM[8], gP[8], lambda;
  int m = o.meqn;
  if (o.eq == EQ_EULER) {
    const int kind = (int)o.eqp[3];
    if (kind == NF_HLL) { *lam = euler_hll(o, n, qM, qP, nf); return; }
    if (kind == NF_ROE) { *lam = euler_roe(o, n, qM, qP, nf); return; }
    if (kind == NF_WAVE) euler_wave_prelude(o, n, qM, qP);
  }
  if (o.eq == EQ_ADVECTION) {
    adv_flux(o, 0, qM, fM); adv_flux(o, 0, qP, fP); adv_flux(o, 1, qM, gM); adv_flux(o, 1, qP, gP);
    lambda = dmax2(std::fabs(o.eqp[0]), std::fabs(o.eqp[1]));
  } else if (o.eq == EQ_EULER) {
    euler_flux(o, 0, qM, fM); euler_flux(o, 0, qP, fP); euler_flux(o, 1, qM, gM); euler_flux(o, 1, qP, gP);
    double pM[5], pP[5];
    euler_prim(o, qM, pM); euler_prim(o, qP, pP);
    double gamma = o.eqp[0];
    double c0M = std::sqrt(pM[1] * pM[1] + pM[2] * pM[2] + pM[3] * pM[3]) + std::sqrt(gamma * pM[4] / pM[0]);
    double c0P = std::sqrt(pP[1] * pP[1] + pP[2] * pP[2] + pP[3] * pP[3]) + std::sqrt(gamma * pP[4] / pP[0]);
    lambda = dmax2(c0M, c0P);
  } else {
    maxwell_flux(o, 0, qM, fM); maxwell_flux(o, 0, qP, fP); maxwell_flux(o, 1, qM, gM); maxwell_flux(o, 1, qP, gP);
    lambda = dmax3(o.eqp[2] * o.eqp[0], o.eqp[1] * o.eqp[0], o.eqp[0]);
  }
  for (int c = 0; c < m; ++c)
    nf[c] = 0.5 * (n[0] * (fM[c] + fP[c]) + n[1] * (gM[c] + gP[c]) + lambda * (qM[c] - qP[c]));
  *lam = lambda;
}

// Wave speeds of the Riemann solver with ql = qr = q (used by init's dt,
// wxnodaldg2dmethod.cc:202-212).  Returns max over waves of max(sx^2, sy^2).
double eq_speed2(const Oracle& o, const double* q) {
  if (o.eq == EQ_ADVECTION) {
    return dmax3(0.0, o.eqp[0] * o.eqp[0], o.eqp[1] * o.eqp[1]);
  } else if (o.eq == EQ_EULER) {
    // Roe averages with ql = qr (wxeulereqn.cc:145-199)
    double gamma = o.eqp[0], g1 = gamma - 1;
    double lam = 0.0;
    double sx[3], sy[3];
    for (int d = 0; d < 2; ++d) {
      int mu = d == 0 ? 1 : 2, mv = d == 0 ? 2 : 3, mw = d == 0 ? 3 : 1;
      double rs = std::sqrt(q[0]);
      double p = g1 * (q[4] - 0.5 * (q[mu] * q[mu] + q[mv] * q[mv] + q[mw] * q[mw]) / q[0]);
      double rsq2 = rs + rs;
      double u = (q[mu] / rs + q[mu] / rs) / rsq2;
      double v = (q[mv] / rs + q[mv] / rs) / rsq2;
      double w = (q[mw] / rs + q[mw] / rs) / rsq2;
      double u2 = u * u + v * v + w * w;
      double enth = ((q[4] + p) / rs + (q[4] + p) / rs) / rsq2;
      double a = std::sqrt(g1 * (enth - 0.5 * u2));
      double* s = d == 0 ? sx : sy;
      s[0] = u - a; s[1] = u; s[2] = u + a;
    }
    for (int mw = 0; mw < 3; ++mw) lam = dmax3(lam, sx[mw] * sx[mw], sy[mw] * sy[mw]);
    return lam;
  } else {
    double c0 = o.eqp[0], g = o.eqp[1], k = o.eqp[2];
    double s[6] = {c0, -c0, c0 * g, -c0 * g, c0 * k, -c0 * k};
    double lam = 0.0;
    for (int mw = 0; mw < 6; ++mw) lam = dmax3(lam, s[mw] * s[mw], s[mw] * s[mw]);
    return lam;
  }
}

// Boundary conditions: wxgridfixedbc.cc:17-20, wxisentropicvortexbc.cc:20-43,
// wxmaxwelltranversemagneticbc.cc:13-23, wxphmaxwellconductingwallbc.cc:12-41
void apply_bc(const Oracle& o, int tag, const double* xc, const double* nx, const double* q, double* qb) {
  int idx = tag - 1;
  int kind = o.bc_kind[idx];
  const double* p = &o.bc_par[(size_t)idx * 8];
  int m = o.meqn;
  if (kind == BC_FIXED) {
    for (int c = 0; c < m; ++c) qb[c] = q[c];
    qb[0] = p[0];
  } else if (kind == BC_VORTEX) {
    double u0 = p[0], v0 = p[1], x0 = p[2], y0 = p[3], gamma = p[4], beta = p[5];
    double t = xc[0], xx = xc[1], yy = xc[2], pi = 3.141592653589793;
    double xmut = xx - u0 * t, ymvt = yy - v0 * t;
    double rr = std::sqrt((xmut - x0) * (xmut - x0) + (ymvt - y0) * (ymvt - y0));
    double u = u0 - beta * std::exp(1. - rr * rr) * (ymvt - y0) / (2. * pi);
    double v = v0 + beta * std::exp(1. - rr * rr) * (xmut - x0) / (2. * pi);
    double base = 1. - ((gamma - 1.) * beta * beta * std::exp(2. * (1. - rr * rr)) / (16. * gamma * pi * pi));
    double rho1 = std::pow(base, 1. / (gamma - 1));
    double p1 = std::pow(rho1, gamma);
    qb[0] = rho1; qb[1] = rho1 * u; qb[2] = rho1 * v; qb[3] = 0.0;
    qb[4] = p1 / (gamma - 1) + 0.5 * rho1 * (u * u + v * v);
  } else if (kind == BC_EULER_WALL) {
    // wxeulerwallbc.cc
    qb[0] = q[0];
    qb[1] = q[1] - 2. * (nx[0] * q[1] + nx[1] * q[2]) * nx[0];
    qb[2] = q[2] - 2. * (nx[0] * q[1] + nx[1] * q[2]) * nx[1];
    qb[3] = 0.0;
    qb[4] = q[4];
  } else if (kind == BC_EULER_INFLOW) {
    // wxeulerinflowbc.cc: Mach_number, Flow_angle, gas_gamma, Pressure, density
    double mach = p[0], angle = p[1], gamma = p[2], pres = p[3], rho = p[4];
    double pi = 3.141592653589793;
    double sound = std::sqrt(gamma * pres / rho);
    double u = mach * sound * std::cos(angle * pi / 180.), v = mach * sound * std::sin(angle * pi / 180.);
    qb[0] = rho; qb[1] = rho * u; qb[2] = rho * v; qb[3] = 0.0;
    qb[4] = pres / (gamma - 1) + 0.5 * rho * (u * u + v * v);
  } else if (kind == BC_EULER_ZEROGRAD) {
    // wxeulerzerogradientbc.cc
    for (int c = 0; c < 5; ++c) qb[c] = q[c];
  } else if (kind == BC_EULER_DIRICHLET) {
    // wxeulerdirichletbc.cc: density, xvelocity, yvelocity, zvelocity, gas_gamma, pressure
    double rho = p[0], u = p[1], v = p[2], w = p[3], gamma = p[4], pres = p[5];
    qb[0] = rho; qb[1] = rho * u; qb[2] = rho * v; qb[3] = rho * w;
    qb[4] = pres / (gamma - 1) + 0.5 * rho * (u * u + v * v + w * w);
  } else if (kind == BC_TM) {
    for (int c = 0; c < m; ++c) qb[c] = q[c];
    qb[2] = -q[2];
  } else {
    double ex = q[0], ey = q[1], ez = q[2], bx = q[3], by = q[4], bz = q[5], phi = q[6], psi = q[7];
    double en = ex * nx[0] + ey * nx[1], et = ex * nx[1] - ey * nx[0];
    qb[0] = en * nx[0] - et * nx[1];
    qb[1] = en * nx[1] + et * nx[0];
    qb[2] = -ez;
    double bn = -bx * nx[0] - by * nx[1], bt = -bx * nx[1] + by * nx[0];
    qb[3] = bn * nx[0] - bt * nx[1];
    qb[4] = bn * nx[1] + bt * nx[0];
    qb[5] = bz;
    qb[6] = -phi;
    qb[7] = psi;
  }
}

// ------------------------------------------------------------- setup ----
void build_operators(Oracle& o) {
  int N = o.N, Np = o.Np;
  o.r.assign(apollo_tables::kNodeR[N], apollo_tables::kNodeR[N] + Np);
  o.s.assign(apollo_tables::kNodeS[N], apollo_tables::kNodeS[N] + Np);
  o.fmask.assign(apollo_tables::kFmask[N], apollo_tables::kFmask[N] + 3 * (N + 1));
  // wxnodaldggeometry2d.cc:59-76
  std::vector<double> Vand = vandermonde(N, o.r, o.s);
  std::vector<double> invV = invert(Vand, Np);
  o.VVT = matmul(Vand, transpose(Vand, Np, Np), Np, Np, Np);
  o.rmin = std::fabs(o.r[1] - o.r[0]);               // :91
  // wxcubature2d.cc:18-108
  o.Nc = apollo_tables::kCubNpts[N];
  std::vector<double> cr(o.Nc), cs(o.Nc);
  o.cw.resize(o.Nc);
  for (int k = 0; k < o.Nc; ++k) {
    cr[k] = apollo_tables::kCubRST[N][3 * k]; cs[k] = apollo_tables::kCubRST[N][3 * k + 1];
    o.cw[k] = apollo_tables::kCubRST[N][3 * k + 2];
  }
  std::vector<double> Vout = vandermonde(N, cr, cs);
  o.Vc = matmul(Vout, invV, o.Nc, Np, Np);
  o.VT = transpose(o.Vc, o.Nc, Np);
  std::vector<double> Vr, Vs;
  grad_vandermonde(N, cr, cs, Vr, Vs);
  o.Drc = matmul(Vr, invV, o.Nc, Np, Np);
  o.Dsc = matmul(Vs, invV, o.Nc, Np, Np);
  o.DrT = transpose(o.Drc, o.Nc, Np);
  o.DsT = transpose(o.Dsc, o.Nc, Np);
  // Gauss points on the three faces (:110-134)
  o.Ng = 2 * (N + 1);
  std::vector<double> gz;
  gauleg(-1.0, 1.0, gz, o.gw, o.Ng);
  std::vector<double> fr(3 * o.Ng), fs(3 * o.Ng);
  for (int k = 0; k < o.Ng; ++k) {
    fr[k] = gz[k];               fs[k] = -1.0;
    fr[o.Ng + k] = -gz[k];       fs[o.Ng + k] = gz[k];
    fr[2 * o.Ng + k] = -1.0;     fs[2 * o.Ng + k] = -gz[k];
  }
  std::vector<double> gV = vandermonde(N, fr, fs);
  o.interp = matmul(gV, invV, 3 * o.Ng, Np, Np);
  o.interpT = transpose(o.interp, 3 * o.Ng, Np);
  o.Nfp3 = 3 * o.Ng;
}

}  // namespace

extern "C" {

// Create an oracle.  Mesh: vertices (vx, vy), CCW triangles etov[K][3],
// face_tag[K][3] (0 = pair by vertices, t > 0 = boundary condition t),
// vert_canon[nverts] canonical vertex id used for pairing (periodicity), or
// NULL.  eq: 0 advection (ux, uy, uz), 1 Euler (gamma, minP, minD),
// 2 Maxwell (c0, gamma, chi).  bc_kind[nbc], bc_par[nbc][8].
void* orc_create(int N, int eq, const double* eqp, int nverts, const double* vx, const double* vy,
                 int K, const int* etov, const int* face_tag, const int* vert_canon,
                 int nbc, const int* bc_kind, const double* bc_par, double cfl) {
  Oracle* o = new Oracle();
  o->N = N; o->Np = (N + 1) * (N + 2) / 2; o->K = K; o->eq = eq; o->cfl = cfl; o->err = 0;
  for (int i = 0; i < 4; ++i) o->eqp[i] = eqp ? eqp[i] : 0.0;
  o->meqn = eq == EQ_ADVECTION ? 1 : (eq == EQ_EULER ? 5 : 8);
  build_operators(*o);
  o->bc_kind.assign(bc_kind, bc_kind + nbc);
  o->bc_par.assign(bc_par, bc_par + (size_t)nbc * 8);
  int Np = o->Np;
  o->x.resize((size_t)K * Np); o->y.resize((size_t)K * Np);
  o->dtscale = 1.0e6;
  // wxnodaldggeometry2d.cc:198-228
  for (int k = 0; k < K; ++k) {
    int a = etov[3 * k], b = etov[3 * k + 1], c = etov[3 * k + 2];
    double p1x = vx[a], p1y = vy[a], p2x = vx[b], p2y = vy[b], p3x = vx[c], p3y = vy[c];
    for (int n = 0; n < Np; ++n) {
      double r = o->r[n], s = o->s[n];
      o->x[(size_t)k * Np + n] = 0.5 * (-p1x * (r + s) + p2x * (1. + r) + p3x * (1. + s));
      o->y[(size_t)k * Np + n] = 0.5 * (-p1y * (r + s) + p2y * (1. + r) + p3y * (1. + s));
    }
    double l1 = std::sqrt(std::pow(p1x - p2x, 2) + std::pow(p1y - p2y, 2));
    double l2 = std::sqrt(std::pow(p2x - p3x, 2) + std::pow(p2y - p3y, 2));
    double l3 = std::sqrt(std::pow(p3x - p1x, 2) + std::pow(p3y - p1y, 2));
    double sp = 0.5 * (l1 + l2 + l3);
    double area = std::sqrt(std::fabs(sp * (sp - l1) * (sp - l2) * (sp - l3)));
    o->dtscale = std::min(o->dtscale, area / sp);
  }
  // face pairing by shared (canonical) vertices, faces (v0v1, v1v2, v2v0)
  // (wxnodaldggeometry2d.cc:263, 279-363)
  o->conn.assign((size_t)K * 6, -1);
  std::map<std::pair<int, int>, int> open;
  static const int vn[3][2] = {{0, 1}, {1, 2}, {2, 0}};
  for (int k = 0; k < K; ++k)
    for (int f = 0; f < 3; ++f) {
      int tag = face_tag ? face_tag[3 * k + f] : 0;
      if (tag > 0) { o->conn[6 * k + 2 * f] = -tag; o->conn[6 * k + 2 * f + 1] = -tag; continue; }
      int va = etov[3 * k + vn[f][0]], vb = etov[3 * k + vn[f][1]];
      if (vert_canon) { va = vert_canon[va]; vb = vert_canon[vb]; }
      std::pair<int, int> key(std::min(va, vb), std::max(va, vb));
      auto it = open.find(key);
      if (it == open.end()) { open[key] = 3 * k + f; continue; }
      int kf = it->second; open.erase(it);
      int k2 = kf / 3, f2 = kf % 3;
      o->conn[6 * k + 2 * f] = k2; o->conn[6 * k + 2 * f + 1] = f2;
      o->conn[6 * k2 + 2 * f2] = k; o->conn[6 * k2 + 2 * f2 + 1] = f;
    }
  o->area_total.assign(o->meqn, 0.0);
  return o;
}

void orc_destroy(void* h) { delete (Oracle*)h; }

// A source plugin (kind 1 tranverseMagneticSrc, 2 pointCurrentSrc) adding into
// field `out` (Apollo's field index); params[9] as add_sources reads them.
int orc_add_source(void* h, int kind, int out, const double* params) {
  Oracle& o = *(Oracle*)h;
  if (kind < 1 || kind > 2 || out < 0 || out >= o.meqn) return 1;
  o.src_kind.push_back(kind);
  o.src_out.push_back(out);
  for (int i = 0; i < 9; ++i) o.src_par.push_back(params ? params[i] : 0.0);
  return 0;
}

// The source terms at (t, x, y) for a state q (the plugins' own value check).
void orc_source_terms(void* h, double t, double x, double y, double* s) {
  Oracle& o = *(Oracle*)h;
  double tx[5] = {t, x, y, 0.0, 0.0};
  for (int c = 0; c < o.meqn; ++c) s[c] = 0.0;
  add_sources(o, tx, s);
}
int orc_meqn(void* h) { return ((Oracle*)h)->meqn; }
int orc_np(void* h) { return ((Oracle*)h)->Np; }
int orc_nc(void* h) { return ((Oracle*)h)->Nc; }
int orc_ng(void* h) { return ((Oracle*)h)->Ng; }
int orc_error(void* h) { return ((Oracle*)h)->err; }
double orc_dtscale(void* h) { return ((Oracle*)h)->dtscale; }
double orc_rmin(void* h) { return ((Oracle*)h)->rmin; }
void orc_set_threads(void* h, int n) { ((Oracle*)h)->nthreads = n < 1 ? 1 : n; }
void orc_set_ref_plugins(void* h, void* flux, void* numflux, void* ctx) {
  Oracle* o = (Oracle*)h;
  o->ref_flux = (flux_fn)flux; o->ref_numflux = (numflux_fn)numflux; o->ref_ctx = ctx;
}
void orc_node_coords(void* h, double* x, double* y) {
  Oracle* o = (Oracle*)h;
  std::memcpy(x, o->x.data(), o->x.size() * sizeof(double));
  std::memcpy(y, o->y.data(), o->y.size() * sizeof(double));
}
void orc_connectivity(void* h, int* conn) {
  Oracle* o = (Oracle*)h;
  std::memcpy(conn, o->conn.data(), o->conn.size() * sizeof(int));
}
// Operator export for tests: which = 0 Vc, 1 Drc, 2 Dsc, 3 interp, 4 VVT, 5 cub w, 6 gauss w,
// 7 the mass matrix inv(V V^T) that the limiters average with
void orc_operator(void* h, int which, double* out) {
  Oracle* o = (Oracle*)h;
  if (which == 7) {
    std::vector<double> mass = invert(o->VVT, o->Np);
    std::memcpy(out, mass.data(), mass.size() * sizeof(double));
    return;
  }
  const std::vector<double>* v[] = {&o->Vc, &o->Drc, &o->Dsc, &o->interp, &o->VVT, &o->cw, &o->gw};
  std::memcpy(out, v[which]->data(), v[which]->size() * sizeof(double));
}

// Face node masks [3][N + 1] (the limiters' face and vertex nodes).
void orc_fmask(void* h, int* out) {
  Oracle* o = (Oracle*)h;
  std::memcpy(out, o->fmask.data(), o->fmask.size() * sizeof(int));
}
// Boundary condition `tag` (1-based, in bcs order) at one point, for tests:
// xc = [t, x, y, 0, 0], nx the unit outward normal.
void orc_apply_bc(void* h, int tag, const double* xc, const double* nx, const double* q, double* qb) {
  apply_bc(*(Oracle*)h, tag, xc, nx, q, qb);
}

// One right-hand-side evaluation, WxNodalDG2dMethod::step
// (wxnodaldg2dmethod.cc:235-542).  u, rhs: [K][Np][meqn].  Returns the
// suggested dt 2/3*cfl*dtscale*rmin/maxSpeed (:523).
double orc_rhs(void* h, double t, double dt, const double* u, double* rhs) {
  Oracle& o = *(Oracle*)h;
  const int Np = o.Np, Nc = o.Nc, Ng = o.Ng, m = o.meqn, K = o.K, NF = 3 * Ng;
  double maxSpeed = 0.0;
  std::vector<double> area(m, 0.0);
  const int nth = o.nthreads;
  std::vector<double> th_speed(nth, 0.0), th_area((size_t)nth * m, 0.0);
  auto worker = [&](int tid) {
    std::vector<double> xc5(5), q_vol(Np * m), volInt(Np * m), vec_rhs(Np * m), Iq(Nc * m), If(Nc * m), Ig(Nc * m),
        Isrc(Nc * m, 0.0), Ixc(Nc), Iyc(Nc), qtemp(Np * m), q_surf(Np * m), QP(NF * m), QM(NF * m), nflux(NF * m),
        Xc(NF), Yc(NF), qg(NF * m), qM(m), qP(m), nfl(m), F(m), G(m), myarea(m, 0.0);
    std::vector<double> xr(Nc), xs(Nc), yr(Nc), ys(Nc), Jc(Nc), rx(Nc), sx(Nc), ry(Nc), sy(Nc), RR(Nc * m), SS(Nc * m),
        CC(Nc * m), ddx(Np * m), ddy(Np * m), src(Np * m), W(NF);
    double mySpeed = 0.0;
    xc5[0] = t; xc5[4] = dt;
    const int k0 = (int)((long long)K * tid / nth), k1 = (int)((long long)K * (tid + 1) / nth);
    for (int k = k0; k < k1; ++k) {
      const double* xk = &o.x[(size_t)k * Np];
      const double* yk = &o.y[(size_t)k * Np];
      for (int i = 0; i < Np * m; ++i) q_vol[i] = u[(size_t)k * Np * m + i];
      // GeometricFactors2d / Normals2d (wxnodaldggeometry2d.cc:382-442)
      const int NpF = o.N + 1;
      double x1 = xk[o.fmask[0]], y1 = yk[o.fmask[0]], x2 = xk[o.fmask[NpF]], y2 = yk[o.fmask[NpF]],
             x3 = xk[o.fmask[2 * NpF]], y3 = yk[o.fmask[2 * NpF]];
      double dxdr = (x2 - x1) / 2, dxds = (x3 - x1) / 2, dydr = (y2 - y1) / 2, dyds = (y3 - y1) / 2;
      double Jel = -dxds * dydr + dxdr * dyds;
      if (Jel <= 0) o.err |= ERR_JAC;
      double nrm[9] = {(y2 - y1), -(x2 - x1), 0, (y3 - y2), -(x3 - x2), 0, (y1 - y3), -(x1 - x3), 0};
      for (int f = 0; f < 3; ++f) {
        double sJ = std::sqrt(nrm[3 * f] * nrm[3 * f] + nrm[3 * f + 1] * nrm[3 * f + 1]);
        nrm[3 * f] /= sJ; nrm[3 * f + 1] /= sJ; nrm[3 * f + 2] = sJ / 2.;
      }
      // volume part (:346-380)
      mat_vec(Nc, Np, m, o.Vc.data(), q_vol.data(), Iq.data());
      mat_vec(Nc, Np, 1, o.Vc.data(), xk, Ixc.data());
      mat_vec(Nc, Np, 1, o.Vc.data(), yk, Iyc.data());
      for (int p = 0; p < Nc; ++p) {
        xc5[1] = Ixc[p]; xc5[2] = Iyc[p];
        eq_flux(o, 0, &Iq[p * m], F.data());
        eq_flux(o, 1, &Iq[p * m], G.data());
        for (int c = 0; c < m; ++c) { If[p * m + c] = F[c]; Ig[p * m + c] = G[c]; Isrc[p * m + c] = 0.0; }
        // sourceTerms (src/hyper/wxhyperbolicsrcset.cc:59-71) at the cubature point
        add_sources(o, xc5.data(), &Isrc[p * m]);
      }
      // evaluatedVolumeIntegrals + geometricFactors2D (wxcubature2d.cc:297-356)
      mat_vec(Nc, Np, 1, o.Drc.data(), xk, xr.data());
      mat_vec(Nc, Np, 1, o.Drc.data(), yk, yr.data());
      mat_vec(Nc, Np, 1, o.Dsc.data(), xk, xs.data());
      mat_vec(Nc, Np, 1, o.Dsc.data(), yk, ys.data());
      for (int p = 0; p < Nc; ++p) {
        Jc[p] = xr[p] * ys[p] - xs[p] * yr[p];
        if (Jc[p] <= 0) o.err |= ERR_JAC;
        rx[p] = ys[p] / Jc[p]; sx[p] = -yr[p] / Jc[p]; ry[p] = -xs[p] / Jc[p]; sy[p] = xr[p] / Jc[p];
      }
      for (int p = 0; p < Nc; ++p)
        for (int c = 0; c < m; ++c) {
          RR[p * m + c] = o.cw[p] * Jc[p] * (rx[p] * If[p * m + c] + ry[p] * Ig[p * m + c]);
          SS[p * m + c] = o.cw[p] * Jc[p] * (sx[p] * If[p * m + c] + sy[p] * Ig[p * m + c]);
          CC[p * m + c] = o.cw[p] * Jc[p] * Isrc[p * m + c];
        }
      mat_vec(Np, Nc, m, o.DrT.data(), RR.data(), ddx.data());
      mat_vec(Np, Nc, m, o.DsT.data(), SS.data(), ddy.data());
      mat_vec(Np, Nc, m, o.VT.data(), CC.data(), src.data());
      for (int i = 0; i < Np * m; ++i) volInt[i] = ddx[i] + ddy[i] + src[i];
      // area integrals of the (zero) area terms, CalculateAreaIntegrals (:463-474)
      for (int c = 0; c < m; ++c) {
        double a = 0.0;
        for (int p = 0; p < Nc; ++p) a += o.cw[p] * 0.0 * Jc[p];
        myarea[c] += a;
      }
      // surface part (:389-472)
      mat_vec(NF, Np, m, o.interp.data(), q_vol.data(), QM.data());
      mat_vec(NF, Np, 1, o.interp.data(), xk, Xc.data());
      mat_vec(NF, Np, 1, o.interp.data(), yk, Yc.data());
      for (int f = 0; f < 3; ++f) {
        int e2 = o.conn[6 * k + 2 * f], f2 = o.conn[6 * k + 2 * f + 1];
        if (f2 < 0) {
          for (int g = 0; g < Ng; ++g) {
            xc5[1] = Xc[f * Ng + g]; xc5[2] = Yc[f * Ng + g];
            double nx[2] = {nrm[3 * f], nrm[3 * f + 1]};
            apply_bc(o, -f2, xc5.data(), nx, &QM[(f * Ng + g) * m], qP.data());
            for (int c = 0; c < m; ++c) QP[(f * Ng + g) * m + c] = qP[c];
          }
        } else {
          for (int i = 0; i < Np * m; ++i) qtemp[i] = u[(size_t)e2 * Np * m + i];
          mat_vec(NF, Np, m, o.interp.data(), qtemp.data(), qg.data());
          for (int g = 0; g < Ng; ++g)
            for (int c = 0; c < m; ++c) QP[(f * Ng + g) * m + c] = qg[(f2 * Ng + Ng - 1 - g) * m + c];
        }
      }
      for (int kk = 0; kk < NF; ++kk) {
        int ce = kk / Ng;
        for (int c = 0; c < m; ++c) { qM[c] = QM[kk * m + c]; qP[c] = QP[kk * m + c]; }
        double nx[2] = {nrm[3 * ce], nrm[3 * ce + 1]}, lambda;
        eq_numflux(o, nx, qM.data(), qP.data(), nfl.data(), &lambda);
        lambda = std::sqrt(lambda * lambda);
        mySpeed = dmax2(mySpeed, lambda);
        for (int c = 0; c < m; ++c) nflux[kk * m + c] = nfl[c] * nrm[3 * ce + 2];
      }
      // calculateSurfaceIntegral (wxcubature2d.cc:367-382)
      for (int f = 0; f < 3; ++f)
        for (int g = 0; g < Ng; ++g) W[f * Ng + g] = o.gw[g];
      for (int kk = 0; kk < NF; ++kk)
        for (int c = 0; c < m; ++c) nflux[kk * m + c] *= W[kk];
      mat_vec(Np, NF, m, o.interpT.data(), nflux.data(), q_surf.data());
      for (int i = 0; i < Np * m; ++i) {
        volInt[i] -= q_surf[i];
        if (q_surf[i] != q_surf[i] || volInt[i] != volInt[i]) o.err |= ERR_NAN;
      }
      // multiplyBYinverseMassMatrix (wxnodaldggeometry2d.cc:444-456), /J (:494-504)
      mat_vec(Np, Np, m, o.VVT.data(), volInt.data(), vec_rhs.data());
      for (int i = 0; i < Np * m; ++i) {
        rhs[(size_t)k * Np * m + i] = vec_rhs[i] / Jel;
        if (vec_rhs[i] != vec_rhs[i]) o.err |= ERR_NAN;
      }
    }
    th_speed[tid] = mySpeed;
    for (int c = 0; c < m; ++c) th_area[(size_t)tid * m + c] = myarea[c];
  };
  if (nth == 1) {
    worker(0);
  } else {
    std::vector<std::thread> pool;
    for (int i = 0; i < nth; ++i) pool.emplace_back(worker, i);
    for (auto& th : pool) th.join();
  }
  for (int i = 0; i < nth; ++i) {
    maxSpeed = dmax2(maxSpeed, th_speed[i]);
    for (int c = 0; c < m; ++c) area[c] += th_area[(size_t)i * m + c];
  }
  o.area_total = area;
  return 2. / 3. * o.cfl * o.dtscale * (o.rmin / maxSpeed);
}

// Initial dt, WxNodalDG2dMethod::init (wxnodaldg2dmethod.cc:183-228).
double orc_init_dt(void* h, const double* u) {
  Oracle& o = *(Oracle*)h;
  double maxSpeed = 0.0;
  for (int k = 0; k < o.K; ++k)
    for (int n = 0; n < o.Np; ++n) {
      double lam = std::sqrt(dmax2(0.0, eq_speed2(o, &u[((size_t)k * o.Np + n) * o.meqn])));
      maxSpeed = dmax2(maxSpeed, lam);
    }
  return 2. / 3. * o.cfl * o.dtscale * (o.rmin / maxSpeed);
}

// ---- Euler limiter "eulerLimiterHW": WxHestavenWarburtonEulerLimiter::applyLimiter
// (src/hyperapps/euler/wxhesthavenwarburtoneulerlimiter.cc:44-330), with
// LimiterElementAVE (wxnodaldggeometry2d.h:84-98) and the limiter's own
// primitiveVariables (:354-362).  5 Euler fields; orders up to 4 (at order 5
// the reference reads past its face-average array).
static void lim_prim(const Oracle& o, const double* qc, double* qp) {
  qp[0] = qc[0];
  qp[1] = qc[1] / qc[0];
  qp[2] = qc[2] / qc[0];
  qp[3] = qc[3] / qc[0];
  qp[4] = (o.lim_gamma - 1.) * (qc[4] - 0.5 * (qc[1] * qc[1] + qc[2] * qc[2] + qc[3] * qc[3]) / qc[0]);
}

// "tuAliabadiLimiter" (WxTuAliabadiLimiter::applyLimiter,
// src/hyperapps/multifluid/aptualiabadilimiter.cc:75-410) is the same patch
// procedure written against the equation set: the primitive variables come
// from the equation's primitiveVariables, which for Euler applies the density
// and pressure floors and rewrites the conserved values it was given
// (wxeulereqn.cc:1326-1341), and the reconstruction is the equation's
// limiterTuAndAliabadi: for Euler the formulas above with the equation's own
// gas_gamma, minPressure and minDensity (wxeulereqn.cc:1345-1450), for
// phMaxwellEqn every node set to the element average (wxphmaxwelleqn.cc:740-755).
static void ta_prim(const Oracle& o, double* qc, double* qp) {
  const double g = o.eqp[0], minP = o.eqp[1], minD = o.eqp[2];
  qp[0] = qc[0];
  if (qp[0] <= 0.) {
    qc[0] = minD;
    qp[0] = minD;
  }
  qp[1] = qc[1] / qc[0];
  qp[2] = qc[2] / qc[0];
  qp[3] = qc[3] / qc[0];
  qp[4] = (g - 1.) * (qc[4] - 0.5 * (qc[1] * qc[1] + qc[2] * qc[2] + qc[3] * qc[3]) / qc[0]);
  if (qp[4] <= 0.) {
    qp[4] = minP;
    qc[4] = minP / (g - 1.) + 0.5 * qp[0] * (qp[1] * qp[1] + qp[2] * qp[2] + qp[3] * qp[3]);
  }
}

// One node's limited conserved state from the cell averages (conserved cc,
// primitive cp) and the node's limited primitive deviations dq: the limiter's
// density and pressure fixes (wxhesthavenwarburtoneulerlimiter.cc:236-318;
// the same arithmetic as WxEulerEqn::limiterTuAndAliabadi, wxeulereqn.cc:1345-1450,
// whose checks ta adds).
static void lim_reconstruct(double g, double minP, double minD, const double* cc, const double* cp, const double* dq,
                            double* out, bool ta, int& err) {
  double averho = cp[0], aveu = cp[1], avev = cp[2], avew = cp[3], avep = cp[4];
  double drho = dq[0], du = dq[1], dv = dq[2], dw = dq[3], dp = dq[4];
  double Lrho = averho + drho;
  if (Lrho < minD) {
    for (int r = 0; r < 4; ++r) {
      drho *= 0.5;
      Lrho = averho + drho;
      if (Lrho > minD) break;
      else if (r == 3) Lrho = cc[0];
    }
  }
  double Lrhou = cc[1] + averho * du + drho * aveu;
  double Lrhov = cc[2] + averho * dv + drho * avev;
  double Lrhow = cc[3] + averho * dw + drho * avew;
  double dEner = dp / (g - 1.) + 0.5 * drho * (aveu * aveu + avev * avev + avew * avew) + averho * (aveu * du + avev * dv + avew * dw);
  double LEner = cc[4] + dEner;
  double Lp = (g - 1.) * (LEner - 0.5 * (Lrhou * Lrhou + Lrhov * Lrhov + Lrhow * Lrhow) / Lrho);
  if (Lp < minP) {
    for (int r = 0; r < 4; ++r) {
      dp *= 0.5;
      dEner = dp / (g - 1.) + 0.5 * drho * (aveu * aveu + avev * avev + avew * avew) + averho * (aveu * du + avev * dv + avew * dw);
      LEner = cc[4] + dEner;
      Lp = (g - 1.) * (LEner - 0.5 * (Lrhou * Lrhou + Lrhov * Lrhov + Lrhow * Lrhow) / Lrho);
      if (Lp > minP) break;
      else if (r == 3) LEner = avep / (g - 1.) + 0.5 * (Lrhou * Lrhou + Lrhov * Lrhov + Lrhow * Lrhow) / Lrho;
    }
  }
  out[0] = Lrho;
  out[1] = Lrhou;
  out[2] = Lrhov;
  out[3] = Lrhow;
  out[4] = LEner;
  if (!std::isfinite(Lrho) || !std::isfinite(LEner)) err |= ERR_NAN;
  if (ta && (!std::isfinite(Lrhou) || !std::isfinite(Lrhov))) err |= ERR_NAN;
  if (ta && Lrho <= 0.) err |= ERR_NONPHYS;
}

static void apply_limiter(Oracle& o, double* u) {
  const int K = o.K, Np = o.Np, NpF = o.N + 1, meqn = 5;
  const std::vector<double>& AVE = o.lim_ave;
  const bool ta = o.lim_kind == 1;
  if (ta && o.eq != EQ_EULER) {
    // every node of an element takes the element average, field by field
    const int m = o.meqn;
    std::vector<double> c(m);
    for (int e = 0; e < K; ++e) {
      double* q = &u[(size_t)e * Np * m];
      for (int f = 0; f < m; ++f) c[f] = 0.;
      for (int f = 0; f < m; ++f)
        for (int n = 0; n < Np; ++n) c[f] += AVE[n] * q[n * m + f];
      for (int n = 0; n < Np; ++n)
        for (int f = 0; f < m; ++f) q[n * m + f] = c[f];
    }
    return;
  }
  auto prim = [&](double* qc, double* qp) {
    if (ta) ta_prim(o, qc, qp);
    else lim_prim(o, qc, qp);
  };
  const double lim_g = ta ? o.eqp[0] : o.lim_gamma;
  const double lim_mP = ta ? o.eqp[1] : o.lim_minP;
  const double lim_mD = ta ? o.eqp[2] : o.lim_minD;
  std::vector<double> dropAVE((size_t)Np * Np);
  {
    int sk = 0;
    for (int k = 0; k < Np; ++k)
      for (int m = 0; m < Np; ++m) dropAVE[sk++] = -AVE[m];
    for (int m = 0; m < Np; ++m) dropAVE[m * Np + m] += 1.;
  }
  // GeometricFactors2d J and Normals2d (nx, ny, len/2) of every element
  std::vector<double> Jel(K), nrm((size_t)K * 9);
  for (int k = 0; k < K; ++k) {
    const double* xk = &o.x[(size_t)k * Np];
    const double* yk = &o.y[(size_t)k * Np];
    double x1 = xk[o.fmask[0]], y1 = yk[o.fmask[0]], x2 = xk[o.fmask[NpF]], y2 = yk[o.fmask[NpF]],
           x3 = xk[o.fmask[2 * NpF]], y3 = yk[o.fmask[2 * NpF]];
    double dxdr = (x2 - x1) / 2, dxds = (x3 - x1) / 2, dydr = (y2 - y1) / 2, dyds = (y3 - y1) / 2;
    Jel[k] = -dxds * dydr + dxdr * dyds;
    double n9[9] = {(y2 - y1), -(x2 - x1), 0, (y3 - y2), -(x3 - x2), 0, (y1 - y3), -(x1 - x3), 0};
    for (int f = 0; f < 3; ++f) {
      double sJ = std::sqrt(n9[3 * f] * n9[3 * f] + n9[3 * f + 1] * n9[3 * f + 1]);
      n9[3 * f] /= sJ; n9[3 * f + 1] /= sJ; n9[3 * f + 2] = sJ / 2.;
    }
    for (int i = 0; i < 9; ++i) nrm[(size_t)k * 9 + i] = n9[i];
  }
  auto X = [&](int k, int node) { return o.x[(size_t)k * Np + node]; };
  auto Y = [&](int k, int node) { return o.y[(size_t)k * Np + node]; };
  auto averages = [&](const double* qIn, double* qCons, double* qPrim) {
    double c[5] = {0., 0., 0., 0., 0.};
    for (int n = 0; n < Np; ++n)
      for (int f = 0; f < 5; ++f) c[f] += AVE[n] * qIn[n * 5 + f];
    for (int f = 0; f < 5; ++f) qCons[f] = c[f];
    prim(qCons, qPrim);
  };
  // the reference hands the boundary conditions two coordinates where they
  // read (t, x, y); only conditions that read none are accepted with the limiter
  auto bc = [&](int tag, double xa, double ya, const double* nx, const double* q, double* qb) {
    double xc[5] = {xa, ya, 0.0, 0.0, 0.0};
    apply_bc(o, tag, xc, nx, q, qb);
  };
  std::vector<double> dVdxE1((size_t)5 * K), dVdyE1((size_t)5 * K), dVdxE2((size_t)5 * K), dVdyE2((size_t)5 * K),
      dVdxE3((size_t)5 * K), dVdyE3((size_t)5 * K), dVdxC0((size_t)5 * K), dVdyC0((size_t)5 * K);
  std::vector<double> cellAVEcons((size_t)meqn * K), cellAVEprim((size_t)meqn * K);
  std::vector<double> QM(3 * NpF * meqn), QP(3 * NpF * meqn), fConsA(3 * NpF * meqn);
  for (int e = 0; e < K; ++e) {
    const int* connect = &o.conn[(size_t)e * 6];
    const double* normals = &nrm[(size_t)e * 9];
    double xc[4] = {0, 0, 0, 0}, yc[4] = {0, 0, 0, 0}, A0[4] = {0, 0, 0, 0};
    for (int kk = 0; kk < 3; ++kk) {
      xc[0] += AVE[kk] * X(e, o.fmask[kk * NpF]);
      yc[0] += AVE[kk] * Y(e, o.fmask[kk * NpF]);
      A0[0] += 2. / 3. * AVE[kk] * Jel[e];
    }
    for (int face = 0; face < 3; ++face) {
      if (connect[2 * face] < 0) {
        double H1 = 2.0 * A0[0] / normals[3 * face + 2];
        xc[face + 1] = xc[0] + 2.0 * normals[3 * face] * H1;
        yc[face + 1] = yc[0] + 2.0 * normals[3 * face + 1] * H1;
      } else {
        int nb = connect[2 * face];
        for (int node = 0; node < 3; ++node) {
          xc[face + 1] += AVE[node] * X(nb, o.fmask[node * NpF]);
          yc[face + 1] += AVE[node] * Y(nb, o.fmask[node * NpF]);
          A0[face + 1] += 2. / 3. * AVE[node] * Jel[nb];
        }
      }
    }
    for (int face = 0; face < 3; ++face) A0[face + 1] += A0[0];
    double ConsAve[5][4], PrimAve[5][4], qCons[5], qPrim[5], qBC[5];
    const double* qIn = &u[(size_t)e * Np * meqn];
    averages(qIn, qCons, qPrim);
    for (int c = 0; c < meqn; ++c) {
      ConsAve[c][0] = qCons[c];
      PrimAve[c][0] = qPrim[c];
      cellAVEprim[(size_t)e * meqn + c] = qPrim[c];
      cellAVEcons[(size_t)e * meqn + c] = qCons[c];
    }
    for (int edge = 0; edge < 3; ++edge)
      for (int n = 0; n < NpF; ++n)
        for (int c = 0; c < meqn; ++c) QM[(edge * NpF + n) * meqn + c] = qIn[o.fmask[edge * NpF + n] * meqn + c];
    // Apollo reads the patch neighbours through the same pointer as the
    // element's own nodes and never points it back
    // (wxhesthavenwarburtoneulerlimiter.cc:158, 221; aptualiabadilimiter.cc:
    // 170, 233): a boundary face listed after an interior face takes its
    // ghost nodes from that neighbour's nodes at this face's node ids.
    const double* qsrc = qIn;
    for (int el = 0; el < 3; ++el) {
      if (connect[2 * el] < 0) {
        double NX[2] = {normals[3 * el], normals[3 * el + 1]};
        for (int c = 0; c < meqn; ++c) qCons[c] = ConsAve[c][0];
        bc(-connect[2 * el], xc[el + 1], yc[el + 1], NX, qCons, qBC);
        prim(qBC, qPrim);
        for (int c = 0; c < meqn; ++c) {
          ConsAve[c][el + 1] = qBC[c];
          PrimAve[c][el + 1] = qPrim[c];
        }
        for (int n = 0; n < NpF; ++n) {
          int node = o.fmask[el * NpF + n];
          for (int c = 0; c < meqn; ++c) qCons[c] = qsrc[node * meqn + c];
          bc(-connect[2 * el], X(e, node), Y(e, node), NX, qCons, qBC);
          for (int c = 0; c < meqn; ++c) QP[(el * NpF + n) * meqn + c] = qBC[c];
        }
      } else {
        const double* qn = &u[(size_t)connect[2 * el] * Np * meqn];
        qsrc = qn;
        averages(qn, qCons, qPrim);
        for (int c = 0; c < meqn; ++c) {
          ConsAve[c][el + 1] = qCons[c];
          PrimAve[c][el + 1] = qPrim[c];
        }
        int faceNum = connect[2 * el + 1];
        for (int n = 0; n < NpF; ++n)
          for (int c = 0; c < meqn; ++c) QP[(el * NpF + n) * meqn + c] = qn[o.fmask[faceNum * NpF + NpF - 1 - n] * meqn + c];
      }
    }
    for (int i = 0; i < 3 * NpF * meqn; ++i) fConsA[i] = 0.5 * (QP[i] + QM[i]);
    int endIDs[6] = {o.fmask[0], o.fmask[NpF - 1], o.fmask[NpF], o.fmask[2 * NpF - 1], o.fmask[2 * NpF], o.fmask[3 * NpF - 1]};
    double fPrimA[6 * 5];
    for (int n = 0; n < 6 && ta; ++n) {
      double Conserved[5];
      for (int c = 0; c < meqn; ++c) Conserved[c] = fConsA[endIDs[n] * meqn + c];
      prim(Conserved, &fPrimA[n * meqn]);
    }
    for (int n = 0; n < 6 && !ta; ++n) {
      double rho = fConsA[endIDs[n] * meqn + 0], rhou = fConsA[endIDs[n] * meqn + 1],
             rhov = fConsA[endIDs[n] * meqn + 2], rhow = fConsA[endIDs[n] * meqn + 3],
             Ener = fConsA[endIDs[n] * meqn + 4];
      fPrimA[n * meqn + 0] = rho;
      fPrimA[n * meqn + 1] = rhou / rho;
      fPrimA[n * meqn + 2] = rhov / rho;
      fPrimA[n * meqn + 3] = rhow / rho;
      fPrimA[n * meqn + 4] = (o.lim_gamma - 1.) * (Ener - 0.5 * (rhou * rhou + rhov * rhov + rhow * rhow) / rho);
    }
    double xv1 = X(e, endIDs[0]), yv1 = Y(e, endIDs[0]);
    double xv2 = X(e, endIDs[2]), yv2 = Y(e, endIDs[2]);
    double xv3 = X(e, endIDs[4]), yv3 = Y(e, endIDs[4]);
    for (int c = 0; c < meqn; ++c) {
      size_t i = (size_t)meqn * e + c;
      dVdxE1[i] = 0.5 * ((PrimAve[c][1] - PrimAve[c][0]) * (yv2 - yv1) + (fPrimA[0 * meqn + c] - fPrimA[1 * meqn + c]) * (yc[1] - yc[0])) / A0[1];
      dVdyE1[i] = -0.5 * ((PrimAve[c][1] - PrimAve[c][0]) * (xv2 - xv1) + (fPrimA[0 * meqn + c] - fPrimA[1 * meqn + c]) * (xc[1] - xc[0])) / A0[1];
      dVdxE2[i] = 0.5 * ((PrimAve[c][2] - PrimAve[c][0]) * (yv3 - yv2) + (fPrimA[2 * meqn + c] - fPrimA[3 * meqn + c]) * (yc[2] - yc[0])) / A0[2];
      dVdyE2[i] = -0.5 * ((PrimAve[c][2] - PrimAve[c][0]) * (xv3 - xv2) + (fPrimA[2 * meqn + c] - fPrimA[3 * meqn + c]) * (xc[2] - xc[0])) / A0[2];
      dVdxE3[i] = 0.5 * ((PrimAve[c][3] - PrimAve[c][0]) * (yv3 - yv2) + (fPrimA[4 * meqn + c] - fPrimA[5 * meqn + c]) * (yc[3] - yc[0])) / A0[3];
      dVdyE3[i] = -0.5 * ((PrimAve[c][3] - PrimAve[c][0]) * (xv3 - xv2) + (fPrimA[4 * meqn + c] - fPrimA[5 * meqn + c]) * (xc[3] - xc[0])) / A0[3];
      dVdxC0[i] = (A0[1] * dVdxE1[i] + A0[2] * dVdxE2[i] + A0[3] * dVdxE3[i]) / (A0[1] + A0[2] + A0[3]);
      dVdyC0[i] = (A0[1] * dVdyE1[i] + A0[2] * dVdyE2[i] + A0[3] * dVdyE3[i]) / (A0[1] + A0[2] + A0[3]);
    }
  }
  std::vector<double> lim_dx(Np), lim_dy(Np), qdv((size_t)meqn * Np);
  for (int e = 0; e < K; ++e) {
    const int* connect = &o.conn[(size_t)e * 6];
    for (int i = 0; i < Np; ++i) { lim_dx[i] = 0.0; lim_dy[i] = 0.0; }
    for (int i = 0; i < Np; ++i)
      for (int j = 0; j < Np; ++j) {
        lim_dx[i] += dropAVE[i * Np + j] * X(e, j);
        lim_dy[i] += dropAVE[i * Np + j] * Y(e, j);
      }
    for (int c = 0; c < meqn; ++c) {
      double gx[3], gy[3];
      for (int edge = 0; edge < 3; ++edge) {
        size_t i = (size_t)e * meqn + c;
        if (connect[2 * edge] < 0) {
          gx[edge] = edge == 0 ? dVdxE1[i] : edge == 1 ? dVdxE2[i] : dVdxE3[i];
          gy[edge] = edge == 0 ? dVdyE1[i] : edge == 1 ? dVdyE2[i] : dVdyE3[i];
        } else {
          size_t a = (size_t)connect[2 * edge] * meqn + c;
          gx[edge] = dVdxC0[a];
          gy[edge] = dVdyC0[a];
        }
      }
      double g1 = (gx[0] * gx[0] + gy[0] * gy[0]);
      double g2 = (gx[1] * gx[1] + gy[1] * gy[1]);
      double g3 = (gx[2] * gx[2] + gy[2] * gy[2]);
      double fac = g1 * g1 + g2 * g2 + g3 * g3;
      double epse = 1.e-14;
      double fac3e = fac + 3.0 * epse;
      double w1 = (g2 * g3 + epse) / fac3e, w2 = (g1 * g3 + epse) / fac3e, w3 = (g1 * g2 + epse) / fac3e;
      double Lx = w1 * gx[0] + w2 * gx[1] + w3 * gx[2];
      double Ly = w1 * gy[0] + w2 * gy[1] + w3 * gy[2];
      for (int n = 0; n < Np; ++n) qdv[n * meqn + c] = lim_dx[n] * Lx + lim_dy[n] * Ly;
    }
    double* qOut = &u[(size_t)e * Np * meqn];
    const double* cp = &cellAVEprim[(size_t)e * meqn];
    const double* cc = &cellAVEcons[(size_t)e * meqn];
    for (int n = 0; n < Np; ++n) {
      double out[5];
      lim_reconstruct(lim_g, lim_mP, lim_mD, cc, cp, &qdv[n * meqn], out, ta, o.err);
      for (int c = 0; c < meqn; ++c) qOut[n * meqn + c] = out[c];
    }
  }
}

// One SSPRK(5,2) step, PETSc TSSSP default "rks2" with 5 stages
// (TSSSPStep_RK_2): w = u; 4x { w += dt/4 L(w) } at t0 + dt*i/4;
// u = 4/5 w + dt/5 L(w) + 1/5 u.  Returns the suggested dt of the last stage
// (ApSolver::ComputeRHSforTS, apsolver.cc:442-480).
double orc_ssp_step(void* h, double* u, double t0, double dt) {
  Oracle& o = *(Oracle*)h;
  size_t n = (size_t)o.K * o.Np * o.meqn;
  std::vector<double> w(u, u + n), F(n);
  const int s = 5;
  double sugg = 0.0;
  Oracle& oo = *(Oracle*)h;
  for (int i = 0; i < s - 1; ++i) {
    double st = t0 + dt * (i / (s - 1.));
    // the limiter rewrites the stage vector the right-hand side receives
    // (WxNodalDG2dMethod::step, wxnodaldg2dmethod.cc:243-247)
    if (oo.lim_on) apply_limiter(oo, w.data());
    orc_rhs(h, st, dt, w.data(), F.data());
    double a = dt / (s - 1.);
    for (size_t j = 0; j < n; ++j) w[j] += a * F[j];
  }
  if (oo.lim_on) apply_limiter(oo, w.data());
  sugg = orc_rhs(h, t0 + dt, dt, w.data(), F.data());
  double al = (s - 1.) / s, be = dt / s, ga = 1. / s;
  for (size_t j = 0; j < n; ++j) u[j] = al * w[j] + be * F[j] + ga * u[j];
  return sugg;
}

// Enables the Euler limiter (5 fields, N <= 4) with its gas_gamma,
// min_pressure and min_density; returns 0, or -1 if not applicable.
int orc_set_limiter(void* h, double gamma, double minP, double minD) {
  Oracle& o = *(Oracle*)h;
  if (o.eq != EQ_EULER || o.N > 4) return -1;
  o.lim_on = true;
  o.lim_kind = 0;
  o.lim_gamma = gamma;
  o.lim_minP = minP;
  o.lim_minD = minD;
  // LimiterElementAVE: half the column sums of the mass matrix inv(V V^T)
  std::vector<double> Mass = invert(o.VVT, o.Np);
  o.lim_ave.assign(o.Np, 0.0);
  for (int k = 0; k < o.Np; ++k)
    for (int m = 0; m < o.Np; ++m) o.lim_ave[k] += 0.5 * Mass[k + m * o.Np];
  return 0;
}

// Enables "tuAliabadiLimiter" (N <= 4): for eulerEqn with the equation's own
// gas_gamma, minPressure and minDensity, for phMaxwellEqn as element
// averaging; returns 0, or -1 if not applicable (advection has no
// limiterTuAndAliabadi in Apollo).
int orc_set_limiter_ta(void* h) {
  Oracle& o = *(Oracle*)h;
  if ((o.eq != EQ_EULER && o.eq != EQ_MAXWELL) || o.N > 4) return -1;
  int r = orc_set_limiter(h, o.eqp[0], o.eqp[1], o.eqp[2]);
  if (o.eq == EQ_MAXWELL) {
    o.lim_on = true;
    std::vector<double> Mass = invert(o.VVT, o.Np);
    o.lim_ave.assign(o.Np, 0.0);
    for (int k = 0; k < o.Np; ++k)
      for (int m = 0; m < o.Np; ++m) o.lim_ave[k] += 0.5 * Mass[k + m * o.Np];
    r = 0;
  }
  if (r == 0) o.lim_kind = 1;
  return r;
}

// Pinning helpers for the tuAliabadiLimiter pieces taken from the equation:
// the Euler primitive variables with their floors (qc rewritten in place), and
// one node's reconstruction with the equation's parameters.
void orc_ta_prim(void* h, double* qc, double* qp) { ta_prim(*(Oracle*)h, qc, qp); }
int orc_ta_node(void* h, const double* cc, const double* cp, const double* dq, double* out) {
  Oracle& o = *(Oracle*)h;
  int err = 0;
  lim_reconstruct(o.eqp[0], o.eqp[1], o.eqp[2], cc, cp, dq, out, true, err);
  return err;
}

// The limiter applied in place to a state u [K][Np][m].
void orc_limit(void* h, double* u) { apply_limiter(*(Oracle*)h, u); }

// Run nsteps steps (stopping early at tend) with Apollo's dt policy: the
// step's dt is min(current dt, the last stage's suggestion) for the next
// step, clipped to the frame end (apsolver.cc:421-440, 442-480).  Updates
// *t and *dt; returns the number of steps taken.
int orc_run(void* h, double* u, int nsteps, double* t, double* dt, double tend) {
  int taken = 0;
  for (int i = 0; i < nsteps; ++i) {
    if (tend > 0 && *t >= tend) break;
    double d = *dt;
    if (tend > 0 && std::fabs(tend - *t) < d) d = std::fabs(tend - *t);
    double sugg = orc_ssp_step(h, u, *t, d);
    *t += d;
    *dt = std::fmin(sugg, d);
    ++taken;
  }
  return taken;
}

}  // extern "C"
