// Reference-element operators for the nodal-DG discretisation on triangles.
//
// The orthonormal simplex basis, its gradients and the Vandermonde matrices
// follow Hesthaven & Warburton, "Nodal Discontinuous Galerkin Methods" (2008),
// sections 6.1-6.2, which is also what Apollo implements in
// src/lib/wxNodalDGMatrices.h and src/lib/wxmath.h (JacobiP, GradJacobiP).
// Nodes and cubature rules are Apollo's tables (dg_tables.inc).
#include "dg_operators.h"

#include <algorithm>
#include <cmath>

#include "dg_tables.inc"

namespace apollo {

Mat matmul(const Mat& A, const Mat& B) {
  Mat C(A.rows, B.cols);
  for (int i = 0; i < A.rows; ++i)
    for (int j = 0; j < B.cols; ++j) {
      double s = 0.0;
      for (int l = 0; l < A.cols; ++l) s += A(i, l) * B(l, j);
      C(i, j) = s;
    }
  return C;
}

Mat transpose(const Mat& A) {
  Mat T(A.cols, A.rows);
  for (int i = 0; i < A.rows; ++i)
    for (int j = 0; j < A.cols; ++j) T(j, i) = A(i, j);
  return T;
}

Mat inverse(const Mat& A0) {
  const int n = A0.rows;
  Mat A = A0, X(n, n);
  for (int i = 0; i < n; ++i) X(i, i) = 1.0;
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(A(r, c)) > std::fabs(A(p, c))) p = r;
    if (p != c)
      for (int j = 0; j < n; ++j) { std::swap(A(c, j), A(p, j)); std::swap(X(c, j), X(p, j)); }
    const double piv = A(c, c);
    for (int j = 0; j < n; ++j) { A(c, j) /= piv; X(c, j) /= piv; }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = A(r, c);
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) { A(r, j) -= f * A(c, j); X(r, j) -= f * X(c, j); }
    }
  }
  return X;
}

namespace {

// Orthonormal Jacobi polynomial P_n^{(alpha,beta)}(x) by the normalised
// three-term recurrence (Hesthaven & Warburton, eq. A.2-A.3).
double jacobi(double x, double alpha, double beta, int n) {
  const double ab = alpha + beta;
  const double g0 = std::pow(2.0, ab + 1.0) / (ab + 1.0) * std::tgamma(alpha + 1.0) * std::tgamma(beta + 1.0) /
                    std::tgamma(ab + 1.0);
  double p_prev = 1.0 / std::sqrt(g0);
  if (n == 0) return p_prev;
  const double g1 = (alpha + 1.0) * (beta + 1.0) / (ab + 3.0) * g0;
  double p = ((ab + 2.0) * x / 2.0 + (alpha - beta) / 2.0) / std::sqrt(g1);
  if (n == 1) return p;
  double a_old = 2.0 / (2.0 + ab) * std::sqrt((alpha + 1.0) * (beta + 1.0) / (ab + 3.0));
  for (int i = 1; i < n; ++i) {
    const double h = 2.0 * i + ab;
    const double a_new = 2.0 / (h + 2.0) *
                         std::sqrt((i + 1) * (i + ab + 1.0) * (i + alpha + 1.0) * (i + beta + 1.0) / (h + 1.0) / (h + 3.0));
    const double b_new = -(alpha * alpha - beta * beta) / h / (h + 2.0);
    const double p_next = (-a_old * p_prev + (x - b_new) * p) / a_new;
    a_old = a_new;
    p_prev = p;
    p = p_next;
  }
  return p;
}

double djacobi(double x, double alpha, double beta, int n) {
  if (n == 0) return 0.0;
  return std::sqrt(n * (n + alpha + beta + 1.0)) * jacobi(x, alpha + 1.0, beta + 1.0, n - 1);
}

void collapse(double r, double s, double& a, double& b) {
  b = s;
  a = (s == 1.0) ? -1.0 : 2.0 * (1.0 + r) / (1.0 - s) - 1.0;
}

// phi_{ij}(r, s) on the reference triangle (mode order i outer, j inner)
double mode(double r, double s, int i, int j) {
  double a, b;
  collapse(r, s, a, b);
  return std::sqrt(2.0) * jacobi(a, 0.0, 0.0, i) * jacobi(b, 2.0 * i + 1.0, 0.0, j) * std::pow(1.0 - b, (double)i);
}

void dmode(double r, double s, int i, int j, double& dr, double& ds) {
  double a, b;
  collapse(r, s, a, b);
  const double fa = jacobi(a, 0.0, 0.0, i), dfa = djacobi(a, 0.0, 0.0, i);
  const double gb = jacobi(b, 2.0 * i + 1.0, 0.0, j), dgb = djacobi(b, 2.0 * i + 1.0, 0.0, j);
  const double h = 0.5 * (1.0 - b);
  double vr = dfa * gb, vs = dfa * gb * 0.5 * (1.0 + a);
  if (i > 0) {
    const double hp = std::pow(h, i - 1.0);
    vr *= hp;
    vs *= hp;
  }
  double tmp = dgb * std::pow(h, (double)i);
  if (i > 0) tmp -= 0.5 * i * gb * std::pow(h, i - 1.0);
  vs += fa * tmp;
  const double scale = std::pow(2.0, i + 0.5);
  dr = vr * scale;
  ds = vs * scale;
}

Mat vandermonde(int N, const std::vector<double>& r, const std::vector<double>& s) {
  const int Np = (N + 1) * (N + 2) / 2;
  Mat V((int)r.size(), Np);
  int col = 0;
  for (int i = 0; i <= N; ++i)
    for (int j = 0; j <= N - i; ++j, ++col)
      for (size_t k = 0; k < r.size(); ++k) V((int)k, col) = mode(r[k], s[k], i, j);
  return V;
}

void grad_vandermonde(int N, const std::vector<double>& r, const std::vector<double>& s, Mat& Vr, Mat& Vs) {
  const int Np = (N + 1) * (N + 2) / 2;
  Vr = Mat((int)r.size(), Np);
  Vs = Mat((int)r.size(), Np);
  int col = 0;
  for (int i = 0; i <= N; ++i)
    for (int j = 0; j <= N - i; ++j, ++col)
      for (size_t k = 0; k < r.size(); ++k) dmode(r[k], s[k], i, j, Vr((int)k, col), Vs((int)k, col));
}

// Gauss-Legendre points (ascending) and weights on [-1, 1] by Newton
// iteration on the Legendre recurrence (Numerical Recipes' gauleg, as Apollo's
// src/lib/wxmath.h:173-209, including its 3e-13 stopping tolerance).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  const double pi = 3.14159265358979323846;
  for (int i = 1; i <= (n + 1) / 2; ++i) {
    double z = std::cos(pi * (i - 0.25) / (n + 0.5)), z1, dp;
    do {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      dp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / dp;
    } while (std::fabs(z - z1) > 3.0e-13);
    x[i - 1] = -z;
    x[n - i] = z;
    w[i - 1] = 2.0 / ((1.0 - z * z) * dp * dp);
    w[n - i] = w[i - 1];
  }
}

}  // namespace

bool build_ref_ops(int N, RefOps& o) {
  if (N < 1 || N > 8) return false;
  o.N = N;
  o.Np = (N + 1) * (N + 2) / 2;
  o.r.assign(apollo_tables::kNodeR[N], apollo_tables::kNodeR[N] + o.Np);
  o.s.assign(apollo_tables::kNodeS[N], apollo_tables::kNodeS[N] + o.Np);
  o.fmask.assign(apollo_tables::kFmask[N], apollo_tables::kFmask[N] + 3 * (N + 1));
  o.rmin = std::fabs(o.r[1] - o.r[0]);
  o.Vand = vandermonde(N, o.r, o.s);
  o.invV = inverse(o.Vand);
  o.VVT = matmul(o.Vand, transpose(o.Vand));
  // cubature rule of order 3(N+1)
  o.Nc = apollo_tables::kCubNpts[N];
  o.cub_r.resize(o.Nc);
  o.cub_s.resize(o.Nc);
  o.cub_w.resize(o.Nc);
  for (int k = 0; k < o.Nc; ++k) {
    o.cub_r[k] = apollo_tables::kCubRST[N][3 * k];
    o.cub_s[k] = apollo_tables::kCubRST[N][3 * k + 1];
    o.cub_w[k] = apollo_tables::kCubRST[N][3 * k + 2];
  }
  o.Vc = matmul(vandermonde(N, o.cub_r, o.cub_s), o.invV);
  Mat Vr, Vs;
  grad_vandermonde(N, o.cub_r, o.cub_s, Vr, Vs);
  o.Drc = matmul(Vr, o.invV);
  o.Dsc = matmul(Vs, o.invV);
  // face Gauss points, faces (v0 v1), (v1 v2), (v2 v0)
  o.Ng = 2 * (N + 1);
  o.Nf = 3 * o.Ng;
  gauss_legendre(o.Ng, o.gz, o.gw);
  std::vector<double> fr(o.Nf), fs(o.Nf);
  for (int k = 0; k < o.Ng; ++k) {
    fr[k] = o.gz[k];
    fs[k] = -1.0;
    fr[o.Ng + k] = -o.gz[k];
    fs[o.Ng + k] = o.gz[k];
    fr[2 * o.Ng + k] = -1.0;
    fs[2 * o.Ng + k] = -o.gz[k];
  }
  o.Interp = matmul(vandermonde(N, fr, fs), o.invV);
  // fused contraction operators
  Mat DrcT = transpose(o.Drc), DscT = transpose(o.Dsc);
  for (int i = 0; i < o.Np; ++i)
    for (int c = 0; c < o.Nc; ++c) {
      DrcT(i, c) *= o.cub_w[c];
      DscT(i, c) *= o.cub_w[c];
    }
  o.DrW = matmul(o.VVT, DrcT);
  o.DsW = matmul(o.VVT, DscT);
  o.Lift = matmul(o.VVT, transpose(o.Interp));
  Mat Mass = inverse(o.VVT);
  o.mass_colsum.assign(o.Np, 0.0);
  for (int j = 0; j < o.Np; ++j)
    for (int i = 0; i < o.Np; ++i) o.mass_colsum[j] += Mass(i, j);
  // node permutations of the three rotations of the reference triangle
  const double vr[3] = {-1.0, 1.0, -1.0}, vs[3] = {-1.0, -1.0, 1.0};
  o.rot.assign(3 * o.Np, -1);
  bool ok = true;
  for (int k = 0; k < 3 && ok; ++k)
    for (int j = 0; j < o.Np && ok; ++j) {
      const double l1 = 0.5 * (1.0 + o.r[j]), l2 = 0.5 * (1.0 + o.s[j]), l0 = 1.0 - l1 - l2;
      const double pr = l0 * vr[k] + l1 * vr[(k + 1) % 3] + l2 * vr[(k + 2) % 3];
      const double ps = l0 * vs[k] + l1 * vs[(k + 1) % 3] + l2 * vs[(k + 2) % 3];
      int best = -1;
      double bd = 1e-9;
      for (int m = 0; m < o.Np; ++m) {
        const double dd = std::fabs(o.r[m] - pr) + std::fabs(o.s[m] - ps);
        if (dd < bd) { bd = dd; best = m; }
      }
      if (best < 0) ok = false;
      else o.rot[k * o.Np + j] = best;
    }
  if (!ok) o.rot.clear();
  return true;
}

}  // namespace apollo
