// Reference-element operators of the nodal-DG discretisation (host, float64).
#pragma once

#include <vector>

namespace apollo {

// Dense row-major matrix.
struct Mat {
  int rows = 0, cols = 0;
  std::vector<double> a;
  Mat() = default;
  Mat(int r, int c) : rows(r), cols(c), a((size_t)r * c, 0.0) {}
  double& operator()(int i, int j) { return a[(size_t)i * cols + j]; }
  double operator()(int i, int j) const { return a[(size_t)i * cols + j]; }
};

Mat matmul(const Mat& A, const Mat& B);
Mat transpose(const Mat& A);
Mat inverse(const Mat& A);  // Gauss-Jordan with partial pivoting

// Everything the kernels need for order N, built the way Apollo builds it
// (wxnodaldggeometry2d.cc:34-91, wxcubature2d.cc:18-134):
//   nodes r, s (tabulated warp-and-blend), face mask, inverse Vandermonde,
//   cubature rule of order 3(N+1), Gauss-Legendre rule with 2(N+1) points per
//   face, and the contraction operators (see DgDev).
struct RefOps {
  int N = 0, Np = 0, Nc = 0, Ng = 0, Nf = 0;
  std::vector<double> r, s;
  std::vector<int> fmask;
  std::vector<double> cub_r, cub_s, cub_w;
  std::vector<double> gz, gw;
  Mat Vand, invV, VVT;
  Mat Vc;         // [Nc][Np]
  Mat Drc, Dsc;   // [Nc][Np] derivatives at cubature points
  Mat Interp;     // [Nf][Np]
  Mat DrW, DsW;   // [Np][Nc] = VVT Drc^T diag(w)
  Mat Lift;       // [Np][Nf] = VVT Interp^T
  std::vector<double> mass_colsum;  // [Np] integrals of the nodal basis on the reference element
  double rmin = 0.0;
  // rot[k][j]: the node at which a field rotated so that face k becomes face 0
  // takes its value (vertex i of the rotated triangle is vertex (i + k) % 3);
  // empty if the node set is not rotation symmetric to 1e-9
  std::vector<int> rot;  // [3][Np]
};

bool build_ref_ops(int N, RefOps& out);

}  // namespace apollo
