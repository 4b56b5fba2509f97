// Apollo's slope limiters "eulerLimiterHW" and "tuAliabadiLimiter"
// (WxHestavenWarburtonEulerLimiter::applyLimiter,
// src/hyperapps/euler/wxhesthavenwarburtoneulerlimiter.cc:44-330), float64,
// one thread per element in two passes:
//   pass 1: the element's four-element patch (centroids, areas), cell averages
//           of the conserved and primitive variables, averages of the face
//           traces at the patch's edge ends, and the primitive-variable
//           gradients of the three sub-triangles and of the element;
//   pass 2: gradients weighted from the neighbours' (or, on a boundary, the
//           element's own edge gradient), and the linear reconstruction of
//           the conserved variables with Apollo's density and pressure fixes.
// The arithmetic follows the reference line by line, including what it does
// that a textbook limiter would not: the patch "centroid" weights the vertex
// coordinates with the averaging weights of nodes 0..2, the third edge's
// gradient uses the second edge's vertex differences, and the face averages
// are read at positions given by element node ids.
//
// tuAliabadiLimiter (WxTuAliabadiLimiter::applyLimiter,
// src/hyperapps/multifluid/aptualiabadilimiter.cc:75-410) runs the same patch
// procedure through the equation set: for Euler the primitive variables come
// from the equation (with its density and pressure floors, which rewrite the
// averages they are given) and the equation's gas_gamma, minPressure and
// minDensity drive the reconstruction; for phMaxwellEqn the reconstruction
// returns the cell averages, so every node takes its element's average.
#include "dg_device.cuh"

namespace apollo {
namespace {

template <int M>
__device__ __forceinline__ void lim_prim(double gamma, const double* c, double* p) {
  // the limiter's primitiveVariables (no floors), 5-field order with rho w = 0 for 4 fields
  const double c3 = M == 5 ? c[3] : 0.0;
  p[0] = c[0];
  p[1] = c[1] / c[0];
  p[2] = c[2] / c[0];
  p[3] = c3 / c[0];
  p[4] = (gamma - 1.) * (c[M - 1] - 0.5 * (c[1] * c[1] + c[2] * c[2] + c3 * c3) / c[0]);
}

// The equation's primitive variables as Apollo's tuAliabadiLimiter obtains
// them (WxEulerEqn::primitiveVariables, src/hyperapps/euler/wxeulereqn.cc:1326-1341):
// density and pressure floors, which also rewrite the conserved values given.
__device__ __forceinline__ void ta_prim(double gamma, double minP, double minD, double* c, double* p) {
  p[0] = c[0];
  if (p[0] <= 0.) {
    c[0] = minD;
    p[0] = minD;
  }
  p[1] = c[1] / c[0];
  p[2] = c[2] / c[0];
  p[3] = c[3] / c[0];
  p[4] = (gamma - 1.) * (c[4] - 0.5 * (c[1] * c[1] + c[2] * c[2] + c[3] * c[3]) / c[0]);
  if (p[4] <= 0.) {
    p[4] = minP;
    c[4] = minP / (gamma - 1.) + 0.5 * p[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
  }
}

// per element: E1x E1y E2x E2y E3x E3y C0x C0y (5 each), cons average, prim average
constexpr int kLimStride = 10 * 5;

template <int EQ, int N>
__global__ void __launch_bounds__(128) k_limiter_grad(DgDev d, LimArgs L, const double* __restrict__ x,
                                                     const double* __restrict__ xn, const double* __restrict__ yn,
                                                     double* __restrict__ work) {
  constexpr int M = Eq<EQ>::M;
  constexpr int NP = Sizes<N>::NP, NPF = N + 1;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.K) return;
  const ElemGeo& g = d.geo[e];
  const double* q = x + (size_t)e * NP * M;
  auto qv = [&](const double* qe, int node, int c) { return qe[node * M + c]; };
  // Step 1: patch geometry
  double xc[4] = {0, 0, 0, 0}, yc[4] = {0, 0, 0, 0}, A0[4] = {0, 0, 0, 0};
  for (int kk = 0; kk < 3; ++kk) {
    xc[0] += L.ave[kk] * xn[(size_t)e * NP + L.fmask[kk * NPF]];
    yc[0] += L.ave[kk] * yn[(size_t)e * NP + L.fmask[kk * NPF]];
    A0[0] += 2. / 3. * L.ave[kk] * g.J;
  }
  int nb[3], nf[3];
  for (int f = 0; f < 3; ++f) {
    nb[f] = d.conn[(size_t)e * 6 + 2 * f];
    nf[f] = d.conn[(size_t)e * 6 + 2 * f + 1];
    if (nb[f] < 0) {
      const double H1 = 2.0 * A0[0] / g.sJ[f];
      xc[f + 1] = xc[0] + 2.0 * g.nx[f] * H1;
      yc[f + 1] = yc[0] + 2.0 * g.ny[f] * H1;
    } else {
      const double Jn = d.geo[nb[f]].J;
      for (int node = 0; node < 3; ++node) {
        xc[f + 1] += L.ave[node] * xn[(size_t)nb[f] * NP + L.fmask[node * NPF]];
        yc[f + 1] += L.ave[node] * yn[(size_t)nb[f] * NP + L.fmask[node * NPF]];
        A0[f + 1] += 2. / 3. * L.ave[node] * Jn;
      }
    }
  }
  for (int f = 0; f < 3; ++f) A0[f + 1] += A0[0];
  // Step 2: cell averages of the patch (5-field order)
  double cons[4][5], prim[4][5];
  auto average = [&](const double* qe, double* c) {
    double acc[M];
    for (int f = 0; f < M; ++f) acc[f] = 0.;
    for (int n = 0; n < NP; ++n)
      for (int f = 0; f < M; ++f) acc[f] += L.ave[n] * qv(qe, n, f);
    c[0] = acc[0]; c[1] = acc[1]; c[2] = acc[2]; c[3] = M == 5 ? acc[3] : 0.0; c[4] = acc[M - 1];
  };
  auto to5 = [&](const double* a, double* b) {
    b[0] = a[0]; b[1] = a[1]; b[2] = a[2]; b[3] = M == 5 ? a[3] : 0.0; b[4] = a[M - 1];
  };
  auto from5 = [&](const double* b, double* a) {
    a[0] = b[0]; a[1] = b[1]; a[2] = b[2];
    if (M == 5) a[3] = b[3];
    a[M - 1] = b[4];
  };
  // eulerLimiterHW: the limiter's own primitive variables; tuAliabadiLimiter:
  // the equation's, whose floors rewrite the averages they are given
  const bool ta = L.kind == 1;
  auto prim_of = [&](double* c, double* p) {
    if (ta) ta_prim(L.gamma, L.minP, L.minD, c, p);
    else lim_prim<5>(L.gamma, c, p);
  };
  average(q, cons[0]);
  prim_of(cons[0], prim[0]);
  for (int f = 0; f < 3; ++f) {
    if (nb[f] < 0) {
      double qa[M], qb[M];
      from5(cons[0], qa);
      apply_bc<EQ, double>(d.bcs, -nb[f], xc[f + 1], yc[f + 1], 0.0, g.nx[f], g.ny[f], qa, qb);
      to5(qb, cons[f + 1]);
      prim_of(cons[f + 1], prim[f + 1]);
    } else {
      average(x + (size_t)nb[f] * NP * M, cons[f + 1]);
      prim_of(cons[f + 1], prim[f + 1]);
    }
  }
  // Step 3: face averages at the six positions Apollo reads (fConsA at index
  // endIDs[n], an element node id, taken as a face-node position)
  double fprim[6][5];
  for (int n = 0; n < 6; ++n) {
    const int end_id = L.fmask[n == 0 ? 0 : n == 1 ? NPF - 1 : n == 2 ? NPF : n == 3 ? 2 * NPF - 1 : n == 4 ? 2 * NPF : 3 * NPF - 1];
    const int edge = end_id / NPF, nd = end_id - edge * NPF;
    const int node = L.fmask[edge * NPF + nd];
    double qm[M], qp[M];
    for (int f = 0; f < M; ++f) qm[f] = qv(q, node, f);
    if (nb[edge] < 0) {
      // Apollo reads the patch neighbours through the pointer that held this
      // element's nodes and never points it back, so the condition sees the
      // nodes of the last neighbour read before this face (faces in order;
      // this element's own where none): wxhesthavenwarburtoneulerlimiter.cc
      // :158, 221, aptualiabadilimiter.cc:170, 233
      const double* qs = q;
      for (int j = 0; j < edge; ++j)
        if (nb[j] >= 0) qs = x + (size_t)nb[j] * NP * M;
      double qin[M];
      for (int f = 0; f < M; ++f) qin[f] = qv(qs, node, f);
      apply_bc<EQ, double>(d.bcs, -nb[edge], xn[(size_t)e * NP + node], yn[(size_t)e * NP + node], 0.0, g.nx[edge],
                           g.ny[edge], qin, qp);
    } else {
      const double* qn = x + (size_t)nb[edge] * NP * M;
      const int pn = L.fmask[nf[edge] * NPF + NPF - 1 - nd];
      for (int f = 0; f < M; ++f) qp[f] = qv(qn, pn, f);
    }
    double fa[M], c5[5];
    for (int f = 0; f < M; ++f) fa[f] = 0.5 * (qp[f] + qm[f]);
    to5(fa, c5);
    if (ta) {
      ta_prim(L.gamma, L.minP, L.minD, c5, fprim[n]);
      continue;
    }
    const double rho = c5[0], rhou = c5[1], rhov = c5[2], rhow = c5[3], en = c5[4];
    fprim[n][0] = rho;
    fprim[n][1] = rhou / rho;
    fprim[n][2] = rhov / rho;
    fprim[n][3] = rhow / rho;
    fprim[n][4] = (L.gamma - 1.) * (en - 0.5 * (rhou * rhou + rhov * rhov + rhow * rhow) / rho);
  }
  // Step 4: gradients
  const double xv1 = xn[(size_t)e * NP + L.fmask[0]], yv1 = yn[(size_t)e * NP + L.fmask[0]];
  const double xv2 = xn[(size_t)e * NP + L.fmask[NPF]], yv2 = yn[(size_t)e * NP + L.fmask[NPF]];
  const double xv3 = xn[(size_t)e * NP + L.fmask[2 * NPF]], yv3 = yn[(size_t)e * NP + L.fmask[2 * NPF]];
  double* w = work + (size_t)e * kLimStride;
  for (int c = 0; c < 5; ++c) {
    const double ex1 = 0.5 * ((prim[1][c] - prim[0][c]) * (yv2 - yv1) + (fprim[0][c] - fprim[1][c]) * (yc[1] - yc[0])) / A0[1];
    const double ey1 = -0.5 * ((prim[1][c] - prim[0][c]) * (xv2 - xv1) + (fprim[0][c] - fprim[1][c]) * (xc[1] - xc[0])) / A0[1];
    const double ex2 = 0.5 * ((prim[2][c] - prim[0][c]) * (yv3 - yv2) + (fprim[2][c] - fprim[3][c]) * (yc[2] - yc[0])) / A0[2];
    const double ey2 = -0.5 * ((prim[2][c] - prim[0][c]) * (xv3 - xv2) + (fprim[2][c] - fprim[3][c]) * (xc[2] - xc[0])) / A0[2];
    // (the reference's third edge repeats the second edge's vertex differences)
    const double ex3 = 0.5 * ((prim[3][c] - prim[0][c]) * (yv3 - yv2) + (fprim[4][c] - fprim[5][c]) * (yc[3] - yc[0])) / A0[3];
    const double ey3 = -0.5 * ((prim[3][c] - prim[0][c]) * (xv3 - xv2) + (fprim[4][c] - fprim[5][c]) * (xc[3] - xc[0])) / A0[3];
    w[0 * 5 + c] = ex1; w[1 * 5 + c] = ey1;
    w[2 * 5 + c] = ex2; w[3 * 5 + c] = ey2;
    w[4 * 5 + c] = ex3; w[5 * 5 + c] = ey3;
    w[6 * 5 + c] = (A0[1] * ex1 + A0[2] * ex2 + A0[3] * ex3) / (A0[1] + A0[2] + A0[3]);
    w[7 * 5 + c] = (A0[1] * ey1 + A0[2] * ey2 + A0[3] * ey3) / (A0[1] + A0[2] + A0[3]);
    w[8 * 5 + c] = cons[0][c];
    w[9 * 5 + c] = prim[0][c];
  }
}

template <int EQ, int N>
__global__ void __launch_bounds__(128) k_limiter_apply(DgDev d, LimArgs L, const double* __restrict__ xn,
                                                      const double* __restrict__ yn,
                                                      const double* __restrict__ work, double* __restrict__ out) {
  constexpr int M = Eq<EQ>::M;
  constexpr int NP = Sizes<N>::NP;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.K) return;
  const double* w = work + (size_t)e * kLimStride;
  double lim_dx[NP], lim_dy[NP];
  for (int i = 0; i < NP; ++i) {
    double sx = 0.0, sy = 0.0;
    for (int j = 0; j < NP; ++j) {
      double drop = -L.ave[j];
      if (i == j) drop += 1.;
      sx += drop * xn[(size_t)e * NP + j];
      sy += drop * yn[(size_t)e * NP + j];
    }
    lim_dx[i] = sx;
    lim_dy[i] = sy;
  }
  double Lx[5], Ly[5];
  for (int c = 0; c < 5; ++c) {
    double gx[3], gy[3];
    for (int edge = 0; edge < 3; ++edge) {
      const int nbr = d.conn[(size_t)e * 6 + 2 * edge];
      if (nbr < 0) {
        gx[edge] = w[(2 * edge) * 5 + c];
        gy[edge] = w[(2 * edge + 1) * 5 + c];
      } else {
        const double* wn = work + (size_t)nbr * kLimStride;
        gx[edge] = wn[6 * 5 + c];
        gy[edge] = wn[7 * 5 + c];
      }
    }
    const double g1 = (gx[0] * gx[0] + gy[0] * gy[0]);
    const double g2 = (gx[1] * gx[1] + gy[1] * gy[1]);
    const double g3 = (gx[2] * gx[2] + gy[2] * gy[2]);
    const double fac = g1 * g1 + g2 * g2 + g3 * g3;
    const double epse = 1.e-14;
    const double fac3e = fac + 3.0 * epse;
    const double w1 = (g2 * g3 + epse) / fac3e;
    const double w2 = (g1 * g3 + epse) / fac3e;
    const double w3 = (g1 * g2 + epse) / fac3e;
    Lx[c] = w1 * gx[0] + w2 * gx[1] + w3 * gx[2];
    Ly[c] = w1 * gy[0] + w2 * gy[1] + w3 * gy[2];
  }
  const double gamma = L.gamma, minD = L.minD, minP = L.minP;
  const double averho = w[45 + 0], aveu = w[45 + 1], avev = w[45 + 2], avew = w[45 + 3], avep = w[45 + 4];
  const double* cons = w + 40;
  double* o = out + (size_t)e * NP * M;
  int err = 0;
  for (int n = 0; n < NP; ++n) {
    double drho = lim_dx[n] * Lx[0] + lim_dy[n] * Ly[0];
    const double du = lim_dx[n] * Lx[1] + lim_dy[n] * Ly[1];
    const double dv = lim_dx[n] * Lx[2] + lim_dy[n] * Ly[2];
    const double dw = lim_dx[n] * Lx[3] + lim_dy[n] * Ly[3];
    double dp = lim_dx[n] * Lx[4] + lim_dy[n] * Ly[4];
    double Lrho = averho + drho;
    if (Lrho < minD) {
      for (int it = 0; it < 4; ++it) {
        drho *= 0.5;
        Lrho = averho + drho;
        if (Lrho > minD) break;
        else if (it == 3) Lrho = cons[0];
      }
    }
    const double Lrhou = cons[1] + averho * du + drho * aveu;
    const double Lrhov = cons[2] + averho * dv + drho * avev;
    const double Lrhow = cons[3] + averho * dw + drho * avew;
    double dEner = dp / (gamma - 1.) + 0.5 * drho * (aveu * aveu + avev * avev + avew * avew) +
                   averho * (aveu * du + avev * dv + avew * dw);
    double LEner = cons[4] + dEner;
    double Lp = (gamma - 1.) * (LEner - 0.5 * (Lrhou * Lrhou + Lrhov * Lrhov + Lrhow * Lrhow) / Lrho);
    if (Lp < minP) {
      for (int it = 0; it < 4; ++it) {
        dp *= 0.5;
        dEner = dp / (gamma - 1.) + 0.5 * drho * (aveu * aveu + avev * avev + avew * avew) +
                averho * (aveu * du + avev * dv + avew * dw);
        LEner = cons[4] + dEner;
        Lp = (gamma - 1.) * (LEner - 0.5 * (Lrhou * Lrhou + Lrhov * Lrhov + Lrhow * Lrhow) / Lrho);
        if (Lp > minP) break;
        else if (it == 3) LEner = avep / (gamma - 1.) + 0.5 * (Lrhou * Lrhou + Lrhov * Lrhov + Lrhow * Lrhow) / Lrho;
      }
    }
    if (!isfinite(Lrho) || !isfinite(Lrhou) || !isfinite(Lrhov) || !isfinite(LEner)) err |= ERRB_NAN;
    // tuAliabadiLimiter's reconstruction (WxEulerEqn::limiterTuAndAliabadi)
    // also stops on a non-positive density
    if (L.kind == 1 && Lrho <= 0.) err |= ERRB_NONPHYS;
    o[n * M + 0] = Lrho;
    o[n * M + 1] = Lrhou;
    o[n * M + 2] = Lrhov;
    if (M == 5) o[n * M + 3] = Lrhow;
    o[n * M + M - 1] = LEner;
  }
  if (err) atomicOr(&d.st->err, err);
}

// tuAliabadiLimiter for phMaxwellEqn (WxPHMaxwellEqn::limiterTuAndAliabadi,
// src/hyperapps/maxwell/wxphmaxwelleqn.cc:740-755, returns the cell averages):
// every node of an element takes the element average, field by field, summed
// in node order.  One thread per (element, field); it reads its row before it
// writes it, so out may be x.
template <int M, int N>
__global__ void __launch_bounds__(128) k_limiter_average(int K, LimArgs L, const double* x, double* out) {
  constexpr int NP = Sizes<N>::NP;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)K * M) return;
  const long long e = t / M;
  const int f = (int)(t - e * M);
  double s = 0.0;
  for (int n = 0; n < NP; ++n) s += L.ave[n] * x[(e * NP + n) * M + f];
  for (int n = 0; n < NP; ++n) out[(e * NP + n) * M + f] = s;
}

template <int M>
cudaError_t average_n(const DgDev& d, const LimArgs& L, const double* x, double* out, cudaStream_t s) {
  const long long n = (long long)d.K * M;
  const int blocks = (int)((n + 127) / 128);
  switch (d.N) {
    case 2: k_limiter_average<M, 2><<<blocks, 128, 0, s>>>(d.K, L, x, out); break;
    case 3: k_limiter_average<M, 3><<<blocks, 128, 0, s>>>(d.K, L, x, out); break;
    case 4: k_limiter_average<M, 4><<<blocks, 128, 0, s>>>(d.K, L, x, out); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int EQ, int N>
cudaError_t limiter_t(const DgDev& d, const LimArgs& L, const double* x, double* out, const double* xn,
                      const double* yn, double* work, cudaStream_t s) {
  const int blocks = (d.K + 127) / 128;
  k_limiter_grad<EQ, N><<<blocks, 128, 0, s>>>(d, L, x, xn, yn, work);
  k_limiter_apply<EQ, N><<<blocks, 128, 0, s>>>(d, L, xn, yn, work, out);
  return cudaGetLastError();
}

template <int EQ>
cudaError_t limiter_n(const DgDev& d, const LimArgs& L, const double* x, double* out, const double* xn,
                      const double* yn, double* work, cudaStream_t s) {
  switch (d.N) {
    case 2: return limiter_t<EQ, 2>(d, L, x, out, xn, yn, work, s);
    case 3: return limiter_t<EQ, 3>(d, L, x, out, xn, yn, work, s);
    case 4: return limiter_t<EQ, 4>(d, L, x, out, xn, yn, work, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

size_t limiter_work_doubles(int K) { return (size_t)K * kLimStride; }

cudaError_t launch_limiter(int eq, const DgDev& d, const LimArgs& L, const double* x, double* out, const double* xn,
                           const double* yn, double* work, cudaStream_t s) {
  if (eq == EQ_EULER) return limiter_n<EQ_EULER>(d, L, x, out, xn, yn, work, s);
  if (eq == EQ_EULER2D) return limiter_n<EQ_EULER2D>(d, L, x, out, xn, yn, work, s);
  if (L.kind == 1 && eq == EQ_MAXWELL) return average_n<Eq<EQ_MAXWELL>::M>(d, L, x, out, s);
  if (L.kind == 1 && eq == EQ_MAXWELL_TM) return average_n<Eq<EQ_MAXWELL_TM>::M>(d, L, x, out, s);
  return cudaErrorInvalidValue;
}

}  // namespace apollo
