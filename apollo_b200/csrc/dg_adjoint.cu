// Derivatives of the float64 right-hand side, for the discrete adjoint of the
// SSPRK(5,2) stepper (no counterpart in Apollo, which has no adjoint).
//
// With q the state, the right-hand side of one element is
//   L(q) = Dr R + Ds S - (1/J) LIFT (w f*),   R = rx F(V q) + ry G(V q),
//   S = sx F(V q) + sy G(V q),  f* = f*(n, I q, partner trace or BC),
// where the face flux of an interior face is evaluated once from its first
// side (face list order) and enters the partner with the opposite sign.
//
// Tangent (forward mode), L'(q) v: the float64 volume kernel's contractions
// applied to both q and v, the pointwise fluxes in Dual<1>, the face flux in
// Dual<1>, then the float64 LIFT kernel unchanged on the tangent buffers
// (the lift and the stage update are linear).
//
// Adjoint (reverse mode), L'(q)^T w:
//   volume: a_R = Dr^T w, a_S = Ds^T w at the cubature points; per point
//           g = (rx JF + ry JG)^T a_R + (sx JF + sy JG)^T a_S with the flux
//           Jacobians JF, JG from Dual<M>; contribution V^T g.
//   faces:  s = -(1/J) LIFT^T w per element and Gauss point (k_adj_pre).
//           The Lax-Friedrichs flux is antisymmetric, f*(n, a, b) =
//           -f*(-n, b, a) (bit for bit in float64), so an element's own trace
//           a sees w_g (s_own - s_partner) d f*(n_own, a, b) / d a, with the
//           partner values gathered (no scattering); on a boundary face the
//           ghost state is differentiated through the boundary hook.
//           Contribution I^T of that.
// Stage combination in the same pass: out = alpha w + beta L'(q)^T w + gamma z.
#include <cuda_runtime.h>

#include "dg_adjoint.h"
#include "dg_dmma.cuh"
#include "dg_dual.cuh"

namespace apollo {

namespace {

constexpr int kDThreads = 256;
constexpr int kDWarps = kDThreads / 32;
constexpr int imax(int a, int b) { return a > b ? a : b; }

int g_sms = 0;
int sm_count() {
  if (g_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_sms <= 0) g_sms = 148;
  }
  return g_sms;
}

// ---------------------------------------------------------------- tangent ----
// The volume kernel's tile with a second right-hand operand (the direction).
template <int N, int M> struct TanTile {
  static constexpr int NP = Sizes<N>::NP, NC = Sizes<N>::NC, NF = Sizes<N>::NF;
  static constexpr int E = M == 1 ? 32 : ((M == 8 || N >= 4) ? 8 : 16);
  static constexpr int COLS = round_up(E * M, 8);
  static constexpr int LDB = pad_ld(COLS);
  static constexpr int NPK = round_up(NP, 4);
  static constexpr int LDA1 = pad_ld(NPK);
  static constexpr int NCR = round_up(NC, 8);
  static constexpr int NFR = round_up(NF, 8);
  static constexpr int NPR = round_up(NP, 8);
  static constexpr int K2 = round_up(2 * NC, 4);
  static constexpr int LDA2 = pad_ld(K2);
  static constexpr int RSR = imax(K2, NCR);
  static constexpr int OFF_V = 0;
  static constexpr int OFF_D = OFF_V + NCR * LDA1;
  static constexpr int OFF_I = OFF_D + NPR * LDA2;
  static constexpr int OFF_Q = OFF_I + NFR * LDA1;   // state
  static constexpr int OFF_DQ = OFF_Q + NPK * LDB;   // direction
  static constexpr int OFF_QC = OFF_DQ + NPK * LDB;  // V q
  static constexpr int OFF_RS = OFF_QC + NCR * LDB;  // V v, then the tangents of R and S
  static constexpr int TOTAL = OFF_RS + RSR * LDB;
  static constexpr size_t BYTES = sizeof(double) * TOTAL;
  static_assert(BYTES <= 227 * 1024, "tangent tile fits shared memory");
};

template <int EQ, int N>
__global__ void __launch_bounds__(kDThreads) k_tan_volume(DgDev d, const double* __restrict__ x,
                                                          const double* __restrict__ dx, double* __restrict__ dtrace,
                                                          double* __restrict__ dvol) {
  using P = Eq<EQ>;
  constexpr int M = P::M;
  using T = TanTile<N, M>;
  constexpr int NP = T::NP, NC = T::NC, NF = T::NF, E = T::E, LDB = T::LDB;
  extern __shared__ double smem[];
  double* sV = smem + T::OFF_V;
  double* sD = smem + T::OFF_D;
  double* sI = smem + T::OFF_I;
  double* sQ = smem + T::OFF_Q;
  double* sDQ = smem + T::OFF_DQ;
  double* sQC = smem + T::OFF_QC;
  double* sRS = smem + T::OFF_RS;
  const int tid = threadIdx.x;
  for (int i = tid; i < T::NCR * T::LDA1; i += kDThreads) {
    const int r = i / T::LDA1, c = i % T::LDA1;
    sV[i] = (r < NC && c < NP) ? d.V[r * NP + c] : 0.0;
  }
  for (int i = tid; i < T::NPR * T::LDA2; i += kDThreads) {
    const int r = i / T::LDA2, c = i % T::LDA2;
    double v = 0.0;
    if (r < NP && c < NC) v = d.Dr[r * NC + c];
    else if (r < NP && c >= NC && c < 2 * NC) v = d.Ds[r * NC + c - NC];
    sD[i] = v;
  }
  for (int i = tid; i < T::NFR * T::LDA1; i += kDThreads) {
    const int r = i / T::LDA1, c = i % T::LDA1;
    sI[i] = (r < NF && c < NP) ? d.I[r * NP + c] : 0.0;
  }
  for (int i = tid; i < (T::TOTAL - T::OFF_Q); i += kDThreads) sQ[i] = 0.0;
  int err = 0;
  const int ntiles = (d.K + E - 1) / E;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int k0 = tile * E;
    const int ne = min(E, d.K - k0);
    __syncthreads();
    for (int i = tid; i < ne * NP * M; i += kDThreads) {
      const int e = i / (NP * M), r = i - e * NP * M, j = r / M, f = r - j * M;
      sQ[j * LDB + e * M + f] = x[(size_t)k0 * NP * M + i];
      sDQ[j * LDB + e * M + f] = dx[(size_t)k0 * NP * M + i];
    }
    __syncthreads();
    block_dgemm<T::NCR, T::COLS, T::NPK, T::LDA1, LDB, kDWarps>(
        sV, sQ, [&](int r, int c, double v) { sQC[r * LDB + c] = v; });
    block_dgemm<T::NCR, T::COLS, T::NPK, T::LDA1, LDB, kDWarps>(
        sV, sDQ, [&](int r, int c, double v) { sRS[r * LDB + c] = v; });
    block_dgemm<T::NFR, T::COLS, T::NPK, T::LDA1, LDB, kDWarps>(sI, sQ, [&](int r, int c, double v) {
      const int e = c / M, f = c - e * M;
      if (r < NF && e < ne) d.trace[((size_t)(k0 + e) * NF + r) * M + f] = v;
    });
    block_dgemm<T::NFR, T::COLS, T::NPK, T::LDA1, LDB, kDWarps>(sI, sDQ, [&](int r, int c, double v) {
      const int e = c / M, f = c - e * M;
      if (r < NF && e < ne) dtrace[((size_t)(k0 + e) * NF + r) * M + f] = v;
    });
    __syncthreads();
    // tangents of R and S at every cubature point (row c: R, row NC + c: S;
    // row c of the direction is read before it is overwritten, by its owner)
    for (int idx = tid; idx < ne * NC; idx += kDThreads) {
      const int e = idx / NC, c = idx - e * NC;
      Dual<1> qc[M], F[M], G[M];
#pragma unroll
      for (int f = 0; f < M; ++f) {
        qc[f].v = sQC[c * LDB + e * M + f];
        qc[f].d[0] = sRS[c * LDB + e * M + f];
      }
      P::flux2(d.eqp, qc, F, G, &err);
      const ElemGeo& g = d.geo[k0 + e];
#pragma unroll
      for (int f = 0; f < M; ++f) {
        sRS[c * LDB + e * M + f] = g.rx * F[f].d[0] + g.ry * G[f].d[0];
        sRS[(NC + c) * LDB + e * M + f] = g.sx * F[f].d[0] + g.sy * G[f].d[0];
      }
    }
    __syncthreads();
    block_dgemm<T::NPR, T::COLS, T::K2, T::LDA2, LDB, kDWarps>(sD, sRS, [&](int r, int c, double v) {
      const int e = c / M, f = c - e * M;
      if (r < NP && e < ne) dvol[((size_t)(k0 + e) * NP + r) * M + f] = v;
    });
  }
  if (err) atomicOr(&d.st->err, err);
}

// Tangent of the face flux at one Gauss point per thread, written to both
// sides (the partner with the opposite sign), times sJ and the Gauss weight.
template <int EQ, int N>
__global__ void __launch_bounds__(kDThreads) k_tan_face(DgDev d, const double* __restrict__ dtrace,
                                                        double* __restrict__ dflux, double t) {
  using P = Eq<EQ>;
  constexpr int M = P::M;
  constexpr int NG = Sizes<N>::NG, NF = Sizes<N>::NF;
  int err = 0;
  const int total = d.nfaces * NG;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int fi = idx / NG, gq = idx - fi * NG;
    const FaceRec fr = d.faces[fi];
    const ElemGeo& g = d.geo[fr.k1];
    const double nx = g.nx[fr.f1], ny = g.ny[fr.f1], sJ = g.sJ[fr.f1];
    Dual<1> qM[M], qP[M], nf[M];
    const size_t om = ((size_t)fr.k1 * NF + fr.f1 * NG + gq) * M;
#pragma unroll
    for (int f = 0; f < M; ++f) {
      qM[f].v = d.trace[om + f];
      qM[f].d[0] = dtrace[om + f];
    }
    size_t op = 0;
    if (fr.k2 >= 0) {
      op = ((size_t)fr.k2 * NF + fr.f2 * NG + (NG - 1 - gq)) * M;
#pragma unroll
      for (int f = 0; f < M; ++f) {
        qP[f].v = d.trace[op + f];
        qP[f].d[0] = dtrace[op + f];
      }
    } else {
      const double z = d.gz[gq];
      double r, s;
      if (fr.f1 == 0) { r = z; s = -1.0; }
      else if (fr.f1 == 1) { r = -z; s = z; }
      else { r = -1.0; s = -z; }
      const double xx = 0.5 * (-g.vx[0] * (r + s) + g.vx[1] * (1. + r) + g.vx[2] * (1. + s));
      const double yy = 0.5 * (-g.vy[0] * (r + s) + g.vy[1] * (1. + r) + g.vy[2] * (1. + s));
      apply_bc<EQ, Dual<1>>(d.bcs, -fr.k2, t, xx, yy, Dual<1>(nx), Dual<1>(ny), qM, qP);
    }
    P::numflux(d.eqp, Dual<1>(nx), Dual<1>(ny), qM, qP, nf, &err);
    const double w = d.gw[gq] * sJ;
#pragma unroll
    for (int f = 0; f < M; ++f) dflux[om + f] = nf[f].d[0] * w;
    if (fr.k2 >= 0 && flux_two_sided<EQ>(d.eqp)) {
      // the partner's own evaluation (its normal, weight and trace as "-")
      const ElemGeo& h2 = d.geo[fr.k2];
#pragma unroll
      for (int f = 0; f < M; ++f) {
        qM[f].v = d.trace[op + f];
        qM[f].d[0] = dtrace[op + f];
        qP[f].v = d.trace[om + f];
        qP[f].d[0] = dtrace[om + f];
      }
      P::numflux(d.eqp, Dual<1>(h2.nx[fr.f2]), Dual<1>(h2.ny[fr.f2]), qM, qP, nf, &err);
      const double w2 = d.gw[NG - 1 - gq] * h2.sJ[fr.f2];
#pragma unroll
      for (int f = 0; f < M; ++f) dflux[op + f] = nf[f].d[0] * w2;
    } else if (fr.k2 >= 0) {
#pragma unroll
      for (int f = 0; f < M; ++f) dflux[op + f] = -(nf[f].d[0] * w);
    }
  }
  (void)err;  // the float64 forward reports non-physical states
}

// ---------------------------------------------------------------- adjoint ----
// Pointwise transposed Jacobian products, all inline (no calls, so the
// kernel's stack size is static).  The generic form differentiates the
// equation's own flux code with Dual<M>: it serves the linear equations
// (advection, Maxwell), where the dual arithmetic is a few multiply-adds.
// The Euler form is the reverse sweep of the same computation graph
// (state -> rho, velocities, pressure -> directional flux; Lax-Friedrichs
// with the wave speed of the primitive variables).
template <int M> struct DVec {
  double v[M];
};

// (d f*(n, a, b) / d a)^T dv and, with want_b, (d f* / d b)^T dv, by forward
// differentiation of the equation's own numerical flux (any Numerical_Flux)
template <int EQ, int M>
__device__ __forceinline__ void dual_face(const EqParams& P, double nx, double ny, const DVec<M>& a,
                                          const DVec<M>& b, const DVec<M>& dv, DVec<M>& abar, DVec<M>& bbar,
                                          bool want_b, int* err) {
  for (int side = 0; side < (want_b ? 2 : 1); ++side) {
    Dual<M> A[M], B[M], nf[M];
#pragma unroll
    for (int f = 0; f < M; ++f) {
      A[f] = Dual<M>(a.v[f]);
      B[f] = Dual<M>(b.v[f]);
      if (side == 0) A[f].d[f] = 1.0;
      else B[f].d[f] = 1.0;
    }
    Eq<EQ>::numflux(P, Dual<M>(nx), Dual<M>(ny), A, B, nf, err);
    DVec<M>& out = side == 0 ? abar : bbar;
#pragma unroll
    for (int j = 0; j < M; ++j) {
      double sum = 0.0;
#pragma unroll
      for (int f = 0; f < M; ++f) sum += dv.v[f] * nf[f].d[j];
      out.v[j] = sum;
    }
  }
}

// The same by one-component forward passes (2 M evaluations of the flux in
// Dual<1>, the instantiation the tangent kernels already use): for the Euler
// fluxes other than Lax-Friedrichs, whose Dual<M> code would be several times
// larger.
template <int EQ, int M>
__device__ __forceinline__ void dual1_face(const EqParams& P, double nx, double ny, const DVec<M>& a,
                                           const DVec<M>& b, const DVec<M>& dv, DVec<M>& abar, DVec<M>& bbar,
                                           bool want_b, int* err) {
#pragma unroll 1
  for (int side = 0; side < (want_b ? 2 : 1); ++side) {
    DVec<M>& out = side == 0 ? abar : bbar;
#pragma unroll 1
    for (int j = 0; j < M; ++j) {
      Dual<1> A[M], B[M], nf[M];
#pragma unroll
      for (int f = 0; f < M; ++f) {
        A[f] = Dual<1>(a.v[f]);
        B[f] = Dual<1>(b.v[f]);
      }
      if (side == 0) A[j].d[0] = 1.0;
      else B[j].d[0] = 1.0;
      Eq<EQ>::numflux(P, Dual<1>(nx), Dual<1>(ny), A, B, nf, err);
      double sum = 0.0;
#pragma unroll
      for (int f = 0; f < M; ++f) sum += dv.v[f] * nf[f].d[0];
      out.v[j] = sum;
    }
  }
}

template <int EQ> struct AdjPhys {
  static constexpr int M = Eq<EQ>::M;
  // (dR/dq)^T aR + (dS/dq)^T aS,  R = rx F + ry G,  S = sx F + sy G
  __device__ __forceinline__ static DVec<M> vol(const EqParams& P, const DVec<M>& q, double rx, double ry,
                                                double sx, double sy, const DVec<M>& aR, const DVec<M>& aS,
                                                int* err) {
    Dual<M> qc[M], F[M], G[M];
#pragma unroll
    for (int f = 0; f < M; ++f) {
      qc[f] = Dual<M>(q.v[f]);
      qc[f].d[f] = 1.0;
    }
    Eq<EQ>::flux2(P, qc, F, G, err);
    DVec<M> r;
#pragma unroll
    for (int j = 0; j < M; ++j) r.v[j] = 0.0;
#pragma unroll
    for (int f = 0; f < M; ++f) {
      const double cF = rx * aR.v[f] + sx * aS.v[f], cG = ry * aR.v[f] + sy * aS.v[f];
#pragma unroll
      for (int j = 0; j < M; ++j) r.v[j] += cF * F[f].d[j] + cG * G[f].d[j];
    }
    return r;
  }
  // (d f*(n, a, b) / d a)^T dv and (d f* / d b)^T dv (LF_ONLY: the caller
  // knows the flux is Lax-Friedrichs; nothing to drop here)
  template <bool LF_ONLY = false>
  __device__ __forceinline__ static void face(const EqParams& P, double nx, double ny, const DVec<M>& a,
                                              const DVec<M>& b, const DVec<M>& dv, DVec<M>& abar, DVec<M>& bbar,
                                              bool want_b, int* err) {
    dual_face<EQ, M>(P, nx, ny, a, b, dv, abar, bbar, want_b, err);
  }
};

template <int MF> struct EulerAdj {
  static constexpr int IE = MF - 1;
  // qbar += (dR/dq)^T r for the flux R along (ax, ay): reverse sweep of the
  // flux's own graph with its clamps (rho = max(q0, minD) as a constant when
  // clamped; p = minP as a constant when clamped),
  // rho, v = m / rho, p = g1 (E - rho |v|^2 / 2), u = v . a,
  // R = (rho u, rho vx u + p ax, rho vy u + p ay, [rho vz u], (E + p) u)
  __device__ __forceinline__ static void dir(const EqParams& P, const double* q, double ax, double ay,
                                             const double* r, double* qbar, int* err) {
    const double g1 = P.p[0] - 1.0, minP = P.p[1], minD = P.p[2];
    double rho = q[0];
    if (minD == 0.0 && rho <= 0.0) *err |= ERRB_NONPHYS;
    const bool rho_c = rho < minD;
    if (rho_c) rho = minD;
    const double ir = 1.0 / rho;
    const double vx = q[1] * ir, vy = q[2] * ir, vz = MF == 5 ? q[3] * ir : 0.0, E = q[IE];
    const double v2 = vx * vx + vy * vy + vz * vz;
    double p = g1 * (E - 0.5 * rho * v2);
    bool p_c = false;
    if (p <= 0.0) {
      if (minP == 0.0) *err |= ERRB_NONPHYS;
      else { p = minP; p_c = true; }
    }
    const double u = vx * ax + vy * ay;
    const double r3 = MF == 5 ? r[3] : 0.0;
    const double ub = r[0] * rho + r[1] * rho * vx + r[2] * rho * vy + r3 * rho * vz + r[IE] * (E + p);
    const double pb = p_c ? 0.0 : r[1] * ax + r[2] * ay + r[IE] * u;
    double rhob = (r[0] + r[1] * vx + r[2] * vy + r3 * vz) * u - 0.5 * g1 * v2 * pb;
    const double vxb = r[1] * rho * u + ub * ax - g1 * rho * vx * pb;
    const double vyb = r[2] * rho * u + ub * ay - g1 * rho * vy * pb;
    const double vzb = r3 * rho * u - g1 * rho * vz * pb;
    rhob -= (vxb * vx + vyb * vy + vzb * vz) * ir;
    if (!rho_c) qbar[0] += rhob;
    qbar[1] += vxb * ir;
    qbar[2] += vyb * ir;
    if (MF == 5) qbar[3] += vzb * ir;
    qbar[IE] += r[IE] * u + g1 * pb;
  }
  // Lax-Friedrichs wave speed of the primitive variables and its gradient.
  // Where the primitive variables clamp (non-physical states) the gradient is
  // taken as zero and NONPHYS is flagged.
  __device__ __forceinline__ static double speed(const EqParams& P, const double* q, double* grad, int* err) {
    const double gamma = P.p[0], g1 = gamma - 1.0, minP = P.p[1], minD = P.p[2];
    const double q3 = MF == 5 ? q[3] : 0.0;
    if (!(q[0] > 0.0)) {
      *err |= ERRB_NONPHYS;
#pragma unroll
      for (int j = 0; j < MF; ++j) grad[j] = 0.0;
      return sqrt(gamma * minP / minD);
    }
    const double rho = q[0], ir = 1.0 / rho;
    const double u = q[1] / rho, v = q[2] / rho, w = q3 / rho;
    double p = g1 * (q[IE] - 0.5 * (q[1] * q[1] + q[2] * q[2] + q3 * q3) / q[0]);
    const double sp = sqrt(u * u + v * v + w * w);
    if (p <= 0.0) {
      *err |= ERRB_NONPHYS;
#pragma unroll
      for (int j = 0; j < MF; ++j) grad[j] = 0.0;
      return sp + sqrt(gamma * minP / rho);
    }
    const double cs = sqrt(gamma * p / rho);
    const double ks = sp > 0.0 ? ir / sp : 0.0;  // d|v|/dm = v / (|v| rho)
    const double kc = 0.5 * gamma / (cs * rho);   // dcs/dp = kc, dcs/drho = -kc p / rho
    grad[0] = -sp * ir + kc * (0.5 * g1 * (u * u + v * v + w * w) - p * ir);
    grad[1] = u * ks - kc * g1 * u;
    grad[2] = v * ks - kc * g1 * v;
    if (MF == 5) grad[3] = w * ks - kc * g1 * w;
    grad[IE] = kc * g1;
    return sp + cs;
  }
};

template <int MF> struct EulerAdjPhys {
  static constexpr int M = MF;
  __device__ __forceinline__ static DVec<M> vol(const EqParams& P, const DVec<M>& q, double rx, double ry,
                                                double sx, double sy, const DVec<M>& aR, const DVec<M>& aS,
                                                int* err) {
    DVec<M> r;
#pragma unroll
    for (int j = 0; j < M; ++j) r.v[j] = 0.0;
    EulerAdj<MF>::dir(P, q.v, rx, ry, aR.v, r.v, err);
    EulerAdj<MF>::dir(P, q.v, sx, sy, aS.v, r.v, err);
    return r;
  }
  // f* = 1/2 [Fn(a) + Fn(b) + lambda (a - b)], lambda = max(c(a), c(b)):
  // abar = 1/2 [ (dFn(a)/da)^T dv + lambda dv + (dv . (a - b)) grad c(a) [a wins] ]
  // bbar = 1/2 [ (dFn(b)/db)^T dv - lambda dv + (dv . (a - b)) grad c(b) [b wins] ]
  template <bool LF_ONLY = false>
  __device__ __forceinline__ static void face(const EqParams& P, double nx, double ny, const DVec<M>& a,
                                              const DVec<M>& b, const DVec<M>& dv, DVec<M>& abar, DVec<M>& bbar,
                                              bool want_b, int* err) {
    if constexpr (!LF_ONLY) {
      if ((int)P.p[3] != NF_LF) {
        // HLL, Roe, Wave: the derivative of Apollo's own flux, quirks included
        dual1_face<MF == 5 ? EQ_EULER : EQ_EULER2D, M>(P, nx, ny, a, b, dv, abar, bbar, want_b, err);
        return;
      }
    }
    double ga[M], gb[M];
    const double ca = EulerAdj<MF>::speed(P, a.v, ga, err), cb = EulerAdj<MF>::speed(P, b.v, gb, err);
    const bool a_wins = ca > cb;  // the branch the forward flux takes
    const double lam = a_wins ? ca : cb;
    double jump = 0.0;
#pragma unroll
    for (int f = 0; f < M; ++f) jump += dv.v[f] * (a.v[f] - b.v[f]);
    double fa[M];
#pragma unroll
    for (int j = 0; j < M; ++j) fa[j] = 0.0;
    EulerAdj<MF>::dir(P, a.v, nx, ny, dv.v, fa, err);
#pragma unroll
    for (int j = 0; j < M; ++j) abar.v[j] = 0.5 * (fa[j] + lam * dv.v[j] + (a_wins ? jump * ga[j] : 0.0));
    if (want_b) {
      double fb[M];
#pragma unroll
      for (int j = 0; j < M; ++j) fb[j] = 0.0;
      EulerAdj<MF>::dir(P, b.v, nx, ny, dv.v, fb, err);
#pragma unroll
      for (int j = 0; j < M; ++j) bbar.v[j] = 0.5 * (fb[j] - lam * dv.v[j] + (a_wins ? 0.0 : jump * gb[j]));
    }
  }
};
template <> struct AdjPhys<EQ_EULER> : EulerAdjPhys<5> {};
template <> struct AdjPhys<EQ_EULER2D> : EulerAdjPhys<4> {};

template <int N, int M> struct AdjTile {
  static constexpr int NP = Sizes<N>::NP, NC = Sizes<N>::NC, NF = Sizes<N>::NF;
  static constexpr int E = M == 1 ? 32 : (M >= 5 ? 4 : 8);  // main tile <= 189 KB up to N = 5
  static constexpr int COLS = round_up(E * M, 8);
  static constexpr int LDB = pad_ld(COLS);
  static constexpr int NPK = round_up(NP, 4);   // K of V q, I q, [Dr Ds]^T w, LIFT^T w
  static constexpr int LDA1 = pad_ld(NPK);
  static constexpr int NCK = round_up(NC, 4);   // K of V^T g
  static constexpr int LDAC = pad_ld(NCK);
  static constexpr int NFK = round_up(NF, 4);   // K of I^T a
  static constexpr int LDAF = pad_ld(NFK);
  static constexpr int NCR = round_up(NC, 8);
  static constexpr int NC2R = round_up(2 * NC, 8);
  static constexpr int NFR = round_up(NF, 8);
  static constexpr int NPR = round_up(NP, 8);
  // k_adj_pre: I [NFR][LDA1], LIFT^T [NFR][LDA1], tiles q, w [NPK][LDB]
  static constexpr int PRE_I = 0, PRE_LT = PRE_I + NFR * LDA1, PRE_Q = PRE_LT + NFR * LDA1;
  static constexpr int PRE_W = PRE_Q + NPK * LDB, PRE_TOTAL = PRE_W + NPK * LDB;
  static constexpr size_t PRE_BYTES = sizeof(double) * PRE_TOTAL;
  // k_adj_main: V [NCR][LDA1], [Dr Ds]^T [NC2R][LDA1], V^T [NPR][LDAC],
  // I^T [NPR][LDAF]; tiles q, w [NPK], V q / g [NCR], a_R; a_S [NC2R],
  // face adjoint [NFR], result [NPR]
  static constexpr int M_V = 0, M_DT = M_V + NCR * LDA1, M_VT = M_DT + NC2R * LDA1;
  static constexpr int M_IT = M_VT + NPR * LDAC, M_Q = M_IT + NPR * LDAF, M_W = M_Q + NPK * LDB;
  static constexpr int M_QC = M_W + NPK * LDB, M_AB = M_QC + NCR * LDB, M_AF = M_AB + NC2R * LDB;
  static constexpr int M_OUT = M_AF + NFR * LDB, M_TOTAL = M_OUT + NPR * LDB;
  static constexpr size_t MAIN_BYTES = sizeof(double) * M_TOTAL;
  static_assert(MAIN_BYTES <= 227 * 1024 && PRE_BYTES <= 227 * 1024, "adjoint tile fits shared memory");
};

template <int M, int NP, int LDB>
__device__ __forceinline__ void load_tile(double* s, const double* __restrict__ g, int ne, int tid) {
  for (int i = tid; i < ne * NP * M; i += kDThreads) {
    const int e = i / (NP * M), r = i - e * NP * M, j = r / M, f = r - j * M;
    s[j * LDB + e * M + f] = g[i];
  }
}

// Traces I x of the stage state (into d.trace) and s = -(1/J) LIFT^T w per
// element, face Gauss point and field.
template <int EQ, int N>
__global__ void __launch_bounds__(kDThreads) k_adj_pre(DgDev d, const double* __restrict__ x,
                                                       const double* __restrict__ wbar, double* __restrict__ sbar) {
  constexpr int M = Eq<EQ>::M;
  using T = AdjTile<N, M>;
  constexpr int NP = T::NP, NF = T::NF, E = T::E, LDB = T::LDB;
  extern __shared__ double smem[];
  double* sI = smem + T::PRE_I;
  double* sLT = smem + T::PRE_LT;
  double* sQ = smem + T::PRE_Q;
  double* sW = smem + T::PRE_W;
  const int tid = threadIdx.x;
  for (int i = tid; i < T::NFR * T::LDA1; i += kDThreads) {
    const int r = i / T::LDA1, c = i % T::LDA1;
    const bool in = r < NF && c < NP;
    sI[i] = in ? d.I[r * NP + c] : 0.0;
    sLT[i] = in ? d.L[c * NF + r] : 0.0;
  }
  for (int i = tid; i < 2 * T::NPK * LDB; i += kDThreads) sQ[i] = 0.0;
  const int ntiles = (d.K + E - 1) / E;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int k0 = tile * E;
    const int ne = min(E, d.K - k0);
    __syncthreads();
    load_tile<M, NP, LDB>(sQ, x + (size_t)k0 * NP * M, ne, tid);
    load_tile<M, NP, LDB>(sW, wbar + (size_t)k0 * NP * M, ne, tid);
    __syncthreads();
    block_dgemm<T::NFR, T::COLS, T::NPK, T::LDA1, LDB, kDWarps>(sI, sQ, [&](int r, int c, double v) {
      const int e = c / M, f = c - e * M;
      if (r < NF && e < ne) d.trace[((size_t)(k0 + e) * NF + r) * M + f] = v;
    });
    block_dgemm<T::NFR, T::COLS, T::NPK, T::LDA1, LDB, kDWarps>(sLT, sW, [&](int r, int c, double v) {
      const int e = c / M, f = c - e * M;
      if (r < NF && e < ne) sbar[((size_t)(k0 + e) * NF + r) * M + f] = -d.geo[k0 + e].invJ * v;
    });
  }
}

// GEN: the general face code (boundary faces, and the Euler fluxes other
// than Lax-Friedrichs); without it, the kernel for meshes with no boundary
// face and a Lax-Friedrichs (or linear) flux, whose smaller code keeps more
// of its state in registers.
template <int EQ, int N, bool GEN>
__global__ void __launch_bounds__(kDThreads, 2) k_adj_main(DgDev d, AdjArgs a) {
  using P = Eq<EQ>;
  constexpr int M = P::M;
  using T = AdjTile<N, M>;
  constexpr int NP = T::NP, NC = T::NC, NF = T::NF, NG = Sizes<N>::NG, E = T::E, LDB = T::LDB;
  extern __shared__ double smem[];
  double* sV = smem + T::M_V;
  double* sDT = smem + T::M_DT;
  double* sVT = smem + T::M_VT;
  double* sIT = smem + T::M_IT;
  double* sQ = smem + T::M_Q;
  double* sW = smem + T::M_W;
  double* sQC = smem + T::M_QC;
  double* sAB = smem + T::M_AB;
  double* sAF = smem + T::M_AF;
  double* sOUT = smem + T::M_OUT;
  const int tid = threadIdx.x;
  for (int i = tid; i < T::NCR * T::LDA1; i += kDThreads) {
    const int r = i / T::LDA1, c = i % T::LDA1;
    sV[i] = (r < NC && c < NP) ? d.V[r * NP + c] : 0.0;
  }
  for (int i = tid; i < T::NC2R * T::LDA1; i += kDThreads) {
    const int r = i / T::LDA1, c = i % T::LDA1;
    double v = 0.0;
    if (c < NP && r < NC) v = d.Dr[c * NC + r];
    else if (c < NP && r >= NC && r < 2 * NC) v = d.Ds[c * NC + r - NC];
    sDT[i] = v;
  }
  for (int i = tid; i < T::NPR * T::LDAC; i += kDThreads) {
    const int r = i / T::LDAC, c = i % T::LDAC;
    sVT[i] = (r < NP && c < NC) ? d.V[c * NP + r] : 0.0;
  }
  for (int i = tid; i < T::NPR * T::LDAF; i += kDThreads) {
    const int r = i / T::LDAF, c = i % T::LDAF;
    sIT[i] = (r < NP && c < NF) ? d.I[c * NP + r] : 0.0;
  }
  for (int i = tid; i < T::M_TOTAL - T::M_Q; i += kDThreads) sQ[i] = 0.0;
  int err = 0;
  const int ntiles = (d.K + E - 1) / E;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int k0 = tile * E;
    const int ne = min(E, d.K - k0);
    __syncthreads();
    load_tile<M, NP, LDB>(sQ, a.x + (size_t)k0 * NP * M, ne, tid);
    load_tile<M, NP, LDB>(sW, a.wbar + (size_t)k0 * NP * M, ne, tid);
    __syncthreads();
    block_dgemm<T::NCR, T::COLS, T::NPK, T::LDA1, LDB, kDWarps>(
        sV, sQ, [&](int r, int c, double v) { sQC[r * LDB + c] = v; });
    block_dgemm<T::NC2R, T::COLS, T::NPK, T::LDA1, LDB, kDWarps>(
        sDT, sW, [&](int r, int c, double v) { sAB[r * LDB + c] = v; });
    __syncthreads();
    // volume: g = (dR/dqc)^T a_R + (dS/dqc)^T a_S at every cubature point
    for (int idx = tid; idx < ne * NC; idx += kDThreads) {
      const int e = idx / NC, c = idx - e * NC;
      const ElemGeo& g = d.geo[k0 + e];
      DVec<M> q, aR, aS;
#pragma unroll
      for (int f = 0; f < M; ++f) {
        q.v[f] = sQC[c * LDB + e * M + f];
        aR.v[f] = sAB[c * LDB + e * M + f];
        aS.v[f] = sAB[(NC + c) * LDB + e * M + f];
      }
      const DVec<M> gbar = AdjPhys<EQ>::vol(d.eqp, q, g.rx, g.ry, g.sx, g.sy, aR, aS, &err);
#pragma unroll
      for (int j = 0; j < M; ++j) sQC[c * LDB + e * M + j] = gbar.v[j];
    }
    // faces: w_g (s_own - s_partner) d f*(n_own, a, b) / d a at every Gauss point
    const bool two_sided = GEN && flux_two_sided<EQ>(d.eqp);
    for (int idx = tid; idx < ne * NF; idx += kDThreads) {
      const int e = idx / NF, fg = idx - e * NF, fc = fg / NG, gq = fg - fc * NG;
      const int k = k0 + e;
      const ElemGeo& g = d.geo[k];
      const int nb = d.conn[(size_t)k * 6 + 2 * fc];
      const size_t own = ((size_t)k * NF + fg) * M;
      DVec<M> abar;
      if (nb >= 0) {
        const int f2 = d.conn[(size_t)k * 6 + 2 * fc + 1];
        const size_t par = ((size_t)nb * NF + f2 * NG + (NG - 1 - gq)) * M;
        // the flux's Gauss weight is its first side's (face list: 3 nb + f2 > 3 k + fc)
        const double w = d.gw[(3 * nb + f2 > 3 * k + fc) ? gq : NG - 1 - gq] * g.sJ[fc];
        DVec<M> qa, qb, dvec;
        if (two_sided) {
          // each side holds its own evaluation f*(n_side, own, partner) times
          // its own weight (the forward face kernel's two-sided form): the
          // own slot differentiated in its first argument, the partner's in
          // its second
          const ElemGeo& h2 = d.geo[nb];
          const double w1 = d.gw[gq] * g.sJ[fc], w2 = d.gw[NG - 1 - gq] * h2.sJ[f2];
          DVec<M> dv2, unused, bbar;
#pragma unroll
          for (int f = 0; f < M; ++f) {
            qa.v[f] = d.trace[own + f];
            qb.v[f] = d.trace[par + f];
            dvec.v[f] = w1 * a.sbar[own + f];
            dv2.v[f] = w2 * a.sbar[par + f];
          }
          AdjPhys<EQ>::face(d.eqp, g.nx[fc], g.ny[fc], qa, qb, dvec, abar, unused, false, &err);
          AdjPhys<EQ>::face(d.eqp, h2.nx[f2], h2.ny[f2], qb, qa, dv2, unused, bbar, true, &err);
#pragma unroll
          for (int j = 0; j < M; ++j) abar.v[j] += bbar.v[j];
        } else {
#pragma unroll
        for (int f = 0; f < M; ++f) {
          qa.v[f] = d.trace[own + f];
          qb.v[f] = d.trace[par + f];
          dvec.v[f] = w * (a.sbar[own + f] - a.sbar[par + f]);
        }
        DVec<M> unused;
        AdjPhys<EQ>::template face<!GEN>(d.eqp, g.nx[fc], g.ny[fc], qa, qb, dvec, abar, unused, false, &err);
        }
      } else if constexpr (!GEN) {
        // (the host launches this form only for meshes without boundary faces)
#pragma unroll
        for (int j = 0; j < M; ++j) abar.v[j] = 0.0;
      } else {
        // boundary: ghost state b = A a + c (every supported boundary hook is
        // affine in the trace); abar = (df*/da)^T dv + A^T (df*/db)^T dv
        const double w = d.gw[gq] * g.sJ[fc];
        const double z = d.gz[gq];
        double r, s;
        if (fc == 0) { r = z; s = -1.0; }
        else if (fc == 1) { r = -z; s = z; }
        else { r = -1.0; s = -z; }
        const double xx = 0.5 * (-g.vx[0] * (r + s) + g.vx[1] * (1. + r) + g.vx[2] * (1. + s));
        const double yy = 0.5 * (-g.vy[0] * (r + s) + g.vy[1] * (1. + r) + g.vy[2] * (1. + s));
        DVec<M> qa, qb, dvec, bbar;
        double unit[M], col[M], base[M], zero[M];
#pragma unroll
        for (int f = 0; f < M; ++f) {
          qa.v[f] = d.trace[own + f];
          dvec.v[f] = w * a.sbar[own + f];
          zero[f] = 0.0;
        }
        apply_bc<EQ, double>(d.bcs, -nb, a.t, xx, yy, g.nx[fc], g.ny[fc], qa.v, qb.v);
        AdjPhys<EQ>::face(d.eqp, g.nx[fc], g.ny[fc], qa, qb, dvec, abar, bbar, true, &err);
        apply_bc<EQ, double>(d.bcs, -nb, a.t, xx, yy, g.nx[fc], g.ny[fc], zero, base);
#pragma unroll
        for (int j = 0; j < M; ++j) {
#pragma unroll
          for (int f = 0; f < M; ++f) unit[f] = f == j ? 1.0 : 0.0;
          apply_bc<EQ, double>(d.bcs, -nb, a.t, xx, yy, g.nx[fc], g.ny[fc], unit, col);
          double sum = 0.0;
#pragma unroll
          for (int f = 0; f < M; ++f) sum += (col[f] - base[f]) * bbar.v[f];
          abar.v[j] += sum;
        }
      }
#pragma unroll
      for (int j = 0; j < M; ++j) sAF[fg * LDB + e * M + j] = abar.v[j];
    }
    __syncthreads();
    block_dgemm<T::NPR, T::COLS, T::NCK, T::LDAC, LDB, kDWarps>(
        sVT, sQC, [&](int r, int c, double v) { sOUT[r * LDB + c] = v; });
    __syncthreads();
    block_dgemm<T::NPR, T::COLS, T::NFK, T::LDAF, LDB, kDWarps>(
        sIT, sAF, [&](int r, int c, double v) { sOUT[r * LDB + c] += v; });
    __syncthreads();
    for (int i = tid; i < ne * NP * M; i += kDThreads) {
      const int e = i / (NP * M), rr = i - e * NP * M, j = rr / M, f = rr - j * M;
      const size_t off = (size_t)k0 * NP * M + i;
      double o = a.beta * sOUT[j * LDB + e * M + f];
      if (a.alpha != 0.0) o += a.alpha * a.wbar[off];
      if (a.z) o += a.gamma * a.z[off];
      a.out[off] = o;
    }
  }
  (void)err;
}

// Shared-memory size of a tile kernel and, once per device, how many of its
// blocks are resident per SM (registers and shared memory): the persistent
// grids launch that many, since a block beyond them would start a late
// second wave.
template <class Kern>
cudaError_t set_smem(Kern k, size_t bytes, unsigned& configured, int& resident) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (configured & (1u << (dev & 31))) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k, kDThreads, bytes);
  if (e == cudaSuccess) configured |= 1u << (dev & 31);
  return e;
}

int tile_grid(int K, int E, int resident) {
  const int per = resident < 1 ? 1 : (resident > 8 ? 8 : resident);
  const int tiles = (K + E - 1) / E;
  const int g = sm_count() * per;
  return g < tiles ? g : tiles;
}

template <int EQ, int N>
cudaError_t tangent_t(const DgDev& d, const TanArgs& a, cudaStream_t s) {
  constexpr int M = Eq<EQ>::M;
  using T = TanTile<N, M>;
  static unsigned configured = 0;
  static int resident = 1;
  cudaError_t e = set_smem(k_tan_volume<EQ, N>, T::BYTES, configured, resident);
  if (e != cudaSuccess) return e;
  k_tan_volume<EQ, N><<<tile_grid(d.K, T::E, resident), kDThreads, T::BYTES, s>>>(d, a.x, a.dx, a.dtrace, a.dvol);
  const int fthreads = d.nfaces * Sizes<N>::NG;
  int gf = (fthreads + kDThreads - 1) / kDThreads;
  if (gf > sm_count() * 8) gf = sm_count() * 8;
  if (gf < 1) gf = 1;
  k_tan_face<EQ, N><<<gf, kDThreads, 0, s>>>(d, a.dtrace, a.dflux, a.t);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // the LIFT kernel and the stage update on the tangent buffers
  DgDev dt = d;
  dt.vol = a.dvol;
  dt.flux = a.dflux;
  StageArgs sa{};
  sa.x = a.dx;
  sa.u0 = a.du0;
  sa.out = a.dout;
  sa.mode = a.mode;
  sa.time_from_state = 0;
  sa.t_arg = a.t;
  sa.dt_arg = a.dt;
  return launch_lift_fp64(EQ, dt, sa, s);
}

template <int EQ, int N>
cudaError_t adjoint_t(const DgDev& d, const AdjArgs& a, cudaStream_t s) {
  constexpr int M = Eq<EQ>::M;
  using T = AdjTile<N, M>;
  static unsigned cpre = 0, cmain = 0;
  static int rpre = 1, rmain = 1;
  cudaError_t e = set_smem(k_adj_pre<EQ, N>, T::PRE_BYTES, cpre, rpre);
  if (e != cudaSuccess) return e;
  static unsigned clean = 0;
  static int rlean = 1;
  e = set_smem(k_adj_main<EQ, N, true>, T::MAIN_BYTES, cmain, rmain);
  if (e != cudaSuccess) return e;
  e = set_smem(k_adj_main<EQ, N, false>, T::MAIN_BYTES, clean, rlean);
  if (e != cudaSuccess) return e;
  k_adj_pre<EQ, N><<<tile_grid(d.K, T::E, rpre), kDThreads, T::PRE_BYTES, s>>>(d, a.x, a.wbar, a.sbar);
  const bool lf = !(EQ == EQ_EULER || EQ == EQ_EULER2D) || (int)d.eqp.p[3] == NF_LF;
  if (d.nbound == 0 && lf)
    k_adj_main<EQ, N, false><<<tile_grid(d.K, T::E, rlean), kDThreads, T::MAIN_BYTES, s>>>(d, a);
  else
    k_adj_main<EQ, N, true><<<tile_grid(d.K, T::E, rmain), kDThreads, T::MAIN_BYTES, s>>>(d, a);
  return cudaGetLastError();
}

template <int EQ>
cudaError_t tangent_n(const DgDev& d, const TanArgs& a, cudaStream_t s) {
  switch (d.N) {
    case 2: return tangent_t<EQ, 2>(d, a, s);
    case 3: return tangent_t<EQ, 3>(d, a, s);
    case 4: return tangent_t<EQ, 4>(d, a, s);
    case 5: return tangent_t<EQ, 5>(d, a, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int EQ>
cudaError_t adjoint_n(const DgDev& d, const AdjArgs& a, cudaStream_t s) {
  switch (d.N) {
    case 2: return adjoint_t<EQ, 2>(d, a, s);
    case 3: return adjoint_t<EQ, 3>(d, a, s);
    case 4: return adjoint_t<EQ, 4>(d, a, s);
    case 5: return adjoint_t<EQ, 5>(d, a, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t launch_tangent_stage(int eq, const DgDev& d, const TanArgs& a, cudaStream_t s) {
  switch (eq) {
    case EQ_ADVECTION: return tangent_n<EQ_ADVECTION>(d, a, s);
    case EQ_EULER: return tangent_n<EQ_EULER>(d, a, s);
    case EQ_MAXWELL: return tangent_n<EQ_MAXWELL>(d, a, s);
    case EQ_EULER2D: return tangent_n<EQ_EULER2D>(d, a, s);
    case EQ_MAXWELL_TM: return tangent_n<EQ_MAXWELL_TM>(d, a, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_adjoint_stage(int eq, const DgDev& d, const AdjArgs& a, cudaStream_t s) {
  switch (eq) {
    case EQ_ADVECTION: return adjoint_n<EQ_ADVECTION>(d, a, s);
    case EQ_EULER: return adjoint_n<EQ_EULER>(d, a, s);
    case EQ_MAXWELL: return adjoint_n<EQ_MAXWELL>(d, a, s);
    case EQ_EULER2D: return adjoint_n<EQ_EULER2D>(d, a, s);
    case EQ_MAXWELL_TM: return adjoint_n<EQ_MAXWELL_TM>(d, a, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace apollo
