// Float64 nodal-DG right-hand side on sm_100a: one volume kernel, one face
// kernel and one LIFT kernel with the SSP stage update fused in, per stage.
//
//  k_volume  : per element tile, q -> cubature values (V), physical flux at
//              every cubature point, volume contraction with the weighted
//              derivative operators (Dr, Ds) and the face traces (I q).
//              Apollo: wxnodaldg2dmethod.cc:346-394 with
//              wxcubature2d.cc:290-363.
//  k_face    : per face Gauss point, both traces through the face map (the
//              partner in reversed Gauss order), boundary hook, Lax-Friedrichs
//              flux, times sJ and the Gauss weight, written to both sides, and
//              the max wave speed.  Apollo: wxnodaldg2dmethod.cc:396-469.
//  k_lift    : per element tile, surface contraction (L = VVT I^T), 1/J,
//              combination with the volume term and the stage update.
//              Apollo: wxcubature2d.cc:367-382, wxnodaldggeometry2d.cc:444-456,
//              wxnodaldg2dmethod.cc:475-504; PETSc TSSSP RK_2 update.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dg_device.cuh"
#include "dg_dmma.cuh"

namespace apollo {

namespace {

constexpr int kThreads = 256;

// Euler fluxes in float64 with one reciprocal of the density per state and
// the flux formed along a direction directly (a n.F + b n.G in one pass): the
// same quantities as WxEulerEqn's flux and Lax-Friedrichs flux
// (wxeulereqn.cc:809-871, :1097-1117) to round-off, for states that need none
// of the reference's clamps; a state that does (density below its floor or
// not positive, pressure not positive) takes the equation's own code, which
// applies them and raises its error flags.
template <int MF> struct EulerFast64 {
  static constexpr int IE = MF - 1;
  struct Side {
    double rho, ir, vx, vy, vz, p;
    bool clean;
  };
  __device__ __forceinline__ static Side side(const EqParams& P, const double* q) {
    const double g1 = P.p[0] - 1.0, minD = P.p[2];
    Side s;
    s.rho = q[0];
    s.ir = 1.0 / s.rho;
    s.vx = q[1] * s.ir;
    s.vy = q[2] * s.ir;
    s.vz = MF == 5 ? q[3] * s.ir : 0.0;
    s.p = g1 * (q[IE] - 0.5 * s.rho * (s.vx * s.vx + s.vy * s.vy + s.vz * s.vz));
    s.clean = s.rho > 0.0 && s.rho >= minD && s.p > 0.0;
    return s;
  }
  // the flux along (ax, ay): ax F + ay G
  __device__ __forceinline__ static void along(const Side& s, const double* q, double ax, double ay, double* R) {
    const double ua = s.vx * ax + s.vy * ay;
    R[0] = s.rho * ua;
    R[1] = s.rho * s.vx * ua + s.p * ax;
    R[2] = s.rho * s.vy * ua + s.p * ay;
    if (MF == 5) R[3] = s.rho * s.vz * ua;
    R[IE] = (q[IE] + s.p) * ua;
  }
};

template <int EQ> constexpr bool kEulerEq = EQ == EQ_EULER || EQ == EQ_EULER2D;

// R = rx F + ry G, S = sx F + sy G of one state
template <int EQ>
__device__ __forceinline__ void volume_flux(const EqParams& P, const double* q, double rx, double ry, double sx,
                                            double sy, double* R, double* S, int* err) {
  constexpr int M = Eq<EQ>::M;
  if constexpr (kEulerEq<EQ>) {
    using X = EulerFast64<M>;
    const typename X::Side sd = X::side(P, q);
    if (sd.clean) {
      X::along(sd, q, rx, ry, R);
      X::along(sd, q, sx, sy, S);
      return;
    }
  }
  double F[M], G[M];
  Eq<EQ>::flux2(P, q, F, G, err);
#pragma unroll
  for (int f = 0; f < M; ++f) {
    R[f] = rx * F[f] + ry * G[f];
    S[f] = sx * F[f] + sy * G[f];
  }
}

// The numerical flux of one face point (qM, qP may be modified as the
// reference modifies them); the Euler Lax-Friedrichs flux of two clean states
// through EulerFast64
template <int EQ>
__device__ __forceinline__ double face_flux(const EqParams& P, double nx, double ny, double* qM, double* qP,
                                            double* nf, int* err) {
  constexpr int M = Eq<EQ>::M;
  if constexpr (kEulerEq<EQ>) {
    const int kind = (int)P.p[3];
    if (kind != NF_HLL && kind != NF_ROE && kind != NF_WAVE) {
      using X = EulerFast64<M>;
      const typename X::Side a = X::side(P, qM), b = X::side(P, qP);
      if (a.clean && b.clean) {
        double FM[M], FP[M];
        X::along(a, qM, nx, ny, FM);
        X::along(b, qP, nx, ny, FP);
        const double gamma = P.p[0];
        const double cM = sqrt(a.vx * a.vx + a.vy * a.vy + a.vz * a.vz) + sqrt(gamma * a.p * a.ir);
        const double cP = sqrt(b.vx * b.vx + b.vy * b.vy + b.vz * b.vz) + sqrt(gamma * b.p * b.ir);
        const double lam = cM > cP ? cM : cP;
#pragma unroll
        for (int c = 0; c < M; ++c) nf[c] = 0.5 * (FM[c] + FP[c] + lam * (qM[c] - qP[c]));
        return lam;
      }
    }
  }
  return Eq<EQ>::numflux(P, nx, ny, qM, qP, nf, err);
}


// Tile of elements for the float64 volume kernel.  Columns of every GEMM are
// (element, field) pairs; rows are cubature points, Gauss points or nodes.
template <int N, int M> struct VolTile {
  static constexpr int NP = Sizes<N>::NP, NC = Sizes<N>::NC, NF = Sizes<N>::NF;
  // 16 elements per tile (8 for 8 fields or N >= 5), 64 for scalar advection,
  // keeping the tile near 110 KB of shared memory (two blocks per SM)
  static constexpr int E = M == 1 ? 64 : ((M == 8 || N >= 5) ? 8 : 16);
  static constexpr int COLS = round_up(E * M, 8);
  static constexpr int LDB = pad_ld(COLS);
  static constexpr int NPK = round_up(NP, 4);    // K of V*q and I*q
  static constexpr int LDA1 = pad_ld(NPK);
  static constexpr int NCR = round_up(NC, 8);    // rows of V*q
  static constexpr int NFR = round_up(NF, 8);    // rows of I*q
  static constexpr int NPR = round_up(NP, 8);    // rows of D*[R;S]
  static constexpr int K2 = round_up(2 * NC, 4); // K of D*[R;S]
  static constexpr int LDA2 = pad_ld(K2);
  static constexpr int RSR = K2 > NCR ? K2 : NCR;
  static constexpr int OFF_V = 0;
  static constexpr int OFF_D = OFF_V + NCR * LDA1;
  static constexpr int OFF_I = OFF_D + NPR * LDA2;
  static constexpr int OFF_Q = OFF_I + NFR * LDA1;
  static constexpr int OFF_RS = OFF_Q + NPK * LDB;
  static constexpr int TOTAL = OFF_RS + RSR * LDB;
  static constexpr size_t BYTES = sizeof(double) * TOTAL;
};

template <int EQ, int N>
__global__ void __launch_bounds__(kThreads) k_volume(DgDev d, StageArgs a) {
  using P = Eq<EQ>;
  constexpr int M = P::M;
  using T = VolTile<N, M>;
  constexpr int NP = T::NP, NC = T::NC, NF = T::NF, E = T::E, LDB = T::LDB;
  constexpr int NWARPS = kThreads / 32;
  extern __shared__ double smem[];
  double* sV = smem + T::OFF_V;
  double* sD = smem + T::OFF_D;
  double* sI = smem + T::OFF_I;
  double* sQ = smem + T::OFF_Q;
  double* sRS = smem + T::OFF_RS;
  const int tid = threadIdx.x;
  if (a.reset_lambda && blockIdx.x == 0)
    for (int i = tid; i < d.ninst; i += kThreads) d.st[i].lam_bits = 0ull;
  // operators, zero-padded: V [NCR][NPK], D = [Dr | Ds] [NPR][K2], I [NFR][NPK]
  for (int i = tid; i < T::NCR * T::LDA1; i += kThreads) {
    const int r = i / T::LDA1, c = i % T::LDA1;
    sV[i] = (r < NC && c < NP) ? d.V[r * NP + c] : 0.0;
  }
  for (int i = tid; i < T::NPR * T::LDA2; i += kThreads) {
    const int r = i / T::LDA2, c = i % T::LDA2;
    double v = 0.0;
    if (r < NP && c < NC) v = d.Dr[r * NC + c];
    else if (r < NP && c >= NC && c < 2 * NC) v = d.Ds[r * NC + c - NC];
    sD[i] = v;
  }
  for (int i = tid; i < T::NFR * T::LDA1; i += kThreads) {
    const int r = i / T::LDA1, c = i % T::LDA1;
    sI[i] = (r < NF && c < NP) ? d.I[r * NP + c] : 0.0;
  }
  // padding rows of the right-hand operands stay zero
  for (int i = tid; i < T::NPK * LDB; i += kThreads) sQ[i] = 0.0;
  for (int i = tid; i < T::RSR * LDB; i += kThreads) sRS[i] = 0.0;
  int err = 0;
  const int ntiles = (d.K + E - 1) / E;
  // q tile, [e][node][field] -> Q[node][e*M + field]: the first tile here, each
  // next one loaded into registers while this one's fluxes are evaluated and
  // stored after them (Q is read only by the first two contractions)
  constexpr int NQ = E * NP * M, QPT = (NQ + kThreads - 1) / kThreads;
  auto put_q = [&](int i, double v) {
    const int e = i / (NP * M), r = i - e * NP * M, j = r / M, f = r - j * M;
    sQ[j * LDB + e * M + f] = v;
  };
  __syncthreads();  // the zero padding above is written before the first tile
  if ((int)blockIdx.x < ntiles) {
    const int k0 = blockIdx.x * E, nq = min(E, d.K - k0) * NP * M;
    const double* src = a.x + (size_t)k0 * NP * M;
    for (int i = tid; i < nq; i += kThreads) put_q(i, src[i]);
  }
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int k0 = tile * E;
    const int ne = min(E, d.K - k0);
    __syncthreads();
    // cubature values Qc = V Q (into the R/S buffer) and face traces I Q (to HBM)
    block_dgemm<T::NCR, T::COLS, T::NPK, T::LDA1, LDB, NWARPS>(
        sV, sQ, [&](int r, int c, double v) { sRS[r * LDB + c] = v; });
    block_dgemm<T::NFR, T::COLS, T::NPK, T::LDA1, LDB, NWARPS>(sI, sQ, [&](int r, int c, double v) {
      const int e = c / M, f = c - e * M;
      if (r < NF && e < ne) d.trace[((size_t)(k0 + e) * NF + r) * M + f] = v;
    });
    __syncthreads();
    // the next tile's states, in flight during the flux evaluation
    const int nxt = tile + (int)gridDim.x;
    const int nq_next = nxt < ntiles ? min(E, d.K - nxt * E) * NP * M : 0;
    double qn[QPT];
#pragma unroll
    for (int u = 0; u < QPT; ++u) {
      const int i = tid + u * kThreads;
      qn[u] = i < nq_next ? a.x[(size_t)nxt * E * NP * M + i] : 0.0;
    }
    // physical flux at every cubature point; R = rx F + ry G into row c,
    // S = sx F + sy G into row NC + c (row c is overwritten by its reader only)
    for (int idx = tid; idx < ne * NC; idx += kThreads) {
      const int e = idx / NC, c = idx - e * NC;
      double qc[M], R[M], S[M];
#pragma unroll
      for (int f = 0; f < M; ++f) qc[f] = sRS[c * LDB + e * M + f];
      const ElemGeo& g = d.geo[k0 + e];
      volume_flux<EQ>(d.eqp, qc, g.rx, g.ry, g.sx, g.sy, R, S, &err);
#pragma unroll
      for (int f = 0; f < M; ++f) {
        sRS[c * LDB + e * M + f] = R[f];
        sRS[(NC + c) * LDB + e * M + f] = S[f];
      }
    }
#pragma unroll
    for (int u = 0; u < QPT; ++u) {
      const int i = tid + u * kThreads;
      if (i < nq_next) put_q(i, qn[u]);
    }
    __syncthreads();
    // volume term: [Dr | Ds] [R; S]
    block_dgemm<T::NPR, T::COLS, T::K2, T::LDA2, LDB, NWARPS, 4>(sD, sRS, [&](int r, int c, double v) {
      const int e = c / M, f = c - e * M;
      if (r < NP && e < ne) d.vol[((size_t)(k0 + e) * NP + r) * M + f] = v;
    });
  }
  if (err) atomicOr(&d.st->err, err);
}

// Tile of the fused float64 stage: the volume and surface terms of E elements
// and the stage update in one pass.  Shared memory (doubles):
//   V  [NCR][LDA1]             nodal values -> cubature points
//   DL [NPR][LDA2]             [Dr | Ds | L], K2 = 2 NC + NF (+ zero padding)
//   I  [NFR][LDA1]             nodal values -> face Gauss points
//   Q  [NPK][LDB]              the tile's states, column e M + f
//   PB [NPK][LDP]              the neighbour across face j of element e, column (3 e + j) M + f
//   T  [NFR][LDB]              the tile's face traces I q
//   TP [E][3][NG][M]           the neighbours' traces on the shared faces, in this side's Gauss order
//   RS [K2][LDB]               cubature values, then R (rows 0..NC-1), S (NC..2NC-1)
//                              and -(1/J) sJ w_g times the numerical flux (2NC..)
//   GS [E][16]                 rx, ry, sx, sy, 1/J, dt, nx[3], ny[3], sJ[3] of each element
//   F2 [E][3] int              the neighbour's face index (-1: boundary)
// E is the largest of a few candidates whose tile leaves two blocks per SM
// (the smallest one otherwise).
template <int N, int M> struct StageTile {
  static constexpr int NP = Sizes<N>::NP, NC = Sizes<N>::NC, NF = Sizes<N>::NF, NG = Sizes<N>::NG;
  static constexpr int NPM = NP * M;
  static constexpr int NPK = round_up(NP, 4);
  static constexpr int LDA1 = pad_ld(NPK);
  static constexpr int NCR = round_up(NC, 8);
  static constexpr int NFR = round_up(NF, 8);
  static constexpr int NPR = round_up(NP, 8);
  static constexpr int K2 = round_up(2 * NC + NF, 4);
  static constexpr int LDA2 = pad_ld(K2);
  static constexpr int RSR = K2 > NCR ? K2 : NCR;
  static constexpr int doubles(int e) {
    return NCR * LDA1 + NPR * LDA2 + NFR * LDA1 + NPK * pad_ld(round_up(e * M, 8)) +
           NPK * pad_ld(round_up(3 * e * M, 8)) + NFR * pad_ld(round_up(e * M, 8)) + e * 3 * NG * M +
           RSR * pad_ld(round_up(e * M, 8)) + e * 16 + (e * 3 + 1) / 2;
  }
  static constexpr int pick() {
    const int c0 = M == 1 ? 64 : 16, c1 = M == 1 ? 32 : 8, c2 = M == 1 ? 16 : 4;
    return doubles(c0) * 8 <= 110 * 1024 ? c0 : doubles(c1) * 8 <= 110 * 1024 ? c1 : c2;
  }
  static constexpr int E = pick();
  static constexpr int COLS = round_up(E * M, 8);
  static constexpr int LDB = pad_ld(COLS);
  static constexpr int PCOLS = round_up(3 * E * M, 8);
  static constexpr int LDP = pad_ld(PCOLS);
  static constexpr int OFF_V = 0;
  static constexpr int OFF_DL = OFF_V + NCR * LDA1;
  static constexpr int OFF_I = OFF_DL + NPR * LDA2;
  static constexpr int OFF_Q = OFF_I + NFR * LDA1;
  static constexpr int OFF_PB = OFF_Q + NPK * LDB;
  static constexpr int OFF_T = OFF_PB + NPK * LDP;
  static constexpr int OFF_TP = OFF_T + NFR * LDB;
  static constexpr int OFF_RS = OFF_TP + E * 3 * NG * M;
  static constexpr int OFF_GS = OFF_RS + RSR * LDB;
  static constexpr int OFF_F2 = OFF_GS + E * 16;
  static constexpr int TOTAL = OFF_F2 + (E * 3 + 1) / 2;
  static constexpr size_t BYTES = sizeof(double) * TOTAL;
  static_assert(TOTAL == doubles(E), "layout");
};

// One SSPRK stage (or right-hand side) in float64, fused: per tile, the states
// of its elements and of their face neighbours into shared memory; DMMA
// contractions for the cubature values V q, the face traces I q of the tile
// and of the neighbours (each element's trace comes out of the same
// contraction on either side of a face, so both sides see the same values);
// the physical flux at every cubature point and, on every face Gauss point,
// the boundary hook and the numerical flux; one contraction
// [Dr | Ds | L] [R; S; -(1/J) sJ w_g f*] for the right-hand side; the stage
// update in its epilogue.  Every element evaluates its own faces, as Apollo
// does (wxnodaldg2dmethod.cc:389-472), so no face buffer makes a round trip
// through HBM.  Reads the neighbours of x: x and out must not overlap.
template <int EQ, int N>
__global__ void __launch_bounds__(kThreads) k_stage64(DgDev d, StageArgs a) {
  using P = Eq<EQ>;
  constexpr int M = P::M;
  using T = StageTile<N, M>;
  constexpr int NP = T::NP, NC = T::NC, NF = T::NF, NG = T::NG, NPM = T::NPM, E = T::E, LDB = T::LDB, LDP = T::LDP;
  constexpr int NWARPS = kThreads / 32;
  extern __shared__ double smem[];
  double* sV = smem + T::OFF_V;
  double* sDL = smem + T::OFF_DL;
  double* sI = smem + T::OFF_I;
  double* sQ = smem + T::OFF_Q;
  double* sPB = smem + T::OFF_PB;
  double* sT = smem + T::OFF_T;
  double* sTP = smem + T::OFF_TP;
  double* sRS = smem + T::OFF_RS;
  double* sGS = smem + T::OFF_GS;
  int* sF2 = (int*)(smem + T::OFF_F2);
  const int tid = threadIdx.x;
  for (int i = tid; i < T::NCR * T::LDA1; i += kThreads) {
    const int r = i / T::LDA1, c = i % T::LDA1;
    sV[i] = (r < NC && c < NP) ? d.V[r * NP + c] : 0.0;
  }
  for (int i = tid; i < T::NPR * T::LDA2; i += kThreads) {
    const int r = i / T::LDA2, c = i % T::LDA2;
    double v = 0.0;
    if (r < NP) {
      if (c < NC) v = d.Dr[r * NC + c];
      else if (c < 2 * NC) v = d.Ds[r * NC + c - NC];
      else if (c < 2 * NC + NF) v = d.L[r * NF + c - 2 * NC];
    }
    sDL[i] = v;
  }
  for (int i = tid; i < T::NFR * T::LDA1; i += kThreads) {
    const int r = i / T::LDA1, c = i % T::LDA1;
    sI[i] = (r < NF && c < NP) ? d.I[r * NP + c] : 0.0;
  }
  // padding rows and columns of the contraction operands stay zero
  for (int i = tid; i < T::NPK * LDB; i += kThreads) sQ[i] = 0.0;
  for (int i = tid; i < T::NPK * LDP; i += kThreads) sPB[i] = 0.0;
  for (int i = tid; i < T::RSR * LDB; i += kThreads) sRS[i] = 0.0;
  int err = 0;
  LamAcc lam_acc;
  const int ntiles = (d.K + E - 1) / E;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int k0 = tile * E;
    const int ne = min(E, d.K - k0);
    __syncthreads();
    const double* src = a.x + (size_t)k0 * NPM;
    for (int i = tid; i < ne * NPM; i += kThreads) {
      const int e = i / NPM, r = i - e * NPM, j = r / M, f = r - j * M;
      sQ[j * LDB + e * M + f] = src[i];
    }
    for (int i = tid; i < ne * 3; i += kThreads) sF2[i] = d.conn[(size_t)k0 * 6 + 2 * i + 1];
    for (int i = tid; i < ne * 16; i += kThreads) {
      const int e = i >> 4, q = i & 15;
      const ElemGeo& g = d.geo[k0 + e];
      double v = 0.0;
      if (q == 0) v = g.rx;
      else if (q == 1) v = g.ry;
      else if (q == 2) v = g.sx;
      else if (q == 3) v = g.sy;
      else if (q == 4) v = g.invJ;
      else if (q == 5) v = a.time_from_state ? d.st[inst_of(d, k0 + e)].dt : a.dt_arg;
      else if (q < 9) v = g.nx[q - 6];
      else if (q < 12) v = g.ny[q - 9];
      else if (q < 15) v = g.sJ[q - 12];
      sGS[i] = v;
    }
    for (int i = tid; i < ne * 3 * NPM; i += kThreads) {
      const int p = i / NPM, r = i - p * NPM, n = r / M, f = r - n * M;
      const int* cn = d.conn + (size_t)(k0 + p / 3) * 6 + 2 * (p % 3);
      if (cn[1] >= 0) sPB[n * LDP + p * M + f] = a.x[(size_t)cn[0] * NPM + r];
    }
    __syncthreads();
    // cubature values (into the R/S rows), the tile's traces and the
    // neighbours' traces on the faces they share with the tile
    block_dgemm<T::NCR, T::COLS, T::NPK, T::LDA1, LDB, NWARPS>(
        sV, sQ, [&](int r, int c, double v) { sRS[r * LDB + c] = v; });
    block_dgemm<T::NFR, T::COLS, T::NPK, T::LDA1, LDB, NWARPS>(
        sI, sQ, [&](int r, int c, double v) { sT[r * LDB + c] = v; });
    block_dgemm<T::NFR, T::PCOLS, T::NPK, T::LDA1, LDP, NWARPS>(sI, sPB, [&](int r, int c, double v) {
      const int p = c / M;
      if (p >= 3 * ne) return;
      const int f2 = sF2[p], g2 = r - f2 * NG;
      if (f2 >= 0 && g2 >= 0 && g2 < NG) sTP[(p * NG + (NG - 1 - g2)) * M + (c - p * M)] = v;
    });
    __syncthreads();
    // physical flux at the cubature points: R into row c, S into row NC + c
    for (int idx = tid; idx < ne * NC; idx += kThreads) {
      const int e = idx / NC, c = idx - e * NC;
      double qc[M], R[M], S[M];
#pragma unroll
      for (int f = 0; f < M; ++f) qc[f] = sRS[c * LDB + e * M + f];
      const double* gs = sGS + e * 16;
      volume_flux<EQ>(d.eqp, qc, gs[0], gs[1], gs[2], gs[3], R, S, &err);
#pragma unroll
      for (int f = 0; f < M; ++f) {
        sRS[c * LDB + e * M + f] = R[f];
        sRS[(NC + c) * LDB + e * M + f] = S[f];
      }
    }
    // numerical flux at the face Gauss points into rows 2 NC + j NG + g
    for (int idx = tid; idx < ne * NF; idx += kThreads) {
      const int e = idx / NF, kk = idx - e * NF, j = kk / NG, gq = kk - j * NG;
      const int k = k0 + e;
      const double* gs = sGS + e * 16;
      const double nx = gs[6 + j], ny = gs[9 + j];
      double qM[M], qP[M], nf[M];
#pragma unroll
      for (int f = 0; f < M; ++f) qM[f] = sT[kk * LDB + e * M + f];
      const int inst = inst_of(d, k);
      if (sF2[e * 3 + j] >= 0) {
#pragma unroll
        for (int f = 0; f < M; ++f) qP[f] = sTP[((e * 3 + j) * NG + gq) * M + f];
      } else {
        const ElemGeo& g = d.geo[k];
        const double t = a.time_from_state ? d.st[inst].t + d.st[inst].dt * a.frac : a.t_arg;
        // Gauss point coordinates on face j (wxcubature2d.cc:118-124)
        const double z = d.gz[gq];
        double r, s;
        if (j == 0) { r = z; s = -1.0; }
        else if (j == 1) { r = -z; s = z; }
        else { r = -1.0; s = -z; }
        const double x = 0.5 * (-g.vx[0] * (r + s) + g.vx[1] * (1. + r) + g.vx[2] * (1. + s));
        const double y = 0.5 * (-g.vy[0] * (r + s) + g.vy[1] * (1. + r) + g.vy[2] * (1. + s));
        apply_bc<EQ, double>(d.bcs, -d.conn[(size_t)k * 6 + 2 * j], t, x, y, nx, ny, qM, qP);
      }
      const double lam = face_flux<EQ>(d.eqp, nx, ny, qM, qP, nf, &err);
      lam_acc.add(d.st, inst, fabs(lam));
      const double w = -(gs[4] * (d.gw[gq] * gs[12 + j]));
#pragma unroll
      for (int f = 0; f < M; ++f) sRS[(2 * NC + kk) * LDB + e * M + f] = nf[f] * w;
    }
    __syncthreads();
    // right-hand side [Dr | Ds | L] [R; S; F] and the stage update
    block_dgemm<T::NPR, T::COLS, T::K2, T::LDA2, LDB, NWARPS, 4>(sDL, sRS, [&](int i, int c, double r) {
      const int e = c / M;
      if (i >= NP || e >= ne) return;
      const int k = k0 + e;
      const size_t off = (size_t)k * NPM + i * M + (c - e * M);
      const double dt = sGS[e * 16 + 5];
      const double c_stage = dt / 4.0;  // dt/(s-1), s = 5
      const double c_al = 4.0 / 5.0, c_be = dt / 5.0, c_ga = 1.0 / 5.0;
      if (r != r) err |= ERRB_NAN;
      const double xv = sQ[i * LDB + c];
      double o;
      if (a.mode == MODE_RHS) o = r;
      else if (a.mode == MODE_STAGE) o = xv + c_stage * r;
      else o = c_al * xv + c_be * r + c_ga * a.u0[off];
      a.out[off] = o;
    });
  }
  lam_acc.flush_warp(d.st);
  if (err) atomicOr(&d.st->err, err);
}

// M consecutive doubles of one Gauss point (a trace or a face flux): 16-byte
// vector accesses when M is even (every point's block then starts on a
// 16-byte boundary), scalar ones otherwise.
template <int M>
__device__ __forceinline__ void load_point(const double* __restrict__ p, double* q) {
  if constexpr (M % 2 == 0) {
#pragma unroll
    for (int f = 0; f < M; f += 2) {
      const double2 v = __ldg(reinterpret_cast<const double2*>(p + f));
      q[f] = v.x;
      q[f + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int f = 0; f < M; ++f) q[f] = __ldg(p + f);
  }
}
template <int M>
__device__ __forceinline__ void store_point(double* __restrict__ p, const double* q, double w) {
  if constexpr (M % 2 == 0) {
#pragma unroll
    for (int f = 0; f < M; f += 2) *reinterpret_cast<double2*>(p + f) = make_double2(q[f] * w, q[f + 1] * w);
  } else {
#pragma unroll
    for (int f = 0; f < M; ++f) p[f] = q[f] * w;
  }
}

template <int EQ, int N>
__global__ void __launch_bounds__(kThreads) k_face(DgDev d, StageArgs a) {
  using P = Eq<EQ>;
  constexpr int M = P::M;
  constexpr int NG = Sizes<N>::NG, NF = Sizes<N>::NF;
  int err = 0;
  LamAcc lam_acc;
  // each block takes a contiguous range of face points, so a thread's points
  // stay within one instance of a batched ensemble
  const bool two_sided = flux_two_sided<EQ>(d.eqp);
  const int total = d.nfaces * NG;
  const int per_block = (total + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per_block, i1 = min(total, i0 + per_block);
  for (int idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
    const int fi = idx / NG, gq = idx - fi * NG;
    const FaceRec fr = d.faces[fi];
    const int inst = inst_of(d, fr.k1);
    const double t = a.time_from_state ? d.st[inst].t + d.st[inst].dt * a.frac : a.t_arg;
    const ElemGeo& g = d.geo[fr.k1];
    const double nx = g.nx[fr.f1], ny = g.ny[fr.f1], sJ = g.sJ[fr.f1];
    double qM[M], qP[M], nf[M];
    const double* tm = d.trace + ((size_t)fr.k1 * NF + fr.f1 * NG + gq) * M;
    load_point<M>(tm, qM);
    if (fr.k2 >= 0) {
      load_point<M>(d.trace + ((size_t)fr.k2 * NF + fr.f2 * NG + (NG - 1 - gq)) * M, qP);
    } else {
      // Gauss point coordinates on face f1: the affine map of the face
      // parametrisation (wxcubature2d.cc:118-124)
      const double z = d.gz[gq];
      double r, s;
      if (fr.f1 == 0) { r = z; s = -1.0; }
      else if (fr.f1 == 1) { r = -z; s = z; }
      else { r = -1.0; s = -z; }
      const double x = 0.5 * (-g.vx[0] * (r + s) + g.vx[1] * (1. + r) + g.vx[2] * (1. + s));
      const double y = 0.5 * (-g.vy[0] * (r + s) + g.vy[1] * (1. + r) + g.vy[2] * (1. + s));
      apply_bc<EQ, double>(d.bcs, -fr.k2, t, x, y, nx, ny, qM, qP);
    }
    double lam = face_flux<EQ>(d.eqp, nx, ny, qM, qP, nf, &err);
    lam_acc.add(d.st, inst, fabs(lam));
    const double w = d.gw[gq] * sJ;
    store_point<M>(d.flux + ((size_t)fr.k1 * NF + fr.f1 * NG + gq) * M, nf, w);
    if (fr.k2 >= 0) {
      const int g2 = NG - 1 - gq;
      double* op = d.flux + ((size_t)fr.k2 * NF + fr.f2 * NG + g2) * M;
      if (two_sided) {
        // the partner's own evaluation: its normal, weight and trace as "-"
        const ElemGeo& h2 = d.geo[fr.k2];
        load_point<M>(d.trace + ((size_t)fr.k2 * NF + fr.f2 * NG + g2) * M, qM);
        load_point<M>(tm, qP);
        const double lam2 = P::numflux(d.eqp, h2.nx[fr.f2], h2.ny[fr.f2], qM, qP, nf, &err);
        lam_acc.add(d.st, inst, fabs(lam2));
        store_point<M>(op, nf, d.gw[g2] * h2.sJ[fr.f2]);
      } else {
        store_point<M>(op, nf, -w);
      }
    }
  }
  lam_acc.flush_warp(d.st);
  if (err) atomicOr(&d.st->err, err);
}

template <int N, int M> struct LiftTile {
  static constexpr int NP = Sizes<N>::NP, NF = Sizes<N>::NF;
  static constexpr int E = M == 1 ? 64 : (M == 8 ? 8 : 16);
  static constexpr int COLS = round_up(E * M, 8);
  static constexpr int LDB = pad_ld(COLS);
  static constexpr int NFK = round_up(NF, 4);  // K: face Gauss points
  static constexpr int LDA = pad_ld(NFK);
  static constexpr int NPR = round_up(NP, 8);
  static constexpr int OFF_L = 0;
  static constexpr int OFF_F = NPR * LDA;
  static constexpr size_t BYTES = sizeof(double) * (OFF_F + NFK * LDB);
};

template <int EQ, int N>
__global__ void __launch_bounds__(kThreads) k_lift(DgDev d, StageArgs a) {
  constexpr int M = Eq<EQ>::M;
  using T = LiftTile<N, M>;
  constexpr int NP = T::NP, NF = T::NF, E = T::E, LDB = T::LDB;
  constexpr int NWARPS = kThreads / 32;
  extern __shared__ double smem[];
  double* sL = smem + T::OFF_L;
  double* sF = smem + T::OFF_F;
  const int tid = threadIdx.x;
  for (int i = tid; i < T::NPR * T::LDA; i += kThreads) {
    const int r = i / T::LDA, c = i % T::LDA;
    sL[i] = (r < NP && c < NF) ? d.L[r * NF + c] : 0.0;
  }
  for (int i = tid; i < T::NFK * LDB; i += kThreads) sF[i] = 0.0;
  int err = 0;
  const int ntiles = (d.K + E - 1) / E;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int k0 = tile * E;
    const int ne = min(E, d.K - k0);
    __syncthreads();
    // numerical-flux tile, [e][gauss][field] -> F[gauss][e*M + field]
    const double* src = d.flux + (size_t)k0 * NF * M;
    for (int i = tid; i < ne * NF * M; i += kThreads) {
      const int e = i / (NF * M), r = i - e * NF * M, g = r / M, f = r - g * M;
      sF[g * LDB + e * M + f] = src[i];
    }
    __syncthreads();
    block_dgemm<T::NPR, T::COLS, T::NFK, T::LDA, LDB, NWARPS>(sL, sF, [&](int i, int c, double v) {
      const int e = c / M, f = c - e * M;
      if (i >= NP || e >= ne) return;
      const int k = k0 + e;
      const size_t off = ((size_t)k * NP + i) * M + f;
      const double dt = a.time_from_state ? d.st[inst_of(d, k)].dt : a.dt_arg;
      const double c_stage = dt / 4.0;  // dt/(s-1), s = 5
      const double c_al = 4.0 / 5.0, c_be = dt / 5.0, c_ga = 1.0 / 5.0;
      const double r = d.vol[off] - d.geo[k].invJ * v;
      if (r != r) err |= ERRB_NAN;
      double o;
      if (a.mode == MODE_RHS) o = r;
      else if (a.mode == MODE_STAGE) o = a.x[off] + c_stage * r;
      else o = c_al * a.x[off] + c_be * r + c_ga * a.u0[off];
      a.out[off] = o;
    });
  }
  if (err) atomicOr(&d.st->err, err);
}

template <int EQ>
__global__ void k_init_speed(DgDev d, const double* u, int nnodes) {
  constexpr int M = Eq<EQ>::M;
  LamAcc lam_acc;
  const int per_block = (nnodes + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per_block, i1 = min(nnodes, i0 + per_block);
  const int np = nnodes / d.K;
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    double q[M];
#pragma unroll
    for (int f = 0; f < M; ++f) q[f] = u[(size_t)i * M + f];
    double s2 = Eq<EQ>::speed2(d.eqp, q);
    lam_acc.add(d.st, inst_of(d, i / np), sqrt(s2 > 0.0 ? s2 : 0.0));
  }
  lam_acc.flush_warp(d.st);
}

// After a step: t += dt; dt = min(dt, suggestion of the last stage), clipped
// to the end time (ApSolver::ComputeRHSforTS + MonitorVTK,
// src/solvers/apsolver.cc:421-480).
__global__ void k_finalize(DgDev d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.ninst) return;
  DevState* st = d.st + i;
  const double lam = __longlong_as_double((long long)st->lam_bits);
  const double sugg = (st->dtfac > 0.0 ? st->dtfac : d.dtfac) * (d.rmin / lam);
  st->last_sugg = sugg;
  const double dt = st->dt;
  const double t = st->t + dt;
  double nd = fmin(sugg, dt);
  if (st->tend > 0.0 && fabs(st->tend - t) < nd) nd = fabs(st->tend - t);
  st->t = t;
  st->dt = nd;
  st->steps += 1;
  st->lam_bits = 0ull;  // the next step's last stage reduces into it afresh
}

template <int EQ>
__global__ void k_integrals(DgDev d, const double* u, const double* wmass, int NP) {
  constexpr int M = Eq<EQ>::M;
  double acc[M];
#pragma unroll
  for (int f = 0; f < M; ++f) acc[f] = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < d.K; k += gridDim.x * blockDim.x) {
    const double J = d.geo[k].J;
    for (int j = 0; j < NP; ++j) {
      const double w = wmass[j] * J;
#pragma unroll
      for (int f = 0; f < M; ++f) acc[f] += w * u[((size_t)k * NP + j) * M + f];
    }
  }
#pragma unroll
  for (int f = 0; f < M; ++f) {
    double v = acc[f];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&d.st->sums[f], v);
  }
}

// Per-field integrals of u^2 over the mesh: sum_k J_k u_k^T Mref u_k with the
// reference-element mass matrix Mref = (V V^T)^-1 (the inverse of Apollo's
// VVT, wxnodaldggeometry2d.cc:71-75), one thread per element.
template <int EQ>
__global__ void k_energy(DgDev d, const double* __restrict__ u, const double* __restrict__ mass, int NP) {
  constexpr int M = Eq<EQ>::M;
  double acc[M];
#pragma unroll
  for (int f = 0; f < M; ++f) acc[f] = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < d.K; k += gridDim.x * blockDim.x) {
    const double J = d.geo[k].J;
    const double* uk = u + (size_t)k * NP * M;
    for (int i = 0; i < NP; ++i) {
      double mu[M];
#pragma unroll
      for (int f = 0; f < M; ++f) mu[f] = 0.0;
      for (int j = 0; j < NP; ++j) {
        const double w = mass[i * NP + j];
#pragma unroll
        for (int f = 0; f < M; ++f) mu[f] += w * uk[j * M + f];
      }
#pragma unroll
      for (int f = 0; f < M; ++f) acc[f] += J * uk[i * M + f] * mu[f];
    }
  }
#pragma unroll
  for (int f = 0; f < M; ++f) {
    double v = acc[f];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&d.st->sums[f], v);
  }
}

// The source plugins at one point (Apollo adds each into its output field,
// WxHyperbolicSrc::compSource, src/hyper/wxhyperbolicsrc.cc:64-80).
__device__ __forceinline__ void source_terms(const SrcTable& T, double t, double x, double y, double* s) {
  for (int i = 0; i < T.n; ++i) {
    const double* p = T.p[i];
    double v = 0.0;
    if (T.kind[i] == SRC_TM) {
      v = exp(t) * (x * (1 - x) * y * (1 - y) + 2. * x * (1 - x) + 2 * y * (1 - y));
    } else if (T.kind[i] == SRC_POINT) {
      const double qbyme = p[6] / (p[7] * p[8]);
      if (sqrt((x - p[0]) * (x - p[0]) + (y - p[1]) * (y - p[1])) < p[2]) v = p[3] * qbyme * sin(p[4] * t + p[5]);
    }
    s[T.out[i]] += v;
  }
}

// Source contribution of a block of kSrcE elements: the sources at every
// cubature point (physical coordinates from the element's affine map), then
// VS times them per (element, node, field).
constexpr int kSrcE = 4;
template <int EQ, int N>
__global__ void __launch_bounds__(128) k_source(DgDev d, StageArgs a, double* __restrict__ dst, int accumulate) {
  constexpr int M = Eq<EQ>::M, NP = Sizes<N>::NP, NC = Sizes<N>::NC;
  __shared__ double S[kSrcE][NC][M];
  const int k0 = blockIdx.x * kSrcE;
  for (int i = threadIdx.x; i < kSrcE * NC; i += blockDim.x) {
    const int e = i / NC, c = i - e * NC, k = k0 + e;
    double sv[M];
#pragma unroll
    for (int f = 0; f < M; ++f) sv[f] = 0.0;
    if (k < d.K) {
      const ElemGeo& g = d.geo[k];
      const double r = d.cub_r[c], q = d.cub_s[c];
      const double x = 0.5 * (-g.vx[0] * (r + q) + g.vx[1] * (1. + r) + g.vx[2] * (1. + q));
      const double y = 0.5 * (-g.vy[0] * (r + q) + g.vy[1] * (1. + r) + g.vy[2] * (1. + q));
      const DevState& st = d.st[inst_of(d, k)];
      const double t = a.time_from_state ? st.t + st.dt * a.frac : a.t_arg;
      source_terms(d.src, t, x, y, sv);
    }
#pragma unroll
    for (int f = 0; f < M; ++f) S[e][c][f] = sv[f];
  }
  __syncthreads();
  unsigned fmask = 0;
  for (int i = 0; i < d.src.n; ++i) fmask |= 1u << d.src.out[i];
  for (int i = threadIdx.x; i < kSrcE * NP * M; i += blockDim.x) {
    const int e = i / (NP * M), r = i - e * NP * M, n = r / M, f = r - n * M, k = k0 + e;
    if (k >= d.K) continue;
    double v = 0.0;
    if (fmask & (1u << f))
      for (int c = 0; c < NC; ++c) v += d.VS[n * NC + c] * S[e][c][f];
    double* o = dst + ((size_t)k * NP + n) * M + f;
    if (accumulate) {
      if (fmask & (1u << f)) *o += v;
    } else {
      *o = v;
    }
  }
}

template <int EQ>
cudaError_t source_dispatch(const DgDev& d, const StageArgs& a, double* dst, int acc, cudaStream_t s) {
  const unsigned g = (unsigned)((d.K + kSrcE - 1) / kSrcE);
  if (g == 0) return cudaSuccess;
  switch (d.N) {
    case 2: k_source<EQ, 2><<<g, 128, 0, s>>>(d, a, dst, acc); break;
    case 3: k_source<EQ, 3><<<g, 128, 0, s>>>(d, a, dst, acc); break;
    case 4: k_source<EQ, 4><<<g, 128, 0, s>>>(d, a, dst, acc); break;
    case 5: k_source<EQ, 5><<<g, 128, 0, s>>>(d, a, dst, acc); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

int g_num_sms = 0;
int num_sms() {
  if (g_num_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

template <int EQ, int N>
cudaError_t launch_rhs_t(const DgDev& d, const StageArgs& a, cudaStream_t s, cudaEvent_t* ev) {
  constexpr int M = Eq<EQ>::M;
  using VT = VolTile<N, M>;
  using LT = LiftTile<N, M>;
  static unsigned configured = 0;  // bit per device
  static int vol_res = 1, lift_res = 1;  // resident blocks per SM
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(configured & (1u << (dev & 31)))) {
    cudaError_t e = cudaFuncSetAttribute(k_volume<EQ, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)VT::BYTES);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_lift<EQ, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LT::BYTES);
    if (e != cudaSuccess) return e;
    // persistent grids of the blocks that are resident at once (registers
    // and shared memory): a block beyond them would start a late second wave
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&vol_res, k_volume<EQ, N>, kThreads, VT::BYTES);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&lift_res, k_lift<EQ, N>, kThreads, LT::BYTES);
    if (e != cudaSuccess) return e;
    configured |= 1u << (dev & 31);
  }
  const int sms = d.grid_div > 1 ? (num_sms() + d.grid_div - 1) / d.grid_div : num_sms();
  // the fused stage where it applies: the whole mesh on this handle (no ghost
  // elements), no sources, and an output that does not overlap the input (it
  // reads the neighbours' states while other blocks write theirs)
  const size_t nbytes = (size_t)d.K * Sizes<N>::NP * M * sizeof(double);
  const char *xb = (const char*)a.x, *ob = (const char*)a.out;
  const bool apart = ob + nbytes <= xb || xb + nbytes <= ob;
  using ST = StageTile<N, M>;
  const bool one_wave = (d.K + ST::E - 1) / ST::E <= sms * 2;  // launch-bound: one launch instead of three
  const bool fuse = d.fp64_fused == 1 || (d.fp64_fused == 2 && one_wave);
  if (fuse && d.nghost == 0 && a.phase == PHASE_ALL && d.src.n == 0 && apart) {
    static unsigned fused_configured = 0;
    static int resident = 1;  // blocks per SM (registers and shared memory)
    if (!(fused_configured & (1u << (dev & 31)))) {
      cudaError_t e = cudaFuncSetAttribute(k_stage64<EQ, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)ST::BYTES);
      if (e != cudaSuccess) return e;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_stage64<EQ, N>, kThreads, ST::BYTES);
      if (e != cudaSuccess) return e;
      fused_configured |= 1u << (dev & 31);
    }
    const int st = (d.K + ST::E - 1) / ST::E;
    // a persistent grid of the blocks that are resident at once
    int per = resident < 1 ? 1 : resident;
    int gs = sms * per;
    if (gs > st) gs = st;
    if (ev) cudaEventRecord(ev[0], s);
    if (a.reset_lambda) launch_reset_lambda(d, s);
    k_stage64<EQ, N><<<gs, kThreads, ST::BYTES, s>>>(d, a);
    if (ev) {
      cudaEventRecord(ev[1], s);
      cudaEventRecord(ev[2], s);
      cudaEventRecord(ev[3], s);
    }
    return cudaGetLastError();
  }
  const int vt = (d.K + VT::E - 1) / VT::E;
  int per_sm = vol_res < 1 ? 1 : (vol_res > 8 ? 8 : vol_res);
  int gv = sms * per_sm;
  if (gv > vt) gv = vt;
  if (a.phase == PHASE_ALL || a.phase == PHASE_VOLUME) {
    if (ev) cudaEventRecord(ev[0], s);
    k_volume<EQ, N><<<gv, kThreads, VT::BYTES, s>>>(d, a);
    // sources enter the volume term (wxcubature2d.cc:297-325: VT (w J S))
    if (d.src.n > 0) {
      cudaError_t e = source_dispatch<EQ>(d, a, d.vol, 1, s);
      if (e != cudaSuccess) return e;
    }
    if (ev) cudaEventRecord(ev[1], s);
  }
  if (a.phase == PHASE_VOLUME) return cudaGetLastError();
  if (a.phase != PHASE_LIFT) {
    // the faces d.faces[0, d.nfaces): all of them, or a range of them
    const int fthreads = d.nfaces * Sizes<N>::NG;
    int gf = (fthreads + kThreads - 1) / kThreads;
    if (gf > sms * 8) gf = sms * 8;
    if (gf < 1) gf = 1;
    if (fthreads > 0) k_face<EQ, N><<<gf, kThreads, 0, s>>>(d, a);
    if (ev) cudaEventRecord(ev[2], s);
  }
  if (a.phase == PHASE_FACE_ONLY) return cudaGetLastError();
  const int lt = (d.K + LT::E - 1) / LT::E;
  int lper = lift_res < 1 ? 1 : (lift_res > 8 ? 8 : lift_res);
  int gl = sms * lper;
  if (gl > lt) gl = lt;
  k_lift<EQ, N><<<gl, kThreads, LT::BYTES, s>>>(d, a);
  if (ev) cudaEventRecord(ev[3], s);
  return cudaGetLastError();
}

// The LIFT kernel alone (surface contraction, 1/J, stage update) on the given
// volume and face-flux buffers: the lift and the stage update are linear, so
// the tangent of a stage applies it to the tangent buffers unchanged.
template <int EQ, int N>
cudaError_t launch_lift_t(const DgDev& d, const StageArgs& a, cudaStream_t s) {
  constexpr int M = Eq<EQ>::M;
  using LT = LiftTile<N, M>;
  static unsigned configured = 0;  // bit per device
  static int lift_res = 1;          // resident blocks per SM
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(configured & (1u << (dev & 31)))) {
    cudaError_t e = cudaFuncSetAttribute(k_lift<EQ, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LT::BYTES);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&lift_res, k_lift<EQ, N>, kThreads, LT::BYTES);
    if (e != cudaSuccess) return e;
    configured |= 1u << (dev & 31);
  }
  const int lt = (d.K + LT::E - 1) / LT::E;
  int lper = lift_res < 1 ? 1 : (lift_res > 8 ? 8 : lift_res);
  int gl = num_sms() * lper;
  if (gl > lt) gl = lt;
  k_lift<EQ, N><<<gl, kThreads, LT::BYTES, s>>>(d, a);
  return cudaGetLastError();
}

template <int EQ>
cudaError_t lift_dispatch_n(const DgDev& d, const StageArgs& a, cudaStream_t s) {
  switch (d.N) {
    case 2: return launch_lift_t<EQ, 2>(d, a, s);
    case 3: return launch_lift_t<EQ, 3>(d, a, s);
    case 4: return launch_lift_t<EQ, 4>(d, a, s);
    case 5: return launch_lift_t<EQ, 5>(d, a, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int EQ>
cudaError_t dispatch_n(const DgDev& d, const StageArgs& a, cudaStream_t s, cudaEvent_t* ev) {
  switch (d.N) {
    case 2: return launch_rhs_t<EQ, 2>(d, a, s, ev);
    case 3: return launch_rhs_t<EQ, 3>(d, a, s, ev);
    case 4: return launch_rhs_t<EQ, 4>(d, a, s, ev);
    case 5: return launch_rhs_t<EQ, 5>(d, a, s, ev);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

int fp64_supported(int eq, int N) { return eq >= 0 && eq <= 4 && N >= 2 && N <= 5; }

cudaError_t launch_rhs_fp64(int eq, const DgDev& d, const StageArgs& a, cudaStream_t s, cudaEvent_t* ev) {
  switch (eq) {
    case EQ_ADVECTION: return dispatch_n<EQ_ADVECTION>(d, a, s, ev);
    case EQ_EULER: return dispatch_n<EQ_EULER>(d, a, s, ev);
    case EQ_MAXWELL: return dispatch_n<EQ_MAXWELL>(d, a, s, ev);
    case EQ_EULER2D: return dispatch_n<EQ_EULER2D>(d, a, s, ev);
    case EQ_MAXWELL_TM: return dispatch_n<EQ_MAXWELL_TM>(d, a, s, ev);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_source(int eq, const DgDev& d, const StageArgs& a, double* dst, int accumulate, cudaStream_t s) {
  switch (eq) {
    case EQ_ADVECTION: return source_dispatch<EQ_ADVECTION>(d, a, dst, accumulate, s);
    case EQ_EULER: return source_dispatch<EQ_EULER>(d, a, dst, accumulate, s);
    case EQ_MAXWELL: return source_dispatch<EQ_MAXWELL>(d, a, dst, accumulate, s);
    case EQ_EULER2D: return source_dispatch<EQ_EULER2D>(d, a, dst, accumulate, s);
    case EQ_MAXWELL_TM: return source_dispatch<EQ_MAXWELL_TM>(d, a, dst, accumulate, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_lift_fp64(int eq, const DgDev& d, const StageArgs& a, cudaStream_t s) {
  switch (eq) {
    case EQ_ADVECTION: return lift_dispatch_n<EQ_ADVECTION>(d, a, s);
    case EQ_EULER: return lift_dispatch_n<EQ_EULER>(d, a, s);
    case EQ_MAXWELL: return lift_dispatch_n<EQ_MAXWELL>(d, a, s);
    case EQ_EULER2D: return lift_dispatch_n<EQ_EULER2D>(d, a, s);
    case EQ_MAXWELL_TM: return lift_dispatch_n<EQ_MAXWELL_TM>(d, a, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_init_speed(int eq, const DgDev& d, const double* u, cudaStream_t s) {
  const int np = (d.N + 1) * (d.N + 2) / 2;
  const int nn = d.K * np;
  int g = (nn + 255) / 256;
  if (g > num_sms() * 8) g = num_sms() * 8;
  if (g < 1) g = 1;
  switch (eq) {
    case EQ_ADVECTION: k_init_speed<EQ_ADVECTION><<<g, 256, 0, s>>>(d, u, nn); break;
    case EQ_EULER: k_init_speed<EQ_EULER><<<g, 256, 0, s>>>(d, u, nn); break;
    case EQ_MAXWELL: k_init_speed<EQ_MAXWELL><<<g, 256, 0, s>>>(d, u, nn); break;
    case EQ_EULER2D: k_init_speed<EQ_EULER2D><<<g, 256, 0, s>>>(d, u, nn); break;
    case EQ_MAXWELL_TM: k_init_speed<EQ_MAXWELL_TM><<<g, 256, 0, s>>>(d, u, nn); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

__global__ void k_reset_lambda(DevState* st, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) st[i].lam_bits = 0ull;
}

cudaError_t launch_finalize(const DgDev& d, cudaStream_t s) {
  k_finalize<<<(d.ninst + 127) / 128, 128, 0, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_reset_lambda(const DgDev& d, cudaStream_t s) {
  k_reset_lambda<<<(d.ninst + 127) / 128, 128, 0, s>>>(d.st, d.ninst);
  return cudaGetLastError();
}

// the value travels as a kernel argument, captured at launch: the caller's
// host copy may change before the stream reaches the write
__global__ void k_put_state(DevState* st, DevState v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *st = v;
}

cudaError_t launch_put_state(DevState* st, const DevState& v, cudaStream_t s) {
  k_put_state<<<1, 32, 0, s>>>(st, v);
  return cudaGetLastError();
}

cudaError_t launch_integrals(int eq, const DgDev& d, const double* u, const double* wmass, cudaStream_t s) {
  const int np = (d.N + 1) * (d.N + 2) / 2;
  int g = (d.K + 255) / 256;
  if (g > num_sms() * 4) g = num_sms() * 4;
  if (g < 1) g = 1;
  switch (eq) {
    case EQ_ADVECTION: k_integrals<EQ_ADVECTION><<<g, 256, 0, s>>>(d, u, wmass, np); break;
    case EQ_EULER: k_integrals<EQ_EULER><<<g, 256, 0, s>>>(d, u, wmass, np); break;
    case EQ_MAXWELL: k_integrals<EQ_MAXWELL><<<g, 256, 0, s>>>(d, u, wmass, np); break;
    case EQ_EULER2D: k_integrals<EQ_EULER2D><<<g, 256, 0, s>>>(d, u, wmass, np); break;
    case EQ_MAXWELL_TM: k_integrals<EQ_MAXWELL_TM><<<g, 256, 0, s>>>(d, u, wmass, np); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_energy(int eq, const DgDev& d, const double* u, const double* mass, cudaStream_t s) {
  const int np = (d.N + 1) * (d.N + 2) / 2;
  int g = (d.K + 127) / 128;
  if (g > num_sms() * 8) g = num_sms() * 8;
  if (g < 1) g = 1;
  switch (eq) {
    case EQ_ADVECTION: k_energy<EQ_ADVECTION><<<g, 128, 0, s>>>(d, u, mass, np); break;
    case EQ_EULER: k_energy<EQ_EULER><<<g, 128, 0, s>>>(d, u, mass, np); break;
    case EQ_MAXWELL: k_energy<EQ_MAXWELL><<<g, 128, 0, s>>>(d, u, mass, np); break;
    case EQ_EULER2D: k_energy<EQ_EULER2D><<<g, 128, 0, s>>>(d, u, mass, np); break;
    case EQ_MAXWELL_TM: k_energy<EQ_MAXWELL_TM><<<g, 128, 0, s>>>(d, u, mass, np); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace apollo
