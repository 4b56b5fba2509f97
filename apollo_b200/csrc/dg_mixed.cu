// Mixed-precision right-hand side and SSP stage on the tcgen05 tensor cores.
//
// One fused kernel per Runge-Kutta stage.  A CTA takes a tile of elements;
// the 128 tensor-core rows are (element, field) pairs, 32 per warp quadrant
// (32 / M elements each, so an element never straddles two warps).  Every
// contraction runs on the tensor cores as kind::tf32 with a three-term split
// (hi*hi + hi*lo + lo*hi, fp32 accumulation in TMEM) and acts only on
// deviations from a float64 reference value per element and field:
//
//   q  = qbar + dq          qbar = nodal mean            (float64)
//   V q      = qbar + V dq                  (cubature values)
//   I q      = qbar + I dq                  (own face traces)
//   I q_nb   = qbar_nb + I dq_nb            (neighbour traces, recomputed from
//                                            the neighbour's state in L2)
//   Dr R     = (Dr 1) R(0) + Dr (R - R(0))  (R = rx F + ry G at cubature points)
//   L f*     = sum_f (L_f 1) f*_f(0) + L (f* - f*_f(0))
//
// so the low-precision products see only the element-local fluctuation.  The
// pointwise flux and the Lax-Friedrichs face flux are fp32; the state, the
// reference values, the operator row sums, the stage accumulation, the dt
// reduction (float64 wave speed, last stage only) stay float64.
//
// Apollo: the RHS of wxnodaldg2dmethod.cc:235-542 (volume :346-380, traces and
// partner gather :389-440, numerical flux :442-469, surface integral and M^-1/J
// :472-504) fused with the TSSSP RK_2 stage update.
#include "dg_mixed.h"
#include "dg_umma.cuh"

#include <vector>

namespace apollo {

struct MixedPlan {
  int eq = 0, N = 0, M = 0;
  double* rowsum = nullptr;  // [NP][5]: Dr 1, Ds 1, L_0 1, L_1 1, L_2 1 (float64)
  int* rot = nullptr;        // [3][NP] node permutations rotating face k onto face 0
};

namespace {

constexpr int kMixThreads = 384;
constexpr int round_up_c(int x, int m) { return (x + m - 1) / m * m; }
constexpr int max_c(int a, int b) { return a > b ? a : b; }

template <int N, int M> struct MixCfg {
  static constexpr int NP = Sizes<N>::NP, NC = Sizes<N>::NC, NG = Sizes<N>::NG, NF = Sizes<N>::NF;
  static constexpr int EPQ = 32 / M;  // elements per warp quadrant
  static constexpr int E = 4 * EPQ;   // elements per tile
  static constexpr int K1 = round_up_c(NP, 8);
  static constexpr int VPC = 12;                      // cubature points per volume chunk
  static constexpr int KV = 2 * VPC;                  // K columns per volume chunk (R, S)
  static constexpr int NV = (NC + VPC - 1) / VPC;     // volume chunks
  static constexpr int NC8 = round_up_c(NC, 8);       // first Gauss-point row of B1
  static constexpr int NC16 = round_up_c(NC, 16);
  static constexpr int NI = round_up_c(NF, 16);
  static constexpr int NA = round_up_c(NC8 + NI, 16);
  static constexpr int N3 = 16;                       // neighbour traces: face 0 of the rotated data
  static constexpr int NPN = round_up_c(NP, 16);
  static constexpr int KB2 = NV * KV + 3 * 16;        // then one 16-column chunk per face
  static constexpr int NBUF = 3;
  // TMEM columns
  static constexpr int T_D1 = 0, T_D3 = NA, T_D2 = NA + 3 * N3;
  static constexpr int TUSED = T_D2 + NPN;
  static constexpr int TCOLS = TUSED <= 64 ? 64 : TUSED <= 128 ? 128 : TUSED <= 256 ? 256 : 512;
  // shared memory, bytes (each operand as a tf32 hi half and lo half)
  static constexpr int SZ_B1 = NA * K1 * 4;
  static constexpr int SZ_B2 = NPN * KB2 * 4;
  static constexpr int SZ_A1 = 128 * K1 * 4;
  static constexpr int SZ_CH = 128 * KV * 4;
  static constexpr int SZ_U = max_c(8 * SZ_A1, NBUF * 2 * SZ_CH);
  static constexpr int SR = 48;  // cubature points staged at a time (a multiple of VPC)
  static constexpr int SZ_ST = max_c(SR, 32) * 128 * 4;
  static constexpr int O_B1H = 0, O_B1L = O_B1H + SZ_B1;
  static constexpr int O_B2H = O_B1L + SZ_B1, O_B2L = O_B2H + SZ_B2;
  static constexpr int O_U = round_up_c(O_B2L + SZ_B2, 128);
  static constexpr int O_ST = O_U + SZ_U;
  static constexpr int O_G0 = O_ST + SZ_ST;                // g = 0 traces: [6][128] float
  static constexpr int O_GEO = O_G0 + 6 * 128 * 4;         // [E][16] float
  static constexpr int O_RS = O_GEO + E * 16 * 4;          // operator row sums [NP][5] double
  static constexpr int O_RB = O_RS + NP * 5 * 8;           // R(0), S(0): [E][2M] double
  static constexpr int O_FB = O_RB + E * 2 * M * 8;        // face references: [E][3][M] double
  static constexpr int O_RBH = O_FB + E * 3 * M * 8;       // fp32 point-0 fluxes F, G, face f*: [E][5M]
  static constexpr int O_CN = O_RBH + E * 5 * M * 4;       // [E][6] int
  static constexpr int O_QB = O_CN + E * 6 * 4;            // means: own [128], neighbours [3][128] double
  static constexpr int O_QF = O_QB + 4 * 128 * 8;          // the same means as float
  static constexpr int O_ROT = O_QF + 4 * 128 * 4;         // [3][NP] int
  static constexpr int O_MB = round_up_c(O_ROT + 3 * NP * 4, 8);  // mbarriers: A, ring[NBUF]
  static constexpr int O_TS = O_MB + 8 * (1 + NBUF);       // TMEM base, abort flag
  static constexpr int BYTES = O_TS + 16;
  static constexpr bool FITS = BYTES <= 227 * 1024;
  static_assert(NG <= 16, "one 16-column chunk per face");
};

// tf32 split, both halves rounded to nearest: x = hi + lo + O(2^-22 |x|).
__device__ __forceinline__ void split_trunc(float x, float& h, float& l) {
  h = umma::to_tf32(x);
  l = umma::to_tf32(x - h);
}

template <int M>
__device__ __forceinline__ void load_fields(const float* p, float* v) {
  if constexpr (M == 4) {
    const float4 t = *(const float4*)p;
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else {
#pragma unroll
    for (int f = 0; f < M; ++f) v[f] = p[f];
  }
}

template <int EQ, int N>
__global__ void __launch_bounds__(kMixThreads, 1)
    k_mixed_stage(DgDev d, StageArgs a, const double* __restrict__ rowsum, const int* __restrict__ rot) {
  using P = Eq<EQ>;
  constexpr int M = P::M;
  using C = MixCfg<N, M>;
  constexpr int NP = C::NP, NC = C::NC, NG = C::NG, NF = C::NF, EPQ = C::EPQ, E = C::E, K1 = C::K1;
  constexpr int VPC = C::VPC, KV = C::KV, SR = C::SR;
  static_assert(SR % VPC == 0 && SR % 16 == 0, "staging waves hold whole chunks");
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* B1h = sm + C::O_B1H;
  unsigned char* B1l = sm + C::O_B1L;
  unsigned char* B2h = sm + C::O_B2H;
  unsigned char* B2l = sm + C::O_B2L;
  unsigned char* U = sm + C::O_U;
  float* ST = (float*)(sm + C::O_ST);
  float* G0 = (float*)(sm + C::O_G0);
  float* GEO = (float*)(sm + C::O_GEO);
  double* RSUM = (double*)(sm + C::O_RS);
  double* Rb = (double*)(sm + C::O_RB);   // [E][2M]: R(0), S(0) in float64
  double* Fb = (double*)(sm + C::O_FB);   // [E][3][M]: face references in float64
  float* P0 = (float*)(sm + C::O_RBH);    // [E][5M]: fp32 F(0), G(0), f*_fc(0)
  int* CN = (int*)(sm + C::O_CN);
  double* QB = (double*)(sm + C::O_QB);  // [0..127] own means, [128 (1 + fc) + r] neighbour means
  float* QF = (float*)(sm + C::O_QF);
  int* ROT = (int*)(sm + C::O_ROT);
  uint64_t* mbar = (uint64_t*)(sm + C::O_MB);
  uint32_t* tslot = (uint32_t*)(sm + C::O_TS);
  volatile int* abort_flag = (volatile int*)(sm + C::O_TS + 4);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // ---- once per CTA: operators split into tf32 halves (K-major), zeroed A region
  for (int i = tid; i < C::NA * K1; i += kMixThreads) {
    const int r = i / K1, k = i % K1;
    double v = 0.0;
    if (k < NP) {
      if (r < NC) v = d.V[r * NP + k];
      else if (r >= C::NC8 && r < C::NC8 + NF) v = d.I[(r - C::NC8) * NP + k];
    }
    const float h = umma::to_tf32((float)v);
    const float l = umma::to_tf32((float)(v - (double)h));
    *(float*)(B1h + umma::kmajor_offset(r, k, K1)) = h;
    *(float*)(B1l + umma::kmajor_offset(r, k, K1)) = l;
  }
  // B2: volume chunks (Dr, Ds at cubature points, weights folded in), then per
  // face the LIFT columns times the Gauss weights
  for (int i = tid; i < C::NPN * C::KB2; i += kMixThreads) {
    const int r = i / C::KB2, k = i % C::KB2;
    double v = 0.0;
    if (r < NP) {
      if (k < C::NV * KV) {
        const int c = VPC * (k / KV) + (k % KV) / 2;
        if (c < NC) v = (k & 1) ? d.Ds[r * NC + c] : d.Dr[r * NC + c];
      } else {
        const int kk = k - C::NV * KV, fc = kk / 16, g = kk % 16;
        if (g < NG) v = d.L[r * NF + fc * NG + g] * d.gw[g];
      }
    }
    const float h = umma::to_tf32((float)v);
    const float l = umma::to_tf32((float)(v - (double)h));
    *(float*)(B2h + umma::kmajor_offset(r, k, C::KB2)) = h;
    *(float*)(B2l + umma::kmajor_offset(r, k, C::KB2)) = l;
  }
  for (int i = tid; i < C::SZ_U / 16; i += kMixThreads) ((float4*)U)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int i = tid; i < NP * 5; i += kMixThreads) RSUM[i] = rowsum[i];
  for (int i = tid; i < 3 * NP; i += kMixThreads) ROT[i] = rot[i];
  if (tid == 0) {
    for (int b = 0; b < 1 + C::NBUF; ++b) umma::mbar_init(umma::smem_u32(mbar + b), 1);
    *abort_flag = 0;
  }
  if (warp == 0) umma::tmem_alloc(umma::smem_u32(tslot), C::TCOLS);
  umma::fence_proxy_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tb = *tslot;
  const uint32_t tlane = tb + ((uint32_t)(32 * (warp & 3)) << 16);

  const uint32_t id_A = umma::idesc_tf32(128, C::NA);
  const uint32_t id_3 = umma::idesc_tf32(128, C::N3);
  const uint32_t id_B = umma::idesc_tf32(128, C::NPN);
  const uint32_t sB1h = umma::smem_u32(B1h), sB1l = umma::smem_u32(B1l);
  const uint32_t sB2h = umma::smem_u32(B2h), sB2l = umma::smem_u32(B2l);
  const uint32_t sU = umma::smem_u32(U);
  const uint32_t sbo1 = K1 * 32, sboB2 = C::KB2 * 32, sboCH = KV * 32;
  const uint32_t b3_off = (C::NC8 / 8) * sbo1;  // B1 from its face-0 Gauss-point rows on

  const double tstage = a.time_from_state ? d.st->t + d.st->dt * a.frac : a.t_arg;
  const double dt = a.time_from_state ? d.st->dt : a.dt_arg;
  const bool want_lambda = a.mode != MODE_STAGE;
  int err = 0;
  double lmax = 0.0;
  uint32_t phA = 0, ring_uses[C::NBUF];
#pragma unroll
  for (int b = 0; b < C::NBUF; ++b) ring_uses[b] = 0;
  uint32_t chunk_counter = 0;

  // row (element, field) of a tile row index
  const int rr = tid & 127, rq = rr >> 5, rln = rr & 31;
  const int rel = rln / M, rf = rln - rel * M, re = rq * EPQ + rel;
  auto rowb_of = [](int e) { return (e / EPQ) * 32 + (e % EPQ) * M; };

  // fp32 pointwise physics, identical wherever it is evaluated
  auto flux32 = [&](const float* qc, float* F, float* G) { P::flux2(d.eqp, qc, F, G, &err); };
  auto bc_coords = [&](int e, int fc, int g, double& x, double& y) {
    const ElemGeo& geo = d.geo[e];
    const double z = d.gz[g];
    double r, s;
    if (fc == 0) { r = z; s = -1.0; }
    else if (fc == 1) { r = -z; s = z; }
    else { r = -1.0; s = -z; }
    x = 0.5 * (-geo.vx[0] * (r + s) + geo.vx[1] * (1. + r) + geo.vx[2] * (1. + s));
    y = 0.5 * (-geo.vy[0] * (r + s) + geo.vy[1] * (1. + r) + geo.vy[2] * (1. + s));
  };
  // Lax-Friedrichs flux on face fc at Gauss point g, fp32, float normals
  auto numflux32 = [&](int e, int k, int fc, int g, const float* qM, float* qP, float* nf) {
    const float* G = GEO + e * 16;
    const float nx = G[5 + fc], ny = G[8 + fc];
    const int nb = CN[e * 6 + 2 * fc];
    if (nb < 0) {
      double x, y;
      bc_coords(k, fc, g, x, y);
      apply_bc<EQ, float>(d.bcs, -nb, tstage, x, y, nx, ny, qM, qP);
    }
    float qMc[M];
#pragma unroll
    for (int f = 0; f < M; ++f) qMc[f] = qM[f];
    return P::numflux(d.eqp, nx, ny, qMc, qP, nf, &err);
  };

  const int ntiles = (d.K + E - 1) / E;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int k0 = tile * E;
    const int ne = min(E, d.K - k0);
    const bool rvalid = rel < EPQ && re < ne;
    // ---- operands: own deviations (A1) and, per face, the neighbour's deviations
    // rotated so that the shared face is its face 0 (A3); 4 x 128 row tasks
    for (int task = tid; task < 4 * 128; task += kMixThreads) {
      const int kind = task >> 7, r = task & 127;  // kind 0: own, 1..3: face kind - 1
      const int q = r >> 5, ln = r & 31, el = ln / M, f = ln - el * M, e = q * EPQ + el;
      const bool valid = el < EPQ && e < ne;
      int src = -1, f2 = 0;
      if (valid) {
        if (kind == 0) {
          src = k0 + e;
        } else {
          src = d.conn[(size_t)(k0 + e) * 6 + 2 * (kind - 1)];
          f2 = d.conn[(size_t)(k0 + e) * 6 + 2 * (kind - 1) + 1];
        }
      }
      double qv[NP], qbar = 0.0;
      if (src >= 0) {
        const int* pr = ROT + f2 * NP;
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          const int jj = kind == 0 ? j : pr[j];
          qv[j] = a.x[((size_t)src * NP + jj) * M + f];
          qbar += qv[j];
        }
        qbar *= 1.0 / NP;
      }
      unsigned char* Ah = U + 2 * kind * C::SZ_A1;
      unsigned char* Al = Ah + C::SZ_A1;
#pragma unroll
      for (int j4 = 0; j4 < K1; j4 += 4) {
        float hv[4], lv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int j = j4 + u;
          float x = 0.f;
          if (src >= 0 && j < NP) x = (float)(qv[j] - qbar);
          split_trunc(x, hv[u], lv[u]);
        }
        const uint32_t off = umma::kmajor_offset(r, j4, K1);
        *(float4*)(Ah + off) = make_float4(hv[0], hv[1], hv[2], hv[3]);
        *(float4*)(Al + off) = make_float4(lv[0], lv[1], lv[2], lv[3]);
      }
      QB[128 * kind + r] = qbar;
      QF[128 * kind + r] = (float)qbar;
      if (kind == 0 && valid && f == 0) {
        const int k = k0 + e;
#pragma unroll
        for (int i = 0; i < 6; ++i) CN[e * 6 + i] = d.conn[(size_t)k * 6 + i];
        const ElemGeo& g = d.geo[k];
        float* G = GEO + e * 16;
        G[0] = (float)g.rx; G[1] = (float)g.ry; G[2] = (float)g.sx; G[3] = (float)g.sy; G[4] = (float)g.invJ;
#pragma unroll
        for (int fc = 0; fc < 3; ++fc) {
          G[5 + fc] = (float)g.nx[fc];
          G[8 + fc] = (float)g.ny[fc];
          G[11 + fc] = (float)(g.sJ[fc] * g.invJ);
        }
      }
    }
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < K1 / 8; ++s) {
        const uint32_t off = s * 2 * umma::kLBO;
        const uint64_t a1h = umma::make_desc(sU + off, umma::kLBO, sbo1);
        const uint64_t a1l = umma::make_desc(sU + C::SZ_A1 + off, umma::kLBO, sbo1);
        const uint64_t b1h = umma::make_desc(sB1h + off, umma::kLBO, sbo1);
        const uint64_t b1l = umma::make_desc(sB1l + off, umma::kLBO, sbo1);
        umma::mma_tf32(tb + C::T_D1, a1h, b1h, id_A, s > 0);
        umma::mma_tf32(tb + C::T_D1, a1h, b1l, id_A, 1);
        umma::mma_tf32(tb + C::T_D1, a1l, b1h, id_A, 1);
        const uint64_t b3h = umma::make_desc(sB1h + b3_off + off, umma::kLBO, sbo1);
        const uint64_t b3l = umma::make_desc(sB1l + b3_off + off, umma::kLBO, sbo1);
#pragma unroll
        for (int fc = 0; fc < 3; ++fc) {
          const uint32_t base = sU + 2 * (1 + fc) * C::SZ_A1;
          const uint64_t a3h = umma::make_desc(base + off, umma::kLBO, sbo1);
          const uint64_t a3l = umma::make_desc(base + C::SZ_A1 + off, umma::kLBO, sbo1);
          const uint32_t td = tb + C::T_D3 + fc * C::N3;
          umma::mma_tf32(td, a3h, b3h, id_3, s > 0);
          umma::mma_tf32(td, a3h, b3l, id_3, 1);
          umma::mma_tf32(td, a3l, b3h, id_3, 1);
        }
      }
      umma::commit(umma::smem_u32(mbar));
    }
    if (!umma::mbar_wait_bounded(umma::smem_u32(mbar), phA & 1)) *abort_flag = 1;
    phA++;
    umma::fence_after_sync();
    // ---- staged cubature values (first wave) and the g = 0 traces, as
    // deviations; the means are added in the precision of use
    auto stage_wave = [&](int c_begin) {
      if (tid < 128) {
#pragma unroll 1
        for (int c0 = 0; c0 < SR && c_begin + c0 < NC; c0 += 16) {
          float v[16];
          umma::tmem_ld16(tlane + C::T_D1 + c_begin + c0, v);
          umma::tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 16; ++j) ST[(c0 + j) * 128 + rr] = v[j];
        }
      }
    };
    stage_wave(0);
    if (tid < 128) {
#pragma unroll 1
      for (int fc = 0; fc < 3; ++fc) {
        float v[16];
        umma::tmem_ld16(tlane + C::T_D1 + C::NC8 + fc * NG, v);
        umma::tmem_wait_ld();
        G0[fc * 128 + rr] = v[0];
      }
    } else if (tid < 256) {
      // the partner's g = 0 is its last Gauss point (reversed order)
#pragma unroll 1
      for (int fc = 0; fc < 3; ++fc) {
        float v[16];
        umma::tmem_ld16(tlane + C::T_D3 + fc * C::N3, v);
        umma::tmem_wait_ld();
        G0[(3 + fc) * 128 + rr] = v[NG - 1];
      }
    }
    __syncthreads();
    if (*abort_flag) break;
    // ---- point-0 references.  The fp32 values are what every other point's
    // deviation is taken from (so a uniform state has zero deviations); the
    // float64 constants multiply the operator row sums with float64 metrics
    // and normals, which keeps a uniform flow exactly steady.
    for (int it = tid; it < ne * 4; it += kMixThreads) {
      const int e = it >> 2, kind = it & 3, rowb = rowb_of(e), k = k0 + e;
      const ElemGeo& geo = d.geo[k];
      float* p0 = P0 + e * 5 * M;
      if (kind == 0) {
        float qc[M], F[M], G[M];
#pragma unroll
        for (int f = 0; f < M; ++f) qc[f] = QF[rowb + f] + ST[rowb + f];
        flux32(qc, F, G);
#pragma unroll
        for (int f = 0; f < M; ++f) {
          p0[f] = F[f];
          p0[M + f] = G[f];
          Rb[e * 2 * M + f] = geo.rx * (double)F[f] + geo.ry * (double)G[f];
          Rb[e * 2 * M + M + f] = geo.sx * (double)F[f] + geo.sy * (double)G[f];
        }
      } else {
        const int fc = kind - 1;
        float qM[M], qP[M], nf[M];
#pragma unroll
        for (int f = 0; f < M; ++f) {
          qM[f] = QF[rowb + f] + G0[fc * 128 + rowb + f];
          qP[f] = QF[128 * (1 + fc) + rowb + f] + G0[(3 + fc) * 128 + rowb + f];
        }
        numflux32(e, k, fc, 0, qM, qP, nf);
        // float64 flux of the same fp32 traces with float64 normals
        double dM[M], dP[M], nf64[M];
#pragma unroll
        for (int f = 0; f < M; ++f) { dM[f] = qM[f]; dP[f] = qP[f]; }
        P::numflux(d.eqp, geo.nx[fc], geo.ny[fc], dM, dP, nf64, &err);
        const double w = -geo.sJ[fc] * geo.invJ;
#pragma unroll
        for (int f = 0; f < M; ++f) {
          p0[(2 + fc) * M + f] = nf[f];
          Fb[(e * 3 + fc) * M + f] = nf64[f] * w;
        }
      }
    }
    __syncthreads();
    // ---- contraction with the weighted derivative and LIFT operators, by chunks
    auto claim = [&](int b) {
      if (ring_uses[b] > 0 &&
          !umma::mbar_wait_bounded(umma::smem_u32(mbar + 1 + b), (ring_uses[b] - 1) & 1))
        *abort_flag = 1;
      ring_uses[b]++;
    };
    auto issue_chunk = [&](int b, uint32_t b2off, int ksteps, bool first) {
      umma::fence_proxy_async();
      umma::fence_before_sync();
      __syncthreads();
      umma::fence_after_sync();
      if (tid == 0) {
        const uint32_t ah0 = sU + b * 2 * C::SZ_CH, al0 = ah0 + C::SZ_CH;
        for (int s = 0; s < ksteps; ++s) {
          const uint32_t off = s * 2 * umma::kLBO;
          const uint64_t ah = umma::make_desc(ah0 + off, umma::kLBO, sboCH);
          const uint64_t al = umma::make_desc(al0 + off, umma::kLBO, sboCH);
          const uint64_t bh = umma::make_desc(sB2h + b2off + off, umma::kLBO, sboB2);
          const uint64_t bl = umma::make_desc(sB2l + b2off + off, umma::kLBO, sboB2);
          umma::mma_tf32(tb + C::T_D2, ah, bh, id_B, (first && s == 0) ? 0u : 1u);
          umma::mma_tf32(tb + C::T_D2, ah, bl, id_B, 1);
          umma::mma_tf32(tb + C::T_D2, al, bh, id_B, 1);
        }
        umma::commit(umma::smem_u32(mbar + 1 + b));
      }
    };
    // volume: deviation of the fp32 flux from its point-0 value, times the metric
    auto vol_item = [&](int e, int cp, int c, unsigned char* bh, unsigned char* bl) {
      const int rowb = rowb_of(e);
      const float* p0 = P0 + e * 5 * M;
      float qc[M], F[M], G[M];
      load_fields<M>(ST + (c % SR) * 128 + rowb, qc);
#pragma unroll
      for (int f = 0; f < M; ++f) qc[f] += QF[rowb + f];
      flux32(qc, F, G);
      const float4 g = *(const float4*)(GEO + e * 16);
#pragma unroll
      for (int f = 0; f < M; ++f) {
        const float dF = F[f] - p0[f], dG = G[f] - p0[M + f];
        float h0, l0, h1, l1;
        split_trunc(g.x * dF + g.y * dG, h0, l0);
        split_trunc(g.z * dF + g.w * dG, h1, l1);
        const uint32_t off = umma::kmajor_offset(rowb + f, 2 * cp, KV);
        *(float2*)(bh + off) = make_float2(h0, h1);
        *(float2*)(bl + off) = make_float2(l0, l1);
      }
    };
    for (int ch = 0; ch < C::NV; ++ch) {
      if (ch > 0 && (ch * VPC) % SR == 0) {
        // next staging wave (the previous chunk's items are done: issue barrier)
        stage_wave(ch * VPC);
        __syncthreads();
      }
      const int b = chunk_counter++ % C::NBUF;
      claim(b);
      unsigned char* bh = U + b * 2 * C::SZ_CH;
      unsigned char* bl = bh + C::SZ_CH;
      for (int it = tid; it < ne * VPC; it += kMixThreads) {
        const int e = it / VPC, cp = it - e * VPC, c = ch * VPC + cp;
        if (c < NC) vol_item(e, cp, c, bh, bl);
      }
      issue_chunk(b, ch * (KV / 4) * umma::kLBO, KV / 8, ch == 0);
    }
    for (int fc = 0; fc < 3; ++fc) {
      // own (rows 0..NG-1) and partner (rows 16..16+NG-1) traces of this face
      if (tid < 128) {
        float v[16];
        umma::tmem_ld16(tlane + C::T_D1 + C::NC8 + fc * NG, v);
        umma::tmem_wait_ld();
        const float qb = QF[rr];
#pragma unroll
        for (int j = 0; j < NG; ++j) ST[j * 128 + rr] = qb + v[j];
      } else if (tid < 256) {
        float v[16];
        umma::tmem_ld16(tlane + C::T_D3 + fc * C::N3, v);
        umma::tmem_wait_ld();
        const float qbn = QF[128 * (1 + fc) + rr];
#pragma unroll
        for (int j = 0; j < NG; ++j) ST[(16 + j) * 128 + rr] = qbn + v[NG - 1 - j];
      }
      const int b = chunk_counter++ % C::NBUF;
      claim(b);
      __syncthreads();
      unsigned char* bh = U + b * 2 * C::SZ_CH;
      unsigned char* bl = bh + C::SZ_CH;
      for (int it = tid; it < ne * NG; it += kMixThreads) {
        const int e = it / NG, g = it - e * NG, rowb = rowb_of(e), k = k0 + e;
        float qM[M], qP[M], nf[M];
        load_fields<M>(ST + g * 128 + rowb, qM);
        load_fields<M>(ST + (16 + g) * 128 + rowb, qP);
        const float lam = numflux32(e, k, fc, g, qM, qP, nf);
        if (want_lambda) {
          const double l = fabs((double)lam);
          lmax = l > lmax ? l : lmax;
        }
        const float w = -GEO[e * 16 + 11 + fc];
        const float* p0 = P0 + e * 5 * M + (2 + fc) * M;
#pragma unroll
        for (int f = 0; f < M; ++f) {
          float h, l;
          split_trunc(w * (nf[f] - p0[f]), h, l);
          const uint32_t off = umma::kmajor_offset(rowb + f, g, KV);
          *(float*)(bh + off) = h;
          *(float*)(bl + off) = l;
        }
      }
      issue_chunk(b, (C::NV * KV + 16 * fc) / 4 * umma::kLBO, 2, false);
    }
    // ---- wait for the last chunk, epilogue ----------------------------------------
    {
      const int blast = (chunk_counter - 1) % C::NBUF;
      if (!umma::mbar_wait_bounded(umma::smem_u32(mbar + 1 + blast), (ring_uses[blast] - 1) & 1)) *abort_flag = 1;
    }
    __syncthreads();
    umma::fence_after_sync();
    if (tid < 128 && !*abort_flag) {
      float dv[C::NPN];
#pragma unroll
      for (int c0 = 0; c0 < C::NPN; c0 += 16) {
        float v[16];
        umma::tmem_ld16(tlane + C::T_D2 + c0, v);
        umma::tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) dv[c0 + j] = v[j];
      }
      if (rvalid) {
        const int k = k0 + re;
        const double Rbar = Rb[re * 2 * M + rf], Sbar = Rb[re * 2 * M + M + rf];
        const double F0 = Fb[(re * 3 + 0) * M + rf], F1 = Fb[(re * 3 + 1) * M + rf], F2 = Fb[(re * 3 + 2) * M + rf];
        const double c_stage = dt / 4.0, c_al = 4.0 / 5.0, c_be = dt / 5.0, c_ga = 1.0 / 5.0;
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          const double* rs = RSUM + i * 5;
          const double r = (double)dv[i] + rs[0] * Rbar + rs[1] * Sbar + rs[2] * F0 + rs[3] * F1 + rs[4] * F2;
          if (r != r) err |= ERRB_NAN;
          const size_t off = ((size_t)k * NP + i) * M + rf;
          double o;
          if (a.mode == MODE_RHS) o = r;
          else if (a.mode == MODE_STAGE) o = a.x[off] + c_stage * r;
          else o = c_al * a.x[off] + c_be * r + c_ga * a.u0[off];
          a.out[off] = o;
        }
      }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (*abort_flag) break;
  }
  if (*abort_flag && tid == 0) atomicOr(&d.st->err, ERRB_TIMEOUT);
  if (want_lambda) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double v = __shfl_xor_sync(0xffffffffu, lmax, o);
      lmax = v > lmax ? v : lmax;
    }
    if (lane == 0 && lmax > 0.0) atomicMax(&d.st->lam_bits, (unsigned long long)__double_as_longlong(lmax));
  }
  if (err) atomicOr(&d.st->err, err);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tb, C::TCOLS);
}

template <int EQ, int N>
cudaError_t launch_mixed_t(MixedPlan* p, const DgDev& d, const StageArgs& a, cudaStream_t s, cudaEvent_t* ev) {
  using C = MixCfg<N, Eq<EQ>::M>;
  if constexpr (!C::FITS) {
    return cudaErrorNotSupported;
  } else {
  static unsigned configured = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(configured & (1u << (dev & 31)))) {
    cudaError_t e = cudaFuncSetAttribute(k_mixed_stage<EQ, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::BYTES);
    if (e != cudaSuccess) return e;
    configured |= 1u << (dev & 31);
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int per_sm = max_c(1, min(512 / C::TCOLS, (228 * 1024) / (C::BYTES + 1024)));
  const int ntiles = (d.K + C::E - 1) / C::E;
  int grid = sms * per_sm;
  if (grid > ntiles) grid = ntiles;
  if (a.reset_lambda && a.mode != MODE_STAGE) {
    cudaError_t e = cudaMemsetAsync(&d.st->lam_bits, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
  }
  if (ev) cudaEventRecord(ev[0], s);
  k_mixed_stage<EQ, N><<<grid, kMixThreads, C::BYTES, s>>>(d, a, p->rowsum, p->rot);
  if (ev) {
    cudaEventRecord(ev[1], s);
    cudaEventRecord(ev[2], s);
    cudaEventRecord(ev[3], s);
  }
  return cudaGetLastError();
  }
}

template <int EQ, int N> constexpr bool mixed_fits() { return MixCfg<N, Eq<EQ>::M>::FITS; }

template <int EQ> bool mixed_fits_n(int N) {
  switch (N) {
    case 2: return mixed_fits<EQ, 2>();
    case 3: return mixed_fits<EQ, 3>();
    case 4: return mixed_fits<EQ, 4>();
    case 5: return mixed_fits<EQ, 5>();
  }
  return false;
}

template <int EQ>
cudaError_t mixed_dispatch_n(MixedPlan* p, const DgDev& d, const StageArgs& a, cudaStream_t s, cudaEvent_t* ev) {
  switch (d.N) {
    case 2: return launch_mixed_t<EQ, 2>(p, d, a, s, ev);
    case 3: return launch_mixed_t<EQ, 3>(p, d, a, s, ev);
    case 4: return launch_mixed_t<EQ, 4>(p, d, a, s, ev);
    case 5: return launch_mixed_t<EQ, 5>(p, d, a, s, ev);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

MixedPlan* mixed_create(int eq, const RefOps& o, int K, int M) {
  if (o.N < 2 || o.N > 5) return nullptr;
  bool fits = false;
  switch (eq) {
    case EQ_ADVECTION: fits = mixed_fits_n<EQ_ADVECTION>(o.N); break;
    case EQ_EULER: fits = mixed_fits_n<EQ_EULER>(o.N); break;
    case EQ_MAXWELL: fits = mixed_fits_n<EQ_MAXWELL>(o.N); break;
    case EQ_EULER2D: fits = mixed_fits_n<EQ_EULER2D>(o.N); break;
    case EQ_MAXWELL_TM: fits = mixed_fits_n<EQ_MAXWELL_TM>(o.N); break;
  }
  if (!fits) return nullptr;
  MixedPlan* p = new MixedPlan();
  p->eq = eq;
  p->N = o.N;
  p->M = M;
  std::vector<double> rs((size_t)o.Np * 5, 0.0);
  for (int i = 0; i < o.Np; ++i) {
    for (int c = 0; c < o.Nc; ++c) {
      rs[i * 5 + 0] += o.DrW(i, c);
      rs[i * 5 + 1] += o.DsW(i, c);
    }
    for (int fc = 0; fc < 3; ++fc)
      for (int g = 0; g < o.Ng; ++g) rs[i * 5 + 2 + fc] += o.Lift(i, fc * o.Ng + g) * o.gw[g];
  }
  if (o.rot.empty() || cudaMalloc((void**)&p->rowsum, rs.size() * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&p->rot, o.rot.size() * sizeof(int)) != cudaSuccess) {
    mixed_destroy(p);
    return nullptr;
  }
  cudaMemcpy(p->rowsum, rs.data(), rs.size() * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(p->rot, o.rot.data(), o.rot.size() * sizeof(int), cudaMemcpyHostToDevice);
  return p;
}

void mixed_destroy(MixedPlan* p) {
  if (!p) return;
  if (p->rowsum) cudaFree(p->rowsum);
  if (p->rot) cudaFree(p->rot);
  delete p;
}

cudaError_t mixed_launch_rhs(MixedPlan* p, int eq, const DgDev& d, const StageArgs& a, cudaStream_t s,
                             cudaEvent_t* ev) {
  switch (eq) {
    case EQ_ADVECTION: return mixed_dispatch_n<EQ_ADVECTION>(p, d, a, s, ev);
    case EQ_EULER: return mixed_dispatch_n<EQ_EULER>(p, d, a, s, ev);
    case EQ_MAXWELL: return mixed_dispatch_n<EQ_MAXWELL>(p, d, a, s, ev);
    case EQ_EULER2D: return mixed_dispatch_n<EQ_EULER2D>(p, d, a, s, ev);
    case EQ_MAXWELL_TM: return mixed_dispatch_n<EQ_MAXWELL_TM>(p, d, a, s, ev);
    default: return cudaErrorInvalidValue;
  }
}

namespace {

// One CTA of 128 threads: D[128 x n] = A[128 x k] * B[n x k]^T on the tensor
// cores, kind::tf32, optionally as the 3-term split Ahi Bhi + Ahi Blo + Alo Bhi.
// Operand regions are followed by zeroed guard space so that every address the
// descriptors can form stays inside the block's shared memory.
__global__ void k_umma_selftest(const float* A, const float* B, float* D, int n, int k, int split, int* info) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int regA = 128 * k * 4, regB = n * k * 4;
  unsigned char* pAh = sm;
  unsigned char* pAl = pAh + 2 * regA;
  unsigned char* pBh = pAl + 2 * regA;
  unsigned char* pBl = pBh + 2 * regB;
  uint64_t* mbar = (uint64_t*)(pBl + 2 * regB);
  uint32_t* tslot = (uint32_t*)(mbar + 1);
  const int total = 4 * regA + 4 * regB;
  for (int i = tid; i < total / 4; i += blockDim.x) ((float*)sm)[i] = 0.f;
  __syncthreads();
  for (int i = tid; i < 128 * k; i += blockDim.x) {
    const int r = i / k, c = i % k;
    const float x = A[i];
    const float h = umma::to_tf32(x);
    const float l = umma::to_tf32(x - h);
    *(float*)(pAh + umma::kmajor_offset(r, c, k)) = split ? h : x;
    *(float*)(pAl + umma::kmajor_offset(r, c, k)) = l;
  }
  for (int i = tid; i < n * k; i += blockDim.x) {
    const int r = i / k, c = i % k;
    const float x = B[i];
    const float h = umma::to_tf32(x);
    const float l = umma::to_tf32(x - h);
    *(float*)(pBh + umma::kmajor_offset(r, c, k)) = split ? h : x;
    *(float*)(pBl + umma::kmajor_offset(r, c, k)) = l;
  }
  if (tid == 0) umma::mbar_init(umma::smem_u32(mbar), 1);
  if (warp == 0) umma::tmem_alloc(umma::smem_u32(tslot), 256);
  umma::fence_proxy_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = *tslot;
  if (tid == 0) {
    const uint32_t idesc = umma::idesc_tf32(128, n);
    const uint32_t sbo_a = k * 32, sbo_b = k * 32;
    const int steps = k / 8;
    uint32_t acc = 0;
    for (int s = 0; s < steps; ++s) {
      const uint32_t off = s * 2 * umma::kLBO;
      const uint64_t ah = umma::make_desc(umma::smem_u32(pAh) + off, umma::kLBO, sbo_a);
      const uint64_t bh = umma::make_desc(umma::smem_u32(pBh) + off, umma::kLBO, sbo_b);
      umma::mma_tf32(tbase, ah, bh, idesc, acc);
      acc = 1;
      if (split) {
        const uint64_t al = umma::make_desc(umma::smem_u32(pAl) + off, umma::kLBO, sbo_a);
        const uint64_t bl = umma::make_desc(umma::smem_u32(pBl) + off, umma::kLBO, sbo_b);
        umma::mma_tf32(tbase, ah, bl, idesc, 1);
        umma::mma_tf32(tbase, al, bh, idesc, 1);
      }
    }
    umma::commit(umma::smem_u32(mbar));
  }
  const bool ok = umma::mbar_wait_bounded(umma::smem_u32(mbar), 0);
  if (!ok && lane == 0) atomicOr(info, 1);
  umma::fence_after_sync();
  if (ok) {
    const int row = 32 * (warp & 3) + lane;
    for (int c0 = 0; c0 < n; c0 += 16) {
      float v[16];
      umma::tmem_ld16(tbase + ((uint32_t)(32 * (warp & 3)) << 16) + c0, v);
      umma::tmem_wait_ld();
      for (int j = 0; j < 16 && c0 + j < n; ++j) D[row * n + c0 + j] = v[j];
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tbase, 256);
}

}  // namespace

}  // namespace apollo

// Tensor-core self-test for the test suite (no counterpart in Apollo):
// D[128 x n] = A[128 x k] B[n x k]^T, host arrays, n in {16..256} step 16,
// k in {8, 16, 24, 32}; returns 0 on success, 1 bad size, 2 CUDA error,
// 3 device wait timed out.
extern "C" int apollo_dg_selftest_umma(int n, int k, const float* A, const float* B, float* D, int split) {
  using namespace apollo;
  if (n < 16 || n > 256 || n % 16 || k < 8 || k > 32 || k % 8) return 1;
  float *dA = nullptr, *dB = nullptr, *dD = nullptr;
  int* dinfo = nullptr;
  int info = 0;
  int rc = 0;
  // operands, their guard copies, the mbarrier and 16 KB of trailing guard
  const size_t smem = 4 * (128 * k * 4) + 4 * (n * k * 4) + 64 + 16384;
  if (cudaMalloc(&dA, 128 * k * 4) || cudaMalloc(&dB, n * k * 4) || cudaMalloc(&dD, 128 * n * 4) ||
      cudaMalloc(&dinfo, 4)) {
    rc = 2;
  } else {
    cudaMemcpy(dA, A, 128 * k * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B, n * k * 4, cudaMemcpyHostToDevice);
    cudaMemset(dD, 0, 128 * n * 4);
    cudaMemset(dinfo, 0, 4);
    cudaFuncSetAttribute(k_umma_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_umma_selftest<<<1, 128, smem>>>(dA, dB, dD, n, k, split, dinfo);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = 2;
    cudaMemcpy(&info, dinfo, 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(D, dD, 128 * n * 4, cudaMemcpyDeviceToHost);
    if (!rc && info) rc = 3;
  }
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dD);
  cudaFree(dinfo);
  return rc;
}
