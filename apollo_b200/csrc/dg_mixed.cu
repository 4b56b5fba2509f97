// Mixed-precision right-hand side and SSP stage on the tcgen05 tensor cores.
//
// One fused kernel per Runge-Kutta stage.  A CTA takes a tile of elements;
// the 128 tensor-core rows are (element, field) pairs, 32 per warp quadrant
// (32 / M elements each, so an element never straddles two warps).  Every
// contraction runs on the tensor cores as kind::tf32 with a three-term split
// (hi*hi + hi*lo + lo*hi, fp32 accumulation in TMEM) and acts only on
// deviations from float64 reference values:
//
//   V q        = qbar + V (q - qbar)              (cubature values; qbar = nodal mean)
//   Dr R + Ds S = (Dr 1) R(qbar) + (Ds 1) S(qbar)
//               + Dr (R - R(qbar)) + Ds (S - S(qbar))   (R = rx F + ry G, S = sx F + sy G)
//   L f*       = sum_f (L_f w 1) f*_f(qbar) + L w (f* - f*_f(qbar))
//
// The reference fluxes are evaluated from the same fp32 mean as the pointwise
// fluxes, so a uniform state has exactly zero deviations, and their float64
// counterparts (float64 metrics and normals) multiply float64 operator row
// sums.  Face traces are not recomputed from the neighbours' states: every
// stage that produces a state also writes its fp32 face traces
//   trace = float(mean) + I float(q - mean)            [K][3][NG][M]
// (k_mixed_traces computes the same values from any state), and the next
// stage reads its own and its partners' traces from that buffer.  A stage
// therefore reads only its own elements' state, so it may update in place.
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
  double* rowsum = nullptr;  // [NP][5]: Dr 1, Ds 1, L_0 w 1, L_1 w 1, L_2 w 1 (float64)
};

namespace {

constexpr int kMixThreads = 384;
constexpr int round_up_c(int x, int m) { return (x + m - 1) / m * m; }
constexpr int tmem_cols(int x) { return x <= 32 ? 32 : x <= 64 ? 64 : x <= 128 ? 128 : x <= 256 ? 256 : 512; }
// floats per (element, face) block of the trace buffer: NG points x M fields,
// padded to 16 bytes so that every block can be moved by a bulk copy
constexpr int trace_stride(int NG, int M) { return round_up_c(NG * M, 4); }

// SH selects the operand chunking: 0 = chunks of 24 K columns (16 at N = 5)
// through a two-buffer ring, 1 = chunks of 16 through a three-buffer ring.
// Both issue the same MMAs in the same K order (chunks start on 8-column
// boundaries), so they compute the same result bit for bit; the batch
// autotuner picks the faster per order.
template <int N, int M, int SH = 0> struct MixCfg {
  static constexpr int NP = Sizes<N>::NP, NC = Sizes<N>::NC, NG = Sizes<N>::NG, NF = Sizes<N>::NF;
  static constexpr int EPQ = 32 / M;  // elements per warp quadrant
  static constexpr int E = 4 * EPQ;   // elements per tile
  static constexpr int K1 = round_up_c(NP, 8);
  static constexpr int GA = K1 / 4 <= 2 ? 2 : K1 / 4 <= 4 ? 4 : 8;  // lanes per row in the operand build
  static constexpr int KV = (SH == 1 || N >= 5) ? 16 : 24;  // K columns per chunk
  static constexpr int VPC = KV / 2;                  // cubature points per volume chunk (R, S each)
  static constexpr int NV = (NC + VPC - 1) / VPC;     // volume chunks
  static constexpr int NFK = round_up_c(NF, 8);       // face columns (fc NG + g, packed)
  static constexpr int NFC = (NFK + KV - 1) / KV;     // face chunks
  static constexpr int NCH = NV + NFC;
  static constexpr int NC16 = round_up_c(NC, 16);
  static constexpr int NPN = round_up_c(NP, 16);
  static constexpr int KB2 = NCH * KV;
  static constexpr int NBUF = SH == 1 ? 3 : 2;
  static constexpr int NWORK = kMixThreads - 32;      // worker threads; the last warp issues MMAs and copies
  static constexpr int TS = trace_stride(NG, M);      // floats per (element, face) trace block
  static constexpr int IFS = round_up_c(NP, 4);       // padded row of the interpolation operator
  // TMEM columns: cubature values, then the right-hand side
  static constexpr int T_D1 = 0, T_D2 = NC16;
  static constexpr int TCOLS = tmem_cols(NC16 + 2 * NPN);  // RHS: [hi part | lo part] of B2
  // K-major operand strides (bytes between 8-row groups)
  static constexpr int SBO1 = K1 * 32;       // B1 = V and the A operand
  static constexpr int SBO2 = KB2 * 32;      // B2 = [Dr Ds | L w], hi rows then lo rows
  static constexpr int SBOC = KV * 32 + 16;  // chunk operands, staggered across banks
  // shared memory, bytes (each operand as a tf32 hi half and lo half)
  static constexpr int SZ_B1 = (NC16 / 8) * SBO1;
  static constexpr int SZ_B2 = (NPN / 8) * SBO2;
  static constexpr int SZ_A = 16 * SBO1;
  static constexpr int SZ_CH = 16 * SBOC;
  static constexpr int SZ_ST = NC * 128 * 4;  // cubature deviations [NC][128] float
  static constexpr int SZ_XD = NP * 128 * 4;  // result deviations [NP][128] float
  static constexpr int XS_N = E * NP * M;     // one tile's state, doubles
  static constexpr int SZ_XS = round_up_c(XS_N * 8, 16);
  static constexpr int SZ_TR = E * 3 * TS * 4;  // one tile's own (or partner) traces
  // per-tile data, two slots (tile parity)
  static constexpr int TD_GEO = 0;                         // [13][E] float: rx ry sx sy, nx[3] ny[3] -sJ/J[3] at 4..12
  static constexpr int TD_CN = TD_GEO + 13 * E * 4;        // [E][6] int
  static constexpr int TD_QF = TD_CN + E * 6 * 4;          // [M][E] float own means
  static constexpr int TD_P0 = TD_QF + M * E * 4;          // [5M][E] float F, G, f*_fc at the mean
  static constexpr int TD_RB = round_up_c(TD_P0 + 5 * M * E * 4, 8);  // [2M][E] double R, S at the mean
  static constexpr int TD_FB = TD_RB + 2 * M * E * 8;      // [3M][E] double face references
  static constexpr int TD_G64 = TD_FB + 3 * M * E * 8;     // [13][E] double: rx ry sx sy, nx[3] ny[3] -sJ/J[3]
  static constexpr int SZ_TD = TD_G64 + 13 * E * 8;
  static constexpr int NMB = 8 + 2 * NBUF;
  static constexpr int LIMIT = 227 * 1024;
  static constexpr int fixed_bytes() {
    return round_up_c(2 * SZ_B1 + 2 * SZ_B2, 128) + 2 * SZ_A + NBUF * 2 * SZ_CH + SZ_ST + SZ_XD + 16 + SZ_XS +
           NF * IFS * 4 + 8 + NP * 5 * 8 + 2 * SZ_TD + 128 * 8 + 8 * NMB + 16;
  }
  // optional buffers, in order of benefit: traces in shared memory, a second state tile
  static constexpr bool TRS = fixed_bytes() + 2 * SZ_TR <= LIMIT;
  static constexpr bool XS2 = fixed_bytes() + (TRS ? 2 * SZ_TR : 0) + SZ_XS <= LIMIT;
  static constexpr int O_B1H = 0, O_B1L = O_B1H + SZ_B1;
  static constexpr int O_B2H = O_B1L + SZ_B1, O_B2L = O_B2H + SZ_B2;
  static constexpr int O_A = round_up_c(O_B2L + SZ_B2, 128);
  static constexpr int O_RING = O_A + 2 * SZ_A;
  static constexpr int O_ST = O_RING + NBUF * 2 * SZ_CH;
  static constexpr int O_XD = O_ST + SZ_ST;
  static constexpr int O_XS = round_up_c(O_XD + SZ_XD, 16);           // [1 or 2][XS_N] double
  static constexpr int O_TO = O_XS + (XS2 ? 2 : 1) * SZ_XS;           // [E][3][TS] float own traces
  static constexpr int O_TP = O_TO + (TRS ? SZ_TR : 0);               // [E][3][TS] float partner traces
  static constexpr int O_IF = O_TP + (TRS ? SZ_TR : 0);               // [NF][IFS] float interpolation
  static constexpr int O_RS = round_up_c(O_IF + NF * IFS * 4, 8);     // [NP][5] double row sums
  static constexpr int O_TD = O_RS + NP * 5 * 8;                      // 2 slots of per-tile data
  static constexpr int O_XB = O_TD + 2 * SZ_TD;                       // [128] double means of the result
  // mbarriers: state copy, A operand, GEMM-A done, tile RHS done, epilogue done,
  // traces landed, drain, (spare), ring full[NBUF], ring empty[NBUF]
  static constexpr int O_MB = O_XB + 128 * 8;
  static constexpr int O_TSL = O_MB + 8 * NMB;                        // TMEM base, abort flag
  static constexpr int BYTES = O_TSL + 16;
  static constexpr bool FITS = BYTES <= LIMIT;
  static_assert(KV % 8 == 0 && SZ_TD % 8 == 0 && (TS * 4) % 16 == 0, "layout");
};

// tf32 split of a per-point operand: hi keeps the top 19 bits of x, lo = x - hi
// is exact in fp32 and the tensor core reads its top 19 bits, so
// x = hi + lo + O(2^-21 |x|).  (The operators are split once per CTA with
// rounding to nearest.)
__device__ __forceinline__ void split_tf32(float x, float& h, float& l) {
  h = __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
  l = x - h;
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

// Nodal mean in a fixed order: sums of four consecutive nodes, then a binary
// tree over the group sums (padded with zeros to 2, 4 or 8 groups).  The
// operand build computes the same sums with lane shuffles, so every path
// gives the mean bit for bit.
template <int NP> constexpr int mean_groups() {
  return (NP + 3) / 4 <= 2 ? 2 : (NP + 3) / 4 <= 4 ? 4 : 8;
}
template <int NP>
__device__ __forceinline__ double group_sum(const double* v, int g) {
  const double a0 = 4 * g + 0 < NP ? v[4 * g + 0] : 0.0, a1 = 4 * g + 1 < NP ? v[4 * g + 1] : 0.0;
  const double a2 = 4 * g + 2 < NP ? v[4 * g + 2] : 0.0, a3 = 4 * g + 3 < NP ? v[4 * g + 3] : 0.0;
  return (a0 + a1) + (a2 + a3);
}
template <int NP>
__device__ __forceinline__ double tree_mean(const double* v) {
  constexpr int G = mean_groups<NP>();
  double s[G];
#pragma unroll
  for (int g = 0; g < G; ++g) s[g] = group_sum<NP>(v, g);
#pragma unroll
  for (int w = 1; w < G; w *= 2)
#pragma unroll
    for (int g = 0; g < G; g += 2 * w) s[g] = s[g] + s[g + w];
  return s[0] * (1.0 / NP);
}

// Face traces of one (element, field) row: for the NG Gauss points of face fc,
// float(m) + sum_j I[fc NG + g][j] dv[j] (fp32 fused multiply-adds in node
// order; IF rows padded to IFS floats).  Both the stage epilogue and
// k_mixed_traces call this, so the values agree bit for bit for one state.
template <int NP, int NG, int IFS>
__device__ __forceinline__ void row_traces(const float* __restrict__ IF, const float (&dv)[NP], double m, int fc,
                                           float* __restrict__ dst, int M) {
  const float mf = (float)m;
#pragma unroll 2
  for (int g = 0; g < NG; ++g) {
    const float4* Ig = (const float4*)(IF + (fc * NG + g) * IFS);
    float acc = 0.f;
#pragma unroll
    for (int q = 0; q < IFS / 4; ++q) {
      const float4 w = Ig[q];
      if (4 * q + 0 < NP) acc = fmaf(w.x, dv[4 * q + 0], acc);
      if (4 * q + 1 < NP) acc = fmaf(w.y, dv[4 * q + 1], acc);
      if (4 * q + 2 < NP) acc = fmaf(w.z, dv[4 * q + 2], acc);
      if (4 * q + 3 < NP) acc = fmaf(w.w, dv[4 * q + 3], acc);
    }
    dst[g * M] = mf + acc;
  }
}

// Worker-only barrier (named barrier 1; the control warp does not take part).
template <int NW>
__device__ __forceinline__ void workers_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(NW) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
// transaction bytes expected on an mbarrier, without an arrival
__device__ __forceinline__ void mbar_expect_tx_only(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// fp32 pointwise physics of the mixed kernel.  dirflux gives the fluxes along
// two directions, R = ax F + ay G and S = bx F + by G (the volume terms with
// the metric rows); lf gives the Lax-Friedrichs normal flux.  The generic form
// calls the equation's own flux2/numflux; the Euler form evaluates each
// state's velocities and pressure once, with one reciprocal, and forms the
// directional fluxes directly (the same quantities in exact arithmetic, with
// the reference's clamps and error flags, wxeulereqn.cc:809-871, :1097-1117).
template <int EQ> struct MixPhys {
  static constexpr int M = Eq<EQ>::M;
  __device__ __forceinline__ static void dirflux(const EqParams& P, const float* q, float ax, float ay, float bx,
                                                 float by, float* R, float* S, int* err) {
    float F[M], G[M];
    Eq<EQ>::flux2(P, q, F, G, err);
#pragma unroll
    for (int f = 0; f < M; ++f) {
      R[f] = ax * F[f] + ay * G[f];
      S[f] = bx * F[f] + by * G[f];
    }
  }
  __device__ __forceinline__ static float lf(const EqParams& P, float nx, float ny, const float* qM, const float* qP,
                                             float* nf, int* err) {
    float a[M], b[M];
#pragma unroll
    for (int f = 0; f < M; ++f) { a[f] = qM[f]; b[f] = qP[f]; }
    return Eq<EQ>::numflux(P, nx, ny, a, b, nf, err);
  }
};

template <int MF> struct MixPhysEuler {
  static constexpr int M = MF, IE = MF - 1;
  struct Side { float rho, ir, vx, vy, vz, p; bool clean; };
  // density and pressure clamped as in the flux of the reference; clean: no
  // clamp was needed and the density is positive
  __device__ __forceinline__ static Side side(const EqParams& P, const float* q, int* err) {
    const float g1 = (float)P.p[0] - 1.f, minP = (float)P.p[1], minD = (float)P.p[2];
    Side s;
    s.rho = q[0];
    s.clean = s.rho > 0.f && s.rho >= minD;
    if (minD == 0.f && s.rho <= 0.f) *err |= ERRB_NONPHYS;
    if (s.rho < minD) s.rho = minD;
    s.ir = 1.f / s.rho;
    s.vx = q[1] * s.ir;
    s.vy = q[2] * s.ir;
    s.vz = MF == 5 ? q[3] * s.ir : 0.f;
    s.p = g1 * (q[IE] - 0.5f * s.rho * (s.vx * s.vx + s.vy * s.vy + s.vz * s.vz));
    if (s.p <= 0.f) {
      s.clean = false;
      if (minP == 0.f) *err |= ERRB_NONPHYS;
      else s.p = minP;
    }
    return s;
  }
  // flux along the direction (ax, ay)
  __device__ __forceinline__ static void along(const Side& s, const float* q, float ax, float ay, float* R) {
    const float ua = s.vx * ax + s.vy * ay;
    R[0] = s.rho * ua;
    R[1] = s.rho * s.vx * ua + s.p * ax;
    R[2] = s.rho * s.vy * ua + s.p * ay;
    if (MF == 5) R[3] = s.rho * s.vz * ua;
    R[IE] = (q[IE] + s.p) * ua;
  }
  __device__ __forceinline__ static void dirflux(const EqParams& P, const float* q, float ax, float ay, float bx,
                                                 float by, float* R, float* S, int* err) {
    const Side s = side(P, q, err);
    along(s, q, ax, ay, R);
    along(s, q, bx, by, S);
  }
  __device__ __forceinline__ static float lf(const EqParams& P, float nx, float ny, const float* qM, const float* qP,
                                             float* nf, int* err) {
    const float gamma = (float)P.p[0];
    const Side a = side(P, qM, err), b = side(P, qP, err);
    // any clamp takes the reference's own path (its wave speeds use the
    // primitive variables with their own clamps)
    if (!(a.clean && b.clean)) {
      float x[M], y[M];
#pragma unroll
      for (int f = 0; f < M; ++f) { x[f] = qM[f]; y[f] = qP[f]; }
      return Eq<MF == 5 ? EQ_EULER : EQ_EULER2D>::numflux(P, nx, ny, x, y, nf, err);
    }
    float FM[M], FP[M];
    along(a, qM, nx, ny, FM);
    along(b, qP, nx, ny, FP);
    const float cM = sqrtf(a.vx * a.vx + a.vy * a.vy + a.vz * a.vz) + sqrtf(gamma * a.p * a.ir);
    const float cP = sqrtf(b.vx * b.vx + b.vy * b.vy + b.vz * b.vz) + sqrtf(gamma * b.p * b.ir);
    const float lam = cM > cP ? cM : cP;
#pragma unroll
    for (int c = 0; c < M; ++c) nf[c] = 0.5f * (FM[c] + FP[c] + lam * (qM[c] - qP[c]));
    return lam;
  }
};
template <> struct MixPhys<EQ_EULER> : MixPhysEuler<5> {};
template <> struct MixPhys<EQ_EULER2D> : MixPhysEuler<4> {};

// 16-byte asynchronous copy global -> shared (L2 only), and an mbarrier
// arrival once this thread's earlier copies have landed
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_arrive(uint32_t mbar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(mbar) : "memory");
}

// Stage kernel.  Warps 0..10 are workers, warp 11 is the control warp: its
// lane 0 issues every tcgen05 MMA and its lanes issue the bulk copies.  Per
// tile the workers build the A operand (state deviations), stage GEMM-A's
// cubature values, produce the chunk operands of GEMM-B into a two-buffer
// ring (full/empty mbarriers), and finish with the float64 epilogue and the
// result's face traces.  The next tile's operand build and GEMM-A overlap
// this tile's epilogue; per-tile data live in two slots by tile parity.
//
// GF (Euler kinds): the face flux is the equation's Numerical_Flux (HLL, Roe,
// Wave) in fp32 instead of the Lax-Friedrichs form, and the float64 face
// constants are that flux's value at the mean (a separate instantiation, so
// the Lax-Friedrichs kernels keep their registers).
template <int EQ, int N, int SH, bool GF = false>
__global__ void __launch_bounds__(kMixThreads, 1)
    k_mixed_stage(DgDev d, StageArgs a, const double* __restrict__ rowsum, int flags) {
  using P = Eq<EQ>;
  using Q = MixPhys<EQ>;
  constexpr int M = P::M;
  using C = MixCfg<N, M, SH>;
  constexpr int NP = C::NP, NC = C::NC, NG = C::NG, NF = C::NF, EPQ = C::EPQ, E = C::E, K1 = C::K1;
  constexpr int KV = C::KV, VPC = C::VPC, NV = C::NV, NW = C::NWORK, NBUF = C::NBUF, TS = C::TS;
  constexpr int IFS = C::IFS, GA = C::GA;
  static_assert(GA == mean_groups<NP>(), "the operand build's shuffle tree is the nodal-mean tree");
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* B1h = sm + C::O_B1H;
  unsigned char* B1l = sm + C::O_B1L;
  unsigned char* B2h = sm + C::O_B2H;
  unsigned char* B2l = sm + C::O_B2L;
  unsigned char* AOP = sm + C::O_A;
  unsigned char* RING = sm + C::O_RING;
  float* ST = (float*)(sm + C::O_ST);
  float* XD = (float*)(sm + C::O_XD);
  float* TO = (float*)(sm + C::O_TO);
  float* TP = (float*)(sm + C::O_TP);
  float* IF = (float*)(sm + C::O_IF);
  double* RSUM = (double*)(sm + C::O_RS);
  double* XB = (double*)(sm + C::O_XB);
  uint64_t* mbar = (uint64_t*)(sm + C::O_MB);
  uint32_t* tslot = (uint32_t*)(sm + C::O_TSL);
  volatile int* abort_flag = (volatile int*)(sm + C::O_TSL + 4);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool x_bulk = flags & 1, u0_prefetch = flags & 2;
  const uint32_t wlim = d.wait_limit ? d.wait_limit : (1u << 22);
  auto xs_buf = [&](int i) { return (double*)(sm + C::O_XS + (C::XS2 ? (i & 1) * C::SZ_XS : 0)); };

  // ---- once per CTA: operators split into tf32 halves (K-major)
  for (int i = tid; i < C::NC16 * K1; i += kMixThreads) {
    const int r = i / K1, k = i % K1;
    const double v = (r < NC && k < NP) ? d.V[r * NP + k] : 0.0;
    const float h = umma::round_tf32((float)v);
    const float l = umma::round_tf32((float)(v - (double)h));
    *(float*)(B1h + umma::kmajor_offset_sbo(r, k, C::SBO1)) = h;
    *(float*)(B1l + umma::kmajor_offset_sbo(r, k, C::SBO1)) = l;
  }
  // B2: volume chunks (Dr, Ds at cubature points, weights folded in), then the
  // face chunks: column fc NG + g is LIFT times the Gauss weight
  for (int i = tid; i < C::NPN * C::KB2; i += kMixThreads) {
    const int r = i / C::KB2, k = i % C::KB2;
    double v = 0.0;
    if (r < NP) {
      if (k < NV * KV) {
        const int c = VPC * (k / KV) + (k % KV) / 2;
        if (c < NC) v = (k & 1) ? d.Ds[r * NC + c] : d.Dr[r * NC + c];
      } else {
        const int col = k - NV * KV;
        if (col < NF) v = d.L[r * NF + col] * d.gw[col % NG];
      }
    }
    const float h = umma::round_tf32((float)v);
    const float l = umma::round_tf32((float)(v - (double)h));
    *(float*)(B2h + umma::kmajor_offset_sbo(r, k, C::SBO2)) = h;
    *(float*)(B2l + umma::kmajor_offset_sbo(r, k, C::SBO2)) = l;
  }
  for (int i = tid; i < (2 * C::SZ_A + NBUF * 2 * C::SZ_CH) / 16; i += kMixThreads)
    ((float4*)AOP)[i] = make_float4(0.f, 0.f, 0.f, 0.f);  // A operand and ring: finite padding
  for (int i = tid; i < NF * IFS; i += kMixThreads) IF[i] = (i % IFS) < NP ? (float)d.I[(i / IFS) * NP + i % IFS] : 0.f;
  for (int i = tid; i < NP * 5; i += kMixThreads) RSUM[i] = rowsum[i];
  // mbarriers: 0 state copy, 1 A operand (all workers), 2 GEMM-A done, 3 RHS
  // done, 4 epilogue done with the state tile (128 threads), 5 own traces
  // landed, 6 drain, 7 partner traces landed (warps 4..10), 8 + b ring buffer b full (all workers), 8 + NBUF + b ring buffer b empty
  const uint32_t mbX = umma::smem_u32(mbar + 0), mbA = umma::smem_u32(mbar + 1);
  const uint32_t mbD1 = umma::smem_u32(mbar + 2), mbD2 = umma::smem_u32(mbar + 3);
  const uint32_t mbE = umma::smem_u32(mbar + 4), mbT = umma::smem_u32(mbar + 5);
  const uint32_t mbDrain = umma::smem_u32(mbar + 6), mbTP = umma::smem_u32(mbar + 7);
  auto mb_full = [&](int b) { return umma::smem_u32(mbar + 8 + b); };
  auto mb_empty = [&](int b) { return umma::smem_u32(mbar + 8 + NBUF + b); };
  if (tid == 0) {
    umma::mbar_init(mbX, 1);
    umma::mbar_init(mbA, NW);
    umma::mbar_init(mbD1, 1);
    umma::mbar_init(mbD2, 1);
    umma::mbar_init(mbE, 128);
    umma::mbar_init(mbT, 1);
    umma::mbar_init(mbDrain, 1);
    umma::mbar_init(mbTP, NW - 128);
    for (int b = 0; b < NBUF; ++b) {
      umma::mbar_init(mb_full(b), NW);
      umma::mbar_init(mb_empty(b), 1);
    }
    *abort_flag = 0;
  }
  if (warp == 0) umma::tmem_alloc(umma::smem_u32(tslot), C::TCOLS);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  umma::fence_proxy_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tb = *tslot;

  const int ntiles = (d.K + E - 1) / E;
  const int my_tiles = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto tile_of = [&](int i) { return (int)blockIdx.x + i * (int)gridDim.x; };
  auto x_copy_doubles = [&](int tile) {
    const int ne = min(E, d.K - tile * E);
    return ((ne * NP * M * 8) & ~15) / 8;
  };
  int err = 0;
  int x_issued = 0;  // state copies issued (control warp)

  if (warp == kMixThreads / 32 - 1) {
    // ======================= control warp =======================
    const uint32_t id_A = umma::idesc_tf32(128, C::NC16);
    // GEMM-B multiplies each A half by B2's hi and lo rows at once (N = 2 NPN):
    // RHS columns [0, NPN) collect the hi products, [NPN, 2 NPN) the lo ones
    const uint32_t id_B = umma::idesc_tf32(128, 2 * C::NPN);
    // descriptors: the start address field advances by (bytes >> 4) per K step
    const uint64_t dAh = umma::make_desc(umma::smem_u32(AOP), umma::kLBO, C::SBO1);
    const uint64_t dAl = umma::make_desc(umma::smem_u32(AOP) + C::SZ_A, umma::kLBO, C::SBO1);
    const uint64_t dB1h = umma::make_desc(umma::smem_u32(B1h), umma::kLBO, C::SBO1);
    const uint64_t dB1l = umma::make_desc(umma::smem_u32(B1l), umma::kLBO, C::SBO1);
    const uint64_t dB2 = umma::make_desc(umma::smem_u32(B2h), umma::kLBO, C::SBO2);  // B2l follows as rows NPN..
    static_assert(C::O_B2L == C::O_B2H + C::SZ_B2, "B2 lo rows continue the hi rows");
    const uint64_t dRh = umma::make_desc(umma::smem_u32(RING), umma::kLBO, C::SBOC);
    constexpr uint64_t KSTEP = (2 * umma::kLBO) >> 4;      // one K step (8 columns)
    constexpr uint64_t RBUF = (2 * C::SZ_CH) >> 4;         // one ring buffer (hi + lo)
    constexpr uint64_t RLO = C::SZ_CH >> 4;                // hi -> lo half
    constexpr uint64_t B2CH = (KV / 4) * umma::kLBO >> 4;  // one chunk of B2 columns
    auto issue_x = [&](int i) {
      const int tile = tile_of(i);
      const uint32_t bytes = (uint32_t)x_copy_doubles(tile) * 8u;
      umma::mbar_expect_tx(mbX, bytes);
      umma::bulk_g2s(umma::smem_u32(xs_buf(i)), a.x + (size_t)tile * E * NP * M, bytes, mbX);
    };
    // this tile's own face traces into TO: one bulk copy
    auto issue_traces = [&](int i) {
      const int k0 = tile_of(i) * E, ne = min(E, d.K - k0);
      const uint32_t bytes = (uint32_t)(ne * 3 * TS * 4);
      umma::mbar_expect_tx(mbT, bytes);
      umma::bulk_g2s(umma::smem_u32(TO), a.tr_in + (size_t)k0 * 3 * TS, bytes, mbT);
    };
    if (x_bulk && my_tiles > 0) {
      if (lane == 0) issue_x(0);
      x_issued = 1;
    }
    uint32_t cc = 0;  // chunk counter
    bool ok = true;
    for (int i = 0; i < my_tiles && ok; ++i) {
      const int tile = tile_of(i);
      // GEMM-A once the workers have written the A operand
      // (debug_stall: the first wait is on the drain barrier, which nothing
      // completes before the abort path, so it runs out)
      const uint32_t mb_a = (d.debug_stall && i == 0) ? mbDrain : mbA;
      ok = __all_sync(0xffffffffu, umma::mbar_wait_bounded(mb_a, i & 1, wlim));  // warp-uniform
      if (!ok) break;
      umma::fence_after_sync();
      if (lane == 0) {
#pragma unroll
        for (int s = 0; s < K1 / 8; ++s) {
          umma::mma_tf32(tb + C::T_D1, dAh + s * KSTEP, dB1h + s * KSTEP, id_A, s > 0);
          umma::mma_tf32(tb + C::T_D1, dAh + s * KSTEP, dB1l + s * KSTEP, id_A, 1);
          umma::mma_tf32(tb + C::T_D1, dAl + s * KSTEP, dB1h + s * KSTEP, id_A, 1);
        }
        umma::commit(mbD1);
        if (u0_prefetch) {
          const int ne = min(E, d.K - tile * E);
          bulk_prefetch_l2(a.u0 + (size_t)tile * E * NP * M, (uint32_t)((ne * NP * M * 8) & ~15));
        }
      }
      // the next state tile: its buffer is free once the operand build (single
      // buffer) or the epilogue two tiles back (two buffers) is done with it
      if (x_bulk && i + 1 < my_tiles) {
        if (C::XS2 && i >= 1) ok = __all_sync(0xffffffffu, umma::mbar_wait_bounded(mbE, (i - 1) & 1, wlim));
        if (!ok) break;
        if (lane == 0) issue_x(i + 1);
        x_issued++;
      }
      // this tile's own face traces: the previous tile's face chunks are done
      if constexpr (C::TRS) {
        if (lane == 0) issue_traces(i);
      }
      // GEMM-B, chunk by chunk as the workers fill the ring
      for (int ch = 0; ch < C::NCH && ok; ++ch, ++cc) {
        const int b = cc % NBUF;
        ok = __all_sync(0xffffffffu, umma::mbar_wait_bounded(mb_full(b), (cc / NBUF) & 1, wlim));
        if (!ok) break;
        umma::fence_after_sync();
        if (lane == 0) {
          const uint64_t ah = dRh + b * RBUF, al = ah + RLO, bb = dB2 + ch * B2CH;
          const int ncols = ch < NV ? 2 * min(VPC, NC - ch * VPC) : min(KV, C::NFK - (ch - NV) * KV);
          const int ns = (ncols + 7) / 8;
          for (int s = 0; s < ns; ++s) {
            const uint64_t o = s * KSTEP;
            umma::mma_tf32(tb + C::T_D2, ah + o, bb + o, id_B, (ch == 0 && s == 0) ? 0u : 1u);
            umma::mma_tf32(tb + C::T_D2, al + o, bb + o, id_B, 1);
          }
          umma::commit(mb_empty(b));
          if (ch == C::NCH - 1) umma::commit(mbD2);
        }
        __syncwarp();
      }
    }
    if (!ok) *abort_flag = 1;
  } else {
    // ======================= workers =======================
    const int wtid = tid;  // 0 .. NW-1
    const uint32_t tlane = tb + ((uint32_t)(32 * (warp & 3)) << 16);
    // stage time and dt of an element's instance (batched ensembles)
    auto stage_t = [&](int k) {
      const DevState& S = d.st[inst_of(d, k)];
      return a.time_from_state ? S.t + S.dt * a.frac : a.t_arg;
    };
    auto stage_dt = [&](int k) { return a.time_from_state ? d.st[inst_of(d, k)].dt : a.dt_arg; };
    const bool want_lambda = a.mode != MODE_STAGE;
    const bool write_traces = a.tr_out != nullptr && a.mode != MODE_RHS;
    LamAcc lam_acc;
    // this thread's tile row (element, field)
    const int rr = tid & 127, rq = rr >> 5, rln = rr & 31;
    const int rel = rln / M, rf = rln - rel * M, re = rq * EPQ + rel;
    auto rowb_of = [](int e) { return (e / EPQ) * 32 + (e % EPQ) * M; };
    auto bc_coords = [&](int k, int fc, int g, double& x, double& y) {
      const ElemGeo& geo = d.geo[k];
      const double z = d.gz[g];
      double r, s;
      if (fc == 0) { r = z; s = -1.0; }
      else if (fc == 1) { r = -z; s = z; }
      else { r = -1.0; s = -z; }
      x = 0.5 * (-geo.vx[0] * (r + s) + geo.vx[1] * (1. + r) + geo.vx[2] * (1. + s));
      y = 0.5 * (-geo.vy[0] * (r + s) + geo.vy[1] * (1. + r) + geo.vy[2] * (1. + s));
    };
    auto slot = [&](int i) { return sm + C::O_TD + (i & 1) * C::SZ_TD; };
    bool ok = true;

    // operand build of tile i: state deviations (A operand), means, geometry.
    // GA lanes share a row: four nodes each, the mean by a shuffle tree.
    auto build_a = [&](int i) {
      const int tile = tile_of(i), k0 = tile * E, ne = min(E, d.K - k0);
      unsigned char* td = slot(i);
      float* GEO = (float*)(td + C::TD_GEO);
      int* CN = (int*)(td + C::TD_CN);
      float* QF = (float*)(td + C::TD_QF);
      const double* xg = a.x + (size_t)k0 * NP * M;
      const double* XSb = xs_buf(i);
      int nx = 0;
      if (x_bulk) {
        if (!umma::mbar_wait_bounded(mbX, i & 1, wlim)) {
          *abort_flag = 1;  // no arrival: the control warp's wait times out as well
          return;
        }
        nx = x_copy_doubles(tile);
      }
      for (int task = wtid; task < 128 * GA; task += NW) {
        const int r = task / GA, grp = task % GA;
        const int q = r >> 5, ln = r & 31, el = ln / M, f = ln - el * M, e = q * EPQ + el;
        const bool valid = el < EPQ && e < ne;
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int j = 4 * grp + u, idx = (e * NP + j) * M + f;
          v[u] = (valid && j < NP) ? (idx < nx ? XSb[idx] : xg[idx]) : 0.0;
        }
        double sum = (v[0] + v[1]) + (v[2] + v[3]);
#pragma unroll
        for (int w = 1; w < GA; w *= 2) sum = sum + __shfl_xor_sync(0xffffffffu, sum, w);
        const double qbar = sum * (1.0 / NP);
        if (4 * grp < K1) {
          float hv[4], lv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float x = (valid && 4 * grp + u < NP) ? (float)(v[u] - qbar) : 0.f;
            split_tf32(x, hv[u], lv[u]);
          }
          const uint32_t off = umma::kmajor_offset_sbo(r, grp * 4, C::SBO1);
          *(float4*)(AOP + off) = make_float4(hv[0], hv[1], hv[2], hv[3]);
          *(float4*)(AOP + C::SZ_A + off) = make_float4(lv[0], lv[1], lv[2], lv[3]);
        }
        if (grp == 0 && valid) QF[f * E + e] = (float)qbar;
      }
      for (int e = NW - 1 - wtid; e < ne; e += NW) {
        const int k = k0 + e;
#pragma unroll
        for (int j = 0; j < 6; ++j) CN[e * 6 + j] = d.conn[(size_t)k * 6 + j];
        const ElemGeo& g = d.geo[k];
        double* G64 = (double*)(td + C::TD_G64);
        G64[0 * E + e] = g.rx; G64[1 * E + e] = g.ry; G64[2 * E + e] = g.sx; G64[3 * E + e] = g.sy;
#pragma unroll
        for (int fc = 0; fc < 3; ++fc) {
          G64[(4 + fc) * E + e] = g.nx[fc];
          G64[(7 + fc) * E + e] = g.ny[fc];
          G64[(10 + fc) * E + e] = -g.sJ[fc] * g.invJ;
        }
#pragma unroll
        for (int j = 0; j < 13; ++j) GEO[j * E + e] = (float)G64[j * E + e];
      }
      umma::fence_proxy_async();
      mbar_arrive(mbA);
    };
    // partner face traces of tile i into TP: 16-byte copies by warps 4..10,
    // each thread arriving on mbTP once its copies have landed
    auto issue_partner = [&](int i, int t0, int nt) {
      if constexpr (C::TRS) {
        const int k0 = tile_of(i) * E, ne = min(E, d.K - k0);
        const int* CN = (const int*)(slot(i) + C::TD_CN);
        constexpr int Q4 = TS / 4;  // 16-byte pieces per block
        for (int t = t0; t < 3 * ne * Q4; t += nt) {
          const int pr = t / Q4, part = t - pr * Q4, e = pr / 3, fc = pr - 3 * e;
          const int nb = CN[e * 6 + 2 * fc];
          if (nb >= 0)
            cp_async16(umma::smem_u32(TP + (e * 3 + fc) * TS + 4 * part),
                       a.tr_in + ((size_t)nb * 3 + CN[e * 6 + 2 * fc + 1]) * TS + 4 * part);
        }
        cp_async_arrive(mbTP);
      }
    };
    // reference fluxes at the fp32 mean of tile i (tasks: volume + 3 faces per element)
    // the fp32 numerical flux of a face point (qa, qb are not modified)
    auto face_nf = [&](float nx, float ny, const float* qa, const float* qb, float* nf) -> float {
      if constexpr (GF) {
        float x[M], y[M];
#pragma unroll
        for (int f = 0; f < M; ++f) { x[f] = qa[f]; y[f] = qb[f]; }
        return P::numflux(d.eqp, nx, ny, x, y, nf, &err);
      } else {
        return Q::lf(d.eqp, nx, ny, qa, qb, nf, &err);
      }
    };
    auto refs = [&](int i, int t0, int nt) {
      const int tile = tile_of(i), k0 = tile * E, ne = min(E, d.K - k0);
      constexpr bool lf_flux = !GF;
      unsigned char* td = slot(i);
      const float* GEO = (const float*)(td + C::TD_GEO);
      const float* QF = (const float*)(td + C::TD_QF);
      float* P0 = (float*)(td + C::TD_P0);
      double* Rb = (double*)(td + C::TD_RB);
      double* Fb = (double*)(td + C::TD_FB);
      for (int task = t0; task < 4 * E; task += nt) {
        const int kind = task / E, e = task - kind * E;
        if (e >= ne) continue;
        const double* G64 = (const double*)(td + C::TD_G64);
        float qc[M];
#pragma unroll
        for (int f = 0; f < M; ++f) qc[f] = QF[f * E + e];
        // the fp32 flux of the mean; every float64 constant uses these same
        // values, so the volume and face constants cancel for a uniform state
        float F[M], G[M];
        P::flux2(d.eqp, qc, F, G, &err);
        if (kind == 0) {
          // fp32 directional fluxes of the mean: what the volume items subtract
          float R0[M], S0[M];
          Q::dirflux(d.eqp, qc, GEO[0 * E + e], GEO[1 * E + e], GEO[2 * E + e], GEO[3 * E + e], R0, S0, &err);
#pragma unroll
          for (int f = 0; f < M; ++f) {
            P0[f * E + e] = R0[f];
            P0[(M + f) * E + e] = S0[f];
            Rb[f * E + e] = G64[0 * E + e] * (double)F[f] + G64[1 * E + e] * (double)G[f];
            Rb[(M + f) * E + e] = G64[2 * E + e] * (double)F[f] + G64[3 * E + e] * (double)G[f];
          }
        } else {
          // face reference: the fp32 Lax-Friedrichs flux with both states at the
          // mean (what a uniform state gives at every Gauss point); its float64
          // constant is the normal flux nx F + ny G of the same F, G (the wave-speed
          // term vanishes for equal states) with float64 normals
          const int fc = kind - 1;
          float nf[M];
          face_nf(GEO[(4 + fc) * E + e], GEO[(7 + fc) * E + e], qc, qc, nf);
          const double w = G64[(10 + fc) * E + e], nx = G64[(4 + fc) * E + e], ny = G64[(7 + fc) * E + e];
          if constexpr (lf_flux) {
#pragma unroll
            for (int f = 0; f < M; ++f) {
              P0[((2 + fc) * M + f) * E + e] = nf[f];
              Fb[(fc * M + f) * E + e] = w * (nx * (double)F[f] + ny * (double)G[f]);
            }
          } else {
            // the other Euler fluxes need not reduce to n.F at equal states
            // (Apollo's Roe flux does not): the float64 constant is the
            // float64 numerical flux of the same fp32 mean on both sides
            double qa[M], qb[M], nd[M];
#pragma unroll
            for (int f = 0; f < M; ++f) { qa[f] = (double)qc[f]; qb[f] = (double)qc[f]; }
            Eq<EQ>::numflux(d.eqp, nx, ny, qa, qb, nd, &err);
#pragma unroll
            for (int f = 0; f < M; ++f) {
              P0[((2 + fc) * M + f) * E + e] = nf[f];
              Fb[(fc * M + f) * E + e] = w * nd[f];
            }
          }
        }
      }
    };
    // cubature deviations of tile i from TMEM to ST (warps by lane quadrant)
    auto stage = [&](int i) {
      if (!umma::mbar_wait_bounded(mbD1, i & 1, wlim)) *abort_flag = 1;
      umma::fence_after_sync();
      const int q = warp & 3, nwq = q < 3 ? 3 : 2;  // workers 0..10: three warps per quadrant, two for the last
#pragma unroll 1
      for (int blk = warp >> 2; blk < C::NC16 / 16; blk += nwq) {
        float v[16];
        umma::tmem_ld16(tlane + C::T_D1 + 16 * blk, v);
        umma::tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (16 * blk + j < NC) ST[(16 * blk + j) * 128 + rr] = v[j];
      }
      umma::fence_before_sync();
    };
    // chunk operands of tile i into the ring; cc counts chunks over all tiles.
    // The warp that takes the odd items rotates from chunk to chunk.
    uint32_t cc = 0;
    auto items = [&](int i) {
      const int tile = tile_of(i), k0 = tile * E, ne = min(E, d.K - k0);
      unsigned char* td = slot(i);
      const float* GEO = (const float*)(td + C::TD_GEO);
      const int* CN = (const int*)(td + C::TD_CN);
      const float* QF = (const float*)(td + C::TD_QF);
      const float* P0 = (const float*)(td + C::TD_P0);
      // When the tile's element count divides a warp (E = 16, 32), a worker's
      // element is wtid % E in every chunk (the rotation moves whole warps), so
      // its per-element volume constants stay in registers.
      constexpr bool ECONST = 32 % E == 0;
      // ... and since the worker count is a multiple of E as well, the item
      // loops can step over a worker's own element only
      constexpr bool FIXED_E = ECONST && NW % E == 0 && (M == 4 || M == 8);
      const int e_me = wtid % E;
      float kQF[M], kG[4], kP[2 * M];
      if constexpr (ECONST) {
        if (e_me < ne) {
#pragma unroll
          for (int f = 0; f < M; ++f) {
            kQF[f] = QF[f * E + e_me];
            kP[f] = P0[f * E + e_me];
            kP[M + f] = P0[(M + f) * E + e_me];
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) kG[j] = GEO[j * E + e_me];
        }
      }
      for (int ch = 0; ch < C::NCH; ++ch, ++cc) {
        const int b = cc % NBUF;
        const int rot = (int)((cc * 32u) % NW);
        const int wid = wtid >= rot ? wtid - rot : wtid + NW - rot;
        if (cc >= NBUF && !umma::mbar_wait_bounded(mb_empty(b), ((cc / NBUF) - 1) & 1, wlim)) *abort_flag = 1;
        unsigned char* bh = RING + b * 2 * C::SZ_CH;
        unsigned char* bl = bh + C::SZ_CH;
        if (ch < NV && FIXED_E) {
          // volume, each worker on its own element e_me (see FIXED_E): the
          // element's row block and the operand offsets are set up once
          const int npts = min(VPC, NC - ch * VPC);
          const int nfill = 4 * ((npts + 3) / 4);
          if (e_me < ne) {
            const int rowb = rowb_of(e_me);
            const uint32_t obase = umma::kmajor_offset_sbo(rowb, 0, C::SBOC);
            const float* stb = ST + rowb;
            for (int cp = wid / E; cp < nfill; cp += NW / E) {
              float R[M], S[M];
              if (cp < npts) {
                float qc[M];
                load_fields<M>(stb + (ch * VPC + cp) * 128, qc);
#pragma unroll
                for (int f = 0; f < M; ++f) qc[f] += kQF[f];
                Q::dirflux(d.eqp, qc, kG[0], kG[1], kG[2], kG[3], R, S, &err);
#pragma unroll
                for (int f = 0; f < M; ++f) {
                  R[f] -= kP[f];
                  S[f] -= kP[M + f];
                }
              } else {
#pragma unroll
                for (int f = 0; f < M; ++f) { R[f] = 0.f; S[f] = 0.f; }
              }
              // rows rowb + f share one 8-row group: offsets step by 16 bytes
              const uint32_t oc = obase + ((2 * cp) >> 2) * umma::kLBO + ((2 * cp) & 3) * 4;
#pragma unroll
              for (int f = 0; f < M; ++f) {
                float h0, l0, h1, l1;
                split_tf32(R[f], h0, l0);
                split_tf32(S[f], h1, l1);
                *(float2*)(bh + oc + 16 * f) = make_float2(h0, h1);
                *(float2*)(bl + oc + 16 * f) = make_float2(l0, l1);
              }
            }
          }
        } else if (ch < NV) {
          // volume: deviation of the fp32 flux from the flux of the mean, times the metric
          const int npts = min(VPC, NC - ch * VPC);
          const int nfill = 4 * ((npts + 3) / 4);
          for (int it = wid; it < nfill * E; it += NW) {
            const int cp = it / E, e = it - cp * E;
            if (e >= ne) continue;
            const int rowb = rowb_of(e);
            float R[M], S[M];
            if (cp < npts) {
              const int c = ch * VPC + cp;
              float qc[M];
              load_fields<M>(ST + c * 128 + rowb, qc);
              if constexpr (ECONST) {
#pragma unroll
                for (int f = 0; f < M; ++f) qc[f] += kQF[f];
                Q::dirflux(d.eqp, qc, kG[0], kG[1], kG[2], kG[3], R, S, &err);
#pragma unroll
                for (int f = 0; f < M; ++f) {
                  R[f] -= kP[f];
                  S[f] -= kP[M + f];
                }
              } else {
#pragma unroll
                for (int f = 0; f < M; ++f) qc[f] += QF[f * E + e];
                Q::dirflux(d.eqp, qc, GEO[0 * E + e], GEO[1 * E + e], GEO[2 * E + e], GEO[3 * E + e], R, S, &err);
#pragma unroll
                for (int f = 0; f < M; ++f) {
                  R[f] -= P0[f * E + e];
                  S[f] -= P0[(M + f) * E + e];
                }
              }
            } else {
#pragma unroll
              for (int f = 0; f < M; ++f) { R[f] = 0.f; S[f] = 0.f; }
            }
#pragma unroll
            for (int f = 0; f < M; ++f) {
              float h0, l0, h1, l1;
              split_tf32(R[f], h0, l0);
              split_tf32(S[f], h1, l1);
              const uint32_t off = umma::kmajor_offset_sbo(rowb + f, 2 * cp, C::SBOC);
              *(float2*)(bh + off) = make_float2(h0, h1);
              *(float2*)(bl + off) = make_float2(l0, l1);
            }
          }
        } else {
          // faces: Lax-Friedrichs flux of the stored traces, deviation from the
          // reference flux, times -sJ/J; column fc NG + g
          if constexpr (C::TRS) {
            if (ch == NV && !(umma::mbar_wait_bounded(mbT, i & 1, wlim) && umma::mbar_wait_bounded(mbTP, i & 1, wlim)))
              *abort_flag = 1;
          }
          const int col0 = (ch - NV) * KV;
          const int ncol = min(KV, C::NFK - col0);
          // with FIXED_E every iteration of a worker has e = e_me
          const int it0 = FIXED_E ? (e_me < ne ? (wid / E) * E + e_me : ncol * E) : wid;
          for (int it = it0; it < ncol * E; it += NW) {
            const int e = FIXED_E ? e_me : it % E, cl = it / E, col = col0 + cl;
            if (!FIXED_E && e >= ne) continue;
            const int rowb = rowb_of(e), k = k0 + e;
            float dev[M];
            if (col < NF) {
              const int fc = col / NG, g = col - fc * NG;
              float qM[M], qP[M], nf[M];
              const int nb = CN[e * 6 + 2 * fc];
              if constexpr (C::TRS) {
                load_fields<M>(TO + (e * 3 + fc) * TS + g * M, qM);
                if (nb >= 0) load_fields<M>(TP + (e * 3 + fc) * TS + (NG - 1 - g) * M, qP);
              } else {
                load_fields<M>(a.tr_in + ((size_t)k * 3 + fc) * TS + g * M, qM);
                if (nb >= 0) {
                  const int f2 = CN[e * 6 + 2 * fc + 1];
                  load_fields<M>(a.tr_in + ((size_t)nb * 3 + f2) * TS + (NG - 1 - g) * M, qP);
                }
              }
              const float nx = GEO[(4 + fc) * E + e], ny = GEO[(7 + fc) * E + e];
              if (nb < 0) {
                double x, y;
                bc_coords(k, fc, g, x, y);
                apply_bc<EQ, float>(d.bcs, -nb, stage_t(k), x, y, nx, ny, qM, qP);
              }
              const float lam = face_nf(nx, ny, qM, qP, nf);
              if (want_lambda) lam_acc.add(d.st, inst_of(d, k), fabs((double)lam));
              const float w = GEO[(10 + fc) * E + e];
#pragma unroll
              for (int f = 0; f < M; ++f) dev[f] = w * (nf[f] - P0[((2 + fc) * M + f) * E + e]);
            } else {
#pragma unroll
              for (int f = 0; f < M; ++f) dev[f] = 0.f;
            }
            const uint32_t oc = umma::kmajor_offset_sbo(rowb, cl, C::SBOC);
#pragma unroll
            for (int f = 0; f < M; ++f) {
              float h, l;
              split_tf32(dev[f], h, l);
              // rows rowb + f share one 8-row group (rowb is a multiple of M, M | 8)
              const uint32_t off = (M == 4 || M == 8) ? oc + 16 * f : umma::kmajor_offset_sbo(rowb + f, cl, C::SBOC);
              *(float*)(bh + off) = h;
              *(float*)(bl + off) = l;
            }
          }
        }
        umma::fence_proxy_async();
        mbar_arrive(mb_full(b));
      }
    };
    // float64 epilogue of tile i (threads 0..127: TMEM lane = tile row)
    auto epilogue = [&](int i) {
      const int tile = tile_of(i), k0 = tile * E, ne = min(E, d.K - k0);
      const bool rvalid = rel < EPQ && re < ne;
      const unsigned char* td = slot(i);
      const double* Rb = (const double*)(td + C::TD_RB);
      const double* Fb = (const double*)(td + C::TD_FB);
      if (!umma::mbar_wait_bounded(mbD2, i & 1, wlim)) *abort_flag = 1;
      umma::fence_after_sync();
      float dv[C::NPN];
#pragma unroll
      for (int c0 = 0; c0 < C::NPN; c0 += 16) {
        float vh[16], vl[16];
        umma::tmem_ld16(tlane + C::T_D2 + c0, vh);
        umma::tmem_ld16(tlane + C::T_D2 + C::NPN + c0, vl);
        umma::tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) dv[c0 + j] = vh[j] + vl[j];
      }
      umma::fence_before_sync();
      double o[NP];
      if (rvalid && !*abort_flag) {
        const int k = k0 + re;
        const double Rbar = Rb[rf * E + re], Sbar = Rb[(M + rf) * E + re];
        const double F0 = Fb[(0 * M + rf) * E + re], F1 = Fb[(1 * M + rf) * E + re], F2 = Fb[(2 * M + rf) * E + re];
        const double dt = stage_dt(k);
        const double c_stage = dt / 4.0, c_al = 4.0 / 5.0, c_be = dt / 5.0, c_ga = 1.0 / 5.0;
        const double* XSb = xs_buf(i);
        const int nx = x_bulk ? x_copy_doubles(tile) : 0;
        const double* xrow = a.x + (size_t)k * NP * M + rf;
        const double* urow = a.u0 + (size_t)k * NP * M + rf;
        double* orow = a.out + (size_t)k * NP * M + rf;
        // out may alias x and u0 (same row, same thread): each batch of nodes is
        // loaded in full before any of it is stored, so the loads overlap
        constexpr int BT = 8;
#pragma unroll
        for (int i0 = 0; i0 < NP; i0 += BT) {
          double xr[BT], ur[BT];
#pragma unroll
          for (int u = 0; u < BT; ++u) {
            const int n = i0 + u;
            if (n < NP && a.mode != MODE_RHS) {
              const int idx = (re * NP + n) * M + rf;
              xr[u] = (C::XS2 && idx < nx) ? XSb[idx] : xrow[n * M];
            }
            if (n < NP && a.mode == MODE_FINAL) ur[u] = urow[n * M];
          }
#pragma unroll
          for (int u = 0; u < BT; ++u) {
            const int n = i0 + u;
            if (n >= NP) break;
            const double* rs = RSUM + n * 5;
            double r = (double)dv[n] + rs[0] * Rbar + rs[1] * Sbar + rs[2] * F0 + rs[3] * F1 + rs[4] * F2;
            if (d.srcv) r += d.srcv[((size_t)k * NP + n) * M + rf];  // the stage's source terms
            if (!isfinite(r)) err |= ERRB_NAN;
            if (a.mode == MODE_RHS) o[n] = r;
            else if (a.mode == MODE_STAGE) o[n] = xr[u] + c_stage * r;
            else o[n] = c_al * xr[u] + c_be * r + c_ga * ur[u];
          }
#pragma unroll
          for (int u = 0; u < BT; ++u) {
            const int n = i0 + u;
            if (n < NP) orow[n * M] = o[n];
          }
        }
      }
      if (C::XS2) mbar_arrive(mbE);  // the state tile is no longer needed
      if (rvalid && !*abort_flag && write_traces) {
        const double m = tree_mean<NP>(o);
#pragma unroll
        for (int n = 0; n < NP; ++n) XD[n * 128 + rr] = (float)(o[n] - m);
        XB[rr] = m;
      }
    };
    // face traces of tile i's result: (face, row) tasks
    auto traces = [&](int i) {
      const int tile = tile_of(i), k0 = tile * E, ne = min(E, d.K - k0);
      for (int task = wtid; task < 3 * 128; task += NW) {
        const int fc = task >> 7, r = task & 127, q = r >> 5, ln = r & 31, el = ln / M, f = ln - el * M;
        const int e = q * EPQ + el;
        if (el >= EPQ || e >= ne) continue;
        float dv[NP];
#pragma unroll
        for (int n = 0; n < NP; ++n) dv[n] = XD[n * 128 + r];
        row_traces<NP, NG, IFS>(IF, dv, XB[r], fc, a.tr_out + ((size_t)(k0 + e) * 3 + fc) * TS + f, M);
      }
    };

    if (my_tiles > 0) {
      build_a(0);
      workers_sync<NW>();
      refs(0, wtid, NW);
      if (wtid >= 128) issue_partner(0, wtid - 128, NW - 128);
      stage(0);
      workers_sync<NW>();
      ok = !*abort_flag;
    }
    for (int i = 0; i < my_tiles && ok; ++i) {
      const bool next = i + 1 < my_tiles;
      items(i);
      if (next) build_a(i + 1);
      workers_sync<NW>();
      if (*abort_flag) { ok = false; break; }
      if (wtid < 128) {
        epilogue(i);
      } else if (next) {
        issue_partner(i + 1, wtid - 128, NW - 128);
        refs(i + 1, wtid - 128, NW - 128);
      }
      workers_sync<NW>();
      if (write_traces && !*abort_flag) traces(i);
      if (next) {
        stage(i + 1);
        workers_sync<NW>();
        // read right after a worker barrier, so every worker leaves together
        if (*abort_flag) ok = false;
      }
    }
    // partner-trace copies still in flight after an abort land before the exit
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (want_lambda) lam_acc.flush_warp(d.st);
  }
  if (err) atomicOr(&d.st->err, err);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (*abort_flag) {
    // after an abort: let every issued MMA complete (a fresh barrier, so its
    // parity is unambiguous) and the copies in flight land
    if (warp == kMixThreads / 32 - 1) {
      if (lane == 0) umma::commit(mbDrain);
      __syncwarp();
      // (the default limit: the drain must not give up while work is in flight)
      umma::mbar_wait_bounded(mbDrain, 0);
      if (x_issued > 0) umma::mbar_wait_bounded(mbX, (x_issued - 1) & 1);
    }
    if (tid == 0) atomicOr(&d.st->err, ERRB_TIMEOUT);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
  }
  if (warp == 0) umma::tmem_dealloc(tb, C::TCOLS);
}

#include "dg_mixed_fused.cuh"

// Face traces [K][3][TS] of a state.  A block of 128 threads takes 128 / M
// elements: their states, one contiguous range of x, are read into shared
// memory with coalesced loads (at most NP per thread, all in flight at once),
// then each thread owns one (element, field) row and writes its traces on all
// three faces, so every state value is read from HBM once.
constexpr int kTraceThreads = 128;
template <int N, int M>
__global__ void __launch_bounds__(kTraceThreads) k_mixed_traces(int K, const double* __restrict__ x,
                                                                const double* __restrict__ I, float* __restrict__ T) {
  constexpr int NP = Sizes<N>::NP, NG = Sizes<N>::NG, NF = Sizes<N>::NF;
  constexpr int IFS = round_up_c(NP, 4), TS = trace_stride(NG, M);
  constexpr int EB = kTraceThreads / M;  // elements per block
  static_assert(EB * NP * M <= NP * kTraceThreads, "NP loads per thread cover the block's states");
  __shared__ __align__(16) float IF[NF * IFS];
  __shared__ double XS[EB * NP * M];
  const long long k0 = (long long)blockIdx.x * EB;
  const int ne = (int)min((long long)EB, (long long)K - k0);
  const int nx = ne * NP * M;
  const double* xb = x + k0 * NP * M;
  double ld[NP];
#pragma unroll
  for (int u = 0; u < NP; ++u) {
    const int i = threadIdx.x + u * kTraceThreads;
    ld[u] = i < nx ? xb[i] : 0.0;
  }
  for (int i = threadIdx.x; i < NF * IFS; i += kTraceThreads)
    IF[i] = (i % IFS) < NP ? (float)I[(i / IFS) * NP + i % IFS] : 0.f;
#pragma unroll
  for (int u = 0; u < NP; ++u) {
    const int i = threadIdx.x + u * kTraceThreads;
    if (i < nx) XS[i] = ld[u];
  }
  __syncthreads();
  const int e = threadIdx.x / M, f = threadIdx.x - e * M;
  if (e >= ne) return;
  double v[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) v[j] = XS[(e * NP + j) * M + f];
  const double m = tree_mean<NP>(v);
  float dv[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) dv[j] = (float)(v[j] - m);
  float* Tk = T + (size_t)(k0 + e) * 3 * TS + f;
#pragma unroll 1
  for (int fc = 0; fc < 3; ++fc) row_traces<NP, NG, IFS>(IF, dv, m, fc, Tk + fc * TS, M);
}

template <int N, int M>
cudaError_t launch_traces_t(const DgDev& d, const double* x, float* T, cudaStream_t s) {
  constexpr int EB = kTraceThreads / M;
  const long long blocks = ((long long)d.K + EB - 1) / EB;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
  if (blocks == 0) return cudaSuccess;
  k_mixed_traces<N, M><<<(unsigned)blocks, kTraceThreads, 0, s>>>(d.K, x, d.I, T);
  return cudaGetLastError();
}

template <int EQ, int N, int SH, bool GF = false>
cudaError_t launch_mixed_sh(MixedPlan* p, const DgDev& d, const StageArgs& a0, cudaStream_t s, cudaEvent_t* ev) {
  using C = MixCfg<N, Eq<EQ>::M, SH>;
  if constexpr (!C::FITS) {
    return cudaErrorNotSupported;
  } else {
    static unsigned configured = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(configured & (1u << (dev & 31)))) {
      cudaError_t e = cudaFuncSetAttribute(k_mixed_stage<EQ, N, SH, GF>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::BYTES);
      if (e != cudaSuccess) return e;
      configured |= 1u << (dev & 31);
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (d.grid_div > 1) sms = (sms + d.grid_div - 1) / d.grid_div;
    const int ntiles = (d.K + C::E - 1) / C::E;
    int grid = sms;
    if (grid > ntiles) grid = ntiles;
    StageArgs a = a0;
    if (a.reset_lambda && a.mode != MODE_STAGE) {
      cudaError_t e = launch_reset_lambda(d, s);
      if (e != cudaSuccess) return e;
    }
    if (ev) cudaEventRecord(ev[0], s);
    if (a.mode == MODE_RHS) {
      // the traces of the input first
      if (!a.tr_scratch) return cudaErrorInvalidValue;
      cudaError_t e = launch_traces_t<N, Eq<EQ>::M>(d, a.x, a.tr_scratch, s);
      if (e != cudaSuccess) return e;
      a.tr_in = a.tr_scratch;
      a.tr_out = nullptr;
    }
    if (!a.tr_in) return cudaErrorInvalidValue;
    if (d.srcv) {  // this stage's source terms, added by the epilogue
      cudaError_t e = launch_source(EQ, d, a, d.srcv, 0, s);
      if (e != cudaSuccess) return e;
    }
    if (ev) cudaEventRecord(ev[1], s);
    // bit 0: the state is bulk-copied (16-byte aligned); bit 1: warm L2 with u0
    const int flags = (((uintptr_t)a.x & 15) == 0 ? 1 : 0) |
                      (a.mode == MODE_FINAL && ((uintptr_t)a.u0 & 15) == 0 ? 2 : 0);
    k_mixed_stage<EQ, N, SH, GF><<<grid, kMixThreads, C::BYTES, s>>>(d, a, p->rowsum, flags);
    if (ev) {
      cudaEventRecord(ev[2], s);
      cudaEventRecord(ev[3], s);
    }
    return cudaGetLastError();
  }
}

// the fused form (dg_mixed_fused.cuh): four-field Euler, Lax-Friedrichs, orders 2..4
template <int EQ, int N>
cudaError_t launch_fused(MixedPlan* p, const DgDev& d, const StageArgs& a0, cudaStream_t s, cudaEvent_t* ev) {
  using C = FusedCfg<N>;
  if constexpr (!C::FITS) {
    return cudaErrorNotSupported;
  } else {
    static unsigned configured = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(configured & (1u << (dev & 31)))) {
      cudaError_t e = cudaFuncSetAttribute(k_mixed_fused<EQ, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::BYTES);
      if (e != cudaSuccess) return e;
      configured |= 1u << (dev & 31);
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (d.grid_div > 1) sms = (sms + d.grid_div - 1) / d.grid_div;
    const int ntiles = (d.K + C::E - 1) / C::E;
    int grid = sms;
    if (grid > ntiles) grid = ntiles;
    StageArgs a = a0;
    if (a.reset_lambda && a.mode != MODE_STAGE) {
      cudaError_t e = launch_reset_lambda(d, s);
      if (e != cudaSuccess) return e;
    }
    if (ev) cudaEventRecord(ev[0], s);
    if (a.mode == MODE_RHS) {
      if (!a.tr_scratch) return cudaErrorInvalidValue;
      cudaError_t e = launch_traces_t<N, 4>(d, a.x, a.tr_scratch, s);
      if (e != cudaSuccess) return e;
      a.tr_in = a.tr_scratch;
      a.tr_out = nullptr;
    }
    if (!a.tr_in) return cudaErrorInvalidValue;
    // the trace bulk stores need a 16-byte aligned destination
    if (a.tr_out && ((uintptr_t)a.tr_out & 15)) return cudaErrorInvalidValue;
    if (d.srcv) {  // this stage's source terms, added by the epilogue
      cudaError_t e = launch_source(EQ, d, a, d.srcv, 0, s);
      if (e != cudaSuccess) return e;
    }
    if (ev) cudaEventRecord(ev[1], s);
    const int flags = (((uintptr_t)a.x & 15) == 0 ? 1 : 0) |
                      (a.mode == MODE_FINAL && ((uintptr_t)a.u0 & 15) == 0 ? 2 : 0);
    k_mixed_fused<EQ, N><<<grid, kFusedThreads, C::BYTES, s>>>(d, a, p->rowsum, flags);
    if (ev) {
      cudaEventRecord(ev[2], s);
      cudaEventRecord(ev[3], s);
    }
    return cudaGetLastError();
  }
}

// the second chunk shape for the Euler kinds (the batched ensembles' equations)
template <int EQ, int N>
cudaError_t launch_mixed_t(MixedPlan* p, const DgDev& d, const StageArgs& a, cudaStream_t s, cudaEvent_t* ev) {
  if constexpr (EQ == EQ_EULER || EQ == EQ_EULER2D) {
    // Apollo's other Euler numerical fluxes: their own instantiation
    if ((int)d.eqp.p[3] != NF_LF) return launch_mixed_sh<EQ, N, 0, true>(p, d, a, s, ev);
  }
  if constexpr (EQ == EQ_EULER2D && N <= 4 && FusedCfg<N>::FITS) {
    if (d.tile_shape == 0) return launch_fused<EQ, N>(p, d, a, s, ev);
  }
  if constexpr ((EQ == EQ_EULER || EQ == EQ_EULER2D) && MixCfg<N, Eq<EQ>::M, 1>::FITS) {
    if (d.tile_shape == 1) return launch_mixed_sh<EQ, N, 1>(p, d, a, s, ev);
  }
  // tile_shape 2 (and 0 where the fused form does not apply): the chunked
  // kernel with 24-column chunks
  return launch_mixed_sh<EQ, N, 0>(p, d, a, s, ev);
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

template <int M>
cudaError_t traces_dispatch_n(const DgDev& d, const double* x, float* T, cudaStream_t s) {
  switch (d.N) {
    case 2: return launch_traces_t<2, M>(d, x, T, s);
    case 3: return launch_traces_t<3, M>(d, x, T, s);
    case 4: return launch_traces_t<4, M>(d, x, T, s);
    case 5: return launch_traces_t<5, M>(d, x, T, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

MixedPlan* mixed_create(int eq, const RefOps& o, int K, int M) {
  (void)K;
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
  if (cudaMalloc((void**)&p->rowsum, rs.size() * sizeof(double)) != cudaSuccess) {
    mixed_destroy(p);
    return nullptr;
  }
  cudaMemcpy(p->rowsum, rs.data(), rs.size() * sizeof(double), cudaMemcpyHostToDevice);
  return p;
}

void mixed_destroy(MixedPlan* p) {
  if (!p) return;
  if (p->rowsum) cudaFree(p->rowsum);
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

size_t mixed_trace_floats(const MixedPlan* p, int K) {
  return (size_t)K * 3 * trace_stride(2 * (p->N + 1), p->M);
}

cudaError_t mixed_launch_traces(MixedPlan* p, const DgDev& d, const double* x, float* T, cudaStream_t s) {
  switch (p->M) {
    case 1: return traces_dispatch_n<1>(d, x, T, s);
    case 3: return traces_dispatch_n<3>(d, x, T, s);
    case 4: return traces_dispatch_n<4>(d, x, T, s);
    case 5: return traces_dispatch_n<5>(d, x, T, s);
    case 8: return traces_dispatch_n<8>(d, x, T, s);
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
