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

template <int N, int M> struct MixCfg {
  static constexpr int NP = Sizes<N>::NP, NC = Sizes<N>::NC, NG = Sizes<N>::NG, NF = Sizes<N>::NF;
  static constexpr int EPQ = 32 / M;  // elements per warp quadrant
  static constexpr int E = 4 * EPQ;   // elements per tile
  static constexpr int K1 = round_up_c(NP, 8);
  static constexpr int KV = N >= 5 ? 16 : 32;         // K columns per chunk
  static constexpr int VPC = KV / 2;                  // cubature points per volume chunk (R, S each)
  static constexpr int NV = (NC + VPC - 1) / VPC;     // volume chunks
  static constexpr int NFK = round_up_c(NF, 8);       // face columns (fc NG + g, packed)
  static constexpr int NFC = (NFK + KV - 1) / KV;     // face chunks
  static constexpr int NCH = NV + NFC;
  static constexpr int NC16 = round_up_c(NC, 16);
  static constexpr int NPN = round_up_c(NP, 16);
  static constexpr int KB2 = NCH * KV;
  static constexpr int NBUF = 2;
  static constexpr int NWORK = kMixThreads - 32;      // worker threads; the last warp issues MMAs and copies
  // TMEM columns: cubature values, then the right-hand side
  static constexpr int T_D1 = 0, T_D2 = NC16;
  static constexpr int TCOLS = tmem_cols(NC16 + NPN);
  // K-major operand strides (bytes between 8-row groups)
  static constexpr int SBO1 = K1 * 32;       // B1 = V and the A operand
  static constexpr int SBO2 = KB2 * 32;      // B2 = [Dr Ds | L w]
  static constexpr int SBOC = KV * 32 + 16;  // chunk operands, staggered across banks
  // shared memory, bytes (each operand as a tf32 hi half and lo half)
  static constexpr int SZ_B1 = (NC16 / 8) * SBO1;
  static constexpr int SZ_B2 = (NPN / 8) * SBO2;
  static constexpr int SZ_A = 16 * SBO1;
  static constexpr int SZ_CH = 16 * SBOC;
  static constexpr int SZ_ST = NC * 128 * 4;  // cubature deviations [NC][128] float
  static constexpr int SZ_XD = NP * 128 * 4;  // result deviations [NP][128] float
  static constexpr int XS_N = E * NP * M;     // one tile's state, doubles
  // per-tile data, two slots (tile parity)
  static constexpr int TD_GEO = 0;                         // [14][E] float: rx ry sx sy, nx[3] ny[3] -sJ/J[3] at 5..13
  static constexpr int TD_CN = TD_GEO + 14 * E * 4;        // [E][6] int
  static constexpr int TD_QF = TD_CN + E * 6 * 4;          // [M][E] float own means
  static constexpr int TD_P0 = TD_QF + M * E * 4;          // [5M][E] float F, G, f*_fc at the mean
  static constexpr int TD_RB = round_up_c(TD_P0 + 5 * M * E * 4, 8);  // [2M][E] double R, S at the mean
  static constexpr int TD_FB = TD_RB + 2 * M * E * 8;      // [3M][E] double face references
  static constexpr int SZ_TD = TD_FB + 3 * M * E * 8;
  static constexpr int O_B1H = 0, O_B1L = O_B1H + SZ_B1;
  static constexpr int O_B2H = O_B1L + SZ_B1, O_B2L = O_B2H + SZ_B2;
  static constexpr int O_A = round_up_c(O_B2L + SZ_B2, 128);
  static constexpr int O_RING = O_A + 2 * SZ_A;
  static constexpr int O_ST = O_RING + NBUF * 2 * SZ_CH;
  static constexpr int O_XD = O_ST + SZ_ST;
  static constexpr int O_XS = round_up_c(O_XD + SZ_XD, 16);
  static constexpr int O_IF = O_XS + XS_N * 8;                      // [NF][NP] float interpolation
  static constexpr int O_RS = round_up_c(O_IF + NF * NP * 4, 8);    // [NP][5] double row sums
  static constexpr int O_TD = O_RS + NP * 5 * 8;                    // 2 slots of per-tile data
  static constexpr int O_XB = O_TD + 2 * SZ_TD;                     // [128] double means of the result
  // mbarriers: state copy, A operand, GEMM-A done, tile RHS done, ring full[NBUF], ring empty[NBUF], drain
  static constexpr int O_MB = O_XB + 128 * 8;
  static constexpr int NMB = 5 + 2 * NBUF;
  static constexpr int O_TS = O_MB + 8 * NMB;                       // TMEM base, abort flag
  static constexpr int BYTES = O_TS + 16;
  static constexpr bool FITS = BYTES <= 227 * 1024;
  static_assert(KV % 16 == 0 && SZ_TD % 8 == 0, "layout");
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

// Face traces of one (element, field) row: for the NG Gauss points of face fc,
// float(m) + sum_j I[fc NG + g][j] dv[j], fp32 fused multiply-adds in node
// order.  Both the stage epilogue and k_mixed_traces call this, so the values
// agree bit for bit for the same state.
template <int NP, int NG>
__device__ __forceinline__ void row_traces(const float* __restrict__ IF, const float* dv, int dstride, double m, int fc,
                                           float* __restrict__ dst, int M) {
  const float mf = (float)m;
#pragma unroll 2
  for (int g = 0; g < NG; ++g) {
    const float* Ig = IF + (fc * NG + g) * NP;
    float acc = 0.f;
#pragma unroll
    for (int j = 0; j < NP; ++j) acc = fmaf(Ig[j], dv[j * dstride], acc);
    dst[g * M] = mf + acc;
  }
}

template <int NP>
__device__ __forceinline__ double nodal_mean(const double* v) {
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < NP; ++j) s += v[j];
  return s * (1.0 / NP);
}

// Worker-only barrier (named barrier 1; the control warp does not take part).
template <int NW>
__device__ __forceinline__ void workers_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(NW) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// Stage kernel.  Warps 0..10 are workers, warp 11 is the control warp: its
// lane 0 issues every tcgen05 MMA and bulk copy.  Per tile the workers build
// the A operand (state deviations), stage GEMM-A's cubature values, produce
// the chunk operands of GEMM-B into a two-buffer ring (full/empty mbarriers),
// and finish with the float64 epilogue and the result's face traces.  The
// next tile's operand build and GEMM-A overlap this tile's epilogue; per-tile
// data live in two slots by tile parity.
template <int EQ, int N>
__global__ void __launch_bounds__(kMixThreads, 1)
    k_mixed_stage(DgDev d, StageArgs a, const double* __restrict__ rowsum, int flags) {
  using P = Eq<EQ>;
  constexpr int M = P::M;
  using C = MixCfg<N, M>;
  constexpr int NP = C::NP, NC = C::NC, NG = C::NG, NF = C::NF, EPQ = C::EPQ, E = C::E, K1 = C::K1;
  constexpr int KV = C::KV, VPC = C::VPC, NV = C::NV, NW = C::NWORK, NBUF = C::NBUF;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* B1h = sm + C::O_B1H;
  unsigned char* B1l = sm + C::O_B1L;
  unsigned char* B2h = sm + C::O_B2H;
  unsigned char* B2l = sm + C::O_B2L;
  unsigned char* AOP = sm + C::O_A;
  unsigned char* RING = sm + C::O_RING;
  float* ST = (float*)(sm + C::O_ST);
  float* XD = (float*)(sm + C::O_XD);
  const double* XS = (const double*)(sm + C::O_XS);
  float* IF = (float*)(sm + C::O_IF);
  double* RSUM = (double*)(sm + C::O_RS);
  double* XB = (double*)(sm + C::O_XB);
  uint64_t* mbar = (uint64_t*)(sm + C::O_MB);
  uint32_t* tslot = (uint32_t*)(sm + C::O_TS);
  volatile int* abort_flag = (volatile int*)(sm + C::O_TS + 4);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool x_bulk = flags & 1, u0_prefetch = flags & 2;

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
  for (int i = tid; i < NF * NP; i += kMixThreads) IF[i] = (float)d.I[i];
  for (int i = tid; i < NP * 5; i += kMixThreads) RSUM[i] = rowsum[i];
  // mbarriers: 0 state copy, 1 A operand (all workers), 2 GEMM-A done, 3 RHS
  // done, 4 + b ring buffer b full (all workers), 4 + NBUF + b ring buffer b empty
  const uint32_t mbX = umma::smem_u32(mbar + 0), mbA = umma::smem_u32(mbar + 1);
  const uint32_t mbD1 = umma::smem_u32(mbar + 2), mbD2 = umma::smem_u32(mbar + 3);
  auto mb_full = [&](int b) { return umma::smem_u32(mbar + 4 + b); };
  auto mb_empty = [&](int b) { return umma::smem_u32(mbar + 4 + NBUF + b); };
  const uint32_t mbDrain = umma::smem_u32(mbar + 4 + 2 * NBUF);
  if (tid == 0) {
    umma::mbar_init(mbDrain, 1);
    umma::mbar_init(mbX, 1);
    umma::mbar_init(mbA, NW);
    umma::mbar_init(mbD1, 1);
    umma::mbar_init(mbD2, 1);
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
    const uint32_t id_B = umma::idesc_tf32(128, C::NPN);
    const uint32_t sB1h = umma::smem_u32(B1h), sB1l = umma::smem_u32(B1l);
    const uint32_t sB2h = umma::smem_u32(B2h), sB2l = umma::smem_u32(B2l);
    const uint32_t sA = umma::smem_u32(AOP), sRing = umma::smem_u32(RING);
    auto issue_x = [&](int tile) {
      const uint32_t bytes = (uint32_t)x_copy_doubles(tile) * 8u;
      umma::mbar_expect_tx(mbX, bytes);
      umma::bulk_g2s(umma::smem_u32(XS), a.x + (size_t)tile * E * NP * M, bytes, mbX);
    };
    if (x_bulk && my_tiles > 0 && lane == 0) issue_x(tile_of(0));
    if (x_bulk && my_tiles > 0) x_issued = 1;
    uint32_t cc = 0;  // chunk counter
    bool ok = true;
    for (int i = 0; i < my_tiles && ok; ++i) {
      const int tile = tile_of(i);
      // GEMM-A once the workers have written the A operand
      ok = __all_sync(0xffffffffu, umma::mbar_wait_bounded(mbA, i & 1));  // warp-uniform
      if (!ok) break;
      umma::fence_after_sync();
      if (lane == 0) {
#pragma unroll
        for (int s = 0; s < K1 / 8; ++s) {
          const uint32_t off = s * 2 * umma::kLBO;
          const uint64_t ah = umma::make_desc(sA + off, umma::kLBO, C::SBO1);
          const uint64_t al = umma::make_desc(sA + C::SZ_A + off, umma::kLBO, C::SBO1);
          const uint64_t bh = umma::make_desc(sB1h + off, umma::kLBO, C::SBO1);
          const uint64_t bl = umma::make_desc(sB1l + off, umma::kLBO, C::SBO1);
          umma::mma_tf32(tb + C::T_D1, ah, bh, id_A, s > 0);
          umma::mma_tf32(tb + C::T_D1, ah, bl, id_A, 1);
          umma::mma_tf32(tb + C::T_D1, al, bh, id_A, 1);
        }
        umma::commit(mbD1);
        // the state tile is consumed: fetch the next one; warm L2 with u0
        if (x_bulk && i + 1 < my_tiles) issue_x(tile_of(i + 1));
        if (u0_prefetch) {
          const int ne = min(E, d.K - tile * E);
          bulk_prefetch_l2(a.u0 + (size_t)tile * E * NP * M, (uint32_t)((ne * NP * M * 8) & ~15));
        }
      }
      if (x_bulk && i + 1 < my_tiles) x_issued++;
      // GEMM-B, chunk by chunk as the workers fill the ring
      for (int ch = 0; ch < C::NCH && ok; ++ch, ++cc) {
        const int b = cc % NBUF;
        ok = __all_sync(0xffffffffu, umma::mbar_wait_bounded(mb_full(b), (cc / NBUF) & 1));
        if (!ok) break;
        umma::fence_after_sync();
        if (lane == 0) {
          const uint32_t ah0 = sRing + b * 2 * C::SZ_CH, al0 = ah0 + C::SZ_CH;
          const uint32_t b2 = ch * (KV / 4) * umma::kLBO;
          const int ncols = ch < NV ? 2 * min(VPC, NC - ch * VPC) : min(KV, C::NFK - (ch - NV) * KV);
          const int ns = (ncols + 7) / 8;
          for (int s = 0; s < ns; ++s) {
            const uint32_t off = s * 2 * umma::kLBO;
            const uint64_t ah = umma::make_desc(ah0 + off, umma::kLBO, C::SBOC);
            const uint64_t al = umma::make_desc(al0 + off, umma::kLBO, C::SBOC);
            const uint64_t bh = umma::make_desc(sB2h + b2 + off, umma::kLBO, C::SBO2);
            const uint64_t bl = umma::make_desc(sB2l + b2 + off, umma::kLBO, C::SBO2);
            umma::mma_tf32(tb + C::T_D2, ah, bh, id_B, (ch == 0 && s == 0) ? 0u : 1u);
            umma::mma_tf32(tb + C::T_D2, ah, bl, id_B, 1);
            umma::mma_tf32(tb + C::T_D2, al, bh, id_B, 1);
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
    const double tstage = a.time_from_state ? d.st->t + d.st->dt * a.frac : a.t_arg;
    const double dt = a.time_from_state ? d.st->dt : a.dt_arg;
    const bool want_lambda = a.mode != MODE_STAGE;
    const bool write_traces = a.tr_out != nullptr && a.mode != MODE_RHS;
    double lmax = 0.0;
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

    // operand build of tile i: state deviations (A operand), means, geometry
    auto build_a = [&](int i) {
      const int tile = tile_of(i), k0 = tile * E, ne = min(E, d.K - k0);
      unsigned char* td = slot(i);
      float* GEO = (float*)(td + C::TD_GEO);
      int* CN = (int*)(td + C::TD_CN);
      float* QF = (float*)(td + C::TD_QF);
      const double* xg = a.x + (size_t)k0 * NP * M;
      int nx = 0;
      if (x_bulk) {
        if (!umma::mbar_wait_bounded(mbX, i & 1)) {
          *abort_flag = 1;  // no arrival: the control warp's wait times out as well
          return;
        }
        nx = x_copy_doubles(tile);
      }
      for (int task = wtid; task < 128 * (K1 / 4); task += NW) {
        const int r = task & 127, grp = task >> 7;
        const int q = r >> 5, ln = r & 31, el = ln / M, f = ln - el * M, e = q * EPQ + el;
        float hv[4] = {0.f, 0.f, 0.f, 0.f}, lv[4] = {0.f, 0.f, 0.f, 0.f};
        if (el < EPQ && e < ne) {
          double v[NP];
#pragma unroll
          for (int j = 0; j < NP; ++j) {
            const int idx = (e * NP + j) * M + f;
            v[j] = idx < nx ? XS[idx] : xg[idx];
          }
          const double qbar = nodal_mean<NP>(v);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int j = grp * 4 + u;
            if (j < NP) {
              const int idx = (e * NP + j) * M + f;
              const double xj = idx < nx ? XS[idx] : xg[idx];
              split_tf32((float)(xj - qbar), hv[u], lv[u]);
            }
          }
          if (grp == 0) QF[f * E + e] = (float)qbar;
        }
        const uint32_t off = umma::kmajor_offset_sbo(r, grp * 4, C::SBO1);
        *(float4*)(AOP + off) = make_float4(hv[0], hv[1], hv[2], hv[3]);
        *(float4*)(AOP + C::SZ_A + off) = make_float4(lv[0], lv[1], lv[2], lv[3]);
      }
      for (int e = NW - 1 - wtid; e < ne; e += NW) {
        const int k = k0 + e;
#pragma unroll
        for (int j = 0; j < 6; ++j) CN[e * 6 + j] = d.conn[(size_t)k * 6 + j];
        const ElemGeo& g = d.geo[k];
        GEO[0 * E + e] = (float)g.rx; GEO[1 * E + e] = (float)g.ry;
        GEO[2 * E + e] = (float)g.sx; GEO[3 * E + e] = (float)g.sy;
#pragma unroll
        for (int fc = 0; fc < 3; ++fc) {
          GEO[(4 + fc) * E + e] = (float)g.nx[fc];
          GEO[(7 + fc) * E + e] = (float)g.ny[fc];
          GEO[(10 + fc) * E + e] = (float)(-g.sJ[fc] * g.invJ);
        }
      }
      umma::fence_proxy_async();
      mbar_arrive(mbA);
    };
    // reference fluxes at the fp32 mean of tile i (tasks: volume + 3 faces per element)
    auto refs = [&](int i, int t0, int nt) {
      const int tile = tile_of(i), k0 = tile * E, ne = min(E, d.K - k0);
      unsigned char* td = slot(i);
      const float* GEO = (const float*)(td + C::TD_GEO);
      const float* QF = (const float*)(td + C::TD_QF);
      float* P0 = (float*)(td + C::TD_P0);
      double* Rb = (double*)(td + C::TD_RB);
      double* Fb = (double*)(td + C::TD_FB);
      for (int task = t0; task < 4 * E; task += nt) {
        const int kind = task / E, e = task - kind * E;
        if (e >= ne) continue;
        const ElemGeo& geo = d.geo[k0 + e];
        float qc[M];
#pragma unroll
        for (int f = 0; f < M; ++f) qc[f] = QF[f * E + e];
        // the fp32 flux of the mean; every float64 constant uses these same
        // values, so the volume and face constants cancel for a uniform state
        float F[M], G[M];
        P::flux2(d.eqp, qc, F, G, &err);
        if (kind == 0) {
#pragma unroll
          for (int f = 0; f < M; ++f) {
            P0[f * E + e] = F[f];
            P0[(M + f) * E + e] = G[f];
            Rb[f * E + e] = geo.rx * (double)F[f] + geo.ry * (double)G[f];
            Rb[(M + f) * E + e] = geo.sx * (double)F[f] + geo.sy * (double)G[f];
          }
        } else {
          // face reference: the fp32 Lax-Friedrichs flux with both states at the
          // mean (what a uniform state gives at every Gauss point); its float64
          // constant is the normal flux nx F + ny G of the same F, G (the wave-speed
          // term vanishes for equal states) with float64 normals
          const int fc = kind - 1;
          float qM[M], qP[M], nf[M];
#pragma unroll
          for (int f = 0; f < M; ++f) { qM[f] = qc[f]; qP[f] = qc[f]; }
          P::numflux(d.eqp, GEO[(4 + fc) * E + e], GEO[(7 + fc) * E + e], qM, qP, nf, &err);
          const double w = -geo.sJ[fc] * geo.invJ, nx = geo.nx[fc], ny = geo.ny[fc];
#pragma unroll
          for (int f = 0; f < M; ++f) {
            P0[((2 + fc) * M + f) * E + e] = nf[f];
            Fb[(fc * M + f) * E + e] = w * (nx * (double)F[f] + ny * (double)G[f]);
          }
        }
      }
    };
    // cubature deviations of tile i from TMEM to ST (warps by lane quadrant)
    auto stage = [&](int i) {
      if (!umma::mbar_wait_bounded(mbD1, i & 1)) *abort_flag = 1;
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
    // chunk operands of tile i into the ring; cc counts chunks over all tiles
    uint32_t cc = 0;
    auto items = [&](int i) {
      const int tile = tile_of(i), k0 = tile * E, ne = min(E, d.K - k0);
      unsigned char* td = slot(i);
      const float* GEO = (const float*)(td + C::TD_GEO);
      const int* CN = (const int*)(td + C::TD_CN);
      const float* QF = (const float*)(td + C::TD_QF);
      const float* P0 = (const float*)(td + C::TD_P0);
      for (int ch = 0; ch < C::NCH; ++ch, ++cc) {
        const int b = cc % NBUF;
        if (cc >= NBUF && !umma::mbar_wait_bounded(mb_empty(b), ((cc / NBUF) - 1) & 1)) *abort_flag = 1;
        unsigned char* bh = RING + b * 2 * C::SZ_CH;
        unsigned char* bl = bh + C::SZ_CH;
        if (ch < NV) {
          // volume: deviation of the fp32 flux from the flux of the mean, times the metric
          const int npts = min(VPC, NC - ch * VPC);
          const int nfill = 4 * ((npts + 3) / 4);
          for (int it = wtid; it < nfill * E; it += NW) {
            const int cp = it / E, e = it - cp * E;
            if (e >= ne) continue;
            const int rowb = rowb_of(e);
            float R[M], S[M];
            if (cp < npts) {
              const int c = ch * VPC + cp;
              float qc[M], F[M], G[M];
              load_fields<M>(ST + c * 128 + rowb, qc);
#pragma unroll
              for (int f = 0; f < M; ++f) qc[f] += QF[f * E + e];
              P::flux2(d.eqp, qc, F, G, &err);
              const float rx = GEO[0 * E + e], ry = GEO[1 * E + e], sx = GEO[2 * E + e], sy = GEO[3 * E + e];
#pragma unroll
              for (int f = 0; f < M; ++f) {
                const float dF = F[f] - P0[f * E + e], dG = G[f] - P0[(M + f) * E + e];
                R[f] = rx * dF + ry * dG;
                S[f] = sx * dF + sy * dG;
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
          const int col0 = (ch - NV) * KV;
          const int ncol = min(KV, C::NFK - col0);
          for (int it = wtid; it < ncol * E; it += NW) {
            const int e = it % E, cl = it / E, col = col0 + cl;
            if (e >= ne) continue;
            const int rowb = rowb_of(e), k = k0 + e;
            float dev[M];
            if (col < NF) {
              const int fc = col / NG, g = col - fc * NG;
              float qM[M], qP[M], nf[M];
              const int nb = CN[e * 6 + 2 * fc];
              load_fields<M>(a.tr_in + ((size_t)(k * 3 + fc) * NG + g) * M, qM);
              if (nb >= 0) {
                const int f2 = CN[e * 6 + 2 * fc + 1];
                load_fields<M>(a.tr_in + ((size_t)(nb * 3 + f2) * NG + (NG - 1 - g)) * M, qP);
              }
              const float nx = GEO[(4 + fc) * E + e], ny = GEO[(7 + fc) * E + e];
              if (nb < 0) {
                double x, y;
                bc_coords(k, fc, g, x, y);
                apply_bc<EQ, float>(d.bcs, -nb, tstage, x, y, nx, ny, qM, qP);
              }
              const float lam = P::numflux(d.eqp, nx, ny, qM, qP, nf, &err);
              if (want_lambda) {
                const double l = fabs((double)lam);
                lmax = l > lmax ? l : lmax;
              }
              const float w = GEO[(10 + fc) * E + e];
#pragma unroll
              for (int f = 0; f < M; ++f) dev[f] = w * (nf[f] - P0[((2 + fc) * M + f) * E + e]);
            } else {
#pragma unroll
              for (int f = 0; f < M; ++f) dev[f] = 0.f;
            }
#pragma unroll
            for (int f = 0; f < M; ++f) {
              float h, l;
              split_tf32(dev[f], h, l);
              const uint32_t off = umma::kmajor_offset_sbo(rowb + f, cl, C::SBOC);
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
      if (!umma::mbar_wait_bounded(mbD2, i & 1)) *abort_flag = 1;
      umma::fence_after_sync();
      float dv[C::NPN];
#pragma unroll
      for (int c0 = 0; c0 < C::NPN; c0 += 16) {
        float v[16];
        umma::tmem_ld16(tlane + C::T_D2 + c0, v);
        umma::tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) dv[c0 + j] = v[j];
      }
      umma::fence_before_sync();
      if (!rvalid || *abort_flag) return;
      const int k = k0 + re;
      const double Rbar = Rb[rf * E + re], Sbar = Rb[(M + rf) * E + re];
      const double F0 = Fb[(0 * M + rf) * E + re], F1 = Fb[(1 * M + rf) * E + re], F2 = Fb[(2 * M + rf) * E + re];
      const double c_stage = dt / 4.0, c_al = 4.0 / 5.0, c_be = dt / 5.0, c_ga = 1.0 / 5.0;
      const double* xrow = a.x + (size_t)k * NP * M + rf;
      const double* urow = a.u0 + (size_t)k * NP * M + rf;
      double* orow = a.out + (size_t)k * NP * M + rf;
      double o[NP];
      // out may alias x and u0 (same row, same thread): each batch of nodes is
      // loaded in full before any of it is stored, so the loads overlap
      constexpr int BT = 8;
#pragma unroll
      for (int i0 = 0; i0 < NP; i0 += BT) {
        double xr[BT], ur[BT];
#pragma unroll
        for (int u = 0; u < BT; ++u) {
          const int n = i0 + u;
          if (n < NP && a.mode != MODE_RHS) xr[u] = xrow[n * M];
          if (n < NP && a.mode == MODE_FINAL) ur[u] = urow[n * M];
        }
#pragma unroll
        for (int u = 0; u < BT; ++u) {
          const int n = i0 + u;
          if (n >= NP) break;
          const double* rs = RSUM + n * 5;
          const double r = (double)dv[n] + rs[0] * Rbar + rs[1] * Sbar + rs[2] * F0 + rs[3] * F1 + rs[4] * F2;
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
      if (write_traces) {
        const double m = nodal_mean<NP>(o);
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
        const int k = k0 + e;
        row_traces<NP, NG>(IF, XD + r, 128, XB[r], fc, a.tr_out + ((size_t)(k * 3 + fc) * NG) * M + f, M);
      }
    };

    if (my_tiles > 0) {
      build_a(0);
      workers_sync<NW>();
      refs(0, wtid, NW);
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
      if (wtid < 128) epilogue(i);
      else if (next) refs(i + 1, wtid - 128, NW - 128);
      workers_sync<NW>();
      if (write_traces && !*abort_flag) traces(i);
      if (next) {
        stage(i + 1);
        workers_sync<NW>();
        // read right after a worker barrier, so every worker leaves together
        if (*abort_flag) ok = false;
      }
    }
    if (want_lambda) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double v = __shfl_xor_sync(0xffffffffu, lmax, o);
        lmax = v > lmax ? v : lmax;
      }
      if (lane == 0 && lmax > 0.0) atomicMax(&d.st->lam_bits, (unsigned long long)__double_as_longlong(lmax));
    }
  }
  if (err) atomicOr(&d.st->err, err);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (*abort_flag) {
    // after an abort: let every issued MMA complete (a fresh barrier, so its
    // parity is unambiguous) and the state copy in flight, if any, land
    if (warp == kMixThreads / 32 - 1) {
      if (lane == 0) umma::commit(mbDrain);
      __syncwarp();
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

// Face traces [K][3][NG][M] of a state: one thread per (element, field, face).
template <int N, int M>
__global__ void __launch_bounds__(256) k_mixed_traces(int K, const double* __restrict__ x,
                                                      const double* __restrict__ I, float* __restrict__ T) {
  constexpr int NP = Sizes<N>::NP, NG = Sizes<N>::NG, NF = Sizes<N>::NF;
  __shared__ float IF[NF * NP];
  for (int i = threadIdx.x; i < NF * NP; i += blockDim.x) IF[i] = (float)I[i];
  __syncthreads();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)K * M * 3) return;
  const int fc = (int)(t % 3);
  const long long rest = t / 3;
  const int f = (int)(rest % M);
  const int k = (int)(rest / M);
  double v[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) v[j] = x[((size_t)k * NP + j) * M + f];
  const double m = nodal_mean<NP>(v);
  float dv[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) dv[j] = (float)(v[j] - m);
  row_traces<NP, NG>(IF, dv, 1, m, fc, T + ((size_t)(k * 3 + fc) * NG) * M + f, M);
}

template <int N, int M>
cudaError_t launch_traces_t(const DgDev& d, const double* x, float* T, cudaStream_t s) {
  const long long n = (long long)d.K * M * 3;
  const int blocks = (int)((n + 255) / 256);
  k_mixed_traces<N, M><<<blocks, 256, 0, s>>>(d.K, x, d.I, T);
  return cudaGetLastError();
}

template <int EQ, int N>
cudaError_t launch_mixed_t(MixedPlan* p, const DgDev& d, const StageArgs& a0, cudaStream_t s, cudaEvent_t* ev) {
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
    const int ntiles = (d.K + C::E - 1) / C::E;
    int grid = sms;
    if (grid > ntiles) grid = ntiles;
    StageArgs a = a0;
    if (a.reset_lambda && a.mode != MODE_STAGE) {
      cudaError_t e = cudaMemsetAsync(&d.st->lam_bits, 0, sizeof(unsigned long long), s);
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
    if (ev) cudaEventRecord(ev[1], s);
    // bit 0: the state is bulk-copied (16-byte aligned); bit 1: warm L2 with u0
    const int flags = (((uintptr_t)a.x & 15) == 0 ? 1 : 0) |
                      (a.mode == MODE_FINAL && ((uintptr_t)a.u0 & 15) == 0 ? 2 : 0);
    k_mixed_stage<EQ, N><<<grid, kMixThreads, C::BYTES, s>>>(d, a, p->rowsum, flags);
    if (ev) {
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
