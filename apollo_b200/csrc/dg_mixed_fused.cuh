// Fused mixed-precision stage for the four-field Euler equations (eulerEqn2d)
// with the Lax-Friedrichs flux at orders 2..4: the whole stage of a tile of 32
// elements in one CTA of 512 threads, every thread a worker, with the tensor
// core's work issued by thread 0 between the phases.  Included by dg_mixed.cu
// (inside its anonymous namespace: MixPhys, split_tf32, trace_stride and the
// StageArgs conventions come from there).
//
// The arithmetic is that of k_mixed_stage (the deviation form with tf32x3
// contractions, fp32 pointwise fluxes, float64 constants and epilogue); what
// differs is the schedule:
//   * the A operand of the second contraction (flux deviations at every
//     cubature and face point, hi and lo halves) is held in shared memory in
//     full, so its 36 MMAs go out in two bursts per tile instead of one
//     hand-off per operand chunk;
//   * tile rows are (element, field) pairs r = 4 e + f, so the 32 threads of a
//     warp cover 8 elements x 4 fields of one TMEM lane quarter, and every
//     item loop has a fixed element per thread (per-element constants stay in
//     registers, no index division in the loops);
//   * a thread reads its own row of the cubature values from TMEM and a 4 x 4
//     exchange through a per-warp scratch block hands it the four fields of
//     one point; the flux deviations it computes land in the K-major operand
//     with conflict-free 8-byte stores;
//   * the result's face traces are a third contraction (interpolation of the
//     result's deviations, tf32x3), staged in shared memory and written with
//     one bulk copy per tile.
//
// Phases of a tile (bar = all 512 threads):
//   S0 operand build: state deviations (A1), means, geometry, connectivity  bar
//   S1 [t0] GEMM-A  D1 = A1 V^T;  volume references per thread;  wait D1 bar
//   S2 volume items -> A2 volume columns; face and float64 references     bar
//   S3 [t0] GEMM-B volume part;  face items -> A2 face columns            bar
//   S4 [t0] GEMM-B face part;  wait D2
//   S5 epilogue (float64 result, RK update), result deviations (A3), means bar
//   S6 [t0] trace GEMM  D3 = A3 I^T;  wait D3
//   S7 traces -> shared staging                                          bar
//   S8 [t0] bulk store of the tile's traces
// Apollo: wxnodaldg2dmethod.cc:235-542 with the TSSSP RK_2 stage update.

constexpr int kFusedThreads = 512;



template <int N> struct FusedCfg {
  static constexpr int M = 4;
  static constexpr int NP = Sizes<N>::NP, NC = Sizes<N>::NC, NG = Sizes<N>::NG, NF = Sizes<N>::NF;
  static constexpr int E = 32;                       // elements per tile
  static constexpr int K1 = round_up_c(NP, 8);       // node columns (GEMM-A, trace GEMM)
  static constexpr int NGRP = K1 / 4;                // node groups of 4 (operand build, epilogue)
  static constexpr int NC16 = round_up_c(NC, 16);    // GEMM-A N
  static constexpr int NPN = round_up_c(NP, 16);     // GEMM-B N per half
  static constexpr int NVG = round_up_c(NC, 4) / 4;  // volume point groups of 4 (with zero padding)
  static constexpr int KV = round_up_c(8 * NVG, 8);  // volume K columns: R, S per point
  static constexpr int KF = round_up_c(NF, 8);       // face K columns
  static constexpr int KB = KV + KF;
  static constexpr int NFN = round_up_c(NF, 16);     // trace GEMM N
  static constexpr int NFG = KF / 4;                 // face column groups of 4
  static constexpr int TS = trace_stride(NG, M);
  static constexpr int SBO1 = K1 * 32;               // A1 / A3 (128 x K1), B1 (NC16 x K1), B3 (NFN x K1)
  static constexpr int SBO2 = KB * 32 + 16;          // A2 (128 x KB), groups staggered across banks
  static constexpr int SBOB = KB * 32;               // B2 (2 NPN x KB)
  static constexpr int SZ_B1 = (NC16 / 8) * SBO1;    // each half
  static constexpr int SZ_B2 = (2 * NPN / 8) * SBOB; // hi rows then lo rows
  static constexpr int SZ_B3 = (NFN / 8) * SBO1;     // each half
  static constexpr int SZ_A1 = 16 * SBO1;            // each half
  static constexpr int SZ_A2 = 16 * SBO2;            // each half
  static constexpr int SZ_XS = E * NP * M * 8;
  static constexpr int SZ_TR = E * 3 * TS * 4;
  static constexpr int SZ_SCR = 16 * 8 * 20 * 4;     // per warp: 8 elements x 4 points x 5 (padded) floats
  // per-tile data
  static constexpr int TD_GEO = 0;                        // [13][E] float
  static constexpr int TD_CN = TD_GEO + 13 * E * 4;       // [E][6] int
  static constexpr int TD_QF = TD_CN + E * 6 * 4;         // [M][E] float means
  static constexpr int TD_P0 = TD_QF + M * E * 4;         // [5M][E] float references
  static constexpr int TD_RB = round_up_c(TD_P0 + 5 * M * E * 4, 8);  // [2M][E] double
  static constexpr int TD_FB = TD_RB + 2 * M * E * 8;     // [3M][E] double
  static constexpr int TD_XB = TD_FB + 3 * M * E * 8;     // [128] double means (state, then result)
  static constexpr int TD_PS = TD_XB + 128 * 8;           // [4][128] double partial sums
  static constexpr int TD_GT = round_up_c(TD_PS + 4 * 128 * 8, 16);  // [E] ElemGeo of the tile (bulk copy)
  static constexpr int TD_CT = TD_GT + E * (int)sizeof(ElemGeo);     // [E][6] int connectivity (bulk copy)
  static constexpr int SZ_TD = TD_CT + E * 6 * 4 + 16;
  // layout
  static constexpr int O_A2 = 0;                                   // hi, lo
  static constexpr int O_B2 = O_A2 + 2 * SZ_A2;
  static constexpr int O_A1 = round_up_c(O_B2 + SZ_B2, 128);       // hi, lo (also A3)
  static constexpr int O_B1 = O_A1 + 2 * SZ_A1;                    // hi, lo
  static constexpr int O_B3 = O_B1 + 2 * SZ_B1;                    // hi, lo
  static constexpr int O_XS = round_up_c(O_B3 + 2 * SZ_B3, 16);
  // the state tile is staged in shared memory (one bulk copy, prefetched a
  // tile ahead) where it fits; otherwise the operand build reads it directly
  static constexpr int FIXED = O_XS + SZ_SCR + NP * 5 * 8 + SZ_TD + 128;
  static constexpr int LIMIT = 227 * 1024;
  static constexpr bool XSM = FIXED + SZ_XS <= LIMIT;
  static constexpr int O_SCR = O_XS + (XSM ? SZ_XS : 0);
  static constexpr int O_RS = O_SCR + SZ_SCR;                      // [NP][5] double row sums
  static constexpr int O_TD = round_up_c(O_RS + NP * 5 * 8, 16);
  static constexpr int O_MB = round_up_c(O_TD + SZ_TD, 8);         // mbarriers: x, D1, D2, D3, drain, geometry
  static constexpr int O_TSL = O_MB + 8 * 8;                       // TMEM base, abort flag
  static constexpr int BYTES = O_TSL + 16;
  static constexpr int T_D1 = 0, T_D2 = NC16, T_D3 = 0;
  static constexpr int TCOLS = tmem_cols(NC16 + 2 * NPN);
  // the form applies where shared memory holds it, the four warps of a quarter
  // cover the cubature columns, the trace accumulator fits in the cubature
  // columns and the trace staging in the A2 hi half
  static constexpr bool FITS = BYTES <= LIMIT && NC16 / 16 <= 4 && NFN <= NC16 && SZ_TR <= SZ_A2;
};

template <int EQ, int N>
__global__ void __launch_bounds__(kFusedThreads, 1)
    k_mixed_fused(DgDev d, StageArgs a, const double* __restrict__ rowsum, int flags) {
  using Q = MixPhys<EQ>;
  using C = FusedCfg<N>;
  constexpr int M = C::M, NP = C::NP, NC = C::NC, NG = C::NG, NF = C::NF, E = C::E, K1 = C::K1, TS = C::TS;
  static_assert(Eq<EQ>::M == 4, "four fields");
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* A2h = sm + C::O_A2;
  unsigned char* A2l = A2h + C::SZ_A2;
  unsigned char* B2 = sm + C::O_B2;
  unsigned char* A1h = sm + C::O_A1;
  unsigned char* A1l = A1h + C::SZ_A1;
  unsigned char* B1h = sm + C::O_B1;
  unsigned char* B1l = B1h + C::SZ_B1;
  unsigned char* B3h = sm + C::O_B3;
  unsigned char* B3l = B3h + C::SZ_B3;
  double* XS = (double*)(sm + C::O_XS);
  float* TRS = (float*)A2h;  // the tile's traces, staged for the bulk store
  double* RSUM = (double*)(sm + C::O_RS);
  unsigned char* td = sm + C::O_TD;
  float* GEO = (float*)(td + C::TD_GEO);
  int* CN = (int*)(td + C::TD_CN);
  float* QF = (float*)(td + C::TD_QF);
  float* P0 = (float*)(td + C::TD_P0);
  double* RB = (double*)(td + C::TD_RB);
  double* FB = (double*)(td + C::TD_FB);
  const ElemGeo* GT = (const ElemGeo*)(td + C::TD_GT);
  const int* CT = (const int*)(td + C::TD_CT);
  double* XB = (double*)(td + C::TD_XB);
  double* PS = (double*)(td + C::TD_PS);
  uint64_t* mbar = (uint64_t*)(sm + C::O_MB);
  uint32_t* tslot = (uint32_t*)(sm + C::O_TSL);
  volatile int* abort_flag = (volatile int*)(sm + C::O_TSL + 4);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool x_bulk = C::XSM && (flags & 1), u0_prefetch = flags & 2;
  const uint32_t wlim = d.wait_limit ? d.wait_limit : (1u << 22);
  const uint32_t mbX = umma::smem_u32(mbar + 0), mbD1 = umma::smem_u32(mbar + 1), mbD2 = umma::smem_u32(mbar + 2),
                 mbD3 = umma::smem_u32(mbar + 3), mbDrain = umma::smem_u32(mbar + 4), mbG = umma::smem_u32(mbar + 5);

  // ---- once per CTA: operators split into tf32 halves (K-major), zeroed operands
  for (int i = tid; i < C::NC16 * K1; i += kFusedThreads) {
    const int r = i / K1, k = i % K1;
    const double v = (r < NC && k < NP) ? d.V[r * NP + k] : 0.0;
    const float h = umma::round_tf32((float)v);
    const float l = umma::round_tf32((float)(v - (double)h));
    *(float*)(B1h + umma::kmajor_offset_sbo(r, k, C::SBO1)) = h;
    *(float*)(B1l + umma::kmajor_offset_sbo(r, k, C::SBO1)) = l;
  }
  // B2 rows 0..NPN-1 hi, NPN..2NPN-1 lo; columns: (Dr, Ds) per cubature point,
  // then LIFT times the Gauss weight per face point (fc NG + g)
  for (int i = tid; i < C::NPN * C::KB; i += kFusedThreads) {
    const int r = i / C::KB, k = i % C::KB;
    double v = 0.0;
    if (r < NP) {
      if (k < C::KV) {
        const int c = k >> 1;
        if (c < NC) v = (k & 1) ? d.Ds[r * NC + c] : d.Dr[r * NC + c];
      } else if (k - C::KV < NF) {
        const int col = k - C::KV;
        v = d.L[r * NF + col] * d.gw[col % NG];
      }
    }
    const float h = umma::round_tf32((float)v);
    const float l = umma::round_tf32((float)(v - (double)h));
    *(float*)(B2 + umma::kmajor_offset_sbo(r, k, C::SBOB)) = h;
    *(float*)(B2 + umma::kmajor_offset_sbo(r + C::NPN, k, C::SBOB)) = l;
  }
  // B3: the face interpolation, rows fc NG + g
  for (int i = tid; i < C::NFN * K1; i += kFusedThreads) {
    const int r = i / K1, k = i % K1;
    const double v = (r < NF && k < NP) ? d.I[r * NP + k] : 0.0;
    const float h = umma::round_tf32((float)v);
    const float l = umma::round_tf32((float)(v - (double)h));
    *(float*)(B3h + umma::kmajor_offset_sbo(r, k, C::SBO1)) = h;
    *(float*)(B3l + umma::kmajor_offset_sbo(r, k, C::SBO1)) = l;
  }
  // A2 (every column a finite value; padding columns stay zero) and A1
  for (int i = tid; i < 2 * C::SZ_A2 / 16; i += kFusedThreads) ((float4*)A2h)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int i = tid; i < 2 * C::SZ_A1 / 16; i += kFusedThreads) ((float4*)A1h)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int i = tid; i < NP * 5; i += kFusedThreads) RSUM[i] = rowsum[i];
  if (tid == 0) {
    for (int b = 0; b < 6; ++b) umma::mbar_init(umma::smem_u32(mbar + b), 1);
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
  auto x_doubles = [&](int tile) {
    const int ne = min(E, d.K - tile * E);
    return ((ne * NP * M * 8) & ~15) / 8;
  };
  auto issue_x = [&](int i) {  // thread 0: the state tile into XS
    const int tile = tile_of(i);
    const uint32_t bytes = (uint32_t)x_doubles(tile) * 8u;
    umma::mbar_expect_tx(mbX, bytes);
    umma::bulk_g2s(umma::smem_u32(XS), a.x + (size_t)tile * E * NP * M, bytes, mbX);
  };
  auto issue_geo = [&](int i) {  // thread 0: geometry and connectivity of tile i into GT, CT
    const int k0 = tile_of(i) * E, ne = min(E, d.K - k0);
    const uint32_t gb = (uint32_t)(ne * (int)sizeof(ElemGeo));  // a multiple of 16
    // (rounded up to 16 bytes: the connectivity array has 16 bytes of slack)
    const uint32_t cb = (uint32_t)((ne * 24 + 15) & ~15);
    umma::mbar_expect_tx(mbG, gb + cb);
    umma::bulk_g2s(umma::smem_u32(GT), d.geo + k0, gb, mbG);
    umma::bulk_g2s(umma::smem_u32(CT), d.conn + (size_t)k0 * 6, cb, mbG);
  };
  // (a single warp waits; it spins, so it passes the phase the moment the
  // tensor core or the copy completes it)
  auto wait = [&](uint32_t mb, uint32_t parity) {
    if (!umma::mbar_spin_bounded(mb, parity, wlim)) *abort_flag = 1;
  };

  auto all_sync = [&]() { asm volatile("bar.sync 1, %0;" ::"n"(kFusedThreads) : "memory"); };

  // descriptors (the start address field advances by 16 per K step of 256 bytes)
  constexpr uint64_t KSTEP = (2 * umma::kLBO) >> 4;
  const uint64_t dA1h = umma::make_desc(umma::smem_u32(A1h), umma::kLBO, C::SBO1);
  const uint64_t dA1l = umma::make_desc(umma::smem_u32(A1l), umma::kLBO, C::SBO1);
  const uint64_t dB1h = umma::make_desc(umma::smem_u32(B1h), umma::kLBO, C::SBO1);
  const uint64_t dB1l = umma::make_desc(umma::smem_u32(B1l), umma::kLBO, C::SBO1);
  const uint64_t dB3h = umma::make_desc(umma::smem_u32(B3h), umma::kLBO, C::SBO1);
  const uint64_t dB3l = umma::make_desc(umma::smem_u32(B3l), umma::kLBO, C::SBO1);
  const uint64_t dA2h = umma::make_desc(umma::smem_u32(A2h), umma::kLBO, C::SBO2);
  const uint64_t dA2l = umma::make_desc(umma::smem_u32(A2l), umma::kLBO, C::SBO2);
  const uint64_t dB2 = umma::make_desc(umma::smem_u32(B2), umma::kLBO, C::SBOB);
  constexpr uint32_t idA = umma::idesc_tf32(128, C::NC16);
  constexpr uint32_t idB = umma::idesc_tf32(128, 2 * C::NPN);
  constexpr uint32_t idC = umma::idesc_tf32(128, C::NFN);

  // this thread's row in the TMEM quarter of its warp: element e_q (0..7 in the
  // quarter), field f; the warp's sub-index g = warp / 4 splits the columns
  const int q = warp & 3, g4 = warp >> 2, f_me = lane & 3, e_me = 8 * q + (lane >> 2);
  const uint32_t tlane = tb + ((uint32_t)(32 * q) << 16);
  float* scr = (float*)(sm + C::O_SCR) + warp * (8 * 20);  // this warp's exchange block
  const int eq_w = lane >> 2;                               // element within the warp's block
  // the operand build and the epilogue: thread (row, node group); it keeps its
  // four state values in registers from the one to the other
  const int r_ep = tid & 127, ng_ep = tid >> 7, e_ep = r_ep >> 2, f_ep = r_ep & 3;
  const bool node_thread = ng_ep < C::NGRP;
  const bool want_lambda = a.mode != MODE_STAGE;
  const bool write_traces = a.tr_out != nullptr && a.mode != MODE_RHS;
  LamAcc lam_acc;
  int err = 0;
  bool ok = true;
  int x_issued = 0, g_issued = 0;
  auto stage_t = [&](int k) {
    const DevState& S = d.st[inst_of(d, k)];
    return a.time_from_state ? S.t + S.dt * a.frac : a.t_arg;
  };
  auto stage_dt = [&](int k) { return a.time_from_state ? d.st[inst_of(d, k)].dt : a.dt_arg; };
  // this thread's state values of tile i straight from global memory (no
  // shared-memory state tile)
  double xv[4] = {0.0, 0.0, 0.0, 0.0};
  double dt_ep = 0.0;  // this thread's element's dt, read in the operand build
  auto load_x = [&](int i) {
    const int k0 = tile_of(i) * E, ne = min(E, d.K - k0);
    const double* xg = a.x + (size_t)k0 * NP * M;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int j = 4 * ng_ep + u;
      xv[u] = (node_thread && e_ep < ne && j < NP) ? xg[(e_ep * NP + j) * M + f_ep] : 0.0;
    }
  };

  if (tid == 0 && my_tiles > 0) {
    issue_geo(0);
    g_issued = 1;
    if (x_bulk) {
      issue_x(0);
      x_issued = 1;
    }
  }
  if (!x_bulk && my_tiles > 0) load_x(0);
  for (int i = 0; i < my_tiles && ok; ++i) {
    const int tile = tile_of(i), k0 = tile * E, ne = min(E, d.K - k0);
    const uint32_t par = i & 1;
    // ---------------- S0: operand build (one warp waits for the copies)
    if (warp == 0) {
      wait(mbG, par);
      if (x_bulk) wait(mbX, par);
    }
    all_sync();
    {
      double v[4];
      if (node_thread) {
        const bool valid = e_ep < ne;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int j = 4 * ng_ep + u;
          v[u] = (valid && j < NP) ? (x_bulk ? XS[(e_ep * NP + j) * M + f_ep] : xv[u]) : 0.0;
          xv[u] = v[u];  // kept for the epilogue
        }
        PS[ng_ep * 128 + r_ep] = (v[0] + v[1]) + (v[2] + v[3]);
        if (valid) dt_ep = stage_dt(k0 + e_ep);
      }
      if (tid >= kFusedThreads - E) {
        // fp32 geometry and connectivity of the tile
        const int e = tid - (kFusedThreads - E);
        const bool valid = e < ne;
        const ElemGeo& gg = GT[e];
        GEO[0 * E + e] = valid ? (float)gg.rx : 0.f;
        GEO[1 * E + e] = valid ? (float)gg.ry : 0.f;
        GEO[2 * E + e] = valid ? (float)gg.sx : 0.f;
        GEO[3 * E + e] = valid ? (float)gg.sy : 0.f;
#pragma unroll
        for (int fc = 0; fc < 3; ++fc) {
          GEO[(4 + fc) * E + e] = valid ? (float)gg.nx[fc] : 0.f;
          GEO[(7 + fc) * E + e] = valid ? (float)gg.ny[fc] : 0.f;
          GEO[(10 + fc) * E + e] = valid ? (float)(-gg.sJ[fc] * gg.invJ) : 0.f;
        }
#pragma unroll
        for (int j = 0; j < 6; ++j) CN[e * 6 + j] = valid ? CT[e * 6 + j] : 0;
      }
      all_sync();
      if (node_thread) {
        // the nodal mean in the fixed order of the mean tree
        double s01 = PS[0 * 128 + r_ep] + PS[1 * 128 + r_ep];
        if (C::NGRP > 2) s01 = s01 + (PS[2 * 128 + r_ep] + PS[3 * 128 + r_ep]);
        const double qbar = s01 * (1.0 / NP);
        const bool valid = e_ep < ne;
        float hv[4], lv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float xd = (valid && 4 * ng_ep + u < NP) ? (float)(v[u] - qbar) : 0.f;
          split_tf32(xd, hv[u], lv[u]);
        }
        const uint32_t off = umma::kmajor_offset_sbo(r_ep, ng_ep * 4, C::SBO1);
        *(float4*)(A1h + off) = make_float4(hv[0], hv[1], hv[2], hv[3]);
        *(float4*)(A1l + off) = make_float4(lv[0], lv[1], lv[2], lv[3]);
        if (ng_ep == 0) QF[f_ep * E + e_ep] = valid ? (float)qbar : 0.f;
      }
      umma::fence_proxy_async();
      all_sync();
      if (*abort_flag) { ok = false; break; }
    }
    // ---------------- S1: GEMM-A, the next state tile, the volume references
    if (tid == 0) {
      umma::fence_after_sync();
#pragma unroll
      for (int s = 0; s < K1 / 8; ++s) {
        umma::mma_tf32(tb + C::T_D1, dA1h + s * KSTEP, dB1h + s * KSTEP, idA, s > 0);
        umma::mma_tf32(tb + C::T_D1, dA1h + s * KSTEP, dB1l + s * KSTEP, idA, 1);
        umma::mma_tf32(tb + C::T_D1, dA1l + s * KSTEP, dB1h + s * KSTEP, idA, 1);
      }
      umma::commit(mbD1);
      if (x_bulk && i + 1 < my_tiles) {  // XS is free again
        issue_x(i + 1);
        x_issued++;
      }
      if (u0_prefetch) bulk_prefetch_l2(a.u0 + (size_t)k0 * NP * M, (uint32_t)((ne * NP * M * 8) & ~15));
      // the previous tile's trace store has read its staging (the A2 hi half),
      // which this tile's volume items overwrite after the next barrier
      if (write_traces) umma::bulk_wait_read();
    }
    // this thread's element's volume references (fp32 directional fluxes of
    // the mean), computed while GEMM-A runs; the face and float64 references
    // are left to the lightest warps of the volume phase
    const bool evalid_me = e_me < ne;
    float kQF[M], kG[4], kP[2 * M];
    {
#pragma unroll
      for (int f = 0; f < M; ++f) kQF[f] = QF[f * E + e_me];
#pragma unroll
      for (int j = 0; j < 4; ++j) kG[j] = GEO[j * E + e_me];
      int e_dummy = 0;
      const typename Q::Side sd = Q::side(d.eqp, kQF, evalid_me ? &err : &e_dummy);
      Q::along(sd, kQF, kG[0], kG[1], kP);
      Q::along(sd, kQF, kG[2], kG[3], kP + M);
    }
    // (the stall switch of the failure tests points the first tile's wait at a
    // barrier that nothing completes before the abort path)
    if (warp == kFusedThreads / 32 - 1) wait((d.debug_stall && i == 0) ? mbDrain : mbD1, par);
    all_sync();  // references visible, cubature values in TMEM
    umma::fence_after_sync();
    // ---------------- S2: volume items.  Warp (q, g4) takes the cubature
    // columns [16 g4, 16 g4 + 16) of its quarter; per group of 4 points a
    // thread computes the fluxes of point 4 j + f_me of its element.
    {
      const bool evalid = evalid_me;
      const int c0 = 16 * g4;
      if (c0 < C::NC16) {
        float v[16];
        umma::tmem_ld16(tlane + C::T_D1 + c0, v);
        umma::tmem_wait_ld();
        const int rowb = 4 * e_me;  // rows of this element: rowb .. rowb + 3
        const uint32_t obase = (uint32_t)((rowb >> 3) * C::SBO2 + (rowb & 7) * 16);
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int j = c0 / 4 + jj;  // point group
          if (j >= C::NVG) break;
          // exchange: this thread holds field f_me at points 4j..4j+3; after
          // it, field 0..3 at point 4 j + f_me
#pragma unroll
          for (int u = 0; u < 4; ++u) scr[eq_w * 20 + u * 5 + f_me] = v[4 * jj + u];
          __syncwarp();
          float qc[M];
#pragma unroll
          for (int f = 0; f < M; ++f) qc[f] = scr[eq_w * 20 + f_me * 5 + f];
          __syncwarp();
          const int c = 4 * j + f_me;
          float R[M], S[M];
          if (c < NC && evalid) {
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
          // rows rowb + f, columns 2c (R) and 2c + 1 (S)
          const uint32_t oc = obase + (uint32_t)((c >> 1) * umma::kLBO + (c & 1) * 8);
#pragma unroll
          for (int f = 0; f < M; ++f) {
            float h0, l0, h1, l1;
            split_tf32(R[f], h0, l0);
            split_tf32(S[f], h1, l1);
            *(float2*)(A2h + oc + 16 * f) = make_float2(h0, h1);
            *(float2*)(A2l + oc + 16 * f) = make_float2(l0, l1);
          }
        }
      }
      // reference fluxes for the faces and the float64 epilogue, by the
      // warps with the fewest volume items (the last four)
      if (tid >= kFusedThreads - 4 * E) {
        // reference fluxes at the fp32 mean (volume + three faces per element).
        // With both traces at the mean the Lax-Friedrichs flux is the normal
        // flux of the mean exactly (0.5 (F + F + lam 0) = F in fp32), so a face
        // takes the directional flux unless a clamp sends the flux down its
        // general path.
        const int kind = (tid - (kFusedThreads - 4 * E)) / E, e = (tid - (kFusedThreads - 4 * E)) % E;
        if (e < ne) {
          const ElemGeo& gg = GT[e];
          float qc[M];
#pragma unroll
          for (int f = 0; f < M; ++f) qc[f] = QF[f * E + e];
          float F[M], G[M];
          Eq<EQ>::flux2(d.eqp, qc, F, G, &err);
          const typename Q::Side sd = Q::side(d.eqp, qc, &err);
          if (kind == 0) {
            float R0[M], S0[M];
            Q::along(sd, qc, GEO[0 * E + e], GEO[1 * E + e], R0);
            Q::along(sd, qc, GEO[2 * E + e], GEO[3 * E + e], S0);
#pragma unroll
            for (int f = 0; f < M; ++f) {
              P0[f * E + e] = R0[f];
              P0[(M + f) * E + e] = S0[f];
              RB[f * E + e] = gg.rx * (double)F[f] + gg.ry * (double)G[f];
              RB[(M + f) * E + e] = gg.sx * (double)F[f] + gg.sy * (double)G[f];
            }
          } else {
            const int fc = kind - 1;
            float nf[M];
            const float nx = GEO[(4 + fc) * E + e], ny = GEO[(7 + fc) * E + e];
            if (sd.clean) Q::along(sd, qc, nx, ny, nf);
            else Q::lf(d.eqp, nx, ny, qc, qc, nf, &err);
            const double w = -gg.sJ[fc] * gg.invJ, nxd = gg.nx[fc], nyd = gg.ny[fc];
#pragma unroll
            for (int f = 0; f < M; ++f) {
              P0[((2 + fc) * M + f) * E + e] = nf[f];
              FB[(fc * M + f) * E + e] = w * (nxd * (double)F[f] + nyd * (double)G[f]);
            }
          }
        }
      }
      umma::fence_before_sync();
      umma::fence_proxy_async();
      all_sync();
      if (*abort_flag) { ok = false; break; }
    }
    // ---------------- S3: GEMM-B volume part; face items
    if (tid == 0) {
      umma::fence_after_sync();
      for (int s = 0; s < C::KV / 8; ++s) {
        umma::mma_tf32(tb + C::T_D2, dA2h + s * KSTEP, dB2 + s * KSTEP, idB, s > 0);
        umma::mma_tf32(tb + C::T_D2, dA2l + s * KSTEP, dB2 + s * KSTEP, idB, 1);
      }
      // the next tile's geometry and connectivity: this tile's copies were
      // read into GEO, CN and the reference fluxes before the last barrier
      if (i + 1 < my_tiles) {
        issue_geo(i + 1);
        g_issued++;
      }
    }
    {
      // warp (q, g4) takes face column groups g4 and g4 + 4; the thread the
      // column 4 j + f_me of its element
      const bool evalid = e_me < ne;
      const int k = k0 + e_me;
      const int rowb = 4 * e_me;
      const uint32_t obase = (uint32_t)((rowb >> 3) * C::SBO2 + (rowb & 7) * 16);
      // this thread's two face columns (groups j = g4 and g4 + 4): traces
      // fetched first, boundary ghosts next, then both Lax-Friedrichs fluxes
      // as one straight-line computation
      static_assert(C::NFG <= 8, "two face column groups per warp");
      float tM[2][M], tP[2][M];
      int fcs[2], nbs[2];
      bool val[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j = g4 + 4 * h, col = 4 * j + f_me;
        val[h] = j < C::NFG && col < NF && evalid;
        const int fc = val[h] ? col / NG : 0, g = col - fc * NG;
        fcs[h] = fc;
        nbs[h] = CN[e_me * 6 + 2 * fc];
#pragma unroll
        for (int f = 0; f < M; ++f) { tM[h][f] = kQF[f]; tP[h][f] = kQF[f]; }  // a physical stand-in
        if (val[h]) {
          load_fields<M>(a.tr_in + ((size_t)k * 3 + fc) * TS + g * M, tM[h]);
          if (nbs[h] >= 0)
            load_fields<M>(a.tr_in + ((size_t)nbs[h] * 3 + CN[e_me * 6 + 2 * fc + 1]) * TS + (NG - 1 - g) * M,
                           tP[h]);
        }
      }
      float nx[2], ny[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        nx[h] = GEO[(4 + fcs[h]) * E + e_me];
        ny[h] = GEO[(7 + fcs[h]) * E + e_me];
        if (val[h] && nbs[h] < 0) {
          const int col = 4 * (g4 + 4 * h) + f_me, g = col - fcs[h] * NG;
          const ElemGeo& geo = d.geo[k];
          const double z = d.gz[g];
          double rr, ss;
          if (fcs[h] == 0) { rr = z; ss = -1.0; }
          else if (fcs[h] == 1) { rr = -z; ss = z; }
          else { rr = -1.0; ss = -z; }
          const double bx = 0.5 * (-geo.vx[0] * (rr + ss) + geo.vx[1] * (1. + rr) + geo.vx[2] * (1. + ss));
          const double by = 0.5 * (-geo.vy[0] * (rr + ss) + geo.vy[1] * (1. + rr) + geo.vy[2] * (1. + ss));
          apply_bc<EQ, float>(d.bcs, -nbs[h], stage_t(k), bx, by, nx[h], ny[h], tM[h], tP[h]);
        }
      }
      float nf[2][M], lam[2];
      {
        int e_ign = 0;  // stand-in columns report nothing
        int* er0 = val[0] ? &err : &e_ign;
        int* er1 = val[1] ? &err : &e_ign;
        const typename Q::Side A0 = Q::side(d.eqp, tM[0], er0), B0 = Q::side(d.eqp, tP[0], er0);
        const typename Q::Side A1 = Q::side(d.eqp, tM[1], er1), B1 = Q::side(d.eqp, tP[1], er1);
        if (A0.clean && B0.clean && A1.clean && B1.clean) {
          const float gamma = (float)d.eqp.p[0];
          float FM0[M], FP0[M], FM1[M], FP1[M];
          Q::along(A0, tM[0], nx[0], ny[0], FM0);
          Q::along(B0, tP[0], nx[0], ny[0], FP0);
          Q::along(A1, tM[1], nx[1], ny[1], FM1);
          Q::along(B1, tP[1], nx[1], ny[1], FP1);
          const float cM0 = sqrtf(A0.vx * A0.vx + A0.vy * A0.vy + A0.vz * A0.vz) + sqrtf(gamma * A0.p * A0.ir);
          const float cP0 = sqrtf(B0.vx * B0.vx + B0.vy * B0.vy + B0.vz * B0.vz) + sqrtf(gamma * B0.p * B0.ir);
          const float cM1 = sqrtf(A1.vx * A1.vx + A1.vy * A1.vy + A1.vz * A1.vz) + sqrtf(gamma * A1.p * A1.ir);
          const float cP1 = sqrtf(B1.vx * B1.vx + B1.vy * B1.vy + B1.vz * B1.vz) + sqrtf(gamma * B1.p * B1.ir);
          lam[0] = cM0 > cP0 ? cM0 : cP0;
          lam[1] = cM1 > cP1 ? cM1 : cP1;
#pragma unroll
          for (int c = 0; c < M; ++c) {
            nf[0][c] = 0.5f * (FM0[c] + FP0[c] + lam[0] * (tM[0][c] - tP[0][c]));
            nf[1][c] = 0.5f * (FM1[c] + FP1[c] + lam[1] * (tM[1][c] - tP[1][c]));
          }
        } else {
          // a clamp: each flux down the reference's own path
          lam[0] = Q::lf(d.eqp, nx[0], ny[0], tM[0], tP[0], nf[0], er0);
          lam[1] = Q::lf(d.eqp, nx[1], ny[1], tM[1], tP[1], nf[1], er1);
        }
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j = g4 + 4 * h;
        if (j >= C::NFG) continue;
        const int col = 4 * j + f_me;
        float dev[M];
        if (val[h]) {
          if (want_lambda) lam_acc.add(d.st, inst_of(d, k), fabs((double)lam[h]));
          const float w = GEO[(10 + fcs[h]) * E + e_me];
#pragma unroll
          for (int f = 0; f < M; ++f) dev[f] = w * (nf[h][f] - P0[((2 + fcs[h]) * M + f) * E + e_me]);
        } else {
#pragma unroll
          for (int f = 0; f < M; ++f) dev[f] = 0.f;
        }
        // rows rowb + f, column KV + col
        const uint32_t oc = obase + (uint32_t)(((C::KV + col) >> 2) * umma::kLBO + (col & 3) * 4);
#pragma unroll
        for (int f = 0; f < M; ++f) {
          float hh, ll;
          split_tf32(dev[f], hh, ll);
          *(float*)(A2h + oc + 16 * f) = hh;
          *(float*)(A2l + oc + 16 * f) = ll;
        }
      }
      umma::fence_proxy_async();
      all_sync();
    }
    // ---------------- S4: GEMM-B face part
    if (tid == 0) {
      umma::fence_after_sync();
      for (int s = C::KV / 8; s < C::KB / 8; ++s) {
        umma::mma_tf32(tb + C::T_D2, dA2h + s * KSTEP, dB2 + s * KSTEP, idB, 1);
        umma::mma_tf32(tb + C::T_D2, dA2l + s * KSTEP, dB2 + s * KSTEP, idB, 1);
      }
      umma::commit(mbD2);
      wait(mbD2, par);
    }
    all_sync();
    umma::fence_after_sync();
    // ---------------- S5: float64 epilogue; thread (row, node group)
    {
      const int r = r_ep, ng = ng_ep, e = e_ep, f = f_ep;
      const bool active = node_thread;
      const bool rvalid = active && e < ne && !*abort_flag;
      float vh[4], vl[4];
      if (active) {
        const uint32_t tl = tb + ((uint32_t)(32 * (r >> 5)) << 16);
        umma::tmem_ld4(tl + C::T_D2 + 4 * ng, vh);
        umma::tmem_ld4(tl + C::T_D2 + C::NPN + 4 * ng, vl);
        umma::tmem_wait_ld();
      }
      double o[4] = {0.0, 0.0, 0.0, 0.0};
      if (rvalid) {
        const int k = k0 + e;
        const double Rbar = RB[f * E + e], Sbar = RB[(M + f) * E + e];
        const double F0 = FB[(0 * M + f) * E + e], F1 = FB[(1 * M + f) * E + e], F2 = FB[(2 * M + f) * E + e];
        const double dt = dt_ep;
        const double c_stage = dt / 4.0, c_al = 4.0 / 5.0, c_be = dt / 5.0, c_ga = 1.0 / 5.0;
        const double* urow = a.u0 + (size_t)k * NP * M + f;
        double* orow = a.out + (size_t)k * NP * M + f;
        double ur[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int n = 4 * ng + u;
          if (n < NP && a.mode == MODE_FINAL) ur[u] = urow[n * M];
        }
        const double* xr = xv;  // this thread's state values, read in the operand build
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int n = 4 * ng + u;
          if (n >= NP) break;
          const double* rs = RSUM + n * 5;
          const double dv = (double)(vh[u] + vl[u]);
          double rr = dv + rs[0] * Rbar + rs[1] * Sbar + rs[2] * F0 + rs[3] * F1 + rs[4] * F2;
          if (d.srcv) rr += d.srcv[((size_t)k * NP + n) * M + f];  // the stage's source terms
          if (!isfinite(rr)) err |= ERRB_NAN;
          if (a.mode == MODE_RHS) o[u] = rr;
          else if (a.mode == MODE_STAGE) o[u] = xr[u] + c_stage * rr;
          else o[u] = c_al * xr[u] + c_be * rr + c_ga * ur[u];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int n = 4 * ng + u;
          if (n < NP) orow[n * M] = o[u];
        }
      }
      // the next tile's state values: their loads overlap the rest of this tile
      if (!x_bulk && i + 1 < my_tiles) load_x(i + 1);
      if (write_traces) {
        // the result's mean (the nodal-mean tree: groups of 4 nodes, then pairs)
        if (active) PS[ng * 128 + r] = (o[0] + o[1]) + (o[2] + o[3]);
        all_sync();
        double m = 0.0;
        if (active) {
          double s01 = PS[0 * 128 + r] + PS[1 * 128 + r];
          if (C::NGRP > 2) s01 = s01 + (PS[2 * 128 + r] + PS[3 * 128 + r]);
          m = s01 * (1.0 / NP);
          if (ng == 0) XB[r] = m;
          float hv[4], lv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float dvv = (rvalid && 4 * ng + u < NP) ? (float)(o[u] - m) : 0.f;
            split_tf32(dvv, hv[u], lv[u]);
          }
          const uint32_t off = umma::kmajor_offset_sbo(r, ng * 4, C::SBO1);
          *(float4*)(A1h + off) = make_float4(hv[0], hv[1], hv[2], hv[3]);
          *(float4*)(A1l + off) = make_float4(lv[0], lv[1], lv[2], lv[3]);
        }
        umma::fence_before_sync();
        umma::fence_proxy_async();
      }
      all_sync();
      if (*abort_flag) { ok = false; break; }
    }
    if (write_traces) {
      // ---------------- S6: the trace GEMM (D3 over the cubature columns)
      if (tid == 0) {
        umma::fence_after_sync();
#pragma unroll
        for (int s = 0; s < K1 / 8; ++s) {
          umma::mma_tf32(tb + C::T_D3, dA1h + s * KSTEP, dB3h + s * KSTEP, idC, s > 0);
          umma::mma_tf32(tb + C::T_D3, dA1h + s * KSTEP, dB3l + s * KSTEP, idC, 1);
          umma::mma_tf32(tb + C::T_D3, dA1l + s * KSTEP, dB3h + s * KSTEP, idC, 1);
        }
        umma::commit(mbD3);
      }
      if (warp == 0) wait(mbD3, par);
      all_sync();
      umma::fence_after_sync();
      // ---------------- S7: traces = float(mean) + interpolated deviations
      {
        const int r = tid & 127, p = tid >> 7, e = r >> 2, f = r & 3;
        float v[8];
        const uint32_t tl = tb + ((uint32_t)(32 * (r >> 5)) << 16);
        umma::tmem_ld8(tl + C::T_D3 + 8 * p, v);
        umma::tmem_wait_ld();
        const float mf = (float)XB[r];
        if (e < ne) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int col = 8 * p + j;
            if (col < NF) {
              const int fc = col / NG, g = col - fc * NG;
              TRS[(e * 3 + fc) * TS + g * M + f] = mf + v[j];
            }
          }
        }
        umma::fence_before_sync();
        umma::fence_proxy_async();
        all_sync();
        if (*abort_flag) { ok = false; break; }
      }
      // ---------------- S8: one bulk store of the tile's traces
      if (tid == 0) {
        umma::bulk_s2g(a.tr_out + (size_t)k0 * 3 * TS, umma::smem_u32(TRS), (uint32_t)(ne * 3 * TS * 4));
        umma::bulk_commit();
      }
    }
  }
  if (want_lambda) lam_acc.flush_warp(d.st);
  if (err) atomicOr(&d.st->err, err);
  if (tid == 0) umma::bulk_wait_all();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (*abort_flag) {
    // let every issued MMA complete (a fresh barrier) and the state copy land
    if (tid == 0) {
      umma::commit(mbDrain);
      umma::mbar_wait_bounded(mbDrain, 0);
      if (x_issued > 0) umma::mbar_wait_bounded(mbX, (uint32_t)((x_issued - 1) & 1));
      if (g_issued > 0) umma::mbar_wait_bounded(mbG, (uint32_t)((g_issued - 1) & 1));
      atomicOr(&d.st->err, ERRB_TIMEOUT);
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
  }
  if (warp == 0) umma::tmem_dealloc(tb, C::TCOLS);
}
