// Device-side data of one nodal-DG discretisation and the kernel interfaces.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dg_physics.cuh"

namespace apollo {

// Per-element geometry, 24 float64 (192 bytes), built on the host from the
// element's vertices exactly as Apollo's GeometricFactors2d / Normals2d do
// (src/lib/wxnodaldggeometry2d.cc:382-442).
struct ElemGeo {
  double rx, ry, sx, sy;  // dr/dx, dr/dy, ds/dx, ds/dy
  double J, invJ;
  double nx[3], ny[3], sJ[3];  // outward unit normal and half edge length per face
  double vx[3], vy[3];         // vertices (for boundary-condition coordinates)
  double pad[3];
};

// Face record: interior (k1, f1, k2, f2) with k1's face f1 paired to k2's face
// f2; boundary (k, f, -tag, -1).
struct FaceRec {
  int k1, f1, k2, f2;
};

// Time-stepper state kept on the device so whole steps run without the host.
struct DevState {
  double t;          // time at the start of the current step
  double dt;         // dt of the current step
  double tend;       // end time (<= 0: none)
  double dtfac;      // 2/3 * cfl * dtscale of this instance (the dt policy's factor)
  unsigned long long lam_bits;  // max numerical-flux speed of the current stage (bits of a double >= 0)
  int err;           // ErrBits
  int steps;         // steps completed
  double last_sugg;  // suggested dt of the last right-hand side
  double sums[8];
};

// Source plugins (Apollo's WxHyperbolicSrc kinds whose value depends on time
// and position only): kind SRC_TM tranverseMagneticSrc
// (src/hyperapps/maxwell/wxtransversemagneticsrc.h:37-44), SRC_POINT
// pointCurrentSrc (src/hyperapps/maxwell/wxpointcurrent.h); out: the field of
// this handle's layout the source adds into; p: the plugin's parameters.
constexpr int kMaxSrc = 4;
enum SrcKind : int { SRC_TM = 1, SRC_POINT = 2 };
struct SrcTable {
  int n;
  int kind[kMaxSrc];
  int out[kMaxSrc];
  double p[kMaxSrc][9];
};

// Operators of one order, float64, row-major, built on the host.
//   V  [NC][NP]  nodal values -> cubature points (Vand_cub * V^-1)
//   Dr [NP][NC]  VVT * Dr_cub^T * diag(w_cub)    (VVT = V V^T, reference-element M^-1)
//   Ds [NP][NC]  VVT * Ds_cub^T * diag(w_cub)
//   I  [NF][NP]  nodal values -> face Gauss points, NF = 3 NG
//   L  [NP][NF]  VVT * I^T (surface "LIFT" without the Gauss weights)
struct DgDev {
  int K, nfaces, N;
  const ElemGeo* geo;
  const FaceRec* faces;
  const int* conn;  // [K][6]: per face (neighbour element, its face) or (-tag, -1) on a boundary
  // batched ensembles: instance of each element (nullptr: one instance) and the
  // number of instances; st then holds one DevState per instance (the error
  // word of st[0] serves them all)
  const int* einst;
  int ninst;
  int grid_div;    // launch shape: persistent grids use SMs / grid_div (>= 1; 0 means 1)
  int tile_shape;  // mixed stage operand chunking (0 or 1), picked by the batch autotuner
  int fp64_fused;  // float64 stages: 0 the three kernels, 1 the fused stage kernel where it applies,
                   // 2 the fused kernel where its tiles fit one resident wave (launch-bound meshes)
  int nghost;      // ghost element slots of a partitioned mesh (their faces' traces come from peers)
  int nbound;      // boundary faces of the local mesh
  // bounded device waits of the mixed stage kernel: polls before a wait gives
  // up (0: the default, about 2 s), and a test switch that points the kernel's
  // first wait at a barrier nothing completes (apollo_dg_debug_set_waits)
  unsigned wait_limit;
  int debug_stall;
  // source terms: the table, VS = VVT V^T diag(w) [NP][NC] (the source's
  // contribution is VS S at the cubature points), the cubature points' reference
  // coordinates [NC] each, and (mixed precision) a [K][NP][M] buffer holding
  // the current stage's source contribution
  SrcTable src;
  const double *VS, *cub_r, *cub_s;
  double* srcv;
  const double *V, *Dr, *Ds, *I, *L, *gz, *gw;
  double *vol, *trace, *flux;  // scratch: [K][NP][M], [K][NF][M], [K][NF][M]
  DevState* st;
  EqParams eqp;
  BcTable bcs;
  double dtfac;  // 2/3 * cfl * dtscale
  double rmin;
};

#if defined(__CUDACC__)
__device__ __forceinline__ int inst_of(const DgDev& d, int k) { return d.einst ? d.einst[k] : 0; }

// Per-instance maximum of non-negative wave speeds: a thread accumulates while
// its points stay in one instance and flushes (atomic max on the bit pattern,
// which orders like the value for non-negative doubles) when the instance
// changes; flush_warp, called by all 32 lanes, combines a warp whose lanes end
// in one instance.
struct LamAcc {
  int inst = -1;
  double v = 0.0;
  __device__ __forceinline__ void add(DevState* st, int i, double l) {
    if (i != inst) {
      if (inst >= 0 && v > 0.0) atomicMax(&st[inst].lam_bits, (unsigned long long)__double_as_longlong(v));
      inst = i;
      v = 0.0;
    }
    v = l > v ? l : v;
  }
  __device__ __forceinline__ void flush_warp(DevState* st) {
    const unsigned grp = __match_any_sync(0xffffffffu, inst);
    if (grp == 0xffffffffu) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, v, o);
        v = t > v ? t : v;
      }
      if ((threadIdx.x & 31) == 0 && inst >= 0 && v > 0.0)
        atomicMax(&st[inst].lam_bits, (unsigned long long)__double_as_longlong(v));
    } else if (inst >= 0 && v > 0.0) {
      atomicMax(&st[inst].lam_bits, (unsigned long long)__double_as_longlong(v));
    }
    inst = -1;
    v = 0.0;
  }
};
#endif

enum StageMode : int { MODE_RHS = 0, MODE_STAGE = 1, MODE_FINAL = 2 };

struct StageArgs {
  const double* x;   // right-hand-side input
  const double* u0;  // step start state (MODE_FINAL)
  double* out;
  int mode;
  int time_from_state;  // 1: t = st->t + st->dt * frac; 0: t = t_arg
  double frac;
  double t_arg;
  double dt_arg;        // dt used when time_from_state == 0
  int reset_lambda;     // volume kernel zeroes st->lam_bits first
  // mixed precision only: fp32 face traces [K][3][NG M, padded] of x (tr_in) and of
  // the stage result (tr_out, nullptr: not needed); for MODE_RHS the launcher
  // first computes the traces of x into tr_scratch and reads them from there
  const float* tr_in;
  float* tr_out;
  float* tr_scratch;
  // float64 launches of a partitioned mesh split around the trace exchange:
  // PHASE_ALL, PHASE_VOLUME (volume term and traces) or PHASE_FACE (face
  // fluxes and LIFT)
  int phase;
};

// PHASE_FACE_ONLY and PHASE_LIFT split PHASE_FACE into the face kernel and
// the lift (a partitioned stage runs its interior faces while the halo is in
// flight, then the cut faces and the lift).
enum { PHASE_ALL = 0, PHASE_VOLUME = 1, PHASE_FACE = 2, PHASE_FACE_ONLY = 3, PHASE_LIFT = 4 };

template <int N> struct Sizes {
  static constexpr int NP = (N + 1) * (N + 2) / 2;
  static constexpr int NG = 2 * (N + 1);
  static constexpr int NF = 3 * NG;
  // cubature points for cubature order 3(N+1) (src/lib/wxcubature2d.cc:26-28)
  static constexpr int NC = N == 1 ? 12 : N == 2 ? 19 : N == 3 ? 36 : N == 4 ? 54 : N == 5 ? 73 : N == 6 ? 93 : N == 7 ? 118 : 145;
};

// Host launchers (dg_fp64.cu).
// ev (optional): 4 events recorded before/between/after the three kernels
cudaError_t launch_rhs_fp64(int eq, const DgDev& d, const StageArgs& a, cudaStream_t s, cudaEvent_t* ev = nullptr);
// k_lift alone on d.vol / d.flux (used by the tangent of a stage)
cudaError_t launch_lift_fp64(int eq, const DgDev& d, const StageArgs& a, cudaStream_t s);
cudaError_t launch_init_speed(int eq, const DgDev& d, const double* u, cudaStream_t s);
cudaError_t launch_finalize(const DgDev& d, cudaStream_t s);
// st[i].lam_bits = 0 for every instance
cudaError_t launch_reset_lambda(const DgDev& d, cudaStream_t s);
// *st = v on the stream (no host staging buffer to race with later calls)
cudaError_t launch_put_state(DevState* st, const DevState& v, cudaStream_t s);
// Apollo's Euler limiter "eulerLimiterHW" (dg_limiter.cu), orders 2..4: the
// averaging weights of the nodal basis (half the reference mass matrix's
// column sums), the face-node mask, and the limiter's own gas_gamma,
// min_pressure and min_density
struct LimArgs {
  double ave[15];
  int fmask[15];
  double gamma, minP, minD;
  int kind;  // 0: eulerLimiterHW; 1: tuAliabadiLimiter (the equation's primitive floors and parameters)
};
size_t limiter_work_doubles(int K);
// limits x into out (may be x), scratch work[limiter_work_doubles(K)]; xn, yn
// are the node coordinates [K][Np]
cudaError_t launch_limiter(int eq, const DgDev& d, const LimArgs& L, const double* x, double* out, const double* xn,
                           const double* yn, double* work, cudaStream_t s);
// Halo trace blocks (dg_halo.cu): gather (dst[j] = src[idx[j]]) or scatter
// (dst[idx[j]] = src[j]) of n blocks of block_bytes (a multiple of 16) each
cudaError_t launch_halo_blocks(const void* src, void* dst, const int* idx, int n, int block_bytes, bool scatter,
                               cudaStream_t s);
cudaError_t launch_integrals(int eq, const DgDev& d, const double* u, const double* wJ, cudaStream_t s);
cudaError_t launch_energy(int eq, const DgDev& d, const double* u, const double* mass, cudaStream_t s);
// Source contribution VS S(t, x_c, y_c) of every element at the stage time of
// `a`: added to dst (accumulate) or written to it (fields without a source: 0).
cudaError_t launch_source(int eq, const DgDev& d, const StageArgs& a, double* dst, int accumulate, cudaStream_t s);
int fp64_supported(int eq, int N);

}  // namespace apollo
