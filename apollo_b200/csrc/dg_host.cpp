// C ABI of the nodal-DG solver: setup (operators, geometry, face map), device
// buffers, the right-hand side and the SSPRK(5,2) stepper with Apollo's dt
// policy.  See include/apollo_dg.h for the contract of each entry point.
#include "apollo_dg.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "dg_device.cuh"
#include "dg_adjoint.h"
#include "dg_mixed.h"
#include "dg_operators.h"
#include "dg_partition.h"
#include "dg_revolve.h"

using namespace apollo;

struct apollo_dg {
  apollo_dg_config cfg{};
  std::string err;
  int eq = -1;
  EqParams eqp{};
  BcTable bcs{};
  RefOps ops;
  int K = 0, M = 0;
  double dtscale = 0.0;
  std::vector<ElemGeo> geo_h;
  std::vector<FaceRec> faces_h;
  std::vector<double> xn, yn;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // device memory
  ElemGeo* geo_d = nullptr;
  FaceRec* faces_d = nullptr;
  int* conn_d = nullptr;
  std::vector<int> conn_h;
  // batched ensembles: instance of each element, number of instances (st_d and
  // st_h then hold one DevState per instance)
  int* einst_d = nullptr;
  int ninst = 1;
  int grid_div = 1;    // launch shape picked by the batch autotuner
  int tile_shape = 0;  // mixed stage operand chunking picked by the batch autotuner
  int fp64_fused = 0;  // float64 stage kernels: 0 three, 1 fused, 2 fused on one-wave meshes
  unsigned wait_limit = 0;  // apollo_dg_debug_set_waits
  int debug_stall = 0;
  // source plugins (apollo_dg_add_source): the table, VS = VVT V^T diag(w),
  // the cubature points, and the mixed stages' source buffer
  SrcTable src{};
  double *VS_d = nullptr, *cubr_d = nullptr, *cubs_d = nullptr, *srcv_d = nullptr;
  double *V_d = nullptr, *Dr_d = nullptr, *Ds_d = nullptr, *I_d = nullptr, *L_d = nullptr, *gz_d = nullptr,
         *gw_d = nullptr, *wmass_d = nullptr, *mass_d = nullptr;
  // W_d, W2_d: stage states, alternating so that a stage's output never
  // overlaps its input (the fused float64 stage reads neighbours' states)
  double *U_d = nullptr, *W_d = nullptr, *W2_d = nullptr, *in_d = nullptr, *out_d = nullptr;
  // mixed precision: fp32 face traces of U (TU) and of the stage states (T0, T1)
  float *TU_d = nullptr, *T0_d = nullptr, *T1_d = nullptr;
  bool tu_valid = false;
  // derivatives (float64): tangent scratch, adjoint scratch and state buffers
  double *dvol_d = nullptr, *dtrace_d = nullptr, *dflux_d = nullptr, *sbar_d = nullptr;
  double *tU_d = nullptr, *tW_d = nullptr, *A_d[3] = {nullptr, nullptr, nullptr};
  // trajectory of the last apollo_dg_forward_fixed: checkpoints every `every`
  // steps, and the stage states of one segment during apollo_dg_backward
  std::vector<double*> ckpt;
  double* seg_d = nullptr;
  int seg_steps = 0;
  int tr_snapshots = 0;  // > 0: the last forward was apollo_dg_forward_revolve with this many slots
  long long tr_forward_steps = 0;  // forward steps the last revolve backward sweep re-ran
  RevolvePlan revolve;
  bool tr_spine_valid = false;  // the slots still hold the first descent's states
  int tr_nsteps = 0, tr_every = 0;
  double tr_t0 = 0.0, tr_dt = 0.0;
  bool tr_valid = false;
  double *vol_d = nullptr, *trace_d = nullptr, *flux_d = nullptr;
  DevState* st_d = nullptr;
  DevState* st_h = nullptr;  // pinned
  bool have_state = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  MixedPlan* mixed = nullptr;
  // partitioned mesh (apollo_dg_set_mesh_partition): KG ghost slots after the
  // K local elements in the geometry and trace/flux buffers; per stage the
  // blocks of halo_src (local face blocks k*3+f) are packed into hsend and the
  // blocks of hrecv unpacked to halo_dst (ghost face blocks)
  bool partitioned = false;
  int KG = 0;
  int nbound = 0;  // boundary faces of the local mesh
  std::vector<int> peers, send_count, recv_count;
  int n_send = 0, n_recv = 0;
  int *halo_src_d = nullptr, *halo_dst_d = nullptr;
  void *hsend = nullptr, *hrecv = nullptr, *hlam = nullptr;
  size_t hsend_bytes = 0, hrecv_bytes = 0;
  // the face list holds the faces between local elements first (nface_int of
  // them), then the cut faces that touch ghost slots; a float64 stage runs the
  // first group on side_stream while the caller's exchange is in flight
  int nface_int = 0;
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_packed = nullptr, ev_interior = nullptr;
  // Euler limiter (apollo_dg_set_limiter): applied to every stage input
  bool lim_on = false;
  LimArgs lim{};
  double *lim_work_d = nullptr, *xn_d = nullptr, *yn_d = nullptr;
};

namespace apollo {
// launch and tile shapes (defined with the batch helpers below)
void handle_set_grid_div(apollo_dg* h, int div);
void handle_set_tile_shape(apollo_dg* h, int shape);
}  // namespace apollo

namespace {

apollo_status fail(apollo_dg* h, apollo_status code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

apollo_status cuda_fail(apollo_dg* h, cudaError_t e, const char* where) {
  return fail(h, e == cudaErrorMemoryAllocation ? APOLLO_ERR_ALLOC : APOLLO_ERR_CUDA,
              std::string(where) + ": " + cudaGetErrorString(e));
}

// Device allocations of the handles go through here, so that a test can make
// the n-th next one fail (apollo_dg_debug_fail_alloc; -1: never).
std::atomic<int> g_alloc_fail_in{-1};
cudaError_t dev_malloc(void** p, size_t bytes) {
  if (g_alloc_fail_in.load() >= 0 && g_alloc_fail_in.fetch_sub(1) == 0) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

#define CK(call, where)                          \
  do {                                           \
    cudaError_t e_ = (call);                     \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, where); \
  } while (0)

int fields_of(int eq) {
  switch (eq) {
    case EQ_ADVECTION: return 1;
    case EQ_EULER: return 5;
    case EQ_MAXWELL: return 8;
    case EQ_EULER2D: return 4;
    case EQ_MAXWELL_TM: return 3;
  }
  return 0;
}

template <class T>
void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

void free_mesh(apollo_dg* h) {
  for (auto& g : h->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  dfree(h->geo_d); dfree(h->faces_d); dfree(h->conn_d); dfree(h->einst_d);
  dfree(h->V_d); dfree(h->Dr_d); dfree(h->Ds_d); dfree(h->I_d); dfree(h->L_d); dfree(h->gz_d); dfree(h->gw_d);
  dfree(h->wmass_d); dfree(h->mass_d);
  dfree(h->VS_d); dfree(h->cubr_d); dfree(h->cubs_d); dfree(h->srcv_d);
  dfree(h->U_d); dfree(h->W_d); dfree(h->W2_d); dfree(h->in_d); dfree(h->out_d);
  dfree(h->TU_d); dfree(h->T0_d); dfree(h->T1_d);
  h->tu_valid = false;
  dfree(h->dvol_d); dfree(h->dtrace_d); dfree(h->dflux_d); dfree(h->sbar_d);
  dfree(h->tU_d); dfree(h->tW_d);
  for (auto& p : h->A_d) dfree(p);
  for (auto& p : h->ckpt) dfree(p);
  h->ckpt.clear();
  dfree(h->seg_d);
  h->seg_steps = 0;
  h->tr_valid = false;
  dfree(h->vol_d); dfree(h->trace_d); dfree(h->flux_d);
  if (h->mixed) { mixed_destroy(h->mixed); h->mixed = nullptr; }
  h->have_state = false;
  h->ninst = 1;
  dfree(h->halo_src_d); dfree(h->halo_dst_d);
  if (h->ev_packed) { cudaEventDestroy(h->ev_packed); h->ev_packed = nullptr; }
  if (h->ev_interior) { cudaEventDestroy(h->ev_interior); h->ev_interior = nullptr; }
  if (h->side_stream) { cudaStreamDestroy(h->side_stream); h->side_stream = nullptr; }
  h->nface_int = 0;
  h->partitioned = false;
  h->KG = 0;
  h->peers.clear(); h->send_count.clear(); h->recv_count.clear();
  h->n_send = h->n_recv = 0;
  h->hsend = h->hrecv = h->hlam = nullptr;
  h->hsend_bytes = h->hrecv_bytes = 0;
  dfree(h->lim_work_d); dfree(h->xn_d); dfree(h->yn_d);
  h->lim_on = false;
}

template <class T>
cudaError_t upload(T** dst, const T* src, size_t n) {
  cudaError_t e = dev_malloc((void**)dst, n * sizeof(T) + 16);
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
}

DgDev make_dev(const apollo_dg* h) {
  DgDev d{};
  d.K = h->K;
  d.nfaces = (int)h->faces_h.size();
  d.N = h->ops.N;
  d.geo = h->geo_d;
  d.faces = h->faces_d;
  d.conn = h->conn_d;
  d.V = h->V_d; d.Dr = h->Dr_d; d.Ds = h->Ds_d; d.I = h->I_d; d.L = h->L_d; d.gz = h->gz_d; d.gw = h->gw_d;
  d.vol = h->vol_d; d.trace = h->trace_d; d.flux = h->flux_d;
  d.st = h->st_d;
  d.einst = h->einst_d;
  d.ninst = h->ninst;
  d.grid_div = h->grid_div;
  d.tile_shape = h->tile_shape;
  d.fp64_fused = h->fp64_fused;
  d.nghost = h->KG;
  d.nbound = h->nbound;
  d.wait_limit = h->wait_limit;
  d.debug_stall = h->debug_stall;
  d.src = h->src;
  d.VS = h->VS_d;
  d.cub_r = h->cubr_d;
  d.cub_s = h->cubs_d;
  d.srcv = h->src.n > 0 ? h->srcv_d : nullptr;
  d.eqp = h->eqp;
  d.bcs = h->bcs;
  d.dtfac = 2. / 3. * h->cfg.cfl * h->dtscale;
  d.rmin = h->ops.rmin;
  return d;
}

apollo_status check_ready(apollo_dg* h) {
  if (!h) return APOLLO_ERR_ARG;
  if (h->eq < 0) return fail(h, APOLLO_ERR_STATE, "no equation set");
  if (h->K == 0) return fail(h, APOLLO_ERR_STATE, "no mesh set");
  return APOLLO_OK;
}


// the derivatives do not differentiate the limiter
apollo_status check_adjoint_flux(apollo_dg* h) {
  if (h->lim_on) return fail(h, APOLLO_ERR_CONFIG, "the derivatives do not support the limiter");
  return APOLLO_OK;
}

// the limiter into out from x (x may be out)
apollo_status enqueue_limiter(apollo_dg* h, const double* x, double* out) {
  DgDev d = make_dev(h);
  CK(launch_limiter(h->eq, d, h->lim, x, out, h->xn_d, h->yn_d, h->lim_work_d, h->stream), "limiter launch");
  return APOLLO_OK;
}

// calls that need the whole mesh on this handle (no trace exchange)
apollo_status check_whole(apollo_dg* h) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (!h->peers.empty())
    return fail(h, APOLLO_ERR_STATE, "partitioned mesh with peers: use the staged calls (apollo_dg_stage_begin/end)");
  return APOLLO_OK;
}

apollo_status read_errors(apollo_dg* h) {
  // a stage that gave up wrote no result, so whatever the later stages of the
  // step flagged on that input says nothing: the timeout is reported first
  if (h->st_h->err & ERRB_TIMEOUT) return fail(h, APOLLO_ERR_TIMEOUT, "device wait timed out");
  if (h->st_h->err & ERRB_NONPHYS) return fail(h, APOLLO_ERR_NONPHYSICAL, "negative density or pressure in the Euler flux");
  if (h->st_h->err & ERRB_NAN) return fail(h, APOLLO_ERR_NAN, "NaN in the right-hand side");
  return APOLLO_OK;
}

// One right-hand side or stage into the handle's stream.
apollo_status enqueue_stage(apollo_dg* h, const StageArgs& a, apollo_precision prec, cudaEvent_t* ev = nullptr) {
  DgDev d = make_dev(h);
  cudaError_t e;
  if (prec == APOLLO_PREC_MIXED) {
    if (!h->mixed) return fail(h, APOLLO_ERR_CONFIG, "mixed precision is not available for this equation/order");
    StageArgs am = a;
    if (am.mode == MODE_RHS) am.tr_scratch = h->T0_d;
    e = mixed_launch_rhs(h->mixed, h->eq, d, am, h->stream, ev);
  } else {
    e = launch_rhs_fp64(h->eq, d, a, h->stream, ev);
  }
  if (e != cudaSuccess) return cuda_fail(h, e, "rhs launch");
  return APOLLO_OK;
}

// Stage i of SSPRK(5,2).  Stages update W in place: the float64 kernels read
// neighbour data only in the volume/face kernels, before the LIFT kernel
// writes, and the mixed kernel reads only its own elements' state plus the
// face traces of the previous stage, which alternate between T0 and T1 (TU
// holds those of U).
StageArgs stage_args(const apollo_dg* h, int i) {
  const int s = 5;
  StageArgs a{};
  a.time_from_state = 1;
  a.reset_lambda = 1;
  double* wb[2] = {h->W_d, h->W2_d};
  if (i < s - 1) {
    a.x = i == 0 ? h->U_d : wb[(i - 1) & 1];
    a.out = wb[i & 1];
    a.mode = MODE_STAGE;
    a.frac = i / (s - 1.);
  } else {
    a.x = wb[(i - 1) & 1];
    a.u0 = h->U_d;
    a.out = h->U_d;
    a.mode = MODE_FINAL;
    a.frac = 1.0;
  }
  a.tr_in = i == 0 ? h->TU_d : (i & 1) ? h->T0_d : h->T1_d;
  a.tr_out = i == s - 1 ? h->TU_d : (i & 1) ? h->T1_d : h->T0_d;
  return a;
}

apollo_status enqueue_step(apollo_dg* h, apollo_precision prec) {
  for (int i = 0; i < 5; ++i) {
    StageArgs a = stage_args(h, i);
    if (h->lim_on) {
      // PETSc's SSP stepper hands the right-hand side its work vector, which
      // Apollo's step limits in place: stage 0 limits a copy of U (into the
      // stage buffer stage 0 does not write), later stages their input
      double* lim = i == 0 ? h->W2_d : const_cast<double*>(a.x);
      apollo_status rl = enqueue_limiter(h, a.x, lim);
      if (rl) return rl;
      a.x = lim;
      if (prec == APOLLO_PREC_MIXED && h->mixed) {
        // the mixed stage reads the face traces of its input, which the
        // previous stage wrote for the unlimited state: those of the limited one
        DgDev d = make_dev(h);
        CK(mixed_launch_traces(h->mixed, d, lim, (float*)a.tr_in, h->stream), "trace launch");
      }
    }
    apollo_status r = enqueue_stage(h, a, prec);
    if (r != APOLLO_OK) return r;
  }
  DgDev d = make_dev(h);
  cudaError_t e = launch_finalize(d, h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "finalize launch");
  return APOLLO_OK;
}

apollo_status step_graph(apollo_dg* h, apollo_precision prec, cudaGraphExec_t* out) {
  int gi = prec == APOLLO_PREC_MIXED ? 1 : 0;
  // the mixed step starts from the face traces of U; a float64 step leaves them stale
  if (prec == APOLLO_PREC_MIXED && h->mixed && !h->tu_valid) {
    DgDev d = make_dev(h);
    CK(mixed_launch_traces(h->mixed, d, h->U_d, h->TU_d, h->stream), "trace launch");
    h->tu_valid = true;
  }
  if (prec != APOLLO_PREC_MIXED) h->tu_valid = false;
  if (!h->graph[gi]) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    apollo_status r = enqueue_step(h, prec);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (r != APOLLO_OK) { if (g) cudaGraphDestroy(g); return r; }
    if (e != cudaSuccess) return cuda_fail(h, e, "end capture");
    e = cudaGraphInstantiate(&h->graph[gi], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(h, e, "graph instantiate");
  }
  *out = h->graph[gi];
  return APOLLO_OK;
}

}  // namespace

extern "C" {

apollo_status apollo_dg_create(const apollo_dg_config* cfg, apollo_dg** out) {
  if (!cfg || !out) return APOLLO_ERR_ARG;
  *out = nullptr;
  if (cfg->polynomial_order < 2 || cfg->polynomial_order > 5) return APOLLO_ERR_CONFIG;
  if (!(cfg->cfl > 0.0)) return APOLLO_ERR_CONFIG;
  apollo_dg* h = new apollo_dg();
  h->cfg = *cfg;
  if (cudaSetDevice(cfg->device) != cudaSuccess) { delete h; return APOLLO_ERR_CUDA; }
  if (!build_ref_ops(cfg->polynomial_order, h->ops)) { delete h; return APOLLO_ERR_CONFIG; }
  if (cfg->stream) {
    h->stream = (cudaStream_t)cfg->stream;
  } else {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) { delete h; return APOLLO_ERR_CUDA; }
    h->own_stream = true;
  }
  if (dev_malloc((void**)&h->st_d, sizeof(DevState)) != cudaSuccess ||
      cudaMallocHost((void**)&h->st_h, sizeof(DevState)) != cudaSuccess) {
    apollo_dg_destroy(h);
    return APOLLO_ERR_ALLOC;
  }
  std::memset(h->st_h, 0, sizeof(DevState));
  cudaMemcpy(h->st_d, h->st_h, sizeof(DevState), cudaMemcpyHostToDevice);
  *out = h;
  return APOLLO_OK;
}

apollo_status apollo_dg_set_equation(apollo_dg* h, const char* kind, const double* params, int nparams) {
  if (!h || !kind) return APOLLO_ERR_ARG;
  if (h->K) return fail(h, APOLLO_ERR_STATE, "set the equation before the mesh");
  std::string k(kind);
  int eq = -1;
  if (k == "advectionEqn") eq = EQ_ADVECTION;
  else if (k == "eulerEqn") eq = EQ_EULER;
  else if (k == "phMaxwellEqn") eq = EQ_MAXWELL;
  else if (k == "eulerEqn2d") eq = EQ_EULER2D;
  else if (k == "maxwellTM") eq = EQ_MAXWELL_TM;
  else return fail(h, APOLLO_ERR_CONFIG, "unknown equation kind " + k);
  if (nparams < 0 || nparams > 4 || (nparams > 0 && !params)) return fail(h, APOLLO_ERR_ARG, "bad parameter list");
  h->src.n = 0;  // sources name fields of the equation they were added for
  // the Euler kinds take three parameters; p[3] holds their numerical flux
  if ((eq == EQ_EULER || eq == EQ_EULER2D) && nparams > 3) return fail(h, APOLLO_ERR_ARG, "eulerEqn takes 3 parameters");
  EqParams p{};
  for (int i = 0; i < nparams; ++i) p.p[i] = params[i];
  if ((eq == EQ_EULER || eq == EQ_EULER2D) && !(p.p[0] > 1.0))
    return fail(h, APOLLO_ERR_CONFIG, "eulerEqn needs gas_gamma > 1");
  if ((eq == EQ_MAXWELL || eq == EQ_MAXWELL_TM) && !(p.p[0] > 0.0))
    return fail(h, APOLLO_ERR_CONFIG, "Maxwell needs c0 > 0");
  if (eq == EQ_MAXWELL_TM && (p.p[1] != 0.0 || p.p[2] != 0.0))
    return fail(h, APOLLO_ERR_CONFIG, "maxwellTM requires gamma = chi = 0");
  h->eq = eq;
  h->eqp = p;
  h->M = fields_of(eq);
  return APOLLO_OK;
}

apollo_status apollo_dg_add_source(apollo_dg* h, const char* kind, const int* out_range, int nout,
                                   const double* params, int nparams) {
  if (!h || !kind || !out_range || nout < 1) return APOLLO_ERR_ARG;
  if (h->eq < 0) return fail(h, APOLLO_ERR_STATE, "set the equation before its sources");
  if (h->src.n >= kMaxSrc) return fail(h, APOLLO_ERR_CONFIG, "too many sources");
  if (nparams < 0 || nparams > 9 || (nparams > 0 && !params)) return fail(h, APOLLO_ERR_ARG, "bad parameter list");
  const std::string k(kind);
  int kd = 0;
  if (k == "tranverseMagneticSrc") {
    kd = SRC_TM;
    if (nparams != 0) return fail(h, APOLLO_ERR_ARG, "tranverseMagneticSrc takes no parameters");
  } else if (k == "pointCurrentSrc") {
    kd = SRC_POINT;
    if (nparams != 9)
      return fail(h, APOLLO_ERR_ARG, "pointCurrentSrc takes xLocation, yLocation, radius, currentDensity, "
                                     "frequency, phase, charge, mass, epsilon0");
  } else {
    return fail(h, APOLLO_ERR_CONFIG, "unknown source " + k);
  }
  // both plugins write their first output only: OutRange[0] is the field, in
  // Apollo's numbering, mapped to this handle's layout
  const int a = out_range[0];
  int f = -1;
  switch (h->eq) {
    case EQ_ADVECTION: f = a == 0 ? 0 : -1; break;
    case EQ_EULER: f = a >= 0 && a < 5 ? a : -1; break;
    case EQ_MAXWELL: f = a >= 0 && a < 8 ? a : -1; break;
    case EQ_EULER2D: f = a == 0 ? 0 : a == 1 ? 1 : a == 2 ? 2 : a == 4 ? 3 : -1; break;
    case EQ_MAXWELL_TM: f = a == 2 ? 0 : a == 3 ? 1 : a == 4 ? 2 : -1; break;
  }
  if (f < 0) return fail(h, APOLLO_ERR_CONFIG, "source output field " + std::to_string(a) + " is not a field of this equation");
  const int i = h->src.n;
  h->src.kind[i] = kd;
  h->src.out[i] = f;
  for (int j = 0; j < 9; ++j) h->src.p[i][j] = j < nparams ? params[j] : 0.0;
  h->src.n = i + 1;
  if (h->K > 0 && h->mixed && !h->srcv_d) {
    const size_t nU = (size_t)h->K * h->ops.Np * h->M;
    CK(dev_malloc((void**)&h->srcv_d, nU * sizeof(double)), "source alloc");
  }
  for (auto& g : h->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return APOLLO_OK;
}

apollo_status apollo_dg_add_bc(apollo_dg* h, const char* kind, const double* params, int nparams) {
  if (!h || !kind) return APOLLO_ERR_ARG;
  if (h->bcs.n >= kMaxBc) return fail(h, APOLLO_ERR_CONFIG, "too many boundary conditions");
  if (nparams < 0 || nparams > 8 || (nparams > 0 && !params)) return fail(h, APOLLO_ERR_ARG, "bad parameter list");
  std::string k(kind);
  int b = -1;
  double bp[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int j = 0; j < nparams; ++j) bp[j] = params[j];
  const bool euler_bc = k == "eulerWallBC" || k == "eulerZeroGradientBC" || k == "eulerInflowBC" || k == "eulerDirichletBC";
  if (euler_bc && h->eq >= 0 && h->eq != EQ_EULER && h->eq != EQ_EULER2D)
    return fail(h, APOLLO_ERR_CONFIG, k + " needs an Euler equation");
  if (k == "gridFixedBC") b = BC_FIXED;
  else if (k == "isentropicVortexBC") b = BC_VORTEX;
  else if (k == "maxwellTransverseMagneticBC") b = BC_TM;
  else if (k == "phmConductingWallBC") b = BC_PEC;
  else if (k == "eulerWallBC") b = BC_EULER_WALL;
  else if (k == "eulerZeroGradientBC") b = BC_EULER_ZEROGRAD;
  else if (k == "eulerInflowBC") {
    // WxEulerInflowBC (wxeulerinflowbc.cc): Mach_number, Flow_angle (degrees),
    // gas_gamma, Pressure, density -> the constant inflow state
    if (nparams != 5) return fail(h, APOLLO_ERR_ARG, "eulerInflowBC takes Mach_number, Flow_angle, gas_gamma, Pressure, density");
    const double mach = bp[0], angle = bp[1], gamma = bp[2], pres = bp[3], rho = bp[4];
    const double pi = 3.141592653589793;
    const double sound = std::sqrt(gamma * pres / rho);
    const double u = mach * sound * std::cos(angle * pi / 180.), v = mach * sound * std::sin(angle * pi / 180.);
    const double st[5] = {rho, rho * u, rho * v, 0.0, pres / (gamma - 1) + 0.5 * rho * (u * u + v * v)};
    b = BC_EULER_STATE;
    for (int j = 0; j < 8; ++j) bp[j] = j < 5 ? st[j] : 0.0;
  } else if (k == "eulerDirichletBC") {
    // WxEulerDirichletBC (wxeulerdirichletbc.cc): density, xvelocity,
    // yvelocity, zvelocity, gas_gamma, pressure -> the constant state
    if (nparams != 6)
      return fail(h, APOLLO_ERR_ARG, "eulerDirichletBC takes density, xvelocity, yvelocity, zvelocity, gas_gamma, pressure");
    const double rho = bp[0], u = bp[1], v = bp[2], w = bp[3], gamma = bp[4], pres = bp[5];
    if (h->eq == EQ_EULER2D && w != 0.0) return fail(h, APOLLO_ERR_CONFIG, "eulerEqn2d has no z velocity");
    const double st[5] = {rho, rho * u, rho * v, rho * w, pres / (gamma - 1) + 0.5 * rho * (u * u + v * v + w * w)};
    b = BC_EULER_STATE;
    for (int j = 0; j < 8; ++j) bp[j] = j < 5 ? st[j] : 0.0;
  } else {
    return fail(h, APOLLO_ERR_CONFIG, "unknown boundary condition kind " + k);
  }
  int i = h->bcs.n++;
  h->bcs.kind[i] = b;
  for (int j = 0; j < 8; ++j) h->bcs.p[i][j] = bp[j];
  return APOLLO_OK;
}

apollo_status apollo_dg_set_numerical_flux(apollo_dg* h, const char* name) {
  if (!h || !name) return APOLLO_ERR_ARG;
  if (h->eq < 0) return fail(h, APOLLO_ERR_STATE, "set the equation first");
  const std::string n(name);
  int kind = NF_LF;
  if (h->eq == EQ_EULER || h->eq == EQ_EULER2D) {
    if (n == "HLL") kind = NF_HLL;
    else if (n == "Roe") kind = NF_ROE;
    else if (n == "Wave") kind = NF_WAVE;
    else if (n != "LF") h->err = "numerical flux " + n + " not recognised: Lax-Friedrichs used";
    h->eqp.p[3] = kind;
  } else if (h->eq == EQ_ADVECTION || h->eq == EQ_MAXWELL_TM) {
    if (n == "upwind") kind = NF_UPWIND;
    else if (n != "LF") h->err = "numerical flux " + n + " not recognised: Lax-Friedrichs used";
    h->eqp.p[3] = kind;
  }
  // captured graphs hold the equation parameters
  for (auto& g : h->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return APOLLO_OK;
}

apollo_status apollo_dg_set_launch_shape(apollo_dg* h, int grid_share, int tile_shape) {
  if (!h || grid_share < 1 || tile_shape < 0 || tile_shape > 2) return APOLLO_ERR_ARG;
  handle_set_grid_div(h, grid_share);
  handle_set_tile_shape(h, tile_shape);
  return APOLLO_OK;
}

apollo_status apollo_dg_set_fp64_kernels(apollo_dg* h, int fused) {
  if (!h || fused < 0 || fused > 2) return APOLLO_ERR_ARG;
  if (fused != h->fp64_fused) {
    h->fp64_fused = fused;
    for (auto& g : h->graph)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  }
  return APOLLO_OK;
}

apollo_status apollo_dg_averaging_weights(const apollo_dg* h, double* w) {
  if (!h || !w || h->ops.Np == 0) return APOLLO_ERR_ARG;
  for (int k = 0; k < h->ops.Np; ++k) w[k] = 0.5 * h->ops.mass_colsum[k];
  return APOLLO_OK;
}

apollo_status apollo_dg_set_limiter(apollo_dg* h, const char* kind, const double* params, int nparams) {
  apollo_status r = check_ready(h);
  if (r) return r;
  for (auto& g : h->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  if (!kind || !*kind) {
    h->lim_on = false;
    return APOLLO_OK;
  }
  const std::string k_name(kind);
  const bool ta = k_name == "tuAliabadiLimiter";
  if (!ta && k_name != "eulerLimiterHW") return fail(h, APOLLO_ERR_CONFIG, std::string("unknown limiter ") + kind);
  const bool euler = h->eq == EQ_EULER || h->eq == EQ_EULER2D;
  const bool maxwell = h->eq == EQ_MAXWELL || h->eq == EQ_MAXWELL_TM;
  if (!ta && !euler) return fail(h, APOLLO_ERR_CONFIG, "eulerLimiterHW needs an Euler equation");
  // Apollo's advection equation has no limiterTuAndAliabadi (it throws)
  if (ta && !euler && !maxwell) return fail(h, APOLLO_ERR_CONFIG, "tuAliabadiLimiter needs an Euler or Maxwell equation");
  if (h->ops.N > 4) return fail(h, APOLLO_ERR_CONFIG, "the limiters support orders up to 4");
  if (!ta && (nparams != 3 || !params))
    return fail(h, APOLLO_ERR_ARG, "eulerLimiterHW takes gas_gamma, min_pressure, min_density");
  if (ta && nparams != 0) return fail(h, APOLLO_ERR_ARG, "tuAliabadiLimiter takes the equation's parameters, none of its own");
  if (!h->peers.empty()) return fail(h, APOLLO_ERR_CONFIG, "partitioned meshes do not support the limiter");
  // Apollo's limiters hand the boundary conditions two coordinates where
  // they read (t, x, y): only conditions that read none are accepted
  for (int i = 0; i < h->bcs.n && euler; ++i) {
    const int k = h->bcs.kind[i];
    if (k != BC_FIXED && k != BC_EULER_WALL && k != BC_EULER_ZEROGRAD && k != BC_EULER_STATE)
      return fail(h, APOLLO_ERR_CONFIG, "the limiter supports wall, zero-gradient, inflow, Dirichlet and fixed boundaries");
  }
  const RefOps& o = h->ops;
  LimArgs L{};
  for (int k = 0; k < o.Np; ++k) L.ave[k] = 0.5 * o.mass_colsum[k];
  for (int i = 0; i < 3 * (o.N + 1); ++i) L.fmask[i] = o.fmask[i];
  L.kind = ta ? 1 : 0;
  // eulerLimiterHW reads its own three parameters; tuAliabadiLimiter takes the
  // Euler equation's gas_gamma, minPressure, minDensity
  L.gamma = ta ? h->eqp.p[0] : params[0];
  L.minP = ta ? h->eqp.p[1] : params[1];
  L.minD = ta ? h->eqp.p[2] : params[2];
  if (!h->lim_work_d) {
    CK(dev_malloc((void**)&h->lim_work_d, limiter_work_doubles(h->K) * sizeof(double)), "limiter alloc");
    CK(upload(&h->xn_d, h->xn.data(), h->xn.size()), "limiter coordinates");
    CK(upload(&h->yn_d, h->yn.data(), h->yn.size()), "limiter coordinates");
  }
  h->lim = L;
  h->lim_on = true;
  return APOLLO_OK;
}

}  // extern "C"

namespace {

// The handle's mesh: the whole mesh (part == nullptr) or the elements of one
// rank plus ghost slots for their remote neighbours' traces.
apollo_status set_mesh_body(apollo_dg* h, int nverts, const double* vx, const double* vy, int Kg, const int* etov,
                            const int* face_tag, const int* vert_canon, const int* part, int rank) {
  if (!h || !vx || !vy || !etov || nverts < 3 || Kg < 1) return APOLLO_ERR_ARG;
  if (h->eq < 0) return fail(h, APOLLO_ERR_STATE, "set the equation before the mesh");
  CK(cudaSetDevice(h->cfg.device), "set device");
  free_mesh(h);
  const RefOps& o = h->ops;
  const int Np = o.Np, M = h->M;
  h->K = 0;
  for (size_t i = 0; i < (size_t)Kg * 3; ++i)
    if (etov[i] < 0 || etov[i] >= nverts) return fail(h, APOLLO_ERR_MESH, "vertex index out of range");
  // smallest inscribed radius over the whole mesh, Apollo
  // CalculateNodeCoordinates2d (wxnodaldggeometry2d.cc:220-227)
  double dtscale = 1.0e6;
  for (int k = 0; k < Kg; ++k) {
    const int* v = etov + 3 * k;
    const double p1x = vx[v[0]], p1y = vy[v[0]], p2x = vx[v[1]], p2y = vy[v[1]], p3x = vx[v[2]], p3y = vy[v[2]];
    const double l1 = std::sqrt(std::pow(p1x - p2x, 2) + std::pow(p1y - p2y, 2));
    const double l2 = std::sqrt(std::pow(p2x - p3x, 2) + std::pow(p2y - p3y, 2));
    const double l3 = std::sqrt(std::pow(p3x - p1x, 2) + std::pow(p3y - p1y, 2));
    const double sp = 0.5 * (l1 + l2 + l3);
    const double area = std::sqrt(std::fabs(sp * (sp - l1) * (sp - l2) * (sp - l3)));
    dtscale = std::min(dtscale, area / sp);
  }
  h->dtscale = dtscale;
  // face map: faces sharing both (canonical) vertices pair up
  std::vector<int> partner;
  std::string perr = pair_faces(nverts, Kg, etov, face_tag, vert_canon, partner);
  if (!perr.empty()) return fail(h, APOLLO_ERR_MESH, perr);
  HaloPlan plan;
  if (part) {
    for (int k = 0; k < Kg; ++k)
      if (part[k] < 0) return fail(h, APOLLO_ERR_ARG, "negative part id");
    perr = build_halo(Kg, partner, part, rank, plan);
    if (!perr.empty()) return fail(h, APOLLO_ERR_ARG, perr);
  } else {
    plan.local.resize(Kg);
    for (int k = 0; k < Kg; ++k) plan.local[k] = k;
  }
  const int K = (int)plan.local.size(), G = (int)plan.ghost.size();
  // slot of every held element: local ones first, then the ghosts
  std::vector<int> slot(Kg, -1);
  for (int i = 0; i < K; ++i) slot[plan.local[i]] = i;
  for (int g = 0; g < G; ++g) slot[plan.ghost[g]] = K + g;
  h->geo_h.assign((size_t)K + G, ElemGeo{});
  h->xn.assign((size_t)K * Np, 0.0);
  h->yn.assign((size_t)K * Np, 0.0);
  std::vector<double> xg(Np), yg(Np);
  for (int i = 0; i < K + G; ++i) {
    const int kg = i < K ? plan.local[i] : plan.ghost[i - K];
    const int* v = etov + 3 * kg;
    const double p1x = vx[v[0]], p1y = vy[v[0]], p2x = vx[v[1]], p2y = vy[v[1]], p3x = vx[v[2]], p3y = vy[v[2]];
    double* xs = i < K ? &h->xn[(size_t)i * Np] : xg.data();
    double* ys = i < K ? &h->yn[(size_t)i * Np] : yg.data();
    for (int n = 0; n < Np; ++n) {
      const double r = o.r[n], s = o.s[n];
      xs[n] = 0.5 * (-p1x * (r + s) + p2x * (1. + r) + p3x * (1. + s));
      ys[n] = 0.5 * (-p1y * (r + s) + p2y * (1. + r) + p3y * (1. + s));
    }
    // GeometricFactors2d and Normals2d from the vertex nodes (:382-442)
    const double x1 = xs[o.fmask[0]], y1 = ys[o.fmask[0]];
    const double x2 = xs[o.fmask[o.N + 1]], y2 = ys[o.fmask[o.N + 1]];
    const double x3 = xs[o.fmask[2 * (o.N + 1)]], y3 = ys[o.fmask[2 * (o.N + 1)]];
    const double dxdr = (x2 - x1) / 2, dxds = (x3 - x1) / 2, dydr = (y2 - y1) / 2, dyds = (y3 - y1) / 2;
    const double J = -dxds * dydr + dxdr * dyds;
    if (!(J > 0)) return fail(h, APOLLO_ERR_MESH, "non-positive Jacobian in element " + std::to_string(kg));
    ElemGeo& g = h->geo_h[i];
    g.rx = dyds / J; g.sx = -dydr / J; g.ry = -dxds / J; g.sy = dxdr / J;
    g.J = J; g.invJ = 1.0 / J;
    double nr[3][2] = {{(y2 - y1), -(x2 - x1)}, {(y3 - y2), -(x3 - x2)}, {(y1 - y3), -(x1 - x3)}};
    for (int f = 0; f < 3; ++f) {
      const double sJ = std::sqrt(nr[f][0] * nr[f][0] + nr[f][1] * nr[f][1]);
      if (!(sJ > 0)) return fail(h, APOLLO_ERR_MESH, "zero edge length in element " + std::to_string(kg));
      g.nx[f] = nr[f][0] / sJ;
      g.ny[f] = nr[f][1] / sJ;
      g.sJ[f] = sJ / 2.;
    }
    g.vx[0] = p1x; g.vx[1] = p2x; g.vx[2] = p3x;
    g.vy[0] = p1y; g.vy[1] = p2y; g.vy[2] = p3y;
  }
  // face list and connectivity of the local elements.  An interior face is
  // listed once, from the side that comes first in the global mesh (the one
  // whose global face id 3k+f is lower), so a cut face is computed by both
  // ranks exactly as one handle on the whole mesh computes it.
  h->faces_h.clear();
  h->faces_h.reserve((size_t)K * 2);
  h->conn_h.assign((size_t)K * 6, -1);
  for (int i = 0; i < K; ++i) {
    const int kg = plan.local[i];
    for (int f = 0; f < 3; ++f) {
      const int tag = face_tag ? face_tag[3 * kg + f] : 0;
      const int p = partner[3 * kg + f];
      if (tag > 0 || p < 0) {
        const int t = tag > 0 ? tag : 1;
        if (t > std::max(1, h->bcs.n)) return fail(h, APOLLO_ERR_MESH, "face tag without a boundary condition");
        if (h->bcs.n == 0) return fail(h, APOLLO_ERR_MESH, "boundary face but no boundary condition added");
        h->faces_h.push_back(FaceRec{i, f, -t, -1});
        h->conn_h[6 * i + 2 * f] = -t;
        h->conn_h[6 * i + 2 * f + 1] = -1;
      } else {
        const int sp = slot[p / 3];
        if (p > 3 * kg + f) h->faces_h.push_back(FaceRec{i, f, sp, p % 3});
        else if (sp >= K) h->faces_h.push_back(FaceRec{sp, p % 3, i, f});
        h->conn_h[6 * i + 2 * f] = sp;
        h->conn_h[6 * i + 2 * f + 1] = p % 3;
      }
    }
  }
  h->nbound = 0;
  for (const FaceRec& fr : h->faces_h)
    if (fr.k2 < 0) ++h->nbound;
  // interior and boundary faces of the local elements first, the cut faces
  // (one side a ghost slot) last; each face is computed on its own, so the
  // order changes no result
  std::stable_partition(h->faces_h.begin(), h->faces_h.end(),
                        [K](const FaceRec& fr) { return fr.k1 < K && fr.k2 < K; });
  h->nface_int = 0;
  for (const FaceRec& fr : h->faces_h)
    if (fr.k1 < K && fr.k2 < K) ++h->nface_int;
  // device buffers: state-sized ones for the local elements, geometry and
  // trace/flux scratch with the ghost slots
  const size_t nU = (size_t)K * Np * M, nT = (size_t)(K + G) * o.Nf * M;
  CK(upload(&h->geo_d, h->geo_h.data(), h->geo_h.size()), "geometry upload");
  CK(upload(&h->faces_d, h->faces_h.data(), h->faces_h.size()), "face map upload");
  CK(upload(&h->conn_d, h->conn_h.data(), h->conn_h.size()), "connectivity upload");
  std::vector<double> DrW(o.DrW.a), DsW(o.DsW.a);
  CK(upload(&h->V_d, o.Vc.a.data(), o.Vc.a.size()), "op upload");
  CK(upload(&h->Dr_d, DrW.data(), DrW.size()), "op upload");
  CK(upload(&h->Ds_d, DsW.data(), DsW.size()), "op upload");
  CK(upload(&h->I_d, o.Interp.a.data(), o.Interp.a.size()), "op upload");
  CK(upload(&h->L_d, o.Lift.a.data(), o.Lift.a.size()), "op upload");
  CK(upload(&h->gz_d, o.gz.data(), o.gz.size()), "op upload");
  CK(upload(&h->gw_d, o.gw.data(), o.gw.size()), "op upload");
  CK(upload(&h->wmass_d, o.mass_colsum.data(), o.mass_colsum.size()), "op upload");
  const Mat mass = inverse(o.VVT);
  CK(upload(&h->mass_d, mass.a.data(), mass.a.size()), "op upload");
  {
    // VS = VVT V^T diag(w): the source's share of the right-hand side
    // (wxcubature2d.cc:297-325 adds VT (w J S) to the volume term, which the
    // step multiplies by VVT / J)
    std::vector<double> vs((size_t)o.Np * o.Nc, 0.0);
    for (int n = 0; n < o.Np; ++n)
      for (int c = 0; c < o.Nc; ++c) {
        double acc = 0.0;
        for (int j = 0; j < o.Np; ++j) acc += o.VVT(n, j) * o.Vc(c, j);
        vs[(size_t)n * o.Nc + c] = acc * o.cub_w[c];
      }
    CK(upload(&h->VS_d, vs.data(), vs.size()), "op upload");
    CK(upload(&h->cubr_d, o.cub_r.data(), o.cub_r.size()), "op upload");
    CK(upload(&h->cubs_d, o.cub_s.data(), o.cub_s.size()), "op upload");
  }
  CK(dev_malloc((void**)&h->U_d, nU * sizeof(double)), "state alloc");
  CK(dev_malloc((void**)&h->W_d, nU * sizeof(double)), "state alloc");
  CK(dev_malloc((void**)&h->W2_d, nU * sizeof(double)), "state alloc");
  CK(dev_malloc((void**)&h->in_d, nU * sizeof(double)), "state alloc");
  CK(dev_malloc((void**)&h->out_d, nU * sizeof(double)), "state alloc");
  CK(dev_malloc((void**)&h->vol_d, nU * sizeof(double)), "scratch alloc");
  CK(dev_malloc((void**)&h->trace_d, nT * sizeof(double)), "scratch alloc");
  CK(dev_malloc((void**)&h->flux_d, nT * sizeof(double)), "scratch alloc");
  CK(cudaMemset(h->U_d, 0, nU * sizeof(double)), "state clear");
  CK(cudaMemset(h->trace_d, 0, nT * sizeof(double)), "scratch clear");
  h->K = K;
  h->mixed = mixed_create(h->eq, o, K, h->M);
  if (h->mixed) {
    const size_t nTr = mixed_trace_floats(h->mixed, K + G);
    CK(dev_malloc((void**)&h->TU_d, nTr * sizeof(float)), "trace alloc");
    CK(dev_malloc((void**)&h->T0_d, nTr * sizeof(float)), "trace alloc");
    CK(dev_malloc((void**)&h->T1_d, nTr * sizeof(float)), "trace alloc");
    CK(cudaMemset(h->TU_d, 0, nTr * sizeof(float)), "trace clear");
    CK(cudaMemset(h->T0_d, 0, nTr * sizeof(float)), "trace clear");
    CK(cudaMemset(h->T1_d, 0, nTr * sizeof(float)), "trace clear");
    if (h->src.n > 0) CK(dev_malloc((void**)&h->srcv_d, nU * sizeof(double)), "source alloc");
  }
  // halo: face-block indices of the blocks sent (local) and received (ghost)
  h->partitioned = part != nullptr;
  h->KG = G;
  h->peers = plan.peers;
  h->send_count = plan.send_count;
  h->recv_count = plan.recv_count;
  h->n_send = (int)plan.send_face.size();
  h->n_recv = (int)plan.recv_face.size();
  if (h->n_send) {
    std::vector<int> src(h->n_send), dst(h->n_recv);
    for (int j = 0; j < h->n_send; ++j) src[j] = slot[plan.send_face[j] / 3] * 3 + plan.send_face[j] % 3;
    for (int j = 0; j < h->n_recv; ++j) dst[j] = slot[plan.recv_face[j] / 3] * 3 + plan.recv_face[j] % 3;
    CK(upload(&h->halo_src_d, src.data(), src.size()), "halo upload");
    CK(upload(&h->halo_dst_d, dst.data(), dst.size()), "halo upload");
  }
  return APOLLO_OK;
}

// A mesh that fails part way (a bad element, a failed allocation) leaves the
// handle with no mesh rather than a partial one.
apollo_status set_mesh_impl(apollo_dg* h, int nverts, const double* vx, const double* vy, int Kg, const int* etov,
                            const int* face_tag, const int* vert_canon, const int* part, int rank) {
  const apollo_status r = set_mesh_body(h, nverts, vx, vy, Kg, etov, face_tag, vert_canon, part, rank);
  if (r != APOLLO_OK && h) {
    free_mesh(h);
    h->K = 0;
    h->have_state = false;
  }
  return r;
}

}  // namespace

extern "C" {

apollo_status apollo_dg_set_mesh(apollo_dg* h, int nverts, const double* vx, const double* vy, int K,
                                 const int* etov, const int* face_tag, const int* vert_canon) {
  return set_mesh_impl(h, nverts, vx, vy, K, etov, face_tag, vert_canon, nullptr, 0);
}

apollo_status apollo_dg_set_mesh_partition(apollo_dg* h, int nverts, const double* vx, const double* vy, int K,
                                           const int* etov, const int* face_tag, const int* vert_canon,
                                           const int* part, int rank) {
  if (!part || rank < 0) return APOLLO_ERR_ARG;
  return set_mesh_impl(h, nverts, vx, vy, K, etov, face_tag, vert_canon, part, rank);
}

int apollo_dg_num_fields(const apollo_dg* h) { return h ? h->M : 0; }
int apollo_dg_num_nodes(const apollo_dg* h) { return h ? h->ops.Np : 0; }
int apollo_dg_num_elements(const apollo_dg* h) { return h ? h->K : 0; }
int apollo_dg_num_cubature(const apollo_dg* h) { return h ? h->ops.Nc : 0; }
int apollo_dg_num_gauss(const apollo_dg* h) { return h ? h->ops.Ng : 0; }

apollo_status apollo_dg_node_coords(apollo_dg* h, double* x, double* y) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (!x || !y) return APOLLO_ERR_ARG;
  std::memcpy(x, h->xn.data(), h->xn.size() * sizeof(double));
  std::memcpy(y, h->yn.data(), h->yn.size() * sizeof(double));
  return APOLLO_OK;
}

namespace {
// The resident state in or out, queued on the handle's stream; `wait` returns
// only once the copy is done.
apollo_status copy_state(apollo_dg* h, double* dst, const double* src, bool in, int where, bool wait,
                         const char* what) {
  const size_t n = (size_t)h->K * h->ops.Np * h->M * sizeof(double);
  const cudaMemcpyKind kind = where == APOLLO_DEVICE_PTR ? cudaMemcpyDeviceToDevice
                              : in                        ? cudaMemcpyHostToDevice
                                                          : cudaMemcpyDeviceToHost;
  CK(cudaMemcpyAsync(dst, src, n, kind, h->stream), what);
  if (wait) CK(cudaStreamSynchronize(h->stream), what);
  if (in) {
    h->have_state = true;
    h->tu_valid = false;
  }
  return APOLLO_OK;
}
}  // namespace

apollo_status apollo_dg_set_state(apollo_dg* h, const double* U, int where) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (!U) return APOLLO_ERR_ARG;
  return copy_state(h, h->U_d, U, true, where, true, "set state");
}

apollo_status apollo_dg_get_state(apollo_dg* h, double* U, int where) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (!U) return APOLLO_ERR_ARG;
  return copy_state(h, U, h->U_d, false, where, true, "get state");
}

apollo_status apollo_dg_set_state_async(apollo_dg* h, const double* U, int where) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (!U) return APOLLO_ERR_ARG;
  return copy_state(h, h->U_d, U, true, where, false, "set state");
}

apollo_status apollo_dg_get_state_async(apollo_dg* h, double* U, int where) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (!U) return APOLLO_ERR_ARG;
  if (!h->have_state) return fail(h, APOLLO_ERR_STATE, "no state set");
  return copy_state(h, U, h->U_d, false, where, false, "get state");
}

apollo_status apollo_dg_init_dt(apollo_dg* h, double* dt) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (!dt) return APOLLO_ERR_ARG;
  if (!h->have_state) return fail(h, APOLLO_ERR_STATE, "no state set");
  CK(cudaMemsetAsync(&h->st_d->lam_bits, 0, sizeof(unsigned long long), h->stream), "init dt");
  DgDev d = make_dev(h);
  CK(launch_init_speed(h->eq, d, h->U_d, h->stream), "init dt");
  CK(cudaMemcpyAsync(h->st_h, h->st_d, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream), "init dt");
  CK(cudaStreamSynchronize(h->stream), "init dt");
  double lam;
  std::memcpy(&lam, &h->st_h->lam_bits, sizeof(double));
  *dt = 2. / 3. * h->cfg.cfl * h->dtscale * (h->ops.rmin / lam);
  return APOLLO_OK;
}

apollo_status apollo_dg_rhs(apollo_dg* h, double t, double dt, const double* in, double* out, double* suggested_dt,
                            int where, apollo_precision prec) {
  apollo_status r = check_whole(h);
  if (r) return r;
  if (!in || !out) return APOLLO_ERR_ARG;
  if (prec == APOLLO_PREC_MIXED && where == APOLLO_DEVICE_PTR && (const double*)out == in)
    return fail(h, APOLLO_ERR_ARG, "the mixed-precision RHS needs distinct in and out buffers");
  const size_t n = (size_t)h->K * h->ops.Np * h->M * sizeof(double);
  const double* x = in;
  double* o = out;
  if (where != APOLLO_DEVICE_PTR) {
    CK(cudaMemcpyAsync(h->in_d, in, n, cudaMemcpyHostToDevice, h->stream), "rhs input copy");
    x = h->in_d;
    o = h->out_d;
  }
  CK(cudaMemsetAsync(&h->st_d->err, 0, sizeof(int), h->stream), "rhs");
  if (h->lim_on) {
    // the limited input, in the handle's input buffer (the caller's array is unchanged)
    r = enqueue_limiter(h, x, h->in_d);
    if (r) return r;
    x = h->in_d;
  }
  StageArgs a{};
  a.x = x;
  a.out = o;
  a.mode = MODE_RHS;
  a.time_from_state = 0;
  a.t_arg = t;
  a.dt_arg = dt;
  a.reset_lambda = 1;
  r = enqueue_stage(h, a, prec);
  if (r) return r;
  if (where != APOLLO_DEVICE_PTR) CK(cudaMemcpyAsync(out, h->out_d, n, cudaMemcpyDeviceToHost, h->stream), "rhs output copy");
  CK(cudaMemcpyAsync(h->st_h, h->st_d, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream), "rhs");
  CK(cudaStreamSynchronize(h->stream), "rhs");
  if (suggested_dt) {
    double lam;
    std::memcpy(&lam, &h->st_h->lam_bits, sizeof(double));
    *suggested_dt = 2. / 3. * h->cfg.cfl * h->dtscale * (h->ops.rmin / lam);
  }
  return read_errors(h);
}

apollo_status apollo_dg_step_async(apollo_dg* h, int nsteps, double t, double dt, apollo_precision prec) {
  apollo_status r = check_whole(h);
  if (r) return r;
  if (nsteps < 0) return APOLLO_ERR_ARG;
  if (!h->have_state) return fail(h, APOLLO_ERR_STATE, "no state set");
  DevState s{};
  s.t = t;
  s.dt = dt;
  s.tend = 0.0;
  s.dtfac = 2. / 3. * h->cfg.cfl * h->dtscale;
  CK(launch_put_state(h->st_d, s, h->stream), "step state");
  cudaGraphExec_t g = nullptr;
  r = step_graph(h, prec, &g);
  if (r) return r;
  for (int i = 0; i < nsteps; ++i) CK(cudaGraphLaunch(g, h->stream), "graph launch");
  return APOLLO_OK;
}

apollo_status apollo_dg_synchronize(apollo_dg* h) {
  if (!h) return APOLLO_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream), "synchronize");
  return APOLLO_OK;
}

apollo_status apollo_dg_get_time(apollo_dg* h, double* t, double* dt) {
  if (!h || !t || !dt) return APOLLO_ERR_ARG;
  CK(cudaMemcpyAsync(h->st_h, h->st_d, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream), "get time");
  CK(cudaStreamSynchronize(h->stream), "get time");
  *t = h->st_h->t;
  *dt = h->st_h->dt;
  return read_errors(h);
}

apollo_status apollo_dg_step(apollo_dg* h, int nsteps, double* t, double* dt, double tend, apollo_precision prec) {
  apollo_status r = check_whole(h);
  if (r) return r;
  if (!t || !dt || nsteps < 0) return APOLLO_ERR_ARG;
  if (tend <= 0.0) {
    r = apollo_dg_step_async(h, nsteps, *t, *dt, prec);
    if (r) return r;
    return apollo_dg_get_time(h, t, dt);
  }
  // with an end time: clip before the first step, then one step at a time
  double tt = *t, dd = *dt;
  if (std::fabs(tend - tt) < dd) dd = std::fabs(tend - tt);
  for (int i = 0; i < nsteps && tt < tend; ++i) {
    DevState s{};
    s.t = tt;
    s.dt = dd;
    s.tend = tend;
    s.dtfac = 2. / 3. * h->cfg.cfl * h->dtscale;
    CK(launch_put_state(h->st_d, s, h->stream), "step state");
    cudaGraphExec_t g = nullptr;
    r = step_graph(h, prec, &g);
    if (r) return r;
    CK(cudaGraphLaunch(g, h->stream), "graph launch");
    r = apollo_dg_get_time(h, &tt, &dd);
    if (r) return r;
  }
  *t = tt;
  *dt = dd;
  return APOLLO_OK;
}

apollo_status apollo_dg_integrals(apollo_dg* h, const double* U, int where, double* sums) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (!sums) return APOLLO_ERR_ARG;
  const double* x = h->U_d;
  if (U) {
    if (where == APOLLO_DEVICE_PTR) {
      x = U;
    } else {
      const size_t n = (size_t)h->K * h->ops.Np * h->M * sizeof(double);
      CK(cudaMemcpyAsync(h->in_d, U, n, cudaMemcpyHostToDevice, h->stream), "integrals input");
      x = h->in_d;
    }
  }
  CK(cudaMemsetAsync(h->st_d->sums, 0, sizeof(h->st_d->sums), h->stream), "integrals");
  DgDev d = make_dev(h);
  CK(launch_integrals(h->eq, d, x, h->wmass_d, h->stream), "integrals");
  CK(cudaMemcpyAsync(h->st_h, h->st_d, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream), "integrals");
  CK(cudaStreamSynchronize(h->stream), "integrals");
  for (int f = 0; f < h->M; ++f) sums[f] = h->st_h->sums[f];
  return APOLLO_OK;
}

apollo_status apollo_dg_energy(apollo_dg* h, const double* U, int where, double* sums) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (!sums) return APOLLO_ERR_ARG;
  const double* x = h->U_d;
  if (U) {
    if (where == APOLLO_DEVICE_PTR) {
      x = U;
    } else {
      const size_t n = (size_t)h->K * h->ops.Np * h->M * sizeof(double);
      CK(cudaMemcpyAsync(h->in_d, U, n, cudaMemcpyHostToDevice, h->stream), "energy input");
      x = h->in_d;
    }
  }
  CK(cudaMemsetAsync(h->st_d->sums, 0, sizeof(h->st_d->sums), h->stream), "energy");
  DgDev d = make_dev(h);
  CK(launch_energy(h->eq, d, x, h->mass_d, h->stream), "energy");
  CK(cudaMemcpyAsync(h->st_h, h->st_d, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream), "energy");
  CK(cudaStreamSynchronize(h->stream), "energy");
  for (int f = 0; f < h->M; ++f) sums[f] = h->st_h->sums[f];
  return APOLLO_OK;
}

apollo_status apollo_dg_kernel_times(apollo_dg* h, apollo_precision prec, int iters, double* ms, int* nk) {
  apollo_status r = check_whole(h);
  if (r) return r;
  if (!ms || !nk || iters < 1) return APOLLO_ERR_ARG;
  cudaEvent_t ev[4];
  for (auto& e : ev) CK(cudaEventCreate(&e), "event");
  double acc[3] = {0, 0, 0};
  StageArgs a{};
  a.x = h->U_d;
  a.out = h->out_d;
  a.mode = MODE_RHS;
  a.reset_lambda = 1;
  for (int i = 0; i < iters; ++i) {
    r = enqueue_stage(h, a, prec, ev);
    if (r) break;
    CK(cudaEventSynchronize(ev[3]), "event sync");
    for (int k = 0; k < 3; ++k) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      acc[k] += t;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (r) return r;
  for (int k = 0; k < 3; ++k) ms[k] = acc[k] / iters;
  *nk = 3;
  return APOLLO_OK;
}

}  // extern "C"

// ------------------------------------------------------ derivatives (float64) --
namespace {

apollo_status ensure_deriv_buffers(apollo_dg* h) {
  if (h->dvol_d) return APOLLO_OK;
  const size_t nU = (size_t)h->K * h->ops.Np * h->M, nT = (size_t)h->K * h->ops.Nf * h->M;
  CK(dev_malloc((void**)&h->dvol_d, nU * sizeof(double)), "derivative scratch");
  CK(dev_malloc((void**)&h->dtrace_d, nT * sizeof(double)), "derivative scratch");
  CK(dev_malloc((void**)&h->dflux_d, nT * sizeof(double)), "derivative scratch");
  CK(dev_malloc((void**)&h->sbar_d, nT * sizeof(double)), "derivative scratch");
  CK(dev_malloc((void**)&h->tU_d, nU * sizeof(double)), "derivative state");
  CK(dev_malloc((void**)&h->tW_d, nU * sizeof(double)), "derivative state");
  for (auto& p : h->A_d) CK(dev_malloc((void**)&p, nU * sizeof(double)), "adjoint state");
  return APOLLO_OK;
}

size_t state_doubles(const apollo_dg* h) { return (size_t)h->K * h->ops.Np * h->M; }

// Time of stage s (0..4) of the SSPRK(5,2) step that starts at tn.
double stage_time(int s, double tn, double dt) { return tn + dt * (s < 4 ? s / 4.0 : 1.0); }

// Stage s of a float64 step of fixed size dt: out = x + dt/4 L(x) (s < 4) or
// 4/5 x + dt/5 L(x) + 1/5 u0 (s = 4).
apollo_status fixed_stage(apollo_dg* h, int s, const double* x, const double* u0, double* out, double tn, double dt) {
  StageArgs a{};
  a.x = x;
  a.u0 = u0;
  a.out = out;
  a.mode = s < 4 ? MODE_STAGE : MODE_FINAL;
  a.time_from_state = 0;
  a.t_arg = stage_time(s, tn, dt);
  a.dt_arg = dt;
  a.reset_lambda = 0;
  DgDev d = make_dev(h);
  cudaError_t e = launch_rhs_fp64(h->eq, d, a, h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "stage launch");
  return APOLLO_OK;
}

// One fixed step in place on u (stages through W and W2 alternately).
apollo_status fixed_step(apollo_dg* h, double* u, double tn, double dt) {
  double* wb[2] = {h->W_d, h->W2_d};
  for (int s = 0; s < 5; ++s) {
    apollo_status r = fixed_stage(h, s, s == 0 ? u : wb[(s - 1) & 1], u, s < 4 ? wb[s & 1] : u, tn, dt);
    if (r) return r;
  }
  return APOLLO_OK;
}

// Tangent of stage s at the state x along dx (and du0 on the last stage).
apollo_status tangent_stage(apollo_dg* h, int s, int mode, const double* x, const double* dx, const double* du0,
                            double* dout, double tn, double dt) {
  TanArgs a{};
  a.x = x;
  a.dx = dx;
  a.du0 = du0;
  a.dout = dout;
  a.dvol = h->dvol_d;
  a.dtrace = h->dtrace_d;
  a.dflux = h->dflux_d;
  a.mode = mode;
  a.t = mode == MODE_RHS ? tn : stage_time(s, tn, dt);
  a.dt = dt;
  DgDev d = make_dev(h);
  cudaError_t e = launch_tangent_stage(h->eq, d, a, h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "tangent launch");
  return APOLLO_OK;
}

// out = alpha wbar + beta L'(x)^T wbar + gamma z at time t.
apollo_status adjoint_stage(apollo_dg* h, const double* x, const double* wbar, const double* z, double* out,
                            double alpha, double beta, double gamma, double t) {
  AdjArgs a{};
  a.x = x;
  a.wbar = wbar;
  a.z = z;
  a.out = out;
  a.sbar = h->sbar_d;
  a.alpha = alpha;
  a.beta = beta;
  a.gamma = gamma;
  a.t = t;
  DgDev d = make_dev(h);
  cudaError_t e = launch_adjoint_stage(h->eq, d, a, h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "adjoint launch");
  return APOLLO_OK;
}

apollo_status copy_in(apollo_dg* h, double* dst, const double* src, int where) {
  const size_t n = state_doubles(h) * sizeof(double);
  CK(cudaMemcpyAsync(dst, src, n, where == APOLLO_DEVICE_PTR ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     h->stream), "copy in");
  return APOLLO_OK;
}

apollo_status copy_out(apollo_dg* h, double* dst, const double* src, int where) {
  const size_t n = state_doubles(h) * sizeof(double);
  CK(cudaMemcpyAsync(dst, src, n, where == APOLLO_DEVICE_PTR ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     h->stream), "copy out");
  return APOLLO_OK;
}

apollo_status finish(apollo_dg* h) {
  CK(cudaMemcpyAsync(h->st_h, h->st_d, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream), "state read");
  CK(cudaStreamSynchronize(h->stream), "synchronize");
  return read_errors(h);
}

apollo_status clear_errors(apollo_dg* h) {
  CK(cudaMemsetAsync(&h->st_d->err, 0, sizeof(int), h->stream), "clear errors");
  return APOLLO_OK;
}

}  // namespace

namespace apollo {

// Read-only view of a handle's discretisation for the no-allocation entry
// point (dg_noalloc.cu); the scratch pointers are left for the caller to set.
const char* handle_device_view(const apollo_dg* h, DgDev* d, int* eq, int* device, size_t* nU, size_t* nT) {
  if (!h) return "null handle";
  if (h->eq < 0) return "no equation set";
  if (h->K == 0) return "no mesh set";
  if (!h->peers.empty()) return "partitioned mesh with peers: use the staged calls (apollo_dg_stage_begin/end)";
  *d = make_dev(h);
  *eq = h->eq;
  *device = h->cfg.device;
  *nU = (size_t)h->K * h->ops.Np * h->M;
  *nT = (size_t)h->K * h->ops.Nf * h->M;
  return nullptr;
}

void handle_set_error(apollo_dg* h, const char* msg) {
  if (h) h->err = msg;
}

bool handle_has_limiter(const apollo_dg* h) { return h && h->lim_on; }

// ---- batched ensembles (dg_batch.cpp): one handle holds several independent
// meshes of one order, element ranges by instance
apollo_status handle_set_instances(apollo_dg* h, int ninst, const int* einst) {
  if (!h || h->K == 0 || ninst < 1) return APOLLO_ERR_ARG;
  DevState* st_d = nullptr;
  DevState* st_h = nullptr;
  CK(dev_malloc((void**)&st_d, (size_t)ninst * sizeof(DevState)), "instance states");
  if (cudaMallocHost((void**)&st_h, (size_t)ninst * sizeof(DevState)) != cudaSuccess) {
    cudaFree(st_d);
    return fail(h, APOLLO_ERR_ALLOC, "instance states");
  }
  std::memset(st_h, 0, (size_t)ninst * sizeof(DevState));
  CK(cudaMemcpy(st_d, st_h, (size_t)ninst * sizeof(DevState), cudaMemcpyHostToDevice), "instance states");
  dfree(h->st_d);
  if (h->st_h) cudaFreeHost(h->st_h);
  h->st_d = st_d;
  h->st_h = st_h;
  dfree(h->einst_d);
  CK(upload(&h->einst_d, einst, (size_t)h->K), "instance map");
  h->ninst = ninst;
  for (auto& g : h->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return APOLLO_OK;
}

cudaStream_t handle_stream(const apollo_dg* h) { return h->stream; }
DevState* handle_states_host(apollo_dg* h) { return h->st_h; }

// host states <-> device states (all instances), on the handle's stream
apollo_status handle_push_states(apollo_dg* h) {
  CK(cudaMemcpyAsync(h->st_d, h->st_h, (size_t)h->ninst * sizeof(DevState), cudaMemcpyHostToDevice, h->stream),
     "states");
  return APOLLO_OK;
}
apollo_status handle_pull_states(apollo_dg* h) {
  CK(cudaMemcpyAsync(h->st_h, h->st_d, (size_t)h->ninst * sizeof(DevState), cudaMemcpyDeviceToHost, h->stream),
     "states");
  return APOLLO_OK;
}

// per-instance wave speed of the resident state (into st_d[i].lam_bits)
apollo_status handle_init_speed(apollo_dg* h) {
  DgDev d = make_dev(h);
  CK(launch_reset_lambda(d, h->stream), "init speed");
  CK(launch_init_speed(h->eq, d, h->U_d, h->stream), "init speed");
  return APOLLO_OK;
}

double handle_rmin(const apollo_dg* h) { return h->ops.rmin; }
double handle_cfl(const apollo_dg* h) { return h->cfg.cfl; }
size_t handle_state_doubles(const apollo_dg* h) { return (size_t)h->K * h->ops.Np * h->M; }
double* handle_state_device(apollo_dg* h) { return h->U_d; }
void handle_mark_state(apollo_dg* h) {
  h->have_state = true;
  h->tu_valid = false;
}

// one step (5 stages + finalize) of every instance into the handle's stream,
// as a captured graph; the mixed form first rebuilds the traces of U if stale
apollo_status handle_enqueue_step(apollo_dg* h, apollo_precision prec) {
  cudaGraphExec_t g = nullptr;
  apollo_status r = step_graph(h, prec, &g);
  if (r) return r;
  CK(cudaGraphLaunch(g, h->stream), "graph launch");
  return APOLLO_OK;
}
apollo_status handle_enqueue_step_raw(apollo_dg* h, apollo_precision prec) { return enqueue_step(h, prec); }
apollo_status handle_prepare_step(apollo_dg* h, apollo_precision prec) {
  if (prec == APOLLO_PREC_MIXED && h->mixed && !h->tu_valid) {
    DgDev d = make_dev(h);
    CK(mixed_launch_traces(h->mixed, d, h->U_d, h->TU_d, h->stream), "trace launch");
    h->tu_valid = true;
  }
  if (prec != APOLLO_PREC_MIXED) h->tu_valid = false;
  if (prec == APOLLO_PREC_MIXED && !h->mixed)
    return fail(h, APOLLO_ERR_CONFIG, "mixed precision is not available for this equation/order");
  return APOLLO_OK;
}
apollo_status handle_read_errors(apollo_dg* h) { return read_errors(h); }
void handle_set_tile_shape(apollo_dg* h, int shape) {
  shape = (shape >= 0 && shape <= 2) ? shape : 0;
  if (shape != h->tile_shape) {
    h->tile_shape = shape;
    for (auto& g : h->graph)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  }
}
void handle_set_grid_div(apollo_dg* h, int div) {
  if (div < 1) div = 1;
  if (div != h->grid_div) {
    h->grid_div = div;
    for (auto& g : h->graph)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  }
}

}  // namespace apollo

extern "C" {

void apollo_dg_debug_fail_alloc(int n) { g_alloc_fail_in.store(n < 0 ? -1 : n); }

apollo_status apollo_dg_debug_set_waits(apollo_dg* h, unsigned polls, int stall_first_wait) {
  if (!h) return APOLLO_ERR_ARG;
  h->wait_limit = polls;
  h->debug_stall = stall_first_wait ? 1 : 0;
  // the step graphs captured the old values
  for (auto& g : h->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return APOLLO_OK;
}

const char* apollo_dg_last_error(const apollo_dg* h) { return h ? h->err.c_str() : "null handle"; }

}  // extern "C"

namespace {

// exactly n checkpoint states (extra ones of an earlier schedule are freed, so
// the derivative memory reported is the current schedule's)
apollo_status size_checkpoints(apollo_dg* h, int n) {
  const size_t nU = state_doubles(h);
  while ((int)h->ckpt.size() > n) {
    dfree(h->ckpt.back());
    h->ckpt.pop_back();
  }
  while ((int)h->ckpt.size() < n) {
    double* p = nullptr;
    CK(dev_malloc((void**)&p, nU * sizeof(double)), "checkpoint alloc");
    h->ckpt.push_back(p);
  }
  return APOLLO_OK;
}

// stage states of `steps` steps (5 each) for the backward sweep
apollo_status size_segment(apollo_dg* h, int steps) {
  if (h->seg_steps == steps) return APOLLO_OK;
  dfree(h->seg_d);
  h->seg_steps = 0;
  const size_t nU = state_doubles(h);
  CK(dev_malloc((void**)&h->seg_d, (size_t)5 * steps * nU * sizeof(double)), "segment alloc");
  h->seg_steps = steps;
  return APOLLO_OK;
}

// the five stage states of step n (time tn) from its input state in S0; the
// stage outputs go to S1..S4 (each stage of the step reads only the previous)
apollo_status record_step(apollo_dg* h, double* const S[5], double tn, double dt) {
  for (int s = 0; s < 4; ++s) {
    apollo_status r = fixed_stage(h, s, S[s], nullptr, S[s + 1], tn, dt);
    if (r) return r;
  }
  return APOLLO_OK;
}

// the adjoint of one step from its recorded stage states: A0 holds the
// adjoint of the step's result on entry and of its input on return
apollo_status reverse_step(apollo_dg* h, double* const S[5], double tn, double dt) {
  const double c = dt / 4.0, c_al = 4.0 / 5.0, c_be = dt / 5.0, c_ga = 1.0 / 5.0;
  double *A0 = h->A_d[0], *A1 = h->A_d[1], *A2 = h->A_d[2];
  apollo_status r = adjoint_stage(h, S[4], A0, nullptr, A1, c_al, c_be, 0.0, stage_time(4, tn, dt));
  if (!r) r = adjoint_stage(h, S[3], A1, nullptr, A2, 1.0, c, 0.0, stage_time(3, tn, dt));
  if (!r) r = adjoint_stage(h, S[2], A2, nullptr, A1, 1.0, c, 0.0, stage_time(2, tn, dt));
  if (!r) r = adjoint_stage(h, S[1], A1, nullptr, A2, 1.0, c, 0.0, stage_time(1, tn, dt));
  if (!r) r = adjoint_stage(h, S[0], A2, A0, A0, 1.0, c, c_ga, stage_time(0, tn, dt));
  return r;
}

// The device executor of the binomial reversal: slots are h->ckpt, the work
// buffer is the tangent's state buffer (free during a backward sweep), and a
// step is recorded into the five stage states of the segment buffer.
struct RevolveDevice {
  apollo_dg* h;
  double t0, dt;
  double* S[5];
  double* work;
  long long forward_steps = 0;
  double* buf(int slot) { return slot < 0 ? work : h->ckpt[slot]; }
  int copy(int dst, int src) {
    const size_t nU = state_doubles(h);
    CK(cudaMemcpyAsync(buf(dst), buf(src), nU * sizeof(double), cudaMemcpyDeviceToDevice, h->stream), "snapshot");
    return APOLLO_OK;
  }
  int advance(int slot, int from, int count) {
    for (int n = 0; n < count; ++n) {
      apollo_status r = fixed_step(h, buf(slot), t0 + (from + n) * dt, dt);
      if (r) return r;
      ++forward_steps;
    }
    return APOLLO_OK;
  }
  int leaf(int j, int slot) {
    const size_t nU = state_doubles(h);
    CK(cudaMemcpyAsync(S[0], buf(slot), nU * sizeof(double), cudaMemcpyDeviceToDevice, h->stream), "restore");
    apollo_status r = record_step(h, S, t0 + j * dt, dt);
    if (r) return r;
    ++forward_steps;
    return reverse_step(h, S, t0 + j * dt, dt);
  }
};

// The host executor: follows the same schedule, checks that every slot holds
// the step it is used for and that the steps are reversed last to first.
struct RevolveCount {
  std::vector<int> pos;
  int work = -1, next;
  long long forward_steps = 0;
  bool ok = true;
  int& at(int slot) { return slot < 0 ? work : pos[slot]; }
  int copy(int dst, int src) {
    at(dst) = at(src);
    return 0;
  }
  int advance(int slot, int from, int count) {
    if (at(slot) != from) ok = false;
    at(slot) += count;
    forward_steps += count;
    return 0;
  }
  int leaf(int j, int slot) {
    if (at(slot) != j || j != next) ok = false;
    --next;
    ++forward_steps;
    return 0;
  }
};

}  // namespace

extern "C" {

apollo_status apollo_dg_forward_revolve(apollo_dg* h, int nsteps, double t0, double dt, int snapshots) {
  apollo_status r = check_whole(h);
  if (r) return r;
  if (h->lim_on) return fail(h, APOLLO_ERR_CONFIG, "the derivatives do not support the limiter");
  if (nsteps < 1 || snapshots < 1 || !(dt > 0.0)) return fail(h, APOLLO_ERR_ARG, "nsteps, snapshots >= 1, dt > 0");
  if (!h->have_state) return fail(h, APOLLO_ERR_STATE, "no state set");
  // a slot per step already stores every state the sweep needs
  if (snapshots > nsteps) snapshots = nsteps;
  r = ensure_deriv_buffers(h);
  if (!r) r = size_checkpoints(h, snapshots);
  if (!r) r = size_segment(h, 1);
  if (r) return r;
  const size_t nU = state_doubles(h);
  h->tr_valid = false;
  h->tu_valid = false;
  r = clear_errors(h);
  if (r) return r;
  h->revolve.build(nsteps, snapshots);
  const std::vector<int> spine = h->revolve.spine();
  size_t next = 0;
  for (int n = 0; n < nsteps; ++n) {
    if (next < spine.size() && spine[next] == n) {
      CK(cudaMemcpyAsync(h->ckpt[next], h->U_d, nU * sizeof(double), cudaMemcpyDeviceToDevice, h->stream),
         "checkpoint");
      ++next;
    }
    r = fixed_step(h, h->U_d, t0 + n * dt, dt);
    if (r) return r;
  }
  r = finish(h);
  if (r) return r;
  h->tr_nsteps = nsteps;
  h->tr_every = 0;
  h->tr_snapshots = snapshots;
  h->tr_spine_valid = true;
  h->tr_t0 = t0;
  h->tr_dt = dt;
  h->tr_valid = true;
  return APOLLO_OK;
}

apollo_status apollo_dg_forward_fixed(apollo_dg* h, int nsteps, double t0, double dt, int checkpoint_every) {
  apollo_status r = check_whole(h);
  if (r) return r;
  if (h->lim_on) return fail(h, APOLLO_ERR_CONFIG, "the derivatives do not support the limiter");
  if (nsteps < 1 || checkpoint_every < 1 || !(dt > 0.0)) return fail(h, APOLLO_ERR_ARG, "nsteps, checkpoint_every >= 1, dt > 0");
  if (!h->have_state) return fail(h, APOLLO_ERR_STATE, "no state set");
  r = ensure_deriv_buffers(h);
  if (r) return r;
  const size_t nU = state_doubles(h);
  const int nck = (nsteps + checkpoint_every - 1) / checkpoint_every;
  r = size_checkpoints(h, nck);
  if (!r) r = size_segment(h, checkpoint_every);
  if (r) return r;
  h->tr_valid = false;
  h->tu_valid = false;
  r = clear_errors(h);
  if (r) return r;
  for (int n = 0; n < nsteps; ++n) {
    if (n % checkpoint_every == 0)
      CK(cudaMemcpyAsync(h->ckpt[n / checkpoint_every], h->U_d, nU * sizeof(double), cudaMemcpyDeviceToDevice,
                         h->stream), "checkpoint");
    r = fixed_step(h, h->U_d, t0 + n * dt, dt);
    if (r) return r;
  }
  r = finish(h);
  if (r) return r;
  h->tr_nsteps = nsteps;
  h->tr_every = checkpoint_every;
  h->tr_snapshots = 0;
  h->tr_t0 = t0;
  h->tr_dt = dt;
  h->tr_valid = true;
  return APOLLO_OK;
}

apollo_status apollo_dg_backward(apollo_dg* h, const double* ubar_T, double* ubar_0, int where) {
  apollo_status r = check_whole(h);
  if (r) return r;
  if ((r = check_adjoint_flux(h))) return r;
  if (!ubar_T || !ubar_0) return APOLLO_ERR_ARG;
  if (!h->tr_valid) return fail(h, APOLLO_ERR_STATE, "no trajectory: call apollo_dg_forward_fixed first");
  const size_t nU = state_doubles(h);
  if (h->tr_snapshots > 0) {
    // binomial schedule from the spine the forward pass stored
    RevolveDevice dev{h, h->tr_t0, h->tr_dt, {}, h->tU_d};
    for (int s = 0; s < 5; ++s) dev.S[s] = h->seg_d + (size_t)s * nU;
    RevolveRun<RevolveDevice> rv{h->revolve, dev};
    r = clear_errors(h);
    if (!r) r = copy_in(h, h->A_d[0], ubar_T, where);
    if (!r && !h->tr_spine_valid) {
      // an earlier sweep reused the slots of the first descent: run it again
      const std::vector<int> p = h->revolve.spine();
      for (size_t k = 1; k < p.size() && !r; ++k) {
        r = (apollo_status)dev.copy((int)k, (int)k - 1);
        if (!r) r = (apollo_status)dev.advance((int)k, p[k - 1], p[k] - p[k - 1]);
      }
    }
    if (!r) {
      h->tr_spine_valid = false;
      r = (apollo_status)rv.run();
    }
    if (!r) r = copy_out(h, ubar_0, h->A_d[0], where);
    if (r) return r;
    h->tr_forward_steps = dev.forward_steps;
    return finish(h);
  }
  const int C = h->tr_every, nsteps = h->tr_nsteps, nseg = (nsteps + C - 1) / C;
  const double dt = h->tr_dt, c = dt / 4.0, c_al = 4.0 / 5.0, c_be = dt / 5.0, c_ga = 1.0 / 5.0;
  if (h->seg_steps < C) {
    r = size_segment(h, C);
    if (r) return r;
  }
  auto S = [&](int j, int s) { return h->seg_d + ((size_t)j * 5 + s) * nU; };
  double *A0 = h->A_d[0], *A1 = h->A_d[1], *A2 = h->A_d[2];
  r = clear_errors(h);
  if (r) return r;
  r = copy_in(h, A0, ubar_T, where);
  if (r) return r;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int n0 = seg * C, ns = std::min(nsteps, n0 + C) - n0;
    // re-run the segment from its checkpoint, keeping every stage state
    CK(cudaMemcpyAsync(S(0, 0), h->ckpt[seg], nU * sizeof(double), cudaMemcpyDeviceToDevice, h->stream), "restore");
    for (int j = 0; j < ns; ++j) {
      const double tn = h->tr_t0 + (n0 + j) * dt;
      for (int s = 0; s < 4; ++s) {
        r = fixed_stage(h, s, S(j, s), nullptr, S(j, s + 1), tn, dt);
        if (r) return r;
      }
      if (j + 1 < ns) {
        r = fixed_stage(h, 4, S(j, 4), S(j, 0), S(j + 1, 0), tn, dt);
        if (r) return r;
      }
    }
    // reverse through the segment's steps: A0 holds the adjoint of the step's result
    for (int j = ns - 1; j >= 0; --j) {
      const double tn = h->tr_t0 + (n0 + j) * dt;
      r = adjoint_stage(h, S(j, 4), A0, nullptr, A1, c_al, c_be, 0.0, stage_time(4, tn, dt));
      if (!r) r = adjoint_stage(h, S(j, 3), A1, nullptr, A2, 1.0, c, 0.0, stage_time(3, tn, dt));
      if (!r) r = adjoint_stage(h, S(j, 2), A2, nullptr, A1, 1.0, c, 0.0, stage_time(2, tn, dt));
      if (!r) r = adjoint_stage(h, S(j, 1), A1, nullptr, A2, 1.0, c, 0.0, stage_time(1, tn, dt));
      if (!r) r = adjoint_stage(h, S(j, 0), A2, A0, A0, 1.0, c, c_ga, stage_time(0, tn, dt));
      if (r) return r;
    }
  }
  r = copy_out(h, ubar_0, A0, where);
  if (r) return r;
  return finish(h);
}

apollo_status apollo_dg_tangent(apollo_dg* h, int nsteps, double t0, double dt, const double* du0, double* duT,
                                int where) {
  apollo_status r = check_whole(h);
  if (r) return r;
  if (h->lim_on) return fail(h, APOLLO_ERR_CONFIG, "the derivatives do not support the limiter");
  if (nsteps < 0 || !(dt > 0.0) || !du0 || !duT) return APOLLO_ERR_ARG;
  if (!h->have_state) return fail(h, APOLLO_ERR_STATE, "no state set");
  r = ensure_deriv_buffers(h);
  if (r) return r;
  h->tu_valid = false;
  r = clear_errors(h);
  if (r) return r;
  r = copy_in(h, h->tU_d, du0, where);
  if (r) return r;
  for (int n = 0; n < nsteps; ++n) {
    const double tn = t0 + n * dt;
    for (int s = 0; s < 5; ++s) {
      // the tangent stage reads the stage's input state before the value stage replaces it
      double* wb[2] = {h->W_d, h->W2_d};
      const double* x = s == 0 ? h->U_d : wb[(s - 1) & 1];
      const double* dx = s == 0 ? h->tU_d : h->tW_d;
      double* dout = s < 4 ? h->tW_d : h->tU_d;
      r = tangent_stage(h, s, s < 4 ? MODE_STAGE : MODE_FINAL, x, dx, s < 4 ? nullptr : h->tU_d, dout, tn, dt);
      if (!r) r = fixed_stage(h, s, x, h->U_d, s < 4 ? wb[s & 1] : h->U_d, tn, dt);
      if (r) return r;
    }
  }
  r = copy_out(h, duT, h->tU_d, where);
  if (r) return r;
  return finish(h);
}

apollo_status apollo_dg_rhs_jvp(apollo_dg* h, double t, const double* x, const double* v, double* out, int where) {
  apollo_status r = check_whole(h);
  if (r) return r;
  if (h->lim_on) return fail(h, APOLLO_ERR_CONFIG, "the derivatives do not support the limiter");
  if (!x || !v || !out) return APOLLO_ERR_ARG;
  r = ensure_deriv_buffers(h);
  if (r) return r;
  r = clear_errors(h);
  if (r) return r;
  const double *xd = x, *vd = v;
  double* od = out;
  if (where != APOLLO_DEVICE_PTR) {
    r = copy_in(h, h->in_d, x, where);
    if (!r) r = copy_in(h, h->tU_d, v, where);
    if (r) return r;
    xd = h->in_d;
    vd = h->tU_d;
    od = h->out_d;
  }
  r = tangent_stage(h, 0, MODE_RHS, xd, vd, nullptr, od, t, 0.0);
  if (r) return r;
  if (where != APOLLO_DEVICE_PTR) {
    r = copy_out(h, out, h->out_d, where);
    if (r) return r;
  }
  return finish(h);
}

apollo_status apollo_dg_rhs_vjp(apollo_dg* h, double t, const double* x, const double* w, double* out, int where) {
  apollo_status r = check_whole(h);
  if (r) return r;
  if ((r = check_adjoint_flux(h))) return r;
  if (!x || !w || !out) return APOLLO_ERR_ARG;
  if (where == APOLLO_DEVICE_PTR && (out == x || out == w))
    return fail(h, APOLLO_ERR_ARG, "the adjoint needs an output distinct from x and w");
  r = ensure_deriv_buffers(h);
  if (r) return r;
  r = clear_errors(h);
  if (r) return r;
  const double *xd = x, *wd = w;
  double* od = out;
  if (where != APOLLO_DEVICE_PTR) {
    r = copy_in(h, h->in_d, x, where);
    if (!r) r = copy_in(h, h->A_d[0], w, where);
    if (r) return r;
    xd = h->in_d;
    wd = h->A_d[0];
    od = h->out_d;
  }
  r = adjoint_stage(h, xd, wd, nullptr, od, 0.0, 1.0, 0.0, t);
  if (r) return r;
  if (where != APOLLO_DEVICE_PTR) {
    r = copy_out(h, out, h->out_d, where);
    if (r) return r;
  }
  return finish(h);
}

apollo_status apollo_dg_revolve_schedule(int nsteps, int snapshots, long long* recomputed_steps, int* spine_states) {
  if (nsteps < 1 || snapshots < 1 || !recomputed_steps) return APOLLO_ERR_ARG;
  if (snapshots > nsteps) snapshots = nsteps;
  RevolvePlan plan;
  plan.build(nsteps, snapshots);
  const std::vector<int> spine = plan.spine();
  RevolveCount cnt;
  cnt.pos.assign(snapshots, -1);
  for (size_t k = 0; k < spine.size(); ++k) cnt.pos[k] = spine[k];
  cnt.next = nsteps - 1;
  RevolveRun<RevolveCount> rv{plan, cnt};
  rv.run();
  if (!cnt.ok || cnt.next != -1) return APOLLO_ERR_STATE;
  *recomputed_steps = cnt.forward_steps;
  if (spine_states) *spine_states = (int)spine.size();
  return APOLLO_OK;
}

apollo_status apollo_dg_adjoint_stats(const apollo_dg* h, long long* recomputed_steps) {
  if (!h || !recomputed_steps) return APOLLO_ERR_ARG;
  *recomputed_steps = h->tr_snapshots > 0 ? h->tr_forward_steps : (long long)h->tr_nsteps;
  return APOLLO_OK;
}

apollo_status apollo_dg_adjoint_memory(const apollo_dg* h, size_t* bytes) {
  if (!h || !bytes) return APOLLO_ERR_ARG;
  const size_t nU = (size_t)h->K * h->ops.Np * h->M, nT = (size_t)h->K * h->ops.Nf * h->M;
  size_t b = 0;
  if (h->dvol_d) b += (nU * 6 + nT * 3) * sizeof(double);
  b += h->ckpt.size() * nU * sizeof(double);
  b += (size_t)5 * h->seg_steps * nU * sizeof(double);
  *bytes = b;
  return APOLLO_OK;
}

apollo_status apollo_dg_destroy(apollo_dg* h) {
  if (!h) return APOLLO_ERR_ARG;
  cudaSetDevice(h->cfg.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_mesh(h);
  dfree(h->st_d);
  if (h->st_h) cudaFreeHost(h->st_h);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return APOLLO_OK;
}


// ---- partitioned meshes: halo info, buffers and staged stepping

apollo_status apollo_dg_halo_info(const apollo_dg* h, apollo_precision prec, int* n_peers, int* peers,
                                  int* send_count, int* recv_count, int* block_bytes) {
  if (!h || h->K == 0) return APOLLO_ERR_ARG;
  if (n_peers) *n_peers = (int)h->peers.size();
  for (size_t i = 0; i < h->peers.size(); ++i) {
    if (peers) peers[i] = h->peers[i];
    if (send_count) send_count[i] = h->send_count[i];
    if (recv_count) recv_count[i] = h->recv_count[i];
  }
  if (block_bytes) {
    if (prec == APOLLO_PREC_MIXED) {
      if (!h->mixed) return APOLLO_ERR_CONFIG;
      *block_bytes = (int)(mixed_trace_floats(h->mixed, 1) / 3 * sizeof(float));
    } else {
      *block_bytes = h->ops.Ng * h->M * (int)sizeof(double);
    }
  }
  return APOLLO_OK;
}

apollo_status apollo_dg_halo_bind(apollo_dg* h, void* send, size_t send_bytes, void* recv, size_t recv_bytes,
                                  void* lam) {
  apollo_status r = check_ready(h);
  if (r) return r;
  const size_t blk = (size_t)h->ops.Ng * h->M * sizeof(double);  // the larger (float64) block
  if ((h->n_send && (!send || send_bytes < blk * h->n_send)) || (h->n_recv && (!recv || recv_bytes < blk * h->n_recv)))
    return fail(h, APOLLO_ERR_ARG, "halo buffers too small");
  if (((uintptr_t)send | (uintptr_t)recv | (uintptr_t)lam) % 16)
    return fail(h, APOLLO_ERR_ARG, "halo buffers must be 16-byte aligned");
  h->hsend = send;
  h->hsend_bytes = send_bytes;
  h->hrecv = recv;
  h->hrecv_bytes = recv_bytes;
  h->hlam = lam;
  return APOLLO_OK;
}

apollo_status apollo_dg_dist_start(apollo_dg* h, double t, double dt, apollo_precision prec) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (!h->have_state) return fail(h, APOLLO_ERR_STATE, "no state set");
  if (prec == APOLLO_PREC_MIXED && !h->mixed)
    return fail(h, APOLLO_ERR_CONFIG, "mixed precision is not available for this equation/order");
  if (!h->peers.empty() && (!h->hsend || !h->hrecv || !h->hlam))
    return fail(h, APOLLO_ERR_STATE, "bind the halo buffers first (apollo_dg_halo_bind)");
  DevState s{};
  s.t = t;
  s.dt = dt;
  s.dtfac = 2. / 3. * h->cfg.cfl * h->dtscale;
  CK(launch_put_state(h->st_d, s, h->stream), "step state");
  return handle_prepare_step(h, prec);
}

apollo_status apollo_dg_stage_begin(apollo_dg* h, int stage, apollo_precision prec) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (h->lim_on) return fail(h, APOLLO_ERR_CONFIG, "partitioned meshes do not support the limiter");
  if (stage < 0 || stage > 4) return APOLLO_ERR_ARG;
  if (prec == APOLLO_PREC_MIXED && !h->mixed) return fail(h, APOLLO_ERR_CONFIG, "mixed precision not available");
  StageArgs a = stage_args(h, stage);
  DgDev d = make_dev(h);
  if (prec == APOLLO_PREC_MIXED) {
    // the stage input's traces were written by the previous stage (or the
    // trace kernel for U)
    const int blk = (int)(mixed_trace_floats(h->mixed, 1) / 3 * sizeof(float));
    CK(launch_halo_blocks(a.tr_in, h->hsend, h->halo_src_d, h->n_send, blk, false, h->stream), "halo pack");
  } else {
    a.phase = PHASE_VOLUME;
    CK(launch_rhs_fp64(h->eq, d, a, h->stream), "volume launch");
    const int blk = h->ops.Ng * h->M * (int)sizeof(double);
    CK(launch_halo_blocks(h->trace_d, h->hsend, h->halo_src_d, h->n_send, blk, false, h->stream), "halo pack");
    if (!h->peers.empty() && h->nface_int > 0) {
      // the faces between local elements need no remote trace: they run on
      // the side stream while the caller's exchange (enqueued on the handle's
      // stream after this call) is in flight; apollo_dg_stage_end joins them
      if (!h->side_stream) {
        CK(cudaStreamCreateWithFlags(&h->side_stream, cudaStreamNonBlocking), "side stream");
        CK(cudaEventCreateWithFlags(&h->ev_packed, cudaEventDisableTiming), "stage event");
        CK(cudaEventCreateWithFlags(&h->ev_interior, cudaEventDisableTiming), "stage event");
      }
      CK(cudaEventRecord(h->ev_packed, h->stream), "stage event");
      CK(cudaStreamWaitEvent(h->side_stream, h->ev_packed, 0), "stage event");
      DgDev di = d;
      di.nfaces = h->nface_int;
      a.phase = PHASE_FACE_ONLY;
      CK(launch_rhs_fp64(h->eq, di, a, h->side_stream), "interior face launch");
      CK(cudaEventRecord(h->ev_interior, h->side_stream), "stage event");
    }
  }
  return APOLLO_OK;
}

apollo_status apollo_dg_stage_end(apollo_dg* h, int stage, apollo_precision prec) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (h->lim_on) return fail(h, APOLLO_ERR_CONFIG, "partitioned meshes do not support the limiter");
  if (stage < 0 || stage > 4) return APOLLO_ERR_ARG;
  if (prec == APOLLO_PREC_MIXED && !h->mixed) return fail(h, APOLLO_ERR_CONFIG, "mixed precision not available");
  StageArgs a = stage_args(h, stage);
  DgDev d = make_dev(h);
  if (prec == APOLLO_PREC_MIXED) {
    const int blk = (int)(mixed_trace_floats(h->mixed, 1) / 3 * sizeof(float));
    CK(launch_halo_blocks(h->hrecv, (void*)a.tr_in, h->halo_dst_d, h->n_recv, blk, true, h->stream), "halo unpack");
    CK(mixed_launch_rhs(h->mixed, h->eq, d, a, h->stream, nullptr), "stage launch");
  } else {
    const int blk = h->ops.Ng * h->M * (int)sizeof(double);
    CK(launch_halo_blocks(h->hrecv, h->trace_d, h->halo_dst_d, h->n_recv, blk, true, h->stream), "halo unpack");
    if (!h->peers.empty() && h->nface_int > 0) {
      // the interior faces ran on the side stream since apollo_dg_stage_begin;
      // the cut faces now, then the lift over all of them
      CK(cudaStreamWaitEvent(h->stream, h->ev_interior, 0), "stage event");
      DgDev dc = d;
      dc.faces = d.faces + h->nface_int;
      dc.nfaces = d.nfaces - h->nface_int;
      a.phase = PHASE_FACE_ONLY;
      CK(launch_rhs_fp64(h->eq, dc, a, h->stream), "cut face launch");
      a.phase = PHASE_LIFT;
      CK(launch_rhs_fp64(h->eq, d, a, h->stream), "lift launch");
    } else {
      a.phase = PHASE_FACE;
      CK(launch_rhs_fp64(h->eq, d, a, h->stream), "face launch");
    }
  }
  if (stage == 4 && h->hlam)
    CK(cudaMemcpyAsync(h->hlam, &h->st_d->lam_bits, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, h->stream),
       "wave speed out");
  return APOLLO_OK;
}

apollo_status apollo_dg_step_end(apollo_dg* h) {
  apollo_status r = check_ready(h);
  if (r) return r;
  if (h->hlam)
    CK(cudaMemcpyAsync(&h->st_d->lam_bits, h->hlam, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, h->stream),
       "wave speed in");
  DgDev d = make_dev(h);
  CK(launch_finalize(d, h->stream), "finalize launch");
  return APOLLO_OK;
}

}  // extern "C"
