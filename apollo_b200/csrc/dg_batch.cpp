// Batched ensembles (include/apollo_dg.h, "Batched ensembles"): independent
// meshes of one equation, any sizes and orders 2..5, stepped together.
//
// The instances of one order are concatenated into one discretisation (one
// apollo_dg handle over the union of their elements, no faces between them),
// with an instance id per element and one DevState per instance, so every
// stage is one persistent launch over all of them and each instance keeps its
// own dt, time and dt policy.  One CUDA graph per step forks the order groups
// onto their streams, so groups of different orders run concurrently.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "apollo_dg.h"
#include "dg_device.cuh"

namespace apollo {
apollo_status handle_set_instances(apollo_dg* h, int ninst, const int* einst);
cudaStream_t handle_stream(const apollo_dg* h);
DevState* handle_states_host(apollo_dg* h);
apollo_status handle_push_states(apollo_dg* h);
apollo_status handle_pull_states(apollo_dg* h);
apollo_status handle_init_speed(apollo_dg* h);
double handle_rmin(const apollo_dg* h);
double handle_cfl(const apollo_dg* h);
size_t handle_state_doubles(const apollo_dg* h);
double* handle_state_device(apollo_dg* h);
void handle_mark_state(apollo_dg* h);
apollo_status handle_enqueue_step_raw(apollo_dg* h, apollo_precision prec);
apollo_status handle_prepare_step(apollo_dg* h, apollo_precision prec);
apollo_status handle_read_errors(apollo_dg* h);
void handle_set_grid_div(apollo_dg* h, int div);
void handle_set_tile_shape(apollo_dg* h, int shape);
}  // namespace apollo

using namespace apollo;

struct apollo_dg_batch {
  apollo_dg_config cfg{};
  std::string eq_kind;
  std::vector<double> eqp;
  std::string numflux;  // Numerical_Flux name, empty: the default
  std::vector<std::pair<std::string, std::vector<double>>> bcs;
  struct MeshIn {
    int N = 0, nverts = 0, K = 0;
    std::vector<double> vx, vy;
    std::vector<int> etov, tag, canon;
    bool has_tag = false, has_canon = false;
  };
  std::vector<MeshIn> meshes;
  struct Group {
    int N = 0;
    apollo_dg* h = nullptr;
    std::vector<int> insts;  // batch instance ids, in element order
    int div = 1;             // persistent-grid share picked by the autotuner
    int shape = 0;           // mixed stage operand chunking picked by the autotuner
  };
  std::vector<Group> groups;
  struct Inst {
    int g = 0, local = 0, k0 = 0, K = 0, Np = 0;
    double dtfac = 0.0;
  };
  std::vector<Inst> inst;
  int M = 0;
  bool finalized = false;
  cudaStream_t master = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  std::string err;
};

namespace {

apollo_status bfail(apollo_dg_batch* b, apollo_status code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}

apollo_status from_handle(apollo_dg_batch* b, apollo_dg* h, apollo_status r) {
  if (r != APOLLO_OK) b->err = apollo_dg_last_error(h);
  return r;
}

#define BCK(call, where)                                                            \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) return bfail(b, APOLLO_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Smallest inscribed radius over a mesh's elements (Apollo's dtscale,
// wxnodaldggeometry2d.cc:220-227), as apollo_dg_set_mesh computes it.
double mesh_dtscale(const apollo_dg_batch::MeshIn& m) {
  double dtscale = 1.0e6;
  for (int k = 0; k < m.K; ++k) {
    const int v0 = m.etov[3 * k], v1 = m.etov[3 * k + 1], v2 = m.etov[3 * k + 2];
    const double p1x = m.vx[v0], p1y = m.vy[v0], p2x = m.vx[v1], p2y = m.vy[v1], p3x = m.vx[v2], p3y = m.vy[v2];
    const double l1 = std::sqrt(std::pow(p1x - p2x, 2) + std::pow(p1y - p2y, 2));
    const double l2 = std::sqrt(std::pow(p2x - p3x, 2) + std::pow(p2y - p3y, 2));
    const double l3 = std::sqrt(std::pow(p3x - p1x, 2) + std::pow(p3y - p1y, 2));
    const double sp = 0.5 * (l1 + l2 + l3);
    const double area = std::sqrt(std::fabs(sp * (sp - l1) * (sp - l2) * (sp - l3)));
    dtscale = std::min(dtscale, area / sp);
  }
  return dtscale;
}

void drop_graphs(apollo_dg_batch* b) {
  for (auto& g : b->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

// Captures one step of every group: fork from the master stream, each group's
// 5 stages + finalize on its own stream, join.
apollo_status build_graph(apollo_dg_batch* b, apollo_precision prec, cudaGraphExec_t* out) {
  const int gi = prec == APOLLO_PREC_MIXED ? 1 : 0;
  if (b->graph[gi]) {
    *out = b->graph[gi];
    return APOLLO_OK;
  }
  cudaGraph_t g = nullptr;
  BCK(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal), "begin capture");
  apollo_status r = APOLLO_OK;
  cudaError_t e = cudaEventRecord(b->fork, b->master);
  for (size_t i = 0; i < b->groups.size() && r == APOLLO_OK && e == cudaSuccess; ++i) {
    apollo_dg* h = b->groups[i].h;
    e = cudaStreamWaitEvent(handle_stream(h), b->fork, 0);
    if (e == cudaSuccess) r = from_handle(b, h, handle_enqueue_step_raw(h, prec));
    if (r == APOLLO_OK && e == cudaSuccess) e = cudaEventRecord(b->join[i], handle_stream(h));
    if (r == APOLLO_OK && e == cudaSuccess) e = cudaStreamWaitEvent(b->master, b->join[i], 0);
  }
  cudaError_t e2 = cudaStreamEndCapture(b->master, &g);
  if (r != APOLLO_OK || e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    if (r != APOLLO_OK) return r;
    return bfail(b, APOLLO_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  e = cudaGraphInstantiate(&b->graph[gi], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return bfail(b, APOLLO_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(e));
  *out = b->graph[gi];
  return APOLLO_OK;
}

}  // namespace

extern "C" {

apollo_status apollo_dg_batch_create(const apollo_dg_config* cfg, const char* eq_kind, const double* eq_params,
                                     int n_params, apollo_dg_batch** out) {
  if (!cfg || !eq_kind || !out || n_params < 0 || (n_params > 0 && !eq_params)) return APOLLO_ERR_ARG;
  if (!(cfg->cfl > 0.0)) return APOLLO_ERR_CONFIG;
  apollo_dg_batch* b = new apollo_dg_batch();
  b->cfg = *cfg;
  b->eq_kind = eq_kind;
  b->eqp.assign(eq_params, eq_params + n_params);
  *out = b;
  return APOLLO_OK;
}

apollo_status apollo_dg_batch_set_numerical_flux(apollo_dg_batch* b, const char* name) {
  if (!b || !name) return APOLLO_ERR_ARG;
  if (b->finalized) return bfail(b, APOLLO_ERR_STATE, "batch already finalized");
  b->numflux = name;
  return APOLLO_OK;
}

apollo_status apollo_dg_batch_add_bc(apollo_dg_batch* b, const char* kind, const double* params, int n_params) {
  if (!b || !kind || n_params < 0 || (n_params > 0 && !params)) return APOLLO_ERR_ARG;
  if (b->finalized) return bfail(b, APOLLO_ERR_STATE, "batch already finalized");
  b->bcs.emplace_back(kind, std::vector<double>(params, params + n_params));
  return APOLLO_OK;
}

apollo_status apollo_dg_batch_add_mesh(apollo_dg_batch* b, int N, int nverts, const double* vx, const double* vy,
                                       int K, const int* etov, const int* face_tag, const int* vert_canon,
                                       int* instance) {
  if (!b || !vx || !vy || !etov || nverts < 3 || K < 1) return APOLLO_ERR_ARG;
  if (b->finalized) return bfail(b, APOLLO_ERR_STATE, "batch already finalized");
  if (N < 2 || N > 5) return bfail(b, APOLLO_ERR_CONFIG, "order must be 2..5");
  apollo_dg_batch::MeshIn m;
  m.N = N;
  m.nverts = nverts;
  m.K = K;
  m.vx.assign(vx, vx + nverts);
  m.vy.assign(vy, vy + nverts);
  m.etov.assign(etov, etov + 3 * (size_t)K);
  for (int v : m.etov)
    if (v < 0 || v >= nverts) return bfail(b, APOLLO_ERR_MESH, "vertex index out of range");
  if (face_tag) {
    m.tag.assign(face_tag, face_tag + 3 * (size_t)K);
    m.has_tag = true;
  }
  if (vert_canon) {
    m.canon.assign(vert_canon, vert_canon + nverts);
    m.has_canon = true;
  }
  if (instance) *instance = (int)b->meshes.size();
  b->meshes.push_back(std::move(m));
  return APOLLO_OK;
}

apollo_status apollo_dg_batch_finalize(apollo_dg_batch* b) {
  if (!b) return APOLLO_ERR_ARG;
  if (b->finalized) return bfail(b, APOLLO_ERR_STATE, "batch already finalized");
  if (b->meshes.empty()) return bfail(b, APOLLO_ERR_STATE, "no meshes");
  BCK(cudaSetDevice(b->cfg.device), "set device");
  b->inst.assign(b->meshes.size(), apollo_dg_batch::Inst{});
  for (int N = 2; N <= 5; ++N) {
    std::vector<int> ids;
    for (size_t i = 0; i < b->meshes.size(); ++i)
      if (b->meshes[i].N == N) ids.push_back((int)i);
    if (ids.empty()) continue;
    // union of the group's meshes: vertices, cells, tags and periodic vertex
    // identities offset per mesh; the instance of every element
    std::vector<double> vx, vy;
    std::vector<int> etov, tag, canon, einst;
    int vo = 0;
    for (size_t l = 0; l < ids.size(); ++l) {
      const auto& m = b->meshes[ids[l]];
      vx.insert(vx.end(), m.vx.begin(), m.vx.end());
      vy.insert(vy.end(), m.vy.begin(), m.vy.end());
      for (int v : m.etov) etov.push_back(v + vo);
      for (int k = 0; k < 3 * m.K; ++k) tag.push_back(m.has_tag ? m.tag[k] : 0);
      for (int v = 0; v < m.nverts; ++v) canon.push_back((m.has_canon ? m.canon[v] : v) + vo);
      einst.insert(einst.end(), m.K, (int)l);
      vo += m.nverts;
    }
    apollo_dg_config c = b->cfg;
    c.polynomial_order = N;
    c.stream = nullptr;
    apollo_dg* h = nullptr;
    apollo_status r = apollo_dg_create(&c, &h);
    if (r) return bfail(b, r, "group create failed");
    b->groups.push_back(apollo_dg_batch::Group{});
    auto& G = b->groups.back();
    G.N = N;
    G.h = h;
    G.insts = ids;
    r = from_handle(b, h, apollo_dg_set_equation(h, b->eq_kind.c_str(), b->eqp.data(), (int)b->eqp.size()));
    if (!r && !b->numflux.empty()) r = from_handle(b, h, apollo_dg_set_numerical_flux(h, b->numflux.c_str()));
    for (size_t j = 0; j < b->bcs.size() && !r; ++j)
      r = from_handle(b, h, apollo_dg_add_bc(h, b->bcs[j].first.c_str(), b->bcs[j].second.data(),
                                             (int)b->bcs[j].second.size()));
    if (!r)
      r = from_handle(b, h, apollo_dg_set_mesh(h, vo, vx.data(), vy.data(), (int)einst.size(), etov.data(),
                                               tag.data(), canon.data()));
    if (!r) r = from_handle(b, h, handle_set_instances(h, (int)ids.size(), einst.data()));
    if (r) return r;
    b->M = apollo_dg_num_fields(h);
    const int Np = apollo_dg_num_nodes(h);
    DevState* st = handle_states_host(h);
    int k0 = 0;
    for (size_t l = 0; l < ids.size(); ++l) {
      auto& I = b->inst[ids[l]];
      I.g = (int)b->groups.size() - 1;
      I.local = (int)l;
      I.k0 = k0;
      I.K = b->meshes[ids[l]].K;
      I.Np = Np;
      I.dtfac = 2. / 3. * b->cfg.cfl * mesh_dtscale(b->meshes[ids[l]]);
      st[l].dtfac = I.dtfac;
      k0 += I.K;
    }
    r = from_handle(b, h, handle_push_states(h));
    if (r) return r;
    BCK(cudaStreamSynchronize(handle_stream(h)), "group setup");
  }
  if (b->cfg.stream) b->master = (cudaStream_t)b->cfg.stream;
  else BCK(cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking), "batch stream");
  BCK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "batch events");
  b->join.assign(b->groups.size(), nullptr);
  for (auto& e : b->join) BCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch events");
  b->meshes.clear();
  b->meshes.shrink_to_fit();
  b->finalized = true;
  return APOLLO_OK;
}

int apollo_dg_batch_size(const apollo_dg_batch* b) { return b ? (int)b->inst.size() : 0; }

apollo_status apollo_dg_batch_instance_info(const apollo_dg_batch* b, int inst, int* N, int* K, int* Np,
                                            int* fields) {
  if (!b || !b->finalized || inst < 0 || inst >= (int)b->inst.size()) return APOLLO_ERR_ARG;
  const auto& I = b->inst[inst];
  if (N) *N = b->groups[I.g].N;
  if (K) *K = I.K;
  if (Np) *Np = I.Np;
  if (fields) *fields = b->M;
  return APOLLO_OK;
}

apollo_status apollo_dg_batch_node_coords(const apollo_dg_batch* b, int inst, double* x, double* y) {
  if (!b || !b->finalized || inst < 0 || inst >= (int)b->inst.size() || !x || !y) return APOLLO_ERR_ARG;
  const auto& I = b->inst[inst];
  apollo_dg* h = b->groups[I.g].h;
  const size_t n = (size_t)apollo_dg_num_elements(h) * I.Np;
  std::vector<double> xa(n), ya(n);
  apollo_status r = apollo_dg_node_coords(h, xa.data(), ya.data());
  if (r) return r;
  std::memcpy(x, xa.data() + (size_t)I.k0 * I.Np, (size_t)I.K * I.Np * sizeof(double));
  std::memcpy(y, ya.data() + (size_t)I.k0 * I.Np, (size_t)I.K * I.Np * sizeof(double));
  return APOLLO_OK;
}

apollo_status apollo_dg_batch_set_state(apollo_dg_batch* b, int inst, const double* U, int where) {
  if (!b || !b->finalized || inst < 0 || inst >= (int)b->inst.size() || !U) return APOLLO_ERR_ARG;
  const auto& I = b->inst[inst];
  apollo_dg* h = b->groups[I.g].h;
  const size_t n = (size_t)I.K * I.Np * b->M;
  double* dst = handle_state_device(h) + (size_t)I.k0 * I.Np * b->M;
  BCK(cudaMemcpyAsync(dst, U, n * sizeof(double),
                      where == APOLLO_DEVICE_PTR ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                      handle_stream(h)),
      "set state");
  BCK(cudaStreamSynchronize(handle_stream(h)), "set state");
  handle_mark_state(h);
  return APOLLO_OK;
}

apollo_status apollo_dg_batch_get_state(apollo_dg_batch* b, int inst, double* U, int where) {
  if (!b || !b->finalized || inst < 0 || inst >= (int)b->inst.size() || !U) return APOLLO_ERR_ARG;
  const auto& I = b->inst[inst];
  apollo_dg* h = b->groups[I.g].h;
  const size_t n = (size_t)I.K * I.Np * b->M;
  const double* src = handle_state_device(h) + (size_t)I.k0 * I.Np * b->M;
  BCK(cudaMemcpyAsync(U, src, n * sizeof(double),
                      where == APOLLO_DEVICE_PTR ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                      handle_stream(h)),
      "get state");
  BCK(cudaStreamSynchronize(handle_stream(h)), "get state");
  return APOLLO_OK;
}

apollo_status apollo_dg_batch_init_dt(apollo_dg_batch* b, double* dt) {
  if (!b || !b->finalized || !dt) return APOLLO_ERR_ARG;
  for (auto& G : b->groups) {
    apollo_status r = from_handle(b, G.h, handle_init_speed(G.h));
    if (!r) r = from_handle(b, G.h, handle_pull_states(G.h));
    if (r) return r;
  }
  for (auto& G : b->groups) {
    BCK(cudaStreamSynchronize(handle_stream(G.h)), "init dt");
    const DevState* st = handle_states_host(G.h);
    for (int id : G.insts) {
      const auto& I = b->inst[id];
      double lam;
      std::memcpy(&lam, &st[I.local].lam_bits, sizeof(double));
      dt[id] = I.dtfac * (handle_rmin(G.h) / lam);
    }
  }
  return APOLLO_OK;
}

apollo_status apollo_dg_batch_step(apollo_dg_batch* b, int nsteps, double* t, double* dt, apollo_precision prec) {
  if (!b || !b->finalized || !t || !dt || nsteps < 0) return APOLLO_ERR_ARG;
  for (auto& G : b->groups) {
    DevState* st = handle_states_host(G.h);
    for (int id : G.insts) {
      const auto& I = b->inst[id];
      DevState s{};
      s.t = t[id];
      s.dt = dt[id];
      s.dtfac = I.dtfac;
      st[I.local] = s;
    }
    apollo_status r = from_handle(b, G.h, handle_push_states(G.h));
    if (!r) r = from_handle(b, G.h, handle_prepare_step(G.h, prec));
    if (r) return r;
  }
  for (auto& G : b->groups) BCK(cudaStreamSynchronize(handle_stream(G.h)), "batch step");
  cudaGraphExec_t g = nullptr;
  apollo_status r = build_graph(b, prec, &g);
  if (r) return r;
  for (int i = 0; i < nsteps; ++i) BCK(cudaGraphLaunch(g, b->master), "batch graph launch");
  BCK(cudaStreamSynchronize(b->master), "batch step");
  for (auto& G : b->groups) {
    r = from_handle(b, G.h, handle_pull_states(G.h));
    if (r) return r;
    BCK(cudaStreamSynchronize(handle_stream(G.h)), "batch step");
    const DevState* st = handle_states_host(G.h);
    for (int id : G.insts) {
      t[id] = st[b->inst[id].local].t;
      dt[id] = st[b->inst[id].local].dt;
    }
    r = from_handle(b, G.h, handle_read_errors(G.h));
    if (r) return r;
  }
  return APOLLO_OK;
}

apollo_status apollo_dg_batch_autotune(apollo_dg_batch* b, apollo_precision prec, int* share, int* shape) {
  if (!b || !b->finalized) return APOLLO_ERR_ARG;
  // keep the states: every trial starts from them
  const size_t ni = b->inst.size();
  std::vector<double> t0(ni), dt0(ni);
  // the saved states and the timing events, released on every return
  struct Scratch {
    std::vector<double*> saved;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Scratch() {
      for (double* p : saved)
        if (p) cudaFree(p);
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
    }
  } sc;
  sc.saved.assign(b->groups.size(), nullptr);
  std::vector<double*>& saved = sc.saved;
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    apollo_dg* h = b->groups[gi].h;
    const DevState* st = handle_states_host(h);
    apollo_status r = from_handle(b, h, handle_pull_states(h));
    if (r) return r;
    BCK(cudaStreamSynchronize(handle_stream(h)), "autotune");
    for (int id : b->groups[gi].insts) {
      t0[id] = st[b->inst[id].local].t;
      dt0[id] = st[b->inst[id].local].dt;
    }
    const size_t n = handle_state_doubles(h);
    BCK(cudaMalloc((void**)&saved[gi], n * sizeof(double)), "autotune");
    BCK(cudaMemcpy(saved[gi], handle_state_device(h), n * sizeof(double), cudaMemcpyDeviceToDevice), "autotune");
  }
  // initial dt where none was set yet
  bool need_dt = false;
  for (size_t i = 0; i < ni; ++i) need_dt |= !(dt0[i] > 0.0);
  std::vector<double> dtinit(ni);
  if (need_dt) {
    apollo_status r = apollo_dg_batch_init_dt(b, dtinit.data());
    if (r) return r;
    for (size_t i = 0; i < ni; ++i)
      if (!(dt0[i] > 0.0)) dt0[i] = dtinit[i];
  }
  BCK(cudaEventCreate(&sc.e0), "autotune");
  BCK(cudaEventCreate(&sc.e1), "autotune");
  cudaEvent_t e0 = sc.e0, e1 = sc.e1;
  auto trial = [&](float* ms) -> apollo_status {
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
      apollo_dg* h = b->groups[gi].h;
      BCK(cudaMemcpy(handle_state_device(h), saved[gi], handle_state_doubles(h) * sizeof(double),
                     cudaMemcpyDeviceToDevice), "autotune");
      handle_mark_state(h);
    }
    std::vector<double> t = t0, dt = dt0;
    apollo_status r = apollo_dg_batch_step(b, 1, t.data(), dt.data(), prec);  // warm-up, graph built
    if (r) return r;
    cudaGraphExec_t g = nullptr;
    r = build_graph(b, prec, &g);
    if (r) return r;
    BCK(cudaEventRecord(e0, b->master), "autotune");
    for (int i = 0; i < 3; ++i) BCK(cudaGraphLaunch(g, b->master), "autotune");
    BCK(cudaEventRecord(e1, b->master), "autotune");
    BCK(cudaEventSynchronize(e1), "autotune");
    BCK(cudaEventElapsedTime(ms, e0, e1), "autotune");
    return APOLLO_OK;
  };
  // coordinate descent over the groups' launch shapes: the persistent-grid
  // share and, in mixed precision, the operand chunking of the stage kernel
  const int divs[3] = {1, 2, 4};
  const int nshape = prec == APOLLO_PREC_MIXED ? 2 : 1;
  apollo_status r = APOLLO_OK;
  for (size_t gi = 0; gi < b->groups.size() && !r; ++gi) {
    float best = 1e30f;
    int best_div = b->groups[gi].div, best_shape = b->groups[gi].shape;
    for (int sh = 0; sh < nshape && !r; ++sh)
      for (int c : divs) {
        handle_set_grid_div(b->groups[gi].h, c);
        handle_set_tile_shape(b->groups[gi].h, sh);
        drop_graphs(b);
        float ms = 0.f;
        r = trial(&ms);
        if (r) break;
        if (ms < best) {
          best = ms;
          best_div = c;
          best_shape = sh;
        }
      }
    b->groups[gi].div = best_div;
    b->groups[gi].shape = best_shape;
    handle_set_grid_div(b->groups[gi].h, best_div);
    handle_set_tile_shape(b->groups[gi].h, best_shape);
    drop_graphs(b);
  }
  // restore the states
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    apollo_dg* h = b->groups[gi].h;
    if (!r) {
      cudaError_t e = cudaMemcpy(handle_state_device(h), saved[gi], handle_state_doubles(h) * sizeof(double),
                                 cudaMemcpyDeviceToDevice);
      if (e != cudaSuccess) r = bfail(b, APOLLO_ERR_CUDA, "autotune restore");
      handle_mark_state(h);
    }
  }
  for (int i = 0; i < 4; ++i) {
    if (share) share[i] = 0;
    if (shape) shape[i] = -1;
  }
  for (auto& G : b->groups) {
    if (share) share[G.N - 2] = G.div;
    if (shape) shape[G.N - 2] = G.shape;
  }
  return r;
}

const char* apollo_dg_batch_last_error(const apollo_dg_batch* b) { return b ? b->err.c_str() : "null batch"; }

apollo_status apollo_dg_batch_destroy(apollo_dg_batch* b) {
  if (!b) return APOLLO_ERR_ARG;
  cudaSetDevice(b->cfg.device);
  if (b->master) cudaStreamSynchronize(b->master);
  drop_graphs(b);
  for (auto& G : b->groups) apollo_dg_destroy(G.h);
  if (b->fork) cudaEventDestroy(b->fork);
  for (auto& e : b->join)
    if (e) cudaEventDestroy(e);
  if (b->master && b->master != (cudaStream_t)b->cfg.stream) cudaStreamDestroy(b->master);
  delete b;
  return APOLLO_OK;
}

}  // extern "C"
