// Mesh partitioning and halo plans (host only): face pairing shared with
// apollo_dg_set_mesh, recursive coordinate bisection, and the per-rank lists
// of cut faces whose traces cross between ranks once per stage.
#include "dg_partition.h"

#include <algorithm>
#include <numeric>
#include <unordered_map>

#include "apollo_dg.h"

namespace apollo {

std::string pair_faces(int nverts, int K, const int* etov, const int* face_tag, const int* vert_canon,
                       std::vector<int>& partner) {
  static const int vn[3][2] = {{0, 1}, {1, 2}, {2, 0}};
  partner.assign((size_t)K * 3, -1);
  std::unordered_map<unsigned long long, int> open;
  open.reserve((size_t)K * 2);
  for (int k = 0; k < K; ++k)
    for (int f = 0; f < 3; ++f) {
      const int tag = face_tag ? face_tag[3 * k + f] : 0;
      if (tag < 0) return "negative face tag";
      if (tag > 0) continue;
      int a = etov[3 * k + vn[f][0]], b = etov[3 * k + vn[f][1]];
      if (a < 0 || a >= nverts || b < 0 || b >= nverts) return "vertex index out of range";
      if (vert_canon) {
        a = vert_canon[a];
        b = vert_canon[b];
      }
      if (a == b) return "degenerate face";
      const unsigned long long key = ((unsigned long long)(unsigned)std::min(a, b) << 32) | (unsigned)std::max(a, b);
      auto it = open.find(key);
      if (it == open.end()) {
        open.emplace(key, 3 * k + f);
      } else {
        const int kf = it->second;
        if (kf < 0) return "face shared by more than two elements";
        partner[3 * k + f] = kf;
        partner[kf] = 3 * k + f;
        it->second = -1;
      }
    }
  return "";
}

namespace {

void rcb(std::vector<int>& ids, size_t lo, size_t hi, int p0, int np, const std::vector<double>& cx,
         const std::vector<double>& cy, int* part) {
  if (np == 1) {
    for (size_t i = lo; i < hi; ++i) part[ids[i]] = p0;
    return;
  }
  double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
  for (size_t i = lo; i < hi; ++i) {
    x0 = std::min(x0, cx[ids[i]]);
    x1 = std::max(x1, cx[ids[i]]);
    y0 = std::min(y0, cy[ids[i]]);
    y1 = std::max(y1, cy[ids[i]]);
  }
  const std::vector<double>& c = (x1 - x0 >= y1 - y0) ? cx : cy;
  const int n1 = np / 2;
  const size_t cnt = hi - lo;
  const size_t c1 = (size_t)((double)cnt * n1 / np + 0.5);
  auto less = [&](int a, int b) { return c[a] < c[b] || (c[a] == c[b] && a < b); };
  std::nth_element(ids.begin() + lo, ids.begin() + lo + c1, ids.begin() + hi, less);
  rcb(ids, lo, lo + c1, p0, n1, cx, cy, part);
  rcb(ids, lo + c1, hi, p0 + n1, np - n1, cx, cy, part);
}

}  // namespace

std::string rcb_partition(const double* vx, const double* vy, int K, const int* etov, int nparts, int* part) {
  if (nparts < 1) return "nparts must be positive";
  if (nparts > K) return "more parts than elements";
  std::vector<double> cx(K), cy(K);
  for (int k = 0; k < K; ++k) {
    const int a = etov[3 * k], b = etov[3 * k + 1], d = etov[3 * k + 2];
    cx[k] = (vx[a] + vx[b] + vx[d]) / 3.0;
    cy[k] = (vy[a] + vy[b] + vy[d]) / 3.0;
  }
  std::vector<int> ids(K);
  std::iota(ids.begin(), ids.end(), 0);
  rcb(ids, 0, (size_t)K, 0, nparts, cx, cy, part);
  return "";
}

std::string build_halo(int K, const std::vector<int>& partner, const int* part, int rank, HaloPlan& plan) {
  plan = HaloPlan{};
  struct Cut {
    int owner, mine, theirs;  // owner rank of the partner; global face ids
  };
  std::vector<Cut> cuts;
  for (int k = 0; k < K; ++k) {
    if (part[k] < 0) return "negative part id";
    if (part[k] != rank) continue;
    plan.local.push_back(k);
    for (int f = 0; f < 3; ++f) {
      const int p = partner[3 * k + f];
      if (p >= 0 && part[p / 3] != rank) cuts.push_back(Cut{part[p / 3], 3 * k + f, p});
    }
  }
  if (plan.local.empty()) return "rank owns no elements";
  // ghost elements by (owner, id)
  std::vector<std::pair<int, int>> gh;
  for (const Cut& c : cuts) gh.emplace_back(c.owner, c.theirs / 3);
  std::sort(gh.begin(), gh.end());
  gh.erase(std::unique(gh.begin(), gh.end()), gh.end());
  for (auto& g : gh) plan.ghost.push_back(g.second);
  for (auto& g : gh)
    if (plan.peers.empty() || plan.peers.back() != g.first) plan.peers.push_back(g.first);
  // per peer: sends by the local face id, receives by the remote face id (the
  // order of that peer's own send list)
  for (int peer : plan.peers) {
    std::vector<int> s, r;
    for (const Cut& c : cuts)
      if (c.owner == peer) {
        s.push_back(c.mine);
        r.push_back(c.theirs);
      }
    std::sort(s.begin(), s.end());
    std::sort(r.begin(), r.end());
    plan.send_count.push_back((int)s.size());
    plan.recv_count.push_back((int)r.size());
    plan.send_face.insert(plan.send_face.end(), s.begin(), s.end());
    plan.recv_face.insert(plan.recv_face.end(), r.begin(), r.end());
  }
  return "";
}

}  // namespace apollo

using namespace apollo;

extern "C" {

apollo_status apollo_dg_partition(int nverts, const double* vx, const double* vy, int K, const int* etov,
                                  int nparts, int* part) {
  if (!vx || !vy || !etov || !part || nverts < 3 || K < 1) return APOLLO_ERR_ARG;
  for (size_t i = 0; i < (size_t)K * 3; ++i)
    if (etov[i] < 0 || etov[i] >= nverts) return APOLLO_ERR_MESH;
  return rcb_partition(vx, vy, K, etov, nparts, part).empty() ? APOLLO_OK : APOLLO_ERR_ARG;
}

apollo_status apollo_dg_halo_plan(int nverts, int K, const int* etov, const int* face_tag, const int* vert_canon,
                                  const int* part, int rank, apollo_dg_halo_sizes* sizes, int* local_elems,
                                  int* ghost_elems, int* peers, int* send_count, int* recv_count, int* send_faces,
                                  int* recv_faces) {
  if (!etov || !part || !sizes || nverts < 3 || K < 1 || rank < 0) return APOLLO_ERR_ARG;
  std::vector<int> partner;
  if (!pair_faces(nverts, K, etov, face_tag, vert_canon, partner).empty()) return APOLLO_ERR_MESH;
  HaloPlan plan;
  if (!build_halo(K, partner, part, rank, plan).empty()) return APOLLO_ERR_ARG;
  sizes->n_local = (int)plan.local.size();
  sizes->n_ghost = (int)plan.ghost.size();
  sizes->n_peers = (int)plan.peers.size();
  sizes->n_send = (int)plan.send_face.size();
  sizes->n_recv = (int)plan.recv_face.size();
  auto put = [](int* dst, const std::vector<int>& v) {
    if (dst) std::copy(v.begin(), v.end(), dst);
  };
  put(local_elems, plan.local);
  put(ghost_elems, plan.ghost);
  put(peers, plan.peers);
  put(send_count, plan.send_count);
  put(recv_count, plan.recv_count);
  put(send_faces, plan.send_face);
  put(recv_faces, plan.recv_face);
  return APOLLO_OK;
}

}  // extern "C"
