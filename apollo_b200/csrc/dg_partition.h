// Mesh partitioning and the halo plan of one rank (host only, no device calls).
#pragma once

#include <string>
#include <vector>

namespace apollo {

// Pairs the faces of a triangle mesh that share both (canonical) vertices:
// partner[3k+f] = 3k'+f' for an interior face, -1 for an unpaired or tagged
// (boundary) face.  Apollo pairs faces by shared vertices
// (wxnodaldggeometry2d.cc:235-367); vert_canon (optional) identifies periodic
// vertices.  Returns an empty string, or the reason the mesh is rejected.
std::string pair_faces(int nverts, int K, const int* etov, const int* face_tag, const int* vert_canon,
                       std::vector<int>& partner);

// Recursive coordinate bisection of the element centroids into nparts parts
// of sizes within one element of K/nparts: each cut halves the part count and
// splits the elements in proportion along the longer side of their bounding
// box (ties broken by element id, so the result is deterministic).
std::string rcb_partition(const double* vx, const double* vy, int K, const int* etov, int nparts, int* part);

// One rank's share of a partitioned mesh.  Elements keep their global order;
// the ghost slots are the remote elements that share a face with a local one.
// A cut face (local element k, face f) with partner face p on peer rank s is
// sent as the trace block of (k, f) and received into the ghost slot of p's
// element at face p % 3.  Both sides order the blocks of one peer by the
// sending side's global face id (3k + f), so a send list and the matching
// receive list agree without any exchange of indices.
struct HaloPlan {
  std::vector<int> local;       // global ids of the local elements, ascending
  std::vector<int> ghost;       // global ids of the ghost elements, by (owner rank, id)
  std::vector<int> peers;       // ranks sharing a face with this rank, ascending
  std::vector<int> send_count;  // blocks per peer
  std::vector<int> recv_count;
  std::vector<int> send_face;   // per send block, peer-major: global face id of the local side
  std::vector<int> recv_face;   // per receive block, peer-major: global face id of the remote side
};

std::string build_halo(int K, const std::vector<int>& partner, const int* part, int rank, HaloPlan& plan);

}  // namespace apollo
