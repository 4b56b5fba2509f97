// Mixed-precision right-hand side (placeholder until the tensor-core kernels land).
#include "dg_mixed.h"

namespace apollo {

struct MixedPlan {
  int dummy;
};

MixedPlan* mixed_create(int, const RefOps&, int, int) { return nullptr; }
void mixed_destroy(MixedPlan* p) { delete p; }
cudaError_t mixed_launch_rhs(MixedPlan*, int, const DgDev&, const StageArgs&, cudaStream_t, cudaEvent_t*) {
  return cudaErrorNotSupported;
}

}  // namespace apollo
