// Mixed-precision right-hand side: contractions on the tcgen05 tensor cores
// with split bf16 operands and fp32 accumulation; state, stage accumulation,
// dt reduction and sums stay float64.
#pragma once

#include <cuda_runtime.h>

#include "dg_device.cuh"
#include "dg_operators.h"

namespace apollo {

struct MixedPlan;

// nullptr when the equation/order has no mixed-precision kernel.
MixedPlan* mixed_create(int eq, const RefOps& ops, int K, int M);
void mixed_destroy(MixedPlan* p);
cudaError_t mixed_launch_rhs(MixedPlan* p, int eq, const DgDev& d, const StageArgs& a, cudaStream_t s,
                             cudaEvent_t* ev = nullptr);

}  // namespace apollo
