// Mixed-precision right-hand side: contractions on the tcgen05 tensor cores
// with split tf32 operands and fp32 accumulation; state, stage accumulation,
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
// One stage (or, for MODE_RHS, the input's traces into a.tr_scratch and then
// the right-hand side); ev[0..3] bracket the trace kernel and the stage kernel.
cudaError_t mixed_launch_rhs(MixedPlan* p, int eq, const DgDev& d, const StageArgs& a, cudaStream_t s,
                             cudaEvent_t* ev = nullptr);
// Floats of one trace buffer: [K][3][NG M padded to a multiple of 4].
size_t mixed_trace_floats(const MixedPlan* p, int K);
// fp32 face traces of the float64 state x.
cudaError_t mixed_launch_traces(MixedPlan* p, const DgDev& d, const double* x, float* T, cudaStream_t s);

}  // namespace apollo
