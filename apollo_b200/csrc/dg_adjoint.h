// Tangent and adjoint of one float64 right-hand-side stage (dg_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include "dg_device.cuh"

namespace apollo {

// Tangent of a stage: dout = tangent of the stage result along dx (and du0
// for MODE_FINAL), at the state x.  d.trace receives the traces of x;
// dtrace, dvol, dflux are scratch ([K][NF][M], [K][NP][M], [K][NF][M]).
struct TanArgs {
  const double* x;
  const double* dx;
  const double* du0;
  double* dout;
  double* dvol;
  double* dtrace;
  double* dflux;
  int mode;  // MODE_RHS, MODE_STAGE, MODE_FINAL
  double t, dt;
};

// Adjoint of a stage: out = alpha * wbar + beta * L'(x)^T wbar + gamma * z
// (z may be null).  d.trace receives the traces of x; sbar is scratch
// [K][NF][M].  out may alias z (each element is read before it is written);
// it may not alias x or wbar.
struct AdjArgs {
  const double* x;
  const double* wbar;
  const double* z;
  double* out;
  double* sbar;
  double alpha, beta, gamma;
  double t;
};

cudaError_t launch_tangent_stage(int eq, const DgDev& d, const TanArgs& a, cudaStream_t s);
cudaError_t launch_adjoint_stage(int eq, const DgDev& d, const AdjArgs& a, cudaStream_t s);

}  // namespace apollo
