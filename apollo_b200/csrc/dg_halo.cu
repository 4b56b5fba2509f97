// Packing and unpacking of the face-trace blocks that cross between ranks of
// a partitioned mesh: one 16-byte word per thread, grid-stride.
#include "dg_device.cuh"

namespace apollo {
namespace {

__global__ void k_halo_blocks(const float4* __restrict__ src, float4* __restrict__ dst, const int* __restrict__ idx,
                              int n, int b4, int scatter) {
  const long long total = (long long)n * b4;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(i / b4), q = (int)(i - (long long)j * b4);
    const size_t far = (size_t)idx[j] * b4 + q, near = (size_t)j * b4 + q;
    if (scatter) dst[far] = src[near];
    else dst[near] = src[far];
  }
}

}  // namespace

cudaError_t launch_halo_blocks(const void* src, void* dst, const int* idx, int n, int block_bytes, bool scatter,
                               cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (block_bytes <= 0 || block_bytes % 16 || ((uintptr_t)src | (uintptr_t)dst) % 16) return cudaErrorInvalidValue;
  const int b4 = block_bytes / 16;
  const long long total = (long long)n * b4;
  long long blocks = (total + 255) / 256;
  const long long cap = 148LL * 8;
  if (blocks > cap) blocks = cap;
  k_halo_blocks<<<(int)blocks, 256, 0, s>>>((const float4*)src, (float4*)dst, idx, n, b4, scatter ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace apollo
