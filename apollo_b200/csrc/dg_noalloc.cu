// The float64 right-hand side with its scratch in a file-scope device array,
// for callers that cannot allocate device memory when they evaluate it.
//
// The three float64 kernels (volume, face, LIFT) pass the volume term, the
// face traces and the face fluxes between them through global memory.  The
// regular entry point keeps those arrays in the handle; this one keeps them in
// g_rhs_scratch below, a fixed 64 MiB array that every GPU loading the library
// holds until the process exits.  Nothing here calls cudaMalloc or cudaFree.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <mutex>
#include <string>

#include "apollo_dg.h"
#include "dg_device.cuh"

namespace apollo {

// Reads the discretisation of a handle (dg_host.cpp); returns why it cannot, or nullptr.
const char* handle_device_view(const apollo_dg* h, DgDev* d, int* eq, int* device, size_t* nU, size_t* nT);
void handle_set_error(apollo_dg* h, const char* msg);
bool handle_has_limiter(const apollo_dg* h);

}  // namespace apollo

namespace {

constexpr size_t kScratchBytes = (size_t)64 << 20;
constexpr size_t kHeader = 256;  // DevState for this call: lambda bits, error word

// Host code must not use this name as an address: it is a host-side stand-in.
// The device address comes from cudaGetSymbolAddress, taken once per device.
static __device__ __align__(256) unsigned char g_rhs_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
std::atomic<void*> g_scratch_ptr[kMaxDevices];

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// The device address of g_rhs_scratch on the current device (set up on first use).
cudaError_t scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  void* p = g_scratch_ptr[device].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    p = g_scratch_ptr[device].load(std::memory_order_relaxed);
    if (!p) {
      cudaError_t e = cudaGetSymbolAddress(&p, g_rhs_scratch);
      if (e != cudaSuccess) return e;
      g_scratch_ptr[device].store(p, std::memory_order_release);
    }
  }
  *out = p;
  return cudaSuccess;
}

}  // namespace

extern "C" apollo_status apollo_dg_rhs_noalloc(apollo_dg* h, double t, double dt, const double* in, double* out,
                                               double* suggested_dt, void* stream) {
  using namespace apollo;
  if (!h || !in || !out) return APOLLO_ERR_ARG;
  DgDev d;
  int eq = 0, device = 0;
  size_t nU = 0, nT = 0;
  if (handle_has_limiter(h)) {
    // the limiter needs scratch of its own; apollo_dg_rhs applies it
    handle_set_error(h, "apollo_dg_rhs_noalloc: the handle has a limiter; use apollo_dg_rhs");
    return APOLLO_ERR_STATE;
  }
  if (const char* why = handle_device_view(h, &d, &eq, &device, &nU, &nT)) {
    handle_set_error(h, (std::string("apollo_dg_rhs_noalloc: ") + why).c_str());
    return APOLLO_ERR_STATE;
  }
  const size_t need = kHeader + align256(nU * sizeof(double)) + 2 * align256(nT * sizeof(double));
  if (need > kScratchBytes) {
    handle_set_error(h, "apollo_dg_rhs_noalloc: this mesh needs more scratch than the 64 MiB static array; "
                        "use apollo_dg_rhs");
    return APOLLO_ERR_ARG;
  }
  if (cudaSetDevice(device) != cudaSuccess) return APOLLO_ERR_CUDA;
  void* base = nullptr;
  if (scratch_address(device, &base) != cudaSuccess) {
    handle_set_error(h, "apollo_dg_rhs_noalloc: cudaGetSymbolAddress failed");
    return APOLLO_ERR_CUDA;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (suggested_dt) {
    // the suggestion is read back after a wait on the stream, which a stream
    // being captured does not allow
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      handle_set_error(h, "apollo_dg_rhs_noalloc: suggested_dt needs a stream the call can wait on; pass NULL");
      return APOLLO_ERR_STATE;
    }
  }
  unsigned char* p = (unsigned char*)base;
  // per-call state starts at zero (wave-speed maximum, error word); the three
  // arrays are written in full by the kernels before they are read
  d.st = (DevState*)p;
  d.einst = nullptr;  // one DevState in the array's header: a single instance
  d.ninst = 1;
  d.vol = (double*)(p + kHeader);
  d.trace = (double*)(p + kHeader + align256(nU * sizeof(double)));
  d.flux = (double*)(p + kHeader + align256(nU * sizeof(double)) + align256(nT * sizeof(double)));
  if (cudaMemsetAsync(d.st, 0, sizeof(DevState), s) != cudaSuccess) return APOLLO_ERR_CUDA;
  StageArgs a{};
  a.x = in;
  a.out = out;
  a.mode = MODE_RHS;
  a.time_from_state = 0;
  a.t_arg = t;
  a.dt_arg = dt;
  a.reset_lambda = 1;
  if (launch_rhs_fp64(eq, d, a, s) != cudaSuccess) {
    handle_set_error(h, "apollo_dg_rhs_noalloc: kernel launch failed");
    return APOLLO_ERR_CUDA;
  }
  if (suggested_dt) {
    DevState st;
    if (cudaMemcpyAsync(&st, d.st, sizeof(DevState), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return APOLLO_ERR_CUDA;
    double lam;
    std::memcpy(&lam, &st.lam_bits, sizeof(double));
    *suggested_dt = d.dtfac * (d.rmin / lam);
    if (st.err & ERRB_NONPHYS) return APOLLO_ERR_NONPHYSICAL;
    if (st.err & ERRB_NAN) return APOLLO_ERR_NAN;
  }
  return APOLLO_OK;
}
