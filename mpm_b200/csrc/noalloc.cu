// noalloc.cu -- Material<Tdim>::compute_stress on a batch of points without
// allocating device memory.
//
// Some callers cannot call cudaMalloc: a constitutive-model plugin invoked from
// inside another solver's time loop that owns all device memory through its own
// arena (an allocation there would bypass the arena's accounting or fail once
// it holds the whole device), or a real-time loop that must not pay for, or
// fail on, an allocation.  This entry point serves them: the points are staged
// in one fixed array that is part of the library's device image, so the call
// allocates nothing.  It copies synchronously and launches on the legacy
// default stream, so it is an ordinary blocking call, not one to make while a
// stream capture is in progress.
//
// The array holds MPM_NOALLOC_MAX_POINTS points (28 doubles each, 7.3 MB).  Every
// GPU that loads the library holds it until the process exits.  All calls on a
// device share it and it keeps the previous call's contents: nothing in it has
// to start at zero (every value the kernel reads is copied in by the same call,
// and every value returned is written by it).  Calls that overlapped on the GPU
// would race on the array; this entry point holds a lock per device and
// finishes its copies before returning, so calls made through it on one device
// never overlap (calls on different devices use different copies of the array
// and run concurrently).  The first call on a device looks up the array's
// device address (cudaGetSymbolAddress) with that device current and keeps
// it; make that first call before any stream capture begins, and do not reset
// the device (cudaDeviceReset) after it, since the reset reloads the device
// image and can move the array.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/mpm_gpu.h"
#include "mpm_kernels.h"

#ifndef MPM_NOALLOC_MAX_POINTS
#define MPM_NOALLOC_MAX_POINTS 32768
#endif

namespace mpm_b200 {
// defined in mpm_gpu.cu: the material factory of the C ABI
MaterialParams material_from_json(int dim, const char* type, const char* json_props);
}  // namespace mpm_b200

namespace {

constexpr int64_t kMaxPoints = MPM_NOALLOC_MAX_POINTS;
// per point: stress 6, strain increment 6, density 1, state 9, result 6
constexpr int64_t kOffStress = 0, kOffDstrain = 6 * kMaxPoints, kOffDensity = 12 * kMaxPoints,
                  kOffState = 13 * kMaxPoints, kOffOut = 22 * kMaxPoints,
                  kScratchDoubles = 28 * kMaxPoints;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_lock[kMaxDevices];    // one per device: its copy of the array
double* g_noalloc_addr[kMaxDevices] = {};  // device address of the array, per device

void set_err(char* err, int64_t errlen, const std::string& msg) {
  if (!err || errlen <= 0) return;
  std::snprintf(err, (size_t)errlen, "%s", msg.c_str());
}

}  // namespace

extern "C" int mpm_gpu_material_stress_batch_noalloc(int32_t device, int32_t dim, const char* type,
                                                     const char* json_props, int64_t n,
                                                     const double* stress, const double* dstrain,
                                                     const double* density, double* state,
                                                     double* out, char* err, int64_t errlen) {
  set_err(err, errlen, "");
  if (dim != 2 && dim != 3) {
    set_err(err, errlen, "dim must be 2 or 3");
    return MPM_ERR_INVALID;
  }
  if (n < 0 || !type || !json_props ||
      (n > 0 && (!stress || !dstrain || !density || !state || !out))) {
    set_err(err, errlen, "null argument or negative point count");
    return MPM_ERR_INVALID;
  }
  if (n > kMaxPoints) {
    set_err(err, errlen,
            "n = " + std::to_string(n) + " exceeds the maximum of " + std::to_string(kMaxPoints) +
                " points of mpm_gpu_material_stress_batch_noalloc; split the batch");
    return MPM_ERR_INVALID;
  }
  if (device < 0 || device >= kMaxDevices) {
    set_err(err, errlen, "device ordinal out of range");
    return MPM_ERR_INVALID;
  }
  mpm_b200::MaterialParams m;
  try {
    m = mpm_b200::material_from_json(dim, type, json_props);
  } catch (const std::exception& e) {
    set_err(err, errlen, e.what());
    return MPM_ERR_INVALID;
  }
  if (n == 0) return MPM_OK;

  std::lock_guard<std::mutex> guard(g_noalloc_lock[device]);
  int prev = -1;
  cudaGetDevice(&prev);
  auto fail = [&](cudaError_t e, const char* what) {
    set_err(err, errlen, std::string(what) + ": " + cudaGetErrorString(e));
    if (prev >= 0) cudaSetDevice(prev);
    return MPM_ERR_CUDA;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(e, "cudaSetDevice");
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(e, "cudaGetSymbolAddress");
    g_noalloc_addr[device] = static_cast<double*>(p);
  }
  double* base = g_noalloc_addr[device];
  double* d_stress = base + kOffStress;
  double* d_dstrain = base + kOffDstrain;
  double* d_density = base + kOffDensity;
  double* d_state = base + kOffState;
  double* d_out = base + kOffOut;
  const size_t b6 = sizeof(double) * 6 * (size_t)n, b1 = sizeof(double) * (size_t)n,
               b9 = sizeof(double) * 9 * (size_t)n;
  if ((e = cudaMemcpy(d_stress, stress, b6, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(d_dstrain, dstrain, b6, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(d_density, density, b1, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(d_state, state, b9, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(e, "staging copy to the device");
  // the same kernel as mpm_gpu_material_stress_batch, on the legacy default stream
  mpm_b200::launch_material_batch_fp64(dim, n, m, d_stress, d_dstrain, d_density, d_state, d_out,
                                       0);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "kernel launch");
  if ((e = cudaMemcpy(out, d_out, b6, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(state, d_state, b9, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail(e, "copy of the results to the host");
  if (prev >= 0) cudaSetDevice(prev);
  return MPM_OK;
}
