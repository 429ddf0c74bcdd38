// Allocation-free internal-force evaluation (dl_internal_force_static).
//
// Some callers cannot allocate device memory at the point where they need the
// internal force: a real-time control loop with a fixed memory budget (a
// cudaMalloc may synchronise the device and blow the loop's deadline), or a
// host framework that owns every device allocation and forbids others once it
// has started.  This entry point runs the same element-force and gather
// kernels as dl_internal_force, but its scratch memory -- the configuration
// in the engine's node layout and the element-end force slots -- lives in one
// file-scope static device array of fixed size (kStaticScratchBytes per GPU,
// held from library load until process exit), and the caller passes device
// input and output arrays.  Nothing is allocated: no cudaMalloc, no cudaFree.
//
// The array is shared by every call on a device and keeps the last call's
// contents; each call overwrites all of the scratch it reads (every slot is
// written by exactly one element end), so nothing needs clearing.  Calls whose
// GPU work overlaps (different streams, or different handles on one device)
// race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>

#include "devtypes.cuh"
#include "engine.hpp"
#include "noalloc.hpp"

namespace dl {

namespace {

__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_ptr[kMaxDevices] = {};

size_t round_up(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

// Makes `dev` the current device for the guard's lifetime and restores the
// caller's device afterwards.
struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      ok = false;
      prev = -1;
      return;
    }
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) {
      cudaGetLastError();
      ok = false;
    }
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

int static_scratch_address(int dev, void **ptr, const char **why) {
  if (dev < 0 || dev >= kMaxDevices) {
    *why = "device index beyond the static scratch table";
    return DL_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    // once per device, with that device current (the caller's DeviceGuard):
    // the host-side name of the array is not a device address
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != dev) {
      cudaGetLastError();
      *why = "static scratch address requested for a device that is not current";
      return DL_ERR_CUDA;
    }
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess) {
      cudaGetLastError();
      *why = "cudaGetSymbolAddress of the static scratch array failed";
      return DL_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *ptr = g_scratch_ptr[dev];
  return DL_OK;
}

template <class T>
int internal_force_static(const KernelSet &ks, const DevModel<T> &model, int device, const double *X0int,
                          const int32_t *node_old, const double *u, const double *theta, double *fint,
                          cudaStream_t stream, const char **why) {
  const int N = model.N, E = model.E;
  const size_t pos_bytes = round_up(static_cast<size_t>(N) * sizeof(double4));
  const size_t ef_bytes = round_up(static_cast<size_t>(E) * 6 * model.nen * sizeof(T));  // a slot per element node
  if (2 * pos_bytes + ef_bytes > kStaticScratchBytes) {
    *why = "lattice too large for the static scratch array (see kStaticScratchBytes)";
    return DL_ERR_INVALID;
  }
  // the handle's arrays and stream belong to the device it was created on
  DeviceGuard guard(device);
  if (!guard.ok) {
    *why = "cannot make the handle's device current";
    return DL_ERR_CUDA;
  }
  void *base = nullptr;
  int rc = static_scratch_address(device, &base, why);
  if (rc) return rc;
  unsigned char *p = static_cast<unsigned char *>(base);
  DevModel<T> m = model;
  m.pos = reinterpret_cast<double4 *>(p);
  m.rot = reinterpret_cast<double4 *>(p + pos_bytes);
  m.ef = reinterpret_cast<T *>(p + 2 * pos_bytes);
  // configuration -> engine layout (same conversion as dl_set_state)
  cudaError_t e = launch_state_in(m.pos, m.rot, nullptr, X0int, node_old, N, u, theta, nullptr, stream);
  if (e != cudaSuccess) {
    *why = cudaGetErrorString(e);
    return DL_ERR_CUDA;
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (sms <= 0) sms = 1;
  const int eb = std::min((E + 255) / 256, sms * 8);
  void *args[] = {&m};
  e = cudaLaunchKernel(ks.internal_force, dim3(eb > 0 ? eb : 1), dim3(256), args, 0, stream);
  if (e != cudaSuccess) {
    *why = cudaGetErrorString(e);
    return DL_ERR_CUDA;
  }
  // the ordinary gather kernel, writing each node's row in the caller's numbering
  const int nb = std::min((N + 255) / 256, sms * 8);
  double *out = fint;
  const int32_t *perm = node_old;
  void *gargs[] = {&m, &out, &perm};
  e = cudaLaunchKernel(ks.gather, dim3(nb > 0 ? nb : 1), dim3(256), gargs, 0, stream);
  if (e != cudaSuccess) {
    *why = cudaGetErrorString(e);
    return DL_ERR_CUDA;
  }
  return DL_OK;
}

template int internal_force_static<float>(const KernelSet &, const DevModel<float> &, int, const double *,
                                          const int32_t *, const double *, const double *, double *,
                                          cudaStream_t, const char **);
template int internal_force_static<double>(const KernelSet &, const DevModel<double> &, int, const double *,
                                           const int32_t *, const double *, const double *, double *,
                                           cudaStream_t, const char **);

}  // namespace dl
