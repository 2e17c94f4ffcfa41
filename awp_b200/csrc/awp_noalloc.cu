// Allocation-free non-finite check of caller-owned device fields.
//
// Who needs it: a caller that already owns every byte of device memory it may
// use and must not ask the CUDA allocator for more -- for example a host code
// that hands this library fields carved out of its own pre-reserved pool (the
// padded wavefield of a large run can take most of the 180 GB), or a watchdog
// thread that checks the wavefield between time steps of a running simulation,
// where a cudaMalloc/cudaFree pair could fail on a full device or (cudaFree)
// wait for the whole device.  awp_check_finite needs a context, and a context
// allocates; this entry point allocates nothing.
//
// Scratch: the k_nonfinite kernel's per-field flags live in the file-scope
// array below, AWP_NOALLOC_MAX_FIELDS words.  Every GPU that loads the library
// holds it until the process exits.  Its device address is looked up once per
// device (on the first call made with that device current) and cached.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "../../include/awp_b200.h"
#include "awp_kernels.cuh"

void awp_internal_set_error(const char* msg);  // awp_capi.cu

namespace {

static __device__ __align__(256) unsigned int g_nonfinite_scratch[AWP_NOALLOC_MAX_FIELDS];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned int* g_scratch_ptr[kMaxDevices] = {};

// the detail goes to the library's last-error text (awp_last_error)
int fail(int status, const char* msg, cudaError_t e = cudaSuccess) {
  char buf[256];
  if (e != cudaSuccess)
    snprintf(buf, sizeof(buf), "awp_check_finite_noalloc: %s: %s", msg, cudaGetErrorString(e));
  else
    snprintf(buf, sizeof(buf), "awp_check_finite_noalloc: %s", msg);
  awp_internal_set_error(buf);
  return status;
}

// Device address of the scratch array on the current device (set-up once per
// device; cudaGetSymbolAddress allocates nothing).
int scratch_on_current_device(unsigned int** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(AWP_ERR_CUDA, "cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDevices) return fail(AWP_ERR_UNSUPPORTED, "device ordinal >= 64");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_nonfinite_scratch);
    if (e != cudaSuccess || !p) return fail(AWP_ERR_CUDA, "cudaGetSymbolAddress", e);
    g_scratch_ptr[dev] = static_cast<unsigned int*>(p);
  }
  *out = g_scratch_ptr[dev];
  return AWP_OK;
}

}  // namespace

extern "C" int awp_check_finite_noalloc(const float* const* fields, int nfields, long long n,
                                        int* ok, void* stream) {
  if (!fields || !ok || n < 0) return fail(AWP_ERR_ARG, "null argument or negative size");
  if (nfields < 1 || nfields > AWP_NOALLOC_MAX_FIELDS)
    return fail(AWP_ERR_ARG, "nfields must be 1..AWP_NOALLOC_MAX_FIELDS (32)");
  // every argument is checked before any work is queued on the stream
  for (int f = 0; f < nfields; ++f)
    if (!fields[f]) return fail(AWP_ERR_ARG, "null field pointer");
  unsigned int* scratch = nullptr;
  int st = scratch_on_current_device(&scratch);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the array keeps the previous call's flags: clear the words this call uses
  cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned int) * nfields, s);
  if (e != cudaSuccess) return fail(AWP_ERR_CUDA, "cudaMemsetAsync", e);
  for (int f = 0; f < nfields; ++f) {
    e = awp_launch_nonfinite(fields[f], n, scratch + f, s);
    if (e != cudaSuccess) return fail(AWP_ERR_CUDA, "k_nonfinite launch", e);
  }
  unsigned int flags[AWP_NOALLOC_MAX_FIELDS];
  e = cudaMemcpyAsync(flags, scratch, sizeof(unsigned int) * nfields, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return fail(AWP_ERR_CUDA, "cudaMemcpyAsync", e);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(AWP_ERR_CUDA, "cudaStreamSynchronize", e);
  for (int f = 0; f < nfields; ++f) ok[f] = flags[f] ? 0 : 1;
  return AWP_OK;
}
