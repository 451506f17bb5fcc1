// mdx_solve_persistent_noalloc: the persistent refill solve for callers that
// cannot allocate device memory.
//
// Some hosts of this library hand it only the input and output buffers of a
// call and own every other byte of device memory themselves: a plugin or
// custom-call handler running inside a framework whose allocator must not be
// bypassed, code running while a memory pool is locked down, or a caller that
// simply has no allocator it is allowed to use at that point.  The ordinary
// persistent launch (mdx_solve with MDX_LAUNCH_PERSISTENT) needs a small caller-
// provided workspace for its work-queue head; this entry point instead takes
// that scratch from a fixed array that lives in the library itself, so the call
// allocates nothing.
//
// The scratch is the file-scope device array below, MDX_NOALLOC_SCRATCH_BYTES
// bytes on every GPU that loads the library, held until the process exits.
// Every call shares it: the queue head is cleared before each launch (on the
// caller's stream), and two calls whose kernels overlap on the GPU race on it.
// Its device address is looked up once per device (cudaGetSymbolAddress, with
// that device current) on the first call made on that device; make that first
// call before any stream capture.  The address is kept together with the ID of
// the context it was looked up in: if that context is torn down and the device
// gets a new one (cudaDeviceReset, or a framework releasing its context), the
// next call repeats the look-up instead of using an address of freed memory, and
// that call is then a first call again.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/menodax.h"
#include "mdx_internal.h"

static __device__ __align__(256) unsigned char mdx_noalloc_scratch[MDX_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct Scratch {
  unsigned long long ctx_id = 0;  // context the address belongs to (IDs start at 1)
  void* ptr = nullptr;
};
Scratch g_scratch[kMaxDevices];

// The scratch array's device address on `device` in the context `ctx_id`, set up
// on first use.  The array's name in host code only stands in for the symbol;
// the address comes from the runtime, with the device current.
int scratch_address(int device, unsigned long long ctx_id, void** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_scratch[device].ptr && g_scratch[device].ctx_id == ctx_id) {
    *out = g_scratch[device].ptr;
    return MDX_OK;
  }
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess)
    return mdx_internal::fail_message(MDX_E_CUDA, cudaGetErrorString(e));
  void* ptr = nullptr;
  e = cudaGetSymbolAddress(&ptr, mdx_noalloc_scratch);
  if (e != cudaSuccess || !ptr)
    return mdx_internal::fail_message(
        MDX_E_CUDA, e != cudaSuccess ? cudaGetErrorString(e) : "cudaGetSymbolAddress returned NULL");
  g_scratch[device].ctx_id = ctx_id;
  g_scratch[device].ptr = ptr;
  *out = ptr;
  return MDX_OK;
}

}  // namespace

extern "C" int mdx_solve_persistent_noalloc(mdx_plan* plan, const mdx_solve_desc* desc, void* stream) {
  if (!plan || !desc)
    return mdx_internal::fail_message(MDX_E_INVALID, "mdx_solve_persistent_noalloc: null argument");
  // The caller's struct must be this library's before any other field is read.
  if (desc->struct_size != (int)sizeof(mdx_solve_desc))
    return mdx_internal::fail_message(MDX_E_INVALID,
                                      "mdx_solve_persistent_noalloc: mdx_solve_desc.struct_size does not match "
                                      "this library's mdx_solve_desc");
  if (desc->mode != MDX_LAUNCH_PERSISTENT)
    return mdx_internal::fail_message(MDX_E_INVALID,
                                      "mdx_solve_persistent_noalloc: mode must be MDX_LAUNCH_PERSISTENT");
  size_t need = 0;
  int rc = mdx_workspace_size(plan, MDX_LAUNCH_PERSISTENT, desc->n_traj, &need);
  if (rc) return rc;
  if (need > (size_t)MDX_NOALLOC_SCRATCH_BYTES)
    return mdx_internal::fail_message(
        MDX_E_INVALID, "mdx_solve_persistent_noalloc: the solve needs more scratch than "
                       "MDX_NOALLOC_SCRATCH_BYTES; use mdx_solve with a caller workspace");
  int device = 0;
  bool primary = false;
  unsigned long long ctx_id = 0;
  if ((rc = mdx_internal::current_device(&device, &primary, &ctx_id))) return rc;
  if (!primary)
    return mdx_internal::fail_message(
        MDX_E_INVALID, "mdx_solve_persistent_noalloc needs the device's primary context to be current");
  if (device < 0 || device >= kMaxDevices)
    return mdx_internal::fail_message(MDX_E_INVALID, "device ordinal out of range");
  void* scratch = nullptr;
  if ((rc = scratch_address(device, ctx_id, &scratch))) return rc;
  return mdx_internal::solve_with_counter(plan, desc, stream, (int*)scratch);
}
