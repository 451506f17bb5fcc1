// menodax_b200 native runtime: NVRTC compilation, module lifetime and launches.
//
// Replaces the reference's native boundary, the XLA FFI handler that marshals
// buffers and calls cuLaunchKernel on XLA's stream
// (modax/_jax_numba_custom_call.py:66-231), and the ctypes cubin loader
// (compile_kernel, modax/_jax_numba_custom_call.py:286-314).
//
// The CUDA driver is reached through dlopen("libcuda.so.1") and
// cuGetProcAddress, resolved once under std::call_once, so the library loads on
// a machine without a GPU (NVRTC compilation works there; launches return
// MDX_E_NO_DRIVER).  A plan loads its cubin lazily, once per CUDA context.
#include "../../include/menodax.h"
#include "kernels/mdx_args.h"
#include "mdx_internal.h"

#include <cuda.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[2048];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

// --- driver entry points -------------------------------------------------------
struct Driver {
  bool ok = false;
  std::string why;
  decltype(&cuInit) init = nullptr;
  decltype(&cuCtxGetCurrent) ctxGetCurrent = nullptr;
  decltype(&cuCtxSetCurrent) ctxSetCurrent = nullptr;
  decltype(&cuCtxGetDevice) ctxGetDevice = nullptr;
  decltype(&cuCtxGetId) ctxGetId = nullptr;
  decltype(&cuCtxPushCurrent) ctxPushCurrent = nullptr;
  decltype(&cuCtxPopCurrent) ctxPopCurrent = nullptr;
  decltype(&cuDevicePrimaryCtxGetState) primaryCtxGetState = nullptr;
  decltype(&cuDeviceGet) deviceGet = nullptr;
  decltype(&cuDevicePrimaryCtxRetain) primaryCtxRetain = nullptr;
  decltype(&cuDevicePrimaryCtxRelease) primaryCtxRelease = nullptr;
  decltype(&cuDeviceGetAttribute) deviceGetAttribute = nullptr;
  decltype(&cuModuleLoadData) moduleLoadData = nullptr;
  decltype(&cuModuleUnload) moduleUnload = nullptr;
  decltype(&cuModuleGetFunction) moduleGetFunction = nullptr;
  decltype(&cuFuncSetAttribute) funcSetAttribute = nullptr;
  decltype(&cuLaunchKernel) launchKernel = nullptr;
  decltype(&cuMemsetD32Async) memsetD32Async = nullptr;
  decltype(&cuOccupancyMaxActiveBlocksPerMultiprocessor) occupancy = nullptr;
  decltype(&cuGetErrorString) getErrorString = nullptr;
  decltype(&cuPointerGetAttribute) pointerGetAttribute = nullptr;
};

Driver g_driver;
std::once_flag g_driver_once;

typedef CUresult (*GetProcFn)(const char*, void**, int, cuuint64_t, CUdriverProcAddressQueryResult*);

void load_driver() {
  void* lib = dlopen("libcuda.so.1", RTLD_NOW | RTLD_GLOBAL);
  if (!lib) {
    g_driver.why = std::string("cannot load libcuda.so.1: ") + dlerror();
    return;
  }
  GetProcFn get = (GetProcFn)dlsym(lib, "cuGetProcAddress_v2");
  if (!get) {
    g_driver.why = "libcuda.so.1 has no cuGetProcAddress_v2 (driver older than CUDA 12)";
    return;
  }
  bool all = true;
  auto resolve = [&](const char* name, void** slot) {
    CUdriverProcAddressQueryResult q;
    if (get(name, slot, 12000, CU_GET_PROC_ADDRESS_DEFAULT, &q) != CUDA_SUCCESS || !*slot) {
      g_driver.why = std::string("driver symbol missing: ") + name;
      all = false;
    }
  };
  resolve("cuInit", (void**)&g_driver.init);
  resolve("cuCtxGetCurrent", (void**)&g_driver.ctxGetCurrent);
  resolve("cuCtxSetCurrent", (void**)&g_driver.ctxSetCurrent);
  resolve("cuCtxGetDevice", (void**)&g_driver.ctxGetDevice);
  resolve("cuCtxGetId", (void**)&g_driver.ctxGetId);
  resolve("cuCtxPushCurrent", (void**)&g_driver.ctxPushCurrent);
  resolve("cuCtxPopCurrent", (void**)&g_driver.ctxPopCurrent);
  resolve("cuDevicePrimaryCtxGetState", (void**)&g_driver.primaryCtxGetState);
  resolve("cuDeviceGet", (void**)&g_driver.deviceGet);
  resolve("cuDevicePrimaryCtxRetain", (void**)&g_driver.primaryCtxRetain);
  resolve("cuDevicePrimaryCtxRelease", (void**)&g_driver.primaryCtxRelease);
  resolve("cuDeviceGetAttribute", (void**)&g_driver.deviceGetAttribute);
  resolve("cuModuleLoadData", (void**)&g_driver.moduleLoadData);
  resolve("cuModuleUnload", (void**)&g_driver.moduleUnload);
  resolve("cuModuleGetFunction", (void**)&g_driver.moduleGetFunction);
  resolve("cuFuncSetAttribute", (void**)&g_driver.funcSetAttribute);
  resolve("cuLaunchKernel", (void**)&g_driver.launchKernel);
  resolve("cuMemsetD32Async", (void**)&g_driver.memsetD32Async);
  resolve("cuOccupancyMaxActiveBlocksPerMultiprocessor", (void**)&g_driver.occupancy);
  resolve("cuGetErrorString", (void**)&g_driver.getErrorString);
  resolve("cuPointerGetAttribute", (void**)&g_driver.pointerGetAttribute);
  if (!all) return;
  if (g_driver.init(0) != CUDA_SUCCESS) {
    g_driver.why = "cuInit failed (no usable GPU)";
    return;
  }
  g_driver.ok = true;
}

int require_driver() {
  std::call_once(g_driver_once, load_driver);
  if (!g_driver.ok) return fail(MDX_E_NO_DRIVER, "%s", g_driver.why.c_str());
  return MDX_OK;
}

int cuda_fail(CUresult r, const char* what) {
  const char* s = nullptr;
  if (g_driver.getErrorString) g_driver.getErrorString(r, &s);
  return fail(MDX_E_CUDA, "%s failed: %s (%d)", what, s ? s : "unknown error", (int)r);
}

// The context launches go to: the calling thread's current one (torch makes the
// device's primary context current on first use).  With none current the call
// is refused rather than a context made current behind the caller's back.
int current_context(CUcontext* ctx) {
  CUresult r = g_driver.ctxGetCurrent(ctx);
  if (r != CUDA_SUCCESS) return cuda_fail(r, "cuCtxGetCurrent");
  if (!*ctx)
    return fail(MDX_E_INVALID,
                "no CUDA context is current on this thread; make the device's context current first "
                "(cudaSetDevice and any runtime call, or any torch CUDA operation)");
  return MDX_OK;
}

// A context's process-unique ID (cuCtxGetId): a context destroyed and created
// again at the same address gets a new one, so modules cached under the old ID
// are never launched in the new context.
int context_id(CUcontext ctx, unsigned long long* id) {
  CUresult r = g_driver.ctxGetId(ctx, id);
  if (r != CUDA_SUCCESS) return cuda_fail(r, "cuCtxGetId");
  return MDX_OK;
}

struct Loaded {
  CUcontext ctx = nullptr;
  CUdevice device = 0;
  bool primary = false;
  CUmodule module = nullptr;
  CUfunction plain = nullptr;
  CUfunction persistent = nullptr;
  CUfunction grad = nullptr;
  CUfunction combine = nullptr;  // thread adjoint modules: the split reverse's composition
  int sm_count = 0;
};

}  // namespace

struct mdx_plan {
  mdx_plan_desc desc;
  std::vector<char> cubin;
  std::mutex mu;
  std::unordered_map<unsigned long long, Loaded> loaded;  // by context ID
};

namespace {

// Unloads a module unless released: every error return after cuModuleLoadData
// leaves nothing loaded behind.
struct ModuleGuard {
  CUmodule module = nullptr;
  ~ModuleGuard() {
    if (module) g_driver.moduleUnload(module);
  }
};

int load_for_context(mdx_plan* plan, Loaded** out) {
  int rc = require_driver();
  if (rc) return rc;
  CUcontext ctx;
  if ((rc = current_context(&ctx))) return rc;
  unsigned long long id = 0;
  if ((rc = context_id(ctx, &id))) return rc;
  std::lock_guard<std::mutex> lock(plan->mu);
  auto it = plan->loaded.find(id);
  if (it != plan->loaded.end()) {
    *out = &it->second;
    return MDX_OK;
  }
  Loaded l;
  l.ctx = ctx;
  ModuleGuard guard;
  CUresult r = g_driver.moduleLoadData(&guard.module, plan->cubin.data());
  if (r != CUDA_SUCCESS) {
    guard.module = nullptr;
    return cuda_fail(r, "cuModuleLoadData");
  }
  if ((r = g_driver.moduleGetFunction(&l.plain, guard.module, "mdx_solve_plain")) != CUDA_SUCCESS)
    return cuda_fail(r, "cuModuleGetFunction(mdx_solve_plain)");
  if ((r = g_driver.moduleGetFunction(&l.persistent, guard.module, "mdx_solve_persistent")) != CUDA_SUCCESS)
    return cuda_fail(r, "cuModuleGetFunction(mdx_solve_persistent)");
  if (plan->desc.flags & MDX_PLAN_ADJOINT) {
    if ((r = g_driver.moduleGetFunction(&l.grad, guard.module, "mdx_grad_reverse")) != CUDA_SUCCESS)
      return cuda_fail(r, "cuModuleGetFunction(mdx_grad_reverse)");
    if (plan->desc.team_size == 1 &&
        (r = g_driver.moduleGetFunction(&l.combine, guard.module, "mdx_grad_combine")) != CUDA_SUCCESS)
      return cuda_fail(r, "cuModuleGetFunction(mdx_grad_combine)");
  }
  // Above the 48 KB default a kernel's dynamic shared memory has to be opted into.
  if (plan->desc.shared_bytes > 48 * 1024) {
    for (CUfunction f : {l.plain, l.persistent}) {
      r = g_driver.funcSetAttribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, plan->desc.shared_bytes);
      if (r != CUDA_SUCCESS) return cuda_fail(r, "cuFuncSetAttribute(MAX_DYNAMIC_SHARED_SIZE_BYTES)");
    }
  }
  if ((r = g_driver.ctxGetDevice(&l.device)) != CUDA_SUCCESS) return cuda_fail(r, "cuCtxGetDevice");
  if ((r = g_driver.deviceGetAttribute(&l.sm_count, CU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT, l.device)) != CUDA_SUCCESS)
    return cuda_fail(r, "cuDeviceGetAttribute");
  CUcontext primary = nullptr;
  if ((r = g_driver.primaryCtxRetain(&primary, l.device)) != CUDA_SUCCESS)
    return cuda_fail(r, "cuDevicePrimaryCtxRetain");
  g_driver.primaryCtxRelease(l.device);
  l.primary = primary == ctx;
  l.module = guard.module;
  guard.module = nullptr;
  auto res = plan->loaded.emplace(id, l);
  *out = &res.first->second;
  return MDX_OK;
}

// Unloads one plan module with its own context current.  A module whose context
// is gone went with it: a primary context that is inactive, or active under a
// new ID, is skipped, not pushed.
int unload_in_context(unsigned long long id, const Loaded& l) {
  CUcontext ctx = l.ctx;
  bool release = false;
  CUresult r;
  if (l.primary) {
    unsigned int flags = 0;
    int active = 0;
    if ((r = g_driver.primaryCtxGetState(l.device, &flags, &active)) != CUDA_SUCCESS)
      return cuda_fail(r, "cuDevicePrimaryCtxGetState");
    if (!active) return MDX_OK;
    if ((r = g_driver.primaryCtxRetain(&ctx, l.device)) != CUDA_SUCCESS)
      return cuda_fail(r, "cuDevicePrimaryCtxRetain");
    release = true;
    unsigned long long now = 0;
    if (g_driver.ctxGetId(ctx, &now) != CUDA_SUCCESS || now != id) {
      g_driver.primaryCtxRelease(l.device);
      return MDX_OK;
    }
  }
  int rc = MDX_OK;
  if ((r = g_driver.ctxPushCurrent(ctx)) != CUDA_SUCCESS) {
    rc = cuda_fail(r, "cuCtxPushCurrent");
  } else {
    if ((r = g_driver.moduleUnload(l.module)) != CUDA_SUCCESS) rc = cuda_fail(r, "cuModuleUnload");
    CUcontext popped;
    g_driver.ctxPopCurrent(&popped);
  }
  if (release) g_driver.primaryCtxRelease(l.device);
  return rc;
}

}  // namespace

extern "C" {

const char* mdx_version(void) { return "menodax_b200 1.0 (abi 1)"; }

int mdx_last_error(char* buf, size_t buf_size) {
  if (buf && buf_size) {
    size_t n = g_last_error.size() < buf_size - 1 ? g_last_error.size() : buf_size - 1;
    memcpy(buf, g_last_error.data(), n);
    buf[n] = '\0';
  }
  return (int)g_last_error.size();
}

void mdx_free(void* ptr) { free(ptr); }

int mdx_compile(const char* source, const char* program_name, const char* const* options,
                int n_options, void** cubin, size_t* cubin_size, char* log, size_t log_size) {
  if (!source || !cubin || !cubin_size) return fail(MDX_E_INVALID, "mdx_compile: null argument");
  if (n_options < 0 || (n_options > 0 && !options)) return fail(MDX_E_INVALID, "mdx_compile: bad options");
  *cubin = nullptr;
  *cubin_size = 0;
  if (log && log_size) log[0] = '\0';
  nvrtcProgram prog;
  nvrtcResult r = nvrtcCreateProgram(&prog, source, program_name ? program_name : "mdx_problem.cu",
                                     0, nullptr, nullptr);
  if (r != NVRTC_SUCCESS) return fail(MDX_E_COMPILE, "nvrtcCreateProgram: %s", nvrtcGetErrorString(r));
  r = nvrtcCompileProgram(prog, n_options, options);
  size_t n_log = 0;
  nvrtcGetProgramLogSize(prog, &n_log);
  std::string text(n_log, '\0');
  if (n_log) nvrtcGetProgramLog(prog, &text[0]);
  if (log && log_size) {
    size_t n = text.size() < log_size - 1 ? text.size() : log_size - 1;
    memcpy(log, text.data(), n);
    log[n] = '\0';
  }
  if (r != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    return fail(MDX_E_COMPILE, "NVRTC: %s\n%s", nvrtcGetErrorString(r), text.c_str());
  }
  size_t n = 0;
  r = nvrtcGetCUBINSize(prog, &n);
  if (r != NVRTC_SUCCESS || n == 0) {
    nvrtcDestroyProgram(&prog);
    return fail(MDX_E_COMPILE, "NVRTC produced no cubin (was -arch=sm_100a given?)");
  }
  void* buf = malloc(n);
  if (!buf) {
    nvrtcDestroyProgram(&prog);
    return fail(MDX_E_NOMEM, "out of host memory for the cubin");
  }
  nvrtcGetCUBIN(prog, (char*)buf);
  nvrtcDestroyProgram(&prog);
  *cubin = buf;
  *cubin_size = n;
  return MDX_OK;
}

int mdx_plan_create(const mdx_plan_desc* desc, mdx_plan** plan) {
  if (!desc || !plan) return fail(MDX_E_INVALID, "mdx_plan_create: null argument");
  if (desc->struct_size != (int)sizeof(mdx_plan_desc))
    return fail(MDX_E_INVALID, "mdx_plan_desc.struct_size %d != %d", desc->struct_size, (int)sizeof(mdx_plan_desc));
  if (desc->solver != MDX_SOLVER_TSIT5 && desc->solver != MDX_SOLVER_RODAS5P)
    return fail(MDX_E_INVALID, "unknown solver %d", desc->solver);
  if (desc->n_vars <= 0 || desc->n_system < desc->n_vars || desc->n_params < 0)
    return fail(MDX_E_INVALID, "bad sizes n_vars=%d n_system=%d n_params=%d", desc->n_vars, desc->n_system, desc->n_params);
  if (desc->threads_per_block <= 0 || desc->threads_per_block % 32 != 0 || desc->threads_per_block > 1024)
    return fail(MDX_E_INVALID, "threads_per_block must be a multiple of 32 in [32, 1024]; got %d", desc->threads_per_block);
  if (!desc->cubin || desc->cubin_size == 0) return fail(MDX_E_INVALID, "mdx_plan_create: empty cubin");
  if ((desc->flags & MDX_PLAN_CHECKPOINT) && desc->ckpt_stride < 1)
    return fail(MDX_E_INVALID, "a checkpointing plan needs ckpt_stride >= 1; got %d", desc->ckpt_stride);
  const int team = desc->team_size;
  if (team != 1 && team != 4 && team != 8 && team != 16 && team != 32)
    return fail(MDX_E_INVALID, "team_size must be 1, 4, 8, 16 or 32; got %d", team);
  if (desc->shared_bytes < 0 || desc->shared_bytes > MDX_MAX_SHARED_BYTES)
    return fail(MDX_E_INVALID, "shared_bytes must be in [0, %d]; got %d", MDX_MAX_SHARED_BYTES, desc->shared_bytes);
  mdx_plan* p = new (std::nothrow) mdx_plan;
  if (!p) return fail(MDX_E_NOMEM, "out of host memory");
  p->desc = *desc;
  p->cubin.assign((const char*)desc->cubin, (const char*)desc->cubin + desc->cubin_size);
  p->desc.cubin = nullptr;
  *plan = p;
  return MDX_OK;
}

int mdx_plan_destroy(mdx_plan* plan) {
  if (!plan) return MDX_OK;
  int rc = MDX_OK;
  if (g_driver.ok) {
    for (auto& kv : plan->loaded) {
      if (!kv.second.module) continue;
      const int r = unload_in_context(kv.first, kv.second);
      if (r && rc == MDX_OK) rc = r;
    }
  }
  delete plan;
  return rc;
}

int mdx_workspace_size(const mdx_plan* plan, int mode, int n_traj, size_t* bytes) {
  if (!plan || !bytes) return fail(MDX_E_INVALID, "mdx_workspace_size: null argument");
  if (n_traj < 0) return fail(MDX_E_INVALID, "n_traj must be non-negative");
  *bytes = mode == MDX_LAUNCH_PERSISTENT ? 256 : 0;
  return MDX_OK;
}

int mdx_checkpoint_size(const mdx_plan* plan, int n_traj, long long capacity, size_t* bytes) {
  if (!plan || !bytes) return fail(MDX_E_INVALID, "mdx_checkpoint_size: null argument");
  if (!(plan->desc.flags & MDX_PLAN_CHECKPOINT)) return fail(MDX_E_INVALID, "the plan records no checkpoints");
  if (n_traj < 0 || capacity < 0) return fail(MDX_E_INVALID, "n_traj and capacity must be non-negative");
  const long long stride = plan->desc.ckpt_stride;
  const long long segments = (capacity + stride - 1) / stride;
  *bytes = (size_t)8 * ((size_t)capacity * (size_t)n_traj +
                        (size_t)segments * (size_t)n_traj * (size_t)(plan->desc.n_vars + 1));
  return MDX_OK;
}

int mdx_occupancy(mdx_plan* plan, int mode, int* blocks_per_sm, int* sm_count) {
  if (!plan || !blocks_per_sm || !sm_count) return fail(MDX_E_INVALID, "mdx_occupancy: null argument");
  Loaded* l;
  int rc = load_for_context(plan, &l);
  if (rc) return rc;
  CUfunction f = mode == MDX_LAUNCH_PERSISTENT ? l->persistent : l->plain;
  CUresult r = g_driver.occupancy(blocks_per_sm, f, plan->desc.threads_per_block, (size_t)plan->desc.shared_bytes);
  if (r != CUDA_SUCCESS) return cuda_fail(r, "cuOccupancyMaxActiveBlocksPerMultiprocessor");
  *sm_count = l->sm_count;
  return MDX_OK;
}

}  // extern "C"

namespace {

// The device address of `bytes` of page-locked host memory at `p`, after
// checking that the whole range lies inside one allocation the driver maps: a
// kernel store to anything else would fault, so it is refused here instead.
int host_mapping(const void* p, size_t bytes, double** device_address) {
  const CUdeviceptr ptr = (CUdeviceptr)p;
  unsigned int type = 0;
  CUresult r = g_driver.pointerGetAttribute(&type, CU_POINTER_ATTRIBUTE_MEMORY_TYPE, ptr);
  if (r != CUDA_SUCCESS || type != CU_MEMORYTYPE_HOST)
    return fail(MDX_E_INVALID, "hist_host %p is not page-locked host memory the driver knows", p);
  CUdeviceptr start = 0;
  size_t size = 0;
  if ((r = g_driver.pointerGetAttribute(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, ptr)) != CUDA_SUCCESS)
    return cuda_fail(r, "cuPointerGetAttribute(hist_host, RANGE_START_ADDR)");
  if ((r = g_driver.pointerGetAttribute(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, ptr)) != CUDA_SUCCESS)
    return cuda_fail(r, "cuPointerGetAttribute(hist_host, RANGE_SIZE)");
  if (ptr < start || bytes > size || ptr - start > size - bytes)
    return fail(MDX_E_INVALID, "hist_host: %zu bytes at %p run past its page-locked allocation (%zu bytes at %p)",
                bytes, p, size, (void*)start);
  CUdeviceptr mapped = 0;
  if ((r = g_driver.pointerGetAttribute(&mapped, CU_POINTER_ATTRIBUTE_DEVICE_POINTER, ptr)) != CUDA_SUCCESS)
    return cuda_fail(r, "cuPointerGetAttribute(hist_host, DEVICE_POINTER)");
  *device_address = (double*)mapped;
  return MDX_OK;
}

}  // namespace

namespace mdx_internal {

// The body of mdx_solve.  `counter` (when not NULL) replaces the caller's
// workspace as the persistent kernel's queue head.
int solve_with_counter(mdx_plan* plan, const mdx_solve_desc* d, void* stream, int* counter) {
  if (!plan || !d) return fail(MDX_E_INVALID, "mdx_solve: null argument");
  if (d->struct_size != (int)sizeof(mdx_solve_desc))
    return fail(MDX_E_INVALID, "mdx_solve_desc.struct_size %d != %d", d->struct_size, (int)sizeof(mdx_solve_desc));
  if (d->n_traj < 0) return fail(MDX_E_INVALID, "n_traj must be non-negative; got %d", d->n_traj);
  if (d->n_save < 1) return fail(MDX_E_INVALID, "times must hold at least one value; got %d", d->n_save);
  if (d->mode != MDX_LAUNCH_PLAIN && d->mode != MDX_LAUNCH_PERSISTENT)
    return fail(MDX_E_INVALID, "unknown launch mode %d", d->mode);
  if (d->n_traj == 0) return MDX_OK;
  if (!d->y0 || !d->times || (plan->desc.n_params > 0 && !d->params) || !d->hist || !d->accepted ||
      !d->rejected || !d->loop_steps)
    return fail(MDX_E_INVALID, "mdx_solve: a required buffer is NULL");
  if ((plan->desc.flags & MDX_PLAN_SAVE_HOOK) && !d->hook_out)
    return fail(MDX_E_INVALID, "the plan calls a save hook: hook_out must not be NULL");
  if ((plan->desc.flags & MDX_PLAN_NO_HISTORY) ? d->n_save_hist != 1 : d->n_save_hist != d->n_save)
    return fail(MDX_E_INVALID, "n_save_hist %d does not match the plan's history (%s)", d->n_save_hist,
                (plan->desc.flags & MDX_PLAN_NO_HISTORY) ? "final state only" : "every save");
  const bool ckpt = (plan->desc.flags & MDX_PLAN_CHECKPOINT) != 0;
  if (ckpt && (!d->ckpt || !d->ckpt_count || d->ckpt_capacity < 1))
    return fail(MDX_E_INVALID, "a checkpointing plan needs ckpt, ckpt_count and ckpt_capacity >= 1");
  if (d->mode == MDX_LAUNCH_PERSISTENT && !counter && (!d->workspace || d->workspace_bytes < 4))
    return fail(MDX_E_INVALID, "the persistent launch needs a workspace of at least 4 bytes");
  double* hist_host = nullptr;
  if (d->hist_host) {
    int rc = require_driver();
    if (rc) return rc;
    const size_t bytes = (size_t)d->n_traj * (size_t)d->n_save_hist * (size_t)plan->desc.n_system * sizeof(double);
    if ((rc = host_mapping(d->hist_host, bytes, &hist_host))) return rc;
  }

  Loaded* l;
  int rc = load_for_context(plan, &l);
  if (rc) return rc;

  MdxSolveArgs a;
  memset(&a, 0, sizeof(a));
  a.y0 = d->y0;
  a.times = d->times;
  a.params = d->params;
  a.weights = d->weights;
  a.hist = d->hist;
  a.accepted = d->accepted;
  a.rejected = d->rejected;
  a.loop_steps = d->loop_steps;
  a.status = d->status;
  a.hook_out = d->hook_out;
  a.order = d->order;
  a.ckpt = ckpt ? d->ckpt : nullptr;
  a.ckpt_count = ckpt ? d->ckpt_count : nullptr;
  a.ckpt_capacity = ckpt ? d->ckpt_capacity : 0;
  a.hist_host = hist_host;
  a.n_traj = d->n_traj;
  a.n_save = d->n_save;
  a.n_save_hist = d->n_save_hist;
  a.max_steps = d->max_steps;
  a.dt0 = d->dt0;
  a.rtol = d->rtol;
  a.atol = d->atol;

  const unsigned tpb = (unsigned)plan->desc.threads_per_block;
  const unsigned smem = (unsigned)plan->desc.shared_bytes;
  // Trajectories per block: one per thread, or one per team of team_size lanes.
  const int per_block = (int)tpb / plan->desc.team_size;
  CUstream s = (CUstream)stream;
  CUfunction f;
  unsigned grid;
  if (d->mode == MDX_LAUNCH_PLAIN) {
    f = l->plain;
    grid = (unsigned)((d->n_traj + per_block - 1) / per_block);
  } else {
    f = l->persistent;
    a.work_counter = counter ? counter : (int*)d->workspace;
    int blocks = d->grid_blocks;
    if (blocks <= 0) {
      int per_sm = 0;
      CUresult r = g_driver.occupancy(&per_sm, f, (int)tpb, (size_t)smem);
      if (r != CUDA_SUCCESS) return cuda_fail(r, "cuOccupancyMaxActiveBlocksPerMultiprocessor");
      if (per_sm < 1) per_sm = 1;
      blocks = per_sm * l->sm_count;
    }
    const int needed = (d->n_traj + per_block - 1) / per_block;
    if (blocks > needed) blocks = needed;
    grid = (unsigned)blocks;
    CUresult r = g_driver.memsetD32Async((CUdeviceptr)a.work_counter, 0u, 1, s);
    if (r != CUDA_SUCCESS) return cuda_fail(r, "cuMemsetD32Async(work counter)");
  }
  void* params[] = {&a};
  CUresult r = g_driver.launchKernel(f, grid, 1, 1, tpb, 1, 1, smem, s, params, nullptr);
  if (r != CUDA_SUCCESS) return cuda_fail(r, "cuLaunchKernel(mdx_solve)");
  return MDX_OK;
}

int current_device(int* device, bool* is_primary, unsigned long long* ctx_id) {
  int rc = require_driver();
  if (rc) return rc;
  CUcontext ctx;
  if ((rc = current_context(&ctx))) return rc;
  if (ctx_id && (rc = context_id(ctx, ctx_id))) return rc;
  CUresult r;
  CUdevice dev;
  if ((r = g_driver.ctxGetDevice(&dev)) != CUDA_SUCCESS) return cuda_fail(r, "cuCtxGetDevice");
  CUcontext primary;
  if ((r = g_driver.primaryCtxRetain(&primary, dev)) != CUDA_SUCCESS) return cuda_fail(r, "cuDevicePrimaryCtxRetain");
  g_driver.primaryCtxRelease(dev);
  *device = (int)dev;
  *is_primary = primary == ctx;
  return MDX_OK;
}

int fail_message(int code, const char* message) { return fail(code, "%s", message); }

}  // namespace mdx_internal

extern "C" {

int mdx_solve(mdx_plan* plan, const mdx_solve_desc* d, void* stream) {
  return mdx_internal::solve_with_counter(plan, d, stream, nullptr);
}

int mdx_grad(mdx_plan* plan, const mdx_grad_desc* d, void* stream) {
  if (!plan || !d) return fail(MDX_E_INVALID, "mdx_grad: null argument");
  if (d->struct_size != (int)sizeof(mdx_grad_desc))
    return fail(MDX_E_INVALID, "mdx_grad_desc.struct_size %d != %d", d->struct_size, (int)sizeof(mdx_grad_desc));
  if (!(plan->desc.flags & MDX_PLAN_ADJOINT)) return fail(MDX_E_INVALID, "the plan was built without the adjoint kernel");
  if (d->n_traj < 0 || d->n_save < 1) return fail(MDX_E_INVALID, "bad sizes n_traj=%d n_save=%d", d->n_traj, d->n_save);
  if (d->count < 0 || d->count > d->n_traj)
    return fail(MDX_E_INVALID, "mdx_grad: count %d outside [0, n_traj = %d]", d->count, d->n_traj);
  const bool split = d->tasks != nullptr;
  if (split) {
    if (plan->desc.team_size != 1)
      return fail(MDX_E_INVALID, "mdx_grad: the split reverse needs a one-thread-per-trajectory plan");
    if (d->n_tasks < 0 || d->n_slots < 0 || d->n_combine < 0 || (d->n_slots > 0 && !d->task_out) ||
        (d->n_combine > 0 && !d->combine))
      return fail(MDX_E_INVALID, "mdx_grad: split reverse needs n_tasks, n_slots, n_combine >= 0 and "
                  "task_out / combine when slots / combinations are used");
    if (d->n_combine > 0 && d->n_combine * (plan->desc.n_vars + 1) > d->n_slots)
      return fail(MDX_E_INVALID, "mdx_grad: %d combinations need at least %d slots; got %d", d->n_combine,
                  d->n_combine * (plan->desc.n_vars + 1), d->n_slots);
  }
  if (d->n_traj == 0) return MDX_OK;
  if (!d->times || !d->ckpt || !d->ckpt_count || !d->grad_hist || !d->grad_y0 || !d->grad_params ||
      d->ckpt_capacity < 1)
    return fail(MDX_E_INVALID, "mdx_grad: a required buffer is NULL");
  Loaded* l;
  int rc = load_for_context(plan, &l);
  if (rc) return rc;
  MdxGradArgs a;
  memset(&a, 0, sizeof(a));
  a.times = d->times;
  a.params = d->params;
  a.ckpt = d->ckpt;
  a.ckpt_count = d->ckpt_count;
  a.grad_hist = d->grad_hist;
  a.grad_y0 = d->grad_y0;
  a.grad_params = d->grad_params;
  a.status = d->status;
  a.order = d->order;
  a.ckpt_capacity = d->ckpt_capacity;
  a.n_traj = d->n_traj;
  a.n_save = d->n_save;
  a.n_run = d->count > 0 ? d->count : d->n_traj;
  if (split) {
    a.order = nullptr;
    a.tasks = d->tasks;
    a.task_out = d->task_out;
    a.combine = d->combine;
    a.n_slots = d->n_slots;
    a.n_combine = d->n_combine;
    a.n_run = d->n_tasks;
  }
  const unsigned tpb = (unsigned)plan->desc.threads_per_block;
  // Trajectories per block: one per thread, or one per team of team_size lanes.
  const unsigned per_block = tpb / (unsigned)plan->desc.team_size;
  void* params[] = {&a};
  CUresult r;
  if (a.n_run > 0) {
    const unsigned grid = (unsigned)((a.n_run + per_block - 1) / per_block);
    r = g_driver.launchKernel(l->grad, grid, 1, 1, tpb, 1, 1, 0, (CUstream)stream, params, nullptr);
    if (r != CUDA_SUCCESS) return cuda_fail(r, "cuLaunchKernel(mdx_grad_reverse)");
  }
  if (split && a.n_combine > 0) {
    const unsigned grid = (unsigned)((a.n_combine + tpb - 1) / tpb);
    r = g_driver.launchKernel(l->combine, grid, 1, 1, tpb, 1, 1, 0, (CUstream)stream, params, nullptr);
    if (r != CUDA_SUCCESS) return cuda_fail(r, "cuLaunchKernel(mdx_grad_combine)");
  }
  return MDX_OK;
}

}  // extern "C"
