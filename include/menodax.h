/* menodax_b200 C ABI: ensemble ODE integration on one B200 (sm_100a).
 *
 * This is the boundary a host framework binds.  It replaces the reference's
 * device-launch boundary, which is
 *   - the XLA FFI handler `modax_numba_cuda_abi_launch`
 *     (modax/_jax_numba_custom_call.py:145-231): buffers + attrs -> cuLaunchKernel
 *     of a numba-compiled cubin on XLA's stream, errors as ffi::Error;
 *   - its Python callers `ensemble_ffi_call` / `ffi_abi_call`
 *     (modax/_numba_common.py:84-130, modax/_jax_numba_custom_call.py:333-371),
 *     which fix the argument order y0, times, params, dt0, rtol, atol, max_steps,
 *     weights -> hist, accepted, rejected, loop_steps (modax/_numba_common.py:27-40);
 *   - cubin loading and function lookup `compile_kernel`
 *     (modax/_jax_numba_custom_call.py:286-314).
 *
 * Conventions: plain C types only; every call returns an int status (MDX_OK or a
 * negative MDX_E_* code) and never aborts or traps; mdx_last_error() gives the
 * calling thread's last message.  Device buffers are owned by the caller; a plan
 * owns its compiled modules.  Arrays are row-major, the trajectory index slowest.
 * `stream` is a CUstream / cudaStream_t (NULL = legacy default stream).
 */
#ifndef MENODAX_H
#define MENODAX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MDX_ABI_VERSION 1

#define MDX_OK 0
#define MDX_E_INVALID (-1)     /* bad argument (ffi::ErrorCode::kInvalidArgument) */
#define MDX_E_COMPILE (-2)     /* NVRTC rejected the source */
#define MDX_E_CUDA (-3)        /* a CUDA driver call failed (ffi::ErrorCode::kInternal) */
#define MDX_E_NO_DRIVER (-4)   /* libcuda.so.1 could not be loaded */
#define MDX_E_NOMEM (-5)

#define MDX_SOLVER_TSIT5 1
#define MDX_SOLVER_RODAS5P 2

#define MDX_LAUNCH_PLAIN 0      /* one trajectory per thread (or team) for its whole life */
#define MDX_LAUNCH_PERSISTENT 1 /* device-sized grid, warps refill from a queue */

/* Largest dynamic shared memory per block a plan may ask for (sm_100 opt-in). */
#define MDX_MAX_SHARED_BYTES (227 * 1024)

#define MDX_PLAN_CHECKPOINT 1   /* the module records accepted step states */
#define MDX_PLAN_ADJOINT 2      /* the module carries the discrete-adjoint kernel */
#define MDX_PLAN_SAVE_HOOK 4    /* the module calls a save hook: hook_out is required */
#define MDX_PLAN_NO_HISTORY 8   /* the module keeps only the final state: n_save_hist == 1 */

/* Per-trajectory status bits written to mdx_solve_desc.status. */
#define MDX_STATUS_OK 0
#define MDX_STATUS_MAX_STEPS 1
#define MDX_STATUS_NONFINITE 2
#define MDX_STATUS_CKPT_OVERFLOW 4

typedef struct mdx_plan mdx_plan;

/* A compiled problem.  `cubin` is the output of mdx_compile for the source the
 * Python host generates from a traced right-hand side; it is copied.  Replaces
 * the cubin + CUfunction pair modax keeps per kernel (compile_kernel,
 * modax/_jax_numba_custom_call.py:286-314). */
typedef struct mdx_plan_desc {
  int struct_size;        /* sizeof(mdx_plan_desc) */
  int solver;             /* MDX_SOLVER_* */
  int n_vars;             /* state components of the base system */
  int n_system;           /* integrated components (n_vars * (1 + n_sens)) */
  int n_params;
  int threads_per_block;  /* the block size the module was compiled for */
  int flags;              /* MDX_PLAN_* */
  int ckpt_stride;        /* MDX_PLAN_CHECKPOINT: steps per recorded start state (>= 1) */
  int team_size;          /* lanes per trajectory: 1 for the thread-per-trajectory kernels, 4, 8,
                             16 or 32 for a team module (threads_per_block / team_size
                             trajectories per block) */
  int shared_bytes;       /* dynamic shared memory per block the module's solve kernels take */
  const void* cubin;
  size_t cubin_size;
} mdx_plan_desc;

/* One ensemble solve: the reference's SOLVER_ARGTYPES plus a status array, an
 * optional persistent-kernel workspace and optional checkpoint buffers. */
typedef struct mdx_solve_desc {
  int struct_size;        /* sizeof(mdx_solve_desc) */
  int mode;               /* MDX_LAUNCH_* */
  int n_traj;
  int n_save;             /* len(times) */
  int n_save_hist;        /* rows of hist per trajectory: n_save, or 1 without history */
  int max_steps;
  double dt0;             /* <= 0: 1e-6 of the integration window */
  double rtol;
  double atol;
  const double* y0;       /* (n_traj, n_system) */
  const double* times;    /* (n_save,) */
  const double* params;   /* (n_traj, n_params) */
  const double* weights;  /* (n_traj, n_system), or NULL for constant weights */
  double* hist;           /* (n_traj, n_save_hist, n_system) */
  int* accepted;          /* (n_traj,) */
  int* rejected;          /* (n_traj,) */
  int* loop_steps;        /* (n_traj,) */
  int* status;            /* (n_traj,) or NULL */
  double* hook_out;       /* MDX_PLAN_SAVE_HOOK: (n_traj, hook_size), zeroed and filled by the kernel */
  const int* order;       /* persistent: optional trajectory visiting order, or NULL */
  void* workspace;        /* persistent: >= mdx_workspace_size() bytes */
  size_t workspace_bytes;
  double* ckpt;           /* MDX_PLAN_CHECKPOINT: mdx_checkpoint_size() bytes */
  int* ckpt_count;        /* MDX_PLAN_CHECKPOINT: (n_traj,) */
  long long ckpt_capacity;
  int grid_blocks;        /* persistent: 0 = occupancy-sized */
  int reserved;
  double* hist_host;      /* optional page-locked host copy of hist, same layout, or NULL.
                             When set, the kernel copies each trajectory's history rows
                             there as soon as they are final (a whole warp's contiguous
                             rows at once in the one-trajectory-per-thread launch), so the
                             transfer over the host link overlaps the trajectories still
                             running; the host copy is complete when the stream is.  The
                             buffer must lie inside one page-locked allocation the driver
                             maps (cudaHostAlloc / cudaHostRegister): anything else is
                             refused with MDX_E_INVALID before the launch. */
} mdx_solve_desc;

/* The reverse pass of the discrete adjoint over checkpoints a MDX_PLAN_CHECKPOINT
 * solve recorded.  No counterpart in the reference, whose gradients come from
 * forward sensitivities (modax/_sensitivity.py:331-413); this is the backward of
 * the torch.autograd.Function / jax.custom_vjp front ends. */
typedef struct mdx_grad_desc {
  int struct_size;        /* sizeof(mdx_grad_desc) */
  int n_traj;
  int n_save;
  int count;              /* trajectories this launch reverses: order[0..count) (or
                             0..count without order); 0 = all n_traj.  Splitting a large
                             ensemble into several launches bounds the reverse kernel's
                             resident working set */
  const double* times;
  const double* params;
  const double* ckpt;
  const int* ckpt_count;
  long long ckpt_capacity;
  const double* grad_hist; /* (n_traj, n_save, n_vars) */
  double* grad_y0;         /* (n_traj, n_vars), overwritten */
  double* grad_params;     /* (n_traj, n_params), overwritten */
  int* status;             /* (n_traj,) or NULL */
  const int* order;        /* (n_traj,) or NULL: a permutation of 0..n_traj-1, the order in
                              which trajectories are handed to threads -- e.g. longest first by
                              ckpt_count, so the longest reverse sweeps start in the first
                              wave of resident blocks */
  /* Split reverse (one thread per trajectory plans only; `order` and `count` are then
   * ignored).  The reverse pass is linear in the cotangent, so a long trajectory's
   * checkpoint segments can be cut into chunks reversed in parallel: a chunk run from
   * the cotangent e_j at its end, with no save cotangents injected, gives column j of
   * its transfer matrix (and the matching parameter rows); run from zero with the
   * injections, its offset.  mdx_grad reverses every task, then composes each split
   * trajectory's chunks last to first into grad_y0 / grad_params. */
  const int* tasks;        /* (n_tasks, 5): trajectory, first segment, end segment, kind, slot.
                              kind -2: the whole trajectory (segments ignored), written to
                              grad_y0 / grad_params; -1: the chunk from zero with injections;
                              j >= 0: the chunk from e_j without them.  Chunk tasks write
                              (n_vars + n_params) doubles to task_out row `slot` */
  int n_tasks;
  int n_slots;             /* rows of task_out */
  double* task_out;
  const int* combine;      /* (n_combine, 3): trajectory, first slot, chunks; chunk c's task of
                              kind k sits at slot first + c (n_vars + 1) + k + 1 */
  int n_combine;
} mdx_grad_desc;

/* NVRTC: compile CUDA C++ `source` to an sm_100a cubin.  Needs no GPU.
 * On success *cubin is malloc'd (release with mdx_free).  `log` (may be NULL)
 * receives the compiler log, truncated to log_size. */
int mdx_compile(const char* source, const char* program_name, const char* const* options,
                int n_options, void** cubin, size_t* cubin_size, char* log, size_t log_size);
void mdx_free(void* ptr);

int mdx_plan_create(const mdx_plan_desc* desc, mdx_plan** plan);
int mdx_plan_destroy(mdx_plan* plan);

/* Bytes of `workspace` a solve in `mode` needs (0 for MDX_LAUNCH_PLAIN). */
int mdx_workspace_size(const mdx_plan* plan, int mode, int n_traj, size_t* bytes);

/* Bytes of the checkpoint buffer a MDX_PLAN_CHECKPOINT solve of n_traj
 * trajectories needs to record up to `capacity` accepted steps each: every step
 * size, plus the start (t, y) of every ckpt_stride-th step. */
int mdx_checkpoint_size(const mdx_plan* plan, int n_traj, long long capacity, size_t* bytes);

/* Resident blocks per SM for the plan's kernel in `mode`, and the SM count of
 * the current device (loads the module on first use). */
int mdx_occupancy(mdx_plan* plan, int mode, int* blocks_per_sm, int* sm_count);

/* Launch one ensemble solve on `stream`.  Asynchronous. */
int mdx_solve(mdx_plan* plan, const mdx_solve_desc* desc, void* stream);

/* The persistent refill solve for callers that cannot allocate device memory
 * (a plugin or custom-call handler that owns only its inputs and outputs, a
 * host whose allocator must not be bypassed).  No counterpart in the reference.
 * Same as mdx_solve with MDX_LAUNCH_PERSISTENT, except that the work-queue
 * scratch comes from a MDX_NOALLOC_SCRATCH_BYTES array inside the library on
 * each GPU (held until exit) instead of desc->workspace, which is ignored; a solve
 * needing more scratch than that is rejected with MDX_E_INVALID.  It calls no
 * allocator.  The first call on a device looks up the array's address (make it
 * before any stream capture); calls share the array, so calls whose kernels
 * overlap on the GPU race.  Needs the device's primary context current. */
#define MDX_NOALLOC_SCRATCH_BYTES 4096
int mdx_solve_persistent_noalloc(mdx_plan* plan, const mdx_solve_desc* desc, void* stream);

/* Launch the discrete-adjoint reverse pass on `stream` (MDX_PLAN_ADJOINT plans). */
int mdx_grad(mdx_plan* plan, const mdx_grad_desc* desc, void* stream);

/* Measured FMA throughput of the current device's CUDA cores, in FLOP/s
 * (an FMA counts two): the roofline denominator of the ensemble kernels, which
 * are bound by FP64/FP32 issue rather than HBM or the tensor cores.  No
 * counterpart in the reference. */
int mdx_measure_fma_peak(int double_precision, double* flops_per_s);

/* The calling thread's last error message. Returns its full length. */
int mdx_last_error(char* buf, size_t buf_size);

const char* mdx_version(void);

#ifdef __cplusplus
}
#endif
#endif
