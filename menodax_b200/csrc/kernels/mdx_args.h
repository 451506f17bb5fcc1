/* Kernel parameter blocks, identical in layout on the host (C++ runtime) and on
 * the device (NVRTC-compiled kernels).  Plain C with fixed-width-free types so the
 * header compiles under NVRTC, which has no standard library headers.
 *
 * Array layouts follow the reference's FFI call (modax/_numba_common.py:24-42):
 * y0 (N, n_system), times (S,), params (N, n_params), weights (N, n_system),
 * hist (N, S_hist, n_system), and three (N,) int32 counters; all row-major.
 */
#ifndef MDX_ARGS_H
#define MDX_ARGS_H

/* Per-trajectory status written by every solve kernel. */
#define MDX_STATUS_OK 0
#define MDX_STATUS_MAX_STEPS 1     /* max_steps reached before the last save time */
#define MDX_STATUS_NONFINITE 2     /* the final state holds a NaN or an infinity */
#define MDX_STATUS_CKPT_OVERFLOW 4 /* more accepted steps than checkpoint capacity */

typedef struct MdxSolveArgs {
  const double* y0;
  const double* times;
  const double* params;
  const double* weights;   /* may be NULL when the kernel was built with constant weights */
  double* hist;
  int* accepted;
  int* rejected;
  int* loop_steps;
  int* status;             /* may be NULL */
  double* hook_out;        /* (N, hook_size) or NULL */
  int* work_counter;       /* persistent kernels: queue head, zeroed before launch */
  const int* order;        /* persistent kernels: optional visiting order (N,) */
  double* ckpt;            /* adjoint forward pass: step sizes (capacity, N), then segment
                              start states (ceil(capacity / MDX_CKPT_SEG), N, n_vars + 1) */
  int* ckpt_count;         /* adjoint forward pass: accepted steps recorded per trajectory */
  long long ckpt_capacity; /* steps per trajectory the checkpoint buffer holds */
  double* hist_host;       /* page-locked host copy of hist (device-mapped address), or NULL */
  int n_traj;
  int n_save;
  int n_save_hist;         /* S, or 1 when only the final state is kept */
  int max_steps;
  double dt0;
  double rtol;
  double atol;
} MdxSolveArgs;

typedef struct MdxGradArgs {
  const double* times;
  const double* params;
  const double* ckpt;      /* as written by the forward pass */
  const int* ckpt_count;
  const double* grad_hist; /* (N, S, n_vars) cotangent of the history */
  double* grad_y0;         /* (N, n_vars) */
  double* grad_params;     /* (N, n_params) */
  int* status;             /* may be NULL */
  const int* order;        /* may be NULL: thread i takes trajectory order[i] */
  long long ckpt_capacity;
  int n_traj;              /* trajectories in the buffers (their stride) */
  int n_save;
  int n_run;               /* threads of this launch: order[0..n_run), or tasks[0..n_run) */
  const int* tasks;        /* split reverse: (n_run, 5) traj, first segment, end segment, kind, slot */
  double* task_out;        /* (n_slots, n_vars + n_params) */
  const int* combine;      /* (n_combine, 3) traj, first slot, chunks */
  int n_slots;
  int n_combine;
} MdxGradArgs;

#endif
