// Kernel entry points for one compiled problem.  MDX_SOLVER names the solver
// struct (mdx::Tsit5 or mdx::Rodas5P) the problem source selected.
//
//  * mdx_solve_plain      -- one trajectory per thread for its whole life, the
//                            reference's launch shape (modax/rodas5P.py:1010-1021).
//  * mdx_solve_persistent -- a grid sized to the device; each warp keeps its 32
//                            lanes busy by handing finished trajectories back and
//                            taking new ones off an atomic queue.  A warp ballot
//                            finds the idle lanes, one atomicAdd per warp claims a
//                            contiguous run of trajectory indices, and lanes take
//                            them in lane order.  No thread ever waits on another:
//                            the queue is a counter, so there is nothing to spin on.
//
// With a host copy of the history (MdxSolveArgs::hist_host) both kernels copy
// finished rows to it while the rest of the ensemble is still stepping.
#pragma once

// Copies `rows` whole trajectories of history, starting at trajectory `first`,
// from the device buffer to the page-locked host copy.  The warp moves them
// together: the rows are contiguous (trajectory index slowest), so every store
// instruction writes 256 consecutive bytes across the host link.  The rows are
// read from L2 (ld.global.cg): the lanes that wrote them are other threads.
__device__ __forceinline__ void stream_rows(const MdxSolveArgs& a, int first, int rows, unsigned lane) {
  const size_t row = (size_t)a.n_save_hist * (size_t)MDX_NS;
  const size_t total = (size_t)rows * row;
  const double* src = a.hist + (size_t)first * row;
  double* dst = a.hist_host + (size_t)first * row;
  size_t k = lane;
  for (; k + 96 < total; k += 128) {
    const double v0 = __ldcg(src + k), v1 = __ldcg(src + k + 32);
    const double v2 = __ldcg(src + k + 64), v3 = __ldcg(src + k + 96);
    dst[k] = v0;
    dst[k + 32] = v1;
    dst[k + 64] = v2;
    dst[k + 96] = v3;
  }
  for (; k < total; k += 32) dst[k] = __ldcg(src + k);
}

extern "C" __global__ void __launch_bounds__(MDX_TPB, MDX_MIN_BLOCKS)
mdx_solve_plain(const MdxSolveArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.n_traj) {
    MDX_SOLVER::State st;
    MDX_SOLVER::init(st, a, i);
    while (MDX_SOLVER::running(st, a)) MDX_SOLVER::step(st, a);
    MDX_SOLVER::finish(st, a);
  }
  if (a.hist_host != nullptr) {
    // Block sizes are multiples of 32, so every lane of the warp arrives here;
    // __syncwarp also orders the other lanes' history stores before the reads.
    __syncwarp();
    const unsigned lane = threadIdx.x & 31u;
    const int first = i - (int)lane;
    const int rows = min(32, a.n_traj - first);
    if (rows > 0) stream_rows(a, first, rows, lane);
  }
}

extern "C" __global__ void __launch_bounds__(MDX_TPB, MDX_MIN_BLOCKS)
mdx_solve_persistent(const MdxSolveArgs a) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lanes_below = (1u << lane) - 1u;
  MDX_SOLVER::State st;
  bool active = false;
  bool drained = false;
  int traj = 0;
  while (true) {
    bool finished = false;
    if (active && !MDX_SOLVER::running(st, a)) {
      MDX_SOLVER::finish(st, a);
      active = false;
      finished = true;
    }
    if (a.hist_host != nullptr) {
      // The warp moves each just-finished lane's row together.
      unsigned done = __ballot_sync(MDX_FULL_MASK, finished);
      if (done != 0u) __syncwarp();
      while (done != 0u) {
        const int from = __ffs(done) - 1;
        done &= done - 1u;
        stream_rows(a, __shfl_sync(MDX_FULL_MASK, traj, from), 1, lane);
      }
    }
    const unsigned idle = __ballot_sync(MDX_FULL_MASK, !active);
    if (idle != 0u && !drained) {
      const int leader = __ffs(idle) - 1;
      const int want = __popc(idle);
      int base = 0;
      if ((int)lane == leader) base = atomicAdd(a.work_counter, want);
      base = __shfl_sync(MDX_FULL_MASK, base, leader);
      if (!active) {
        const int slot = base + __popc(idle & lanes_below);
        if (slot < a.n_traj) {
          traj = a.order ? a.order[slot] : slot;
          MDX_SOLVER::init(st, a, traj);
          active = true;
        }
      }
      if (base + want >= a.n_traj) drained = true;
    }
    if (!__any_sync(MDX_FULL_MASK, active)) break;
    if (active && MDX_SOLVER::running(st, a)) MDX_SOLVER::step(st, a);
  }
}
