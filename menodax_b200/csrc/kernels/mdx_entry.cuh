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
#pragma once

extern "C" __global__ void __launch_bounds__(MDX_TPB, MDX_MIN_BLOCKS)
mdx_solve_plain(const MdxSolveArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_traj) return;
  MDX_SOLVER::State st;
  MDX_SOLVER::init(st, a, i);
  while (MDX_SOLVER::running(st, a)) MDX_SOLVER::step(st, a);
  MDX_SOLVER::finish(st, a);
}

extern "C" __global__ void __launch_bounds__(MDX_TPB, MDX_MIN_BLOCKS)
mdx_solve_persistent(const MdxSolveArgs a) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lanes_below = (1u << lane) - 1u;
  MDX_SOLVER::State st;
  bool active = false;
  bool drained = false;
  while (true) {
    if (active && !MDX_SOLVER::running(st, a)) {
      MDX_SOLVER::finish(st, a);
      active = false;
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
          MDX_SOLVER::init(st, a, a.order ? a.order[slot] : slot);
          active = true;
        }
      }
      if (base + want >= a.n_traj) drained = true;
    }
    if (!__any_sync(MDX_FULL_MASK, active)) break;
    if (active && MDX_SOLVER::running(st, a)) MDX_SOLVER::step(st, a);
  }
}
