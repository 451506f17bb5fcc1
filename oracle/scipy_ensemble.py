"""TEST INFRASTRUCTURE -- the reference's CPU ensemble solver, restated.

The reference times its "no GPU" baseline with
``reference/solvers/python/scipy_solve_ivp.py:165-255``: every trajectory is an
independent ``scipy.integrate.solve_ivp`` call (LSODA by default, saves through
``t_eval``), spread over a ``spawn`` process pool of one worker per core with
BLAS pinned to one thread each.  That file needs JAX for its right-hand side
(a CPU-jitted ``jax.numpy`` function) and cannot run here; this module does the
same with the tuple-form Python right-hand side evaluated on floats.

Only ``tests/`` and ``bench.py``'s CPU-baseline leg use it.
"""

from __future__ import annotations

import multiprocessing as mp
import os
import time

import numpy as np

_POOLS: dict = {}
_RHS = None


def _init(ode_fn):
    global _RHS
    for key in ("OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS", "OMP_NUM_THREADS"):
        os.environ.setdefault(key, "1")
    _RHS = ode_fn


def _one(args):
    from scipy.integrate import solve_ivp

    y0, p, times, method, rtol, atol, first_step = args
    p = [float(v) for v in p]

    def f(t, y):
        return np.array(_RHS(y, t, p), dtype=np.float64)

    out = np.full((len(times), len(y0)), np.nan)
    sol = solve_ivp(f, (float(times[0]), float(times[-1])), y0, method=method, t_eval=times, rtol=rtol,
                    atol=atol, first_step=first_step)
    got = sol.y.T
    out[: got.shape[0]] = got
    return out


def _pool(ode_fn, workers):
    key = (ode_fn, workers)
    if key not in _POOLS:
        _POOLS[key] = mp.get_context("spawn").Pool(workers, initializer=_init, initargs=(ode_fn,))
    return _POOLS[key]


def solve(ode_fn, y0, t_span, params, *, method="LSODA", rtol=1e-8, atol=1e-10, first_step=None,
          workers=None):
    """``(N, S, n)`` history, one ``solve_ivp`` per trajectory over a process pool."""
    params = np.asarray(params, dtype=np.float64)
    n = params.shape[0]
    y0 = np.asarray(y0, dtype=np.float64)
    if y0.ndim == 1:
        y0 = np.broadcast_to(y0, (n, y0.shape[0]))
    times = np.asarray(t_span, dtype=np.float64)
    workers = min(n, workers or os.cpu_count() or 1)
    jobs = [(y0[i].copy(), params[i], times, method, rtol, atol, first_step) for i in range(n)]
    if workers <= 1:
        _init(ode_fn)
        return np.stack([_one(j) for j in jobs])
    pool = _pool(ode_fn, workers)
    return np.stack(pool.map(_one, jobs, chunksize=max(1, n // (workers * 4))))


def timed_rate(ode_fn, y0, t_span, params, **kw):
    """Solves per second on this sample (the pool is started and warmed first)."""
    solve(ode_fn, y0[:64], t_span, params[:64], **kw)
    t0 = time.perf_counter()
    hist = solve(ode_fn, y0, t_span, params, **kw)
    return len(params) / (time.perf_counter() - t0), hist


def close():
    for pool in _POOLS.values():
        pool.terminate()
    _POOLS.clear()
