"""Benchmark and test systems in the reference's tuple callback form, with seeded scenarios.

The systems follow ``reference/systems/python``: a right-hand side is a plain
function ``ode_fn(y, t, p)`` returning a tuple, and systems whose size is a
parameter are generated from one expression string per component, each wrapped
as ``(expr) + 0.0`` (``reference/systems/python/_tuple_codegen.py:17-35``).
Scenario builders draw from ``np.random.default_rng(seed)`` as the reference's
``make_params`` do (``reference/systems/python/lorenz.py:46-52``).

The ensembles of the five benchmark configurations are built here:
Lorenz Tsit5 (4096), Robertson Rodas5P (65536), the stiff Van der Pol ring
(32768), the periodic Brusselator with a sparsity pattern (16384) and the
Van der Pol gradient problem (65536).
"""

from __future__ import annotations

import math

import numpy as np


def make_tuple_callback(name: str, components):
    """``def name(y, t, p): return ((c0) + 0.0, ...)`` from expression strings."""
    body = ",\n        ".join(f"({expr}) + 0.0" for expr in components)
    source = f"def {name}(y, t, p):\n    return (\n        {body},\n    )\n"
    namespace: dict = {"math": math}
    exec(compile(source, f"<generated {name}>", "exec"), namespace)  # noqa: S102
    fn = namespace[name]
    fn._generated_source = source
    return fn


# --- Lorenz (reference/systems/python/lorenz.py) ------------------------------------
def lorenz(y, t, p):
    sigma = 10.0
    beta = 8.0 / 3.0
    return (
        sigma * (y[1] - y[0]),
        y[0] * (p[0] - y[2]) - y[1],
        y[0] * y[1] - beta * y[2],
    )


LORENZ_Y0 = np.array([1000.0, -500.0, 500.0])
LORENZ_PARAMS = np.array([0.5])


def lorenz_divergence_scenario(size: int, seed: int = 42, divergence: float = 1.0):
    """The reference's ``make_scenario`` (lorenz.py:55-100): y0 = Y0 (1 - U(0, div)), rho ~ 0.5 +- 5% div."""
    rng = np.random.default_rng(seed)
    rho = 0.5 * (1.0 + 0.05 * (2.0 * rng.random((size, 1)) - 1.0))
    params = LORENZ_PARAMS + divergence * (rho - LORENZ_PARAMS)
    rng = np.random.default_rng(seed)
    t = rng.uniform(0.0, divergence, size=(size, 1))
    return LORENZ_Y0 * (1.0 - t), params


def lorenz_config(size: int = 4096, seed: int = 42):
    """Lorenz ensemble: sigma=10, beta=8/3, rho ~ U[0, 28), y0 = (1, 0, 0), t in [0, 1], 10 saves."""
    rng = np.random.default_rng(seed)
    params = rng.uniform(0.0, 28.0, size=(size, 1))
    y0 = np.broadcast_to(np.array([1.0, 0.0, 0.0]), (size, 3)).copy()
    times = np.linspace(0.0, 1.0, 10)
    return dict(ode_fn=lorenz, y0=y0, t_span=times, params=params, rtol=1e-8, atol=1e-10)


# --- Robertson (reference/systems/python/robertson.py) ------------------------------
def robertson(y, t, p):
    """Reference module order: p = [k1, k3, k2] with k3 on y1*y2 and k2 on y1**2."""
    return (
        -p[0] * y[0] + p[1] * y[1] * y[2],
        p[0] * y[0] - p[1] * y[1] * y[2] - p[2] * y[1] ** 2,
        p[2] * y[1] ** 2,
    )


ROBERTSON_TIMES = np.array((0.0, 1e-6, 1e-2, 1e2, 1e5))
ROBERTSON_Y0 = np.array([(1 - 0.1) * 0.99, 0.1, (1 - 0.1) * (1 - 0.99)])
ROBERTSON_PARAMS = np.array([0.04, 1e4, 3e7])


def robertson_config(size: int = 65536, seed: int = 42):
    """Robertson kinetics ensemble: k1=0.04, k2=3e7, k3=1e4 each x log-uniform[0.5, 2]; y0=(1,0,0);
    20 save times on [0, 1e5] (0 then 19 log-spaced from 1e-5); rtol 1e-6, atol 1e-10.

    The rates are mapped onto the module's ``[k1, k3, k2]`` column order."""
    rng = np.random.default_rng(seed)
    scale = np.exp(rng.uniform(math.log(0.5), math.log(2.0), size=(size, 3)))
    k1, k2, k3 = 0.04 * scale[:, 0], 3e7 * scale[:, 1], 1e4 * scale[:, 2]
    params = np.stack([k1, k3, k2], axis=1)
    y0 = np.broadcast_to(np.array([1.0, 0.0, 0.0]), (size, 3)).copy()
    times = np.concatenate([[0.0], np.logspace(-5, 5, 19)])
    return dict(ode_fn=robertson, y0=y0, t_span=times, params=params, rtol=1e-6, atol=1e-10)


# --- Van der Pol ring (reference/systems/python/vdp.py) -----------------------------
def vdp_neighbours(n_osc: int, osc: int, coupling_range: int = 1):
    found = []
    for offset in range(1, coupling_range + 1):
        for other in ((osc - offset) % n_osc, (osc + offset) % n_osc):
            if other != osc:
                found.append(other)
    return found


def make_vdp_system(n_osc: int, *, mu: float = 100.0, d: float = 10.0, omega: float = 1.0,
                    coupling_range: int = 1):
    """``(ode_fn, y0)`` for a ring of coupled Van der Pol oscillators (vdp.py:50-81)."""
    y0 = np.array([2.0, 0.0] * n_osc)
    strength = d / coupling_range
    comps = []
    for osc in range(n_osc):
        base = 2 * osc
        x, v = f"y[{base}]", f"y[{base + 1}]"
        others = vdp_neighbours(n_osc, osc, coupling_range)
        laplacian = " + ".join([f"y[{2 * o}]" for o in others] + [f"-{float(len(others))!r} * {x}"])
        comps += [
            v,
            f"p[0] * {mu!r} * (1.0 - {x} * {x}) * {v} + -{omega * omega!r} * {x} + {strength!r} * ({laplacian})",
        ]
    return make_tuple_callback("ode_fn", comps), y0


def vdp_sparsity(n_osc: int, coupling_range: int = 1) -> np.ndarray:
    n = 2 * n_osc
    mask = np.zeros((n, n), dtype=bool)
    for osc in range(n_osc):
        x, v = 2 * osc, 2 * osc + 1
        mask[x, v] = True
        mask[v, x] = mask[v, v] = True
        for other in vdp_neighbours(n_osc, osc, coupling_range):
            mask[v, 2 * other] = True
    return mask


def vdp_ring_config(n_osc: int, size: int = 32768, seed: int = 42):
    """Stiff Van der Pol ring ensemble: mu ~ log-uniform[10, 1000] as p0, epsilon = 0.1 coupling, omega = 1,
    y0 = (2, 0) + N(0, 0.1) per oscillator, t in [0, 3000], 50 saves, rtol 1e-6, atol 1e-8."""
    ode_fn, base = make_vdp_system(n_osc, mu=1.0, d=0.1, omega=1.0)
    rng = np.random.default_rng(seed)
    mu = np.exp(rng.uniform(math.log(10.0), math.log(1000.0), size=(size, 1)))
    y0 = base[None, :] + rng.normal(0.0, 0.1, size=(size, 2 * n_osc))
    times = np.linspace(0.0, 3000.0, 50)
    return dict(ode_fn=ode_fn, y0=y0, t_span=times, params=mu, rtol=1e-6, atol=1e-8,
                sparsity=vdp_sparsity(n_osc))


# --- Brusselator (reference/systems/python/brusselator.py) --------------------------
def make_brusselator_b(n_grid: int, *, a: float = 1.0, alpha: float = 1.0 / 50.0, length: float = 1.0):
    """Periodic 1-D Brusselator with ``p[0] = B`` and ``A`` fixed, interleaved (u_i, v_i)."""
    dx = length / n_grid
    diff = alpha / (dx * dx)
    comps = []
    for g in range(n_grid):
        left, right = (g - 1) % n_grid, (g + 1) % n_grid
        u, v = 2 * g, 2 * g + 1
        u2v = f"y[{u}] * y[{u}] * y[{v}]"
        comps += [
            f"{a!r} + {u2v} - (p[0] + 1.0) * y[{u}] + {diff!r} * (y[{2 * left}] + -2.0 * y[{u}] + y[{2 * right}])",
            f"p[0] * y[{u}] - {u2v} + {diff!r} * (y[{2 * left + 1}] + -2.0 * y[{v}] + y[{2 * right + 1}])",
        ]
    return make_tuple_callback("ode_fn", comps)


def brusselator_pattern(n_grid: int) -> np.ndarray:
    """``(nnz, 2)``: u_i -> {u_i-1, u_i, u_i+1, v_i}, v_i -> {v_i-1, v_i, v_i+1, u_i}."""
    pairs = set()
    for g in range(n_grid):
        left, right = (g - 1) % n_grid, (g + 1) % n_grid
        u, v = 2 * g, 2 * g + 1
        for c in (2 * left, u, 2 * right, v):
            pairs.add((u, c))
        for c in (2 * left + 1, v, 2 * right + 1, u):
            pairs.add((v, c))
    return np.array(sorted(pairs), dtype=np.int64)


def brusselator_config(n_grid: int = 32, size: int = 16384, seed: int = 42):
    """Brusselator ensemble: 32 points (64 states), alpha = 1/50, A = 1, B ~ U[2.5, 3.5], periodic;
    u = 1 + sin(2 pi x) + N(0, 0.01), v = 3; t in [0, 10], 10 saves; rtol 1e-6, atol 1e-8."""
    rng = np.random.default_rng(seed)
    b = rng.uniform(2.5, 3.5, size=(size, 1))
    x = np.arange(n_grid) / n_grid
    y0 = np.empty((size, 2 * n_grid))
    y0[:, 0::2] = 1.0 + np.sin(2.0 * np.pi * x)[None, :] + rng.normal(0.0, 0.01, size=(size, n_grid))
    y0[:, 1::2] = 3.0
    return dict(ode_fn=make_brusselator_b(n_grid), y0=y0, t_span=np.linspace(0.0, 10.0, 10),
                params=b, rtol=1e-6, atol=1e-8, sparsity=brusselator_pattern(n_grid))


# --- Van der Pol adjoint problem ----------------------------------------------------
def vdp_gradient_config(n_osc: int, size: int = 65536, seed: int = 42):
    """Stiff Van der Pol gradient ensemble: mu ~ log-uniform[10, 500]; differentiate y0 and mu; 20 saves on [0, 1000];
    targets from mu x 1.05 (computed by the caller); rtol 1e-6, atol 1e-8, FP64."""
    ode_fn, base = make_vdp_system(n_osc, mu=1.0, d=0.1, omega=1.0)
    rng = np.random.default_rng(seed)
    mu = np.exp(rng.uniform(math.log(10.0), math.log(500.0), size=(size, 1)))
    y0 = base[None, :] + rng.normal(0.0, 0.1, size=(size, 2 * n_osc))
    return dict(ode_fn=ode_fn, y0=y0, t_span=np.linspace(0.0, 1000.0, 20), params=mu,
                rtol=1e-6, atol=1e-8)


# --- closed-form problems of the reference tests -----------------------------------
def exp_decay(y, t, p):
    return (-p[0] * y[0],)


def cascade(y, t, p):
    return (-p[0] * y[0], p[0] * y[0] - p[1] * y[1])


def forced_decay(y, t, p):
    return (-p[0] * y[0] + p[1] * t,)


def decay_chain(y, t, p):
    """A -> B -> C -> D with rates p[0], p[1], p[2] (the reference's
    tests/test_sparsity.py:40-46); D is stable, so the total is conserved."""
    return (
        -p[0] * y[0],
        p[0] * y[0] - p[1] * y[1],
        p[1] * y[1] - p[2] * y[2],
        p[2] * y[2],
    )


DECAY_CHAIN_PATTERN = [(0, 0), (1, 0), (1, 1), (2, 1), (2, 2), (3, 2)]


def decay_chain_exact(t: float, a: float, b: float, c: float) -> np.ndarray:
    """The chain's state at t from (1, 0, 0, 0), distinct rates a, b, c:
    the Bateman sums over exp(-rate t) for B and C, D from conservation."""
    ea, eb, ec = math.exp(-a * t), math.exp(-b * t), math.exp(-c * t)
    y0 = ea
    y1 = a / (b - a) * (ea - eb)
    y2 = a * b * (ea / ((b - a) * (c - a)) + eb / ((a - b) * (c - b)) + ec / ((a - c) * (b - c)))
    return np.array([y0, y1, y2, 1.0 - y0 - y1 - y2])


def rate_scale_params(size: int, seed: int = 42) -> np.ndarray:
    """p[0] = 1 + 0.1 * U[-1, 1) per trajectory: the rate scale of the linear
    closed-form systems below (reference/systems/python/{kaps,bateman,heat}.py)."""
    rng = np.random.default_rng(seed)
    return 1.0 + 0.1 * (2.0 * rng.random((size, 1)) - 1.0)


def _linear_system(matrix: np.ndarray):
    """y' = p[0] * M y as a tuple-form callback (only the nonzero terms)."""
    comps = []
    for row in matrix:
        terms = " + ".join(f"{float(v)!r} * y[{j}]" for j, v in enumerate(row) if v != 0.0)
        comps.append(f"p[0] * ({terms or '0.0'})")
    return make_tuple_callback("ode_fn", comps)


def _log_spaced_ratios(count: int, ratio: float) -> np.ndarray:
    """ratio ** (i / (count - 1)) for i = 0 .. count - 1."""
    return np.array([10.0 ** (math.log10(ratio) * i / (count - 1)) for i in range(count)])


KAPS_TIMES = np.array((0.0, 0.5, 1.0, 2.0))


def make_kaps_system(n_pairs: int, epsilon_min: float):
    """Independent Kaps pairs (reference/systems/python/kaps.py:23-56): pair i has
    stiffness 1/eps_i with eps_i log-spaced from 1 to epsilon_min, y0 = (1, 1) on
    the slow manifold, and for every eps the exact solution
    y1 = exp(-2 p0 t), y2 = exp(-p0 t) (kaps_exact)."""
    comps = []
    for pair, eps in enumerate(_log_spaced_ratios(n_pairs, epsilon_min)):
        inv = 1.0 / float(eps)
        y1, y2 = f"y[{2 * pair}]", f"y[{2 * pair + 1}]"
        comps += [
            f"p[0] * (-{inv + 2.0!r} * {y1} + {inv!r} * ({y2} * {y2}))",
            f"p[0] * (({y1} - {y2}) - {y2} * {y2})",
        ]
    return make_tuple_callback("ode_fn", comps), np.ones(2 * n_pairs)


def kaps_exact(times, params, n_pairs: int) -> np.ndarray:
    rate = np.outer(np.asarray(params)[:, 0], np.asarray(times, dtype=float))
    pair = np.stack([np.exp(-2.0 * rate), np.exp(-rate)], axis=-1)
    return np.tile(pair, (1, 1, n_pairs))


BATEMAN_TIMES = np.array((0.0, 0.2, 0.5, 1.0, 2.0))


def make_bateman_system(n_vars: int, stiffness: float):
    """A decay chain A_1 -> ... -> A_n with A_n stable
    (reference/systems/python/bateman.py:49-84): rates lambda_i log-spaced from 1
    to `stiffness`, y' = p0 M y with M lower bidiagonal, y0 = (1, 0, ..., 0).
    Returns (ode_fn, y0, M)."""
    lam = _log_spaced_ratios(n_vars - 1, stiffness)
    matrix = np.zeros((n_vars, n_vars))
    for i, rate in enumerate(lam):
        matrix[i, i] = -rate
        matrix[i + 1, i] = rate
    y0 = np.zeros(n_vars)
    y0[0] = 1.0
    return _linear_system(matrix), y0, matrix


def linear_exact(matrix: np.ndarray, y0: np.ndarray, times, params) -> np.ndarray:
    """expm(p0 M t) y0 for every trajectory and time, through M's eigenvectors
    (M has distinct real eigenvalues here)."""
    eigval, eigvec = np.linalg.eig(matrix)
    eigval, eigvec = np.real(eigval), np.real(eigvec)
    coeff = np.linalg.solve(eigvec, y0)
    rate = np.outer(np.asarray(params)[:, 0], np.asarray(times, dtype=float))
    return (np.exp(rate[:, :, None] * eigval) * coeff) @ eigvec.T


HEAT_TIMES = np.array((0.0, 0.025, 0.05, 0.075, 0.1))


def make_heat_system(n_vars: int):
    """The heat equation u_t = p0 u_xx on (0, 1) with zero boundary values, on n
    interior points (reference/systems/python/heat.py:40-69).  y0 = sin(pi x) is
    the first eigenmode of the discrete Laplacian, so y(t) = y0 exp(p0 l1 t) with
    l1 = 2 (cos(pi dx) - 1) / dx^2 (heat_exact).  Returns (ode_fn, y0)."""
    if n_vars < 3:
        raise ValueError(f"n_vars must be at least 3, got {n_vars}")
    dx = 1.0 / (n_vars + 1)
    inv_dx2 = 1.0 / dx ** 2
    matrix = (np.diag(np.full(n_vars, -2.0 * inv_dx2)) + np.diag(np.full(n_vars - 1, inv_dx2), 1)
              + np.diag(np.full(n_vars - 1, inv_dx2), -1))
    x = np.arange(1, n_vars + 1) * dx
    return _linear_system(matrix), np.sin(np.pi * x)


def heat_exact(n_vars: int, times, params) -> np.ndarray:
    dx = 1.0 / (n_vars + 1)
    y0 = np.sin(np.pi * np.arange(1, n_vars + 1) * dx)
    l1 = 2.0 * (math.cos(math.pi * dx) - 1.0) / dx ** 2
    decay = np.exp(l1 * np.outer(np.asarray(params)[:, 0], np.asarray(times, dtype=float)))
    return y0[None, None, :] * decay[:, :, None]


VDP_TIMES = np.array((0.0, 0.25, 0.5, 0.75, 1.0))


def vdp_divergence_scenario(n_osc: int, size: int, seed: int = 42, divergence: float = 1.0):
    """The reference's ``vdp.make_scenario`` (vdp.py:116-150) restated."""
    rng = np.random.default_rng(seed)
    amplitudes = rng.uniform(0.25, 3.0, size=(size, n_osc))
    signs = rng.choice(np.array([-1.0, 1.0]), size=(size, n_osc))
    target_x = amplitudes * signs
    x = 2.0 + min(divergence, 1.0) * (target_x - 2.0)
    v = rng.normal(0.0, 2.0 * divergence, size=(size, n_osc))
    y0 = np.empty((size, 2 * n_osc))
    y0[:, 0::2] = x
    y0[:, 1::2] = v
    rng2 = np.random.default_rng(seed)
    base = 1.0 + 0.2 * (2.0 * rng2.random((size, 1)) - 1.0)
    params = np.maximum(max(divergence, 1.0) + divergence * (base - 1.0), 1e-6)
    return y0, params
