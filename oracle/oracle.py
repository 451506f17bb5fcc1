"""TEST INFRASTRUCTURE -- Python side of the CPU oracle (``oracle/mdx_oracle.cpp``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module.  It is the checker, never the thing measured or shipped.

``build()`` compiles the C++ restatement with g++ (OpenMP) into
``oracle/libmdx_oracle.so``.  Systems are either built into the oracle as C++
templates (exact dual-number derivatives, parallel over trajectories) or given as
a Python tuple-form callback, differentiated here with dual numbers and run on one
thread.  Nothing here touches the product's tracer or code generator.
"""

from __future__ import annotations

import ctypes
import math
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "mdx_oracle.cpp"


def _host_has_fma() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return " fma " in f" {line.split(':', 1)[1].strip()} "
    except OSError:
        pass
    return False


# The reference's GPU compiler contracts a*b + c into fused multiply-adds; the
# oracle is compiled the same way where the host CPU has FMA, which is what
# makes its FP32-LU step counts land on the reference's published ones.
FMA = _host_has_fma()
LIB = HERE / ("libmdx_oracle_fma.so" if FMA else "libmdx_oracle.so")

SYS_LORENZ, SYS_ROBERTSON, SYS_VDP_RING, SYS_BRUSSELATOR = 1, 2, 3, 4
SYS_CASCADE, SYS_FORCED, SYS_EXP_DECAY, SYS_CALLBACK = 5, 6, 7, 100


def build(force: bool = False) -> Path:
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    flags = ["-mfma", "-ffp-contract=fast"] if FMA else ["-ffp-contract=off"]
    subprocess.run(
        ["g++", "-O2", "-std=c++17", "-fopenmp", "-shared", "-fPIC", *flags, str(SRC), "-o", str(LIB)],
        check=True,
    )
    return LIB


F_CB = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                        ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double))
JVP_CB = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                          ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                          ctypes.POINTER(ctypes.c_double))
JVP2_CB = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                           ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                           ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                           ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                           ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double))


class _SystemDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("n", ctypes.c_int), ("np", ctypes.c_int),
                ("cfg", ctypes.POINTER(ctypes.c_double)), ("n_cfg", ctypes.c_int),
                ("f_cb", F_CB), ("jvp_cb", JVP_CB), ("jvp2_cb", JVP2_CB)]


class _Sens(ctypes.Structure):
    _fields_ = [("n_sens", ctypes.c_int), ("n_y0_dirs", ctypes.c_int),
                ("param_cols", ctypes.POINTER(ctypes.c_int)), ("error_control", ctypes.c_int)]


class _Controls(ctypes.Structure):
    _fields_ = [("dt0", ctypes.c_double), ("rtol", ctypes.c_double), ("atol", ctypes.c_double),
                ("max_steps", ctypes.c_int), ("pcoeff", ctypes.c_double),
                ("icoeff", ctypes.c_double), ("dcoeff", ctypes.c_double), ("tf_index", ctypes.c_int)]


class _Ensemble(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("n_system", ctypes.c_int), ("np", ctypes.c_int),
                ("S", ctypes.c_int), ("y0", ctypes.c_void_p), ("times", ctypes.c_void_p),
                ("params", ctypes.c_void_p), ("weights", ctypes.c_void_p), ("hist", ctypes.c_void_p),
                ("accepted", ctypes.c_void_p), ("rejected", ctypes.c_void_p), ("loop", ctypes.c_void_p)]


class _Layout(ctypes.Structure):
    _fields_ = [("n_colours", ctypes.c_int), ("colour", ctypes.c_void_p), ("lu_size", ctypes.c_int),
                ("store", ctypes.c_void_p), ("diag", ctypes.c_void_p), ("sparse", ctypes.c_int),
                ("row_ptr", ctypes.c_void_p), ("col_ind", ctypes.c_void_p),
                ("diag_ptr", ctypes.c_void_p), ("order", ctypes.c_void_p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        L.oracle_tsit5.argtypes = [ctypes.POINTER(_SystemDesc), ctypes.POINTER(_Sens),
                                   ctypes.POINTER(_Controls), ctypes.POINTER(_Ensemble), ctypes.c_int]
        L.oracle_rodas5p.argtypes = [ctypes.POINTER(_SystemDesc), ctypes.POINTER(_Sens),
                                     ctypes.POINTER(_Layout), ctypes.POINTER(_Controls),
                                     ctypes.POINTER(_Ensemble), ctypes.c_int, ctypes.c_int]
        L.oracle_eval.argtypes = [ctypes.POINTER(_SystemDesc)] + [ctypes.c_void_p, ctypes.c_double,
                                                                  ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_max_threads.restype = ctypes.c_int
        L.oracle_jvp2.argtypes = [ctypes.POINTER(_SystemDesc), ctypes.c_void_p, ctypes.c_double,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_jvp.argtypes = [ctypes.POINTER(_SystemDesc), ctypes.c_void_p, ctypes.c_double,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                 ctypes.c_void_p]
        _lib = L
    return _lib


def max_threads() -> int:
    return int(lib().oracle_max_threads())


# --- dual numbers for Python callbacks -------------------------------------------
class Dual:
    """Forward-mode dual number; nests (Dual of Dual) for second derivatives."""

    __slots__ = ("v", "d")

    def __init__(self, v, d=0.0):
        self.v, self.d = v, d

    @staticmethod
    def lift(x):
        return x if isinstance(x, Dual) else Dual(x, 0.0)

    def __add__(self, o):
        o = Dual.lift(o)
        return Dual(self.v + o.v, self.d + o.d)

    __radd__ = __add__

    def __sub__(self, o):
        o = Dual.lift(o)
        return Dual(self.v - o.v, self.d - o.d)

    def __rsub__(self, o):
        return Dual.lift(o) - self

    def __mul__(self, o):
        o = Dual.lift(o)
        return Dual(self.v * o.v, self.d * o.v + self.v * o.d)

    __rmul__ = __mul__

    def __truediv__(self, o):
        o = Dual.lift(o)
        q = self.v / o.v
        return Dual(q, (self.d - q * o.d) / o.v)

    def __rtruediv__(self, o):
        return Dual.lift(o) / self

    def __neg__(self):
        return Dual(-self.v, -self.d)

    def __pos__(self):
        return self

    def __pow__(self, o):
        if isinstance(o, int):
            r = Dual(1.0)
            for _ in range(abs(o)):
                r = r * self
            return Dual(1.0) / r if o < 0 else r
        if isinstance(o, Dual):
            return dexp(o * dlog(self))
        return Dual(self.v ** o, o * self.v ** (o - 1) * self.d)

    def __abs__(self):
        return self if _val(self) >= 0 else -self


def _val(x):
    while isinstance(x, Dual):
        x = x.v
    return x


def dexp(x):
    if isinstance(x, Dual):
        e = dexp(x.v)
        return Dual(e, e * x.d)
    return math.exp(x)


def dlog(x):
    if isinstance(x, Dual):
        return Dual(dlog(x.v), x.d / x.v)
    return math.log(x)


def _dual_math():
    import types

    m = types.ModuleType("math")
    for k in dir(math):
        setattr(m, k, getattr(math, k))

    def unary(fn, dfn):
        def g(x):
            if isinstance(x, Dual):
                return Dual(g(x.v), dfn(x.v) * x.d)
            return fn(x)
        return g

    m.exp = dexp
    m.log = dlog
    m.sqrt = unary(math.sqrt, lambda v: 0.5 / m.sqrt(v))
    m.sin = unary(math.sin, lambda v: m.cos(v))
    m.cos = unary(math.cos, lambda v: -m.sin(v))
    m.tanh = unary(math.tanh, lambda v: 1.0 - m.tanh(v) * m.tanh(v))
    return m


_DMATH = _dual_math()


def _rebind(fn):
    import types

    g = dict(fn.__globals__)
    for k, v in list(g.items()):
        if v is math:
            g[k] = _DMATH
    return types.FunctionType(fn.__code__, g, fn.__name__, fn.__defaults__, fn.__closure__)


@dataclass
class System:
    """A right-hand side the oracle can run."""

    kind: int
    n: int
    np: int
    cfg: tuple = ()
    fn: object = None

    @staticmethod
    def lorenz():
        return System(SYS_LORENZ, 3, 1)

    @staticmethod
    def robertson():
        return System(SYS_ROBERTSON, 3, 3)

    @staticmethod
    def vdp_ring(n_osc, mu, d, omega=1.0):
        return System(SYS_VDP_RING, 2 * n_osc, 1, (float(n_osc), float(mu), float(d), float(omega)))

    @staticmethod
    def brusselator(n_grid, a=1.0, alpha=1.0 / 50.0):
        return System(SYS_BRUSSELATOR, 2 * n_grid, 1, (float(n_grid), float(a), float(alpha)))

    @staticmethod
    def cascade():
        return System(SYS_CASCADE, 2, 2)

    @staticmethod
    def forced():
        return System(SYS_FORCED, 1, 2)

    @staticmethod
    def exp_decay(n=1):
        return System(SYS_EXP_DECAY, n, 1)

    @staticmethod
    def callback(fn, n, np_):
        return System(SYS_CALLBACK, n, np_, (), fn)

    def _desc(self):
        """The C descriptor plus what must outlive the call: buffers, the ctypes
        callbacks and ``errors``, where a Python callback records any exception
        it raises (ctypes would otherwise print and swallow it, leaving the
        output undefined); ``_raise_recorded`` turns it into a failed solve."""
        keep = []
        cfg = (ctypes.c_double * max(1, len(self.cfg)))(*self.cfg)
        keep.append(cfg)
        d = _SystemDesc(kind=self.kind, n=self.n, np=self.np, cfg=cfg, n_cfg=len(self.cfg))
        errors: list[BaseException] = []
        keep.append(errors)
        if self.kind == SYS_CALLBACK:
            fn = _rebind(self.fn)
            n, np_ = self.n, self.np

            def guarded(body):
                # IEEE arithmetic as the C side has it: numpy scalars give inf or
                # nan where Python floats would raise (OverflowError on x ** 2).
                def run(*args):
                    out = args[-1]
                    try:
                        with np.errstate(all="ignore"):
                            body(*args)
                    except BaseException as e:  # noqa: BLE001 -- recorded and re-raised after the solve
                        errors.append(e)
                        for i in range(n):
                            out[i] = math.nan
                return run

            def f_cb(y, t, p, out):
                vals = fn([np.float64(y[i]) for i in range(n)], np.float64(t),
                          [np.float64(p[k]) for k in range(np_)])
                for i in range(n):
                    out[i] = float(vals[i])

            def jvp_cb(y, t, p, vy, vt, vp, out):
                yy = [Dual(y[i], vy[i] if vy else 0.0) for i in range(n)]
                pp = [Dual(p[k], vp[k] if vp else 0.0) for k in range(np_)]
                vals = fn(yy, Dual(t, vt), pp)
                for i in range(n):
                    out[i] = float(Dual.lift(vals[i]).d)

            def jvp2_cb(y, t, p, uy, ut, up, vy, vt, vp, out):
                yy = [Dual(Dual(y[i], uy[i] if uy else 0.0), Dual(vy[i] if vy else 0.0)) for i in range(n)]
                pp = [Dual(Dual(p[k], up[k] if up else 0.0), Dual(vp[k] if vp else 0.0)) for k in range(np_)]
                vals = fn(yy, Dual(Dual(t, ut), Dual(vt)), pp)
                for i in range(n):
                    v = Dual.lift(vals[i])
                    out[i] = float(Dual.lift(v.d).d)

            cbs = (F_CB(guarded(f_cb)), JVP_CB(guarded(jvp_cb)), JVP2_CB(guarded(jvp2_cb)))
            keep.extend(cbs)
            d.f_cb, d.jvp_cb, d.jvp2_cb = cbs
        return d, keep


def _raise_recorded(keep) -> None:
    """Fail the oracle call if a Python callback raised during it."""
    errors = keep[1]
    if errors:
        raise RuntimeError(f"the system's Python callback raised {len(errors)} time(s) during the oracle "
                           f"call; first: {errors[0]!r}") from errors[0]


def _ptr(a):
    return a.ctypes.data if a is not None else None


def _layout_dense(n):
    colour = np.arange(n, dtype=np.int32)
    diag = (np.arange(n) * (n + 1)).astype(np.int32)
    return dict(n_colours=n, colour=colour, lu_size=n * n, store=None, diag=diag, sparse=0)


def sparse_layout(pattern_mask, order):
    """The oracle's own CSR image of L + U for a mask and an elimination order.

    Computed here from scratch (symbolic elimination on the permuted pattern) so
    the oracle does not lean on the product's analysis.
    """
    mask = np.asarray(pattern_mask, dtype=bool)
    n = mask.shape[0]
    order = np.asarray(order, dtype=np.int64)
    inv = np.empty(n, dtype=np.int64)
    inv[order] = np.arange(n)
    filled = mask[np.ix_(order, order)].copy()
    np.fill_diagonal(filled, True)
    for k in range(n):
        for i in range(k + 1, n):
            if filled[i, k]:
                filled[i, k + 1:] |= filled[k, k + 1:]
    row_ptr = np.zeros(n + 1, dtype=np.int32)
    row_ptr[1:] = np.cumsum(filled.sum(axis=1))
    col_ind = np.concatenate([np.flatnonzero(filled[i]) for i in range(n)]).astype(np.int32)
    diag_ptr = np.array([row_ptr[i] + int(np.flatnonzero(col_ind[row_ptr[i]:row_ptr[i + 1]] == i)[0])
                         for i in range(n)], dtype=np.int32)
    slot = -np.ones((n, n), dtype=np.int64)
    for i in range(n):
        for p in range(row_ptr[i], row_ptr[i + 1]):
            slot[order[i], order[col_ind[p]]] = p
    return dict(row_ptr=row_ptr, col_ind=col_ind, diag_ptr=diag_ptr, order=order.astype(np.int32),
                slot=slot, nnz=int(row_ptr[-1]))


def _layout_sparse(mask, colour, order):
    n = mask.shape[0]
    lay = sparse_layout(mask, order)
    n_colours = int(max(colour)) + 1
    store = -np.ones(n * n_colours, dtype=np.int32)
    for r, c in zip(*np.nonzero(mask)):
        store[r * n_colours + colour[c]] = lay["slot"][r, c]
    diag = np.array([lay["slot"][i, i] for i in range(n)], dtype=np.int32)
    return dict(n_colours=n_colours, colour=np.asarray(colour, dtype=np.int32), lu_size=lay["nnz"],
                store=store, diag=diag, sparse=1, row_ptr=lay["row_ptr"], col_ind=lay["col_ind"],
                diag_ptr=lay["diag_ptr"], order=lay["order"])


def _broadcast(y0, params):
    y0 = np.asarray(y0, dtype=np.float64)
    params = np.asarray(params, dtype=np.float64)
    if y0.ndim == 1 and params.ndim == 1:
        n = 1
    elif y0.ndim == 2:
        n = y0.shape[0]
    else:
        n = params.shape[0]
    if y0.ndim == 1:
        y0 = np.broadcast_to(y0, (n, y0.shape[0]))
    if params.ndim == 1:
        params = np.broadcast_to(params, (n, params.shape[0]))
    return np.ascontiguousarray(y0), np.ascontiguousarray(params), n


def _sens_struct(system, sens):
    if sens is None:
        return _Sens(n_sens=0, n_y0_dirs=0, param_cols=None, error_control=1), None
    wrt_y0, param_cols, error_control = sens
    cols = np.asarray(param_cols, dtype=np.int32)
    n_y0 = system.n if wrt_y0 else 0
    s = _Sens(n_sens=n_y0 + len(cols), n_y0_dirs=n_y0,
              param_cols=cols.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if len(cols) else None,
              error_control=1 if error_control else 0)
    return s, cols


def augmented_y0(system, y0, sens):
    """``[y0, S(t0)]``: identity for the y0 block, zeros for parameter columns."""
    if sens is None:
        return y0
    wrt_y0, cols, _ = sens
    n = system.n
    blocks = [y0]
    if wrt_y0:
        blocks.append(np.broadcast_to(np.eye(n).reshape(1, -1), (y0.shape[0], n * n)))
    if len(cols):
        blocks.append(np.zeros((y0.shape[0], n * len(cols))))
    return np.ascontiguousarray(np.concatenate(blocks, axis=1))


def solve(solver, system: System, y0, t_span, params, *, rtol=1e-8, atol=1e-10, first_step=None,
          max_steps=100000, error_weights=None, pcoeff=0.0, icoeff=1.0, dcoeff=0.0,
          lu_precision="fp64", sparsity_mask=None, colour=None, order=None, tf_index=None,
          sens=None, threads=0):
    """Run the oracle; returns ``(hist, accepted, rejected, loop_steps)``.

    ``sens = (wrt_y0, param_columns, error_control)`` integrates the joint
    forward-sensitivity system (hist then has ``n * (1 + n_sens)`` components).
    """
    y0, params, n_traj = _broadcast(y0, params)
    y0 = augmented_y0(system, y0, sens)
    times = np.ascontiguousarray(np.asarray(t_span, dtype=np.float64))
    n_system = y0.shape[1]
    hist = np.empty((n_traj, times.shape[0], n_system))
    acc = np.empty(n_traj, dtype=np.int32)
    rej = np.empty(n_traj, dtype=np.int32)
    loop = np.empty(n_traj, dtype=np.int32)
    weights = None
    if error_weights is not None:
        weights = np.ascontiguousarray(np.broadcast_to(np.asarray(error_weights, dtype=np.float64), (n_traj, n_system)))
    desc, keep = system._desc()
    s, cols = _sens_struct(system, sens)
    ctl = _Controls(dt0=0.0 if first_step is None else float(first_step), rtol=rtol, atol=atol,
                    max_steps=int(max_steps), pcoeff=pcoeff, icoeff=icoeff, dcoeff=dcoeff,
                    tf_index=-1 if tf_index is None else int(tf_index))
    ens = _Ensemble(N=n_traj, n_system=n_system, np=params.shape[1], S=times.shape[0], y0=_ptr(y0),
                    times=_ptr(times), params=_ptr(params), weights=_ptr(weights), hist=_ptr(hist),
                    accepted=_ptr(acc), rejected=_ptr(rej), loop=_ptr(loop))
    if solver == "tsit5":
        lib().oracle_tsit5(ctypes.byref(desc), ctypes.byref(s), ctypes.byref(ctl), ctypes.byref(ens), threads)
    else:
        if sparsity_mask is None:
            lay = _layout_dense(system.n)
        else:
            lay = _layout_sparse(np.asarray(sparsity_mask, dtype=bool), colour, order)
        arrays = {k: (np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v) for k, v in lay.items()}
        L = _Layout(n_colours=arrays["n_colours"], colour=_ptr(arrays["colour"]), lu_size=arrays["lu_size"],
                    store=_ptr(arrays.get("store")), diag=_ptr(arrays["diag"]), sparse=arrays["sparse"],
                    row_ptr=_ptr(arrays.get("row_ptr")), col_ind=_ptr(arrays.get("col_ind")),
                    diag_ptr=_ptr(arrays.get("diag_ptr")), order=_ptr(arrays.get("order")))
        lib().oracle_rodas5p(ctypes.byref(desc), ctypes.byref(s), ctypes.byref(L), ctypes.byref(ctl),
                             ctypes.byref(ens), 1 if lu_precision == "fp32" else 0, threads)
    _raise_recorded(keep)
    del keep, cols
    return hist, acc, rej, loop


def jvp(system: System, y, t, p, vy, vt=0.0, vp=None):
    """Directional derivative of the system's right-hand side (host check of traced code)."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    p = np.ascontiguousarray(p, dtype=np.float64)
    vy = np.ascontiguousarray(vy, dtype=np.float64)
    vp = np.ascontiguousarray(np.zeros(system.np) if vp is None else vp, dtype=np.float64)
    out = np.empty(system.n)
    desc, keep = system._desc()
    lib().oracle_jvp(ctypes.byref(desc), _ptr(y), float(t), _ptr(p), _ptr(vy), float(vt), _ptr(vp), _ptr(out))
    _raise_recorded(keep)
    del keep
    return out


def jvp2(system: System, y, t, p, uy, ut, up, vy, vt, vp):
    """Second directional derivative D^2 f(y, t, p)[u, v] of the system's right-hand side."""
    arr = [np.ascontiguousarray(a, dtype=np.float64) for a in (y, p, uy, up, vy, vp)]
    y, p, uy, up, vy, vp = arr
    out = np.empty(system.n)
    desc, keep = system._desc()
    lib().oracle_jvp2(ctypes.byref(desc), _ptr(y), float(t), _ptr(p), _ptr(uy), float(ut), _ptr(up),
                      _ptr(vy), float(vt), _ptr(vp), _ptr(out))
    _raise_recorded(keep)
    del keep
    return out
