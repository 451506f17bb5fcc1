"""ctypes binding of the C ABI in ``include/menodax.h`` and the library build.

The library is built in-tree (``menodax_b200/libmenodax_b200.so``) by
``build_library``; nothing here falls back to anything else when it is missing:
every entry point raises.  This is the Python counterpart of the reference's
``ffi_abi_call`` (``modax/_jax_numba_custom_call.py:333-371``).
"""

from __future__ import annotations

import ctypes
import hashlib
import os
import re
import subprocess
import threading
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
REPO_DIR = PKG_DIR.parent
CSRC = PKG_DIR / "csrc"
KERNEL_DIR = CSRC / "kernels"
INCLUDE_DIR = REPO_DIR / "include"
LIB_PATH = PKG_DIR / "libmenodax_b200.so"
CUBIN_CACHE = PKG_DIR / "_cubin_cache"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))

MDX_OK = 0
MDX_SOLVER_TSIT5 = 1
MDX_SOLVER_RODAS5P = 2
MDX_LAUNCH_PLAIN = 0
MDX_LAUNCH_PERSISTENT = 1
MDX_PLAN_CHECKPOINT = 1
MDX_PLAN_ADJOINT = 2
MDX_PLAN_SAVE_HOOK = 4
MDX_PLAN_NO_HISTORY = 8
MDX_MAX_SHARED_BYTES = 227 * 1024
MDX_STATUS_MAX_STEPS = 1
MDX_STATUS_NONFINITE = 2
MDX_STATUS_CKPT_OVERFLOW = 4

EXPORTED = (
    "mdx_compile", "mdx_free", "mdx_plan_create", "mdx_plan_destroy", "mdx_workspace_size",
    "mdx_occupancy", "mdx_solve", "mdx_grad", "mdx_last_error", "mdx_version",
    "mdx_measure_fma_peak", "mdx_solve_persistent_noalloc", "mdx_checkpoint_size",
)


class NativeError(RuntimeError):
    """A call into the native library failed; the message is the library's."""


class PlanDesc(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int), ("solver", ctypes.c_int), ("n_vars", ctypes.c_int),
        ("n_system", ctypes.c_int), ("n_params", ctypes.c_int),
        ("threads_per_block", ctypes.c_int), ("flags", ctypes.c_int), ("ckpt_stride", ctypes.c_int),
        ("team_size", ctypes.c_int), ("shared_bytes", ctypes.c_int),
        ("cubin", ctypes.c_void_p), ("cubin_size", ctypes.c_size_t),
    ]


class SolveDesc(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int), ("mode", ctypes.c_int), ("n_traj", ctypes.c_int),
        ("n_save", ctypes.c_int), ("n_save_hist", ctypes.c_int), ("max_steps", ctypes.c_int),
        ("dt0", ctypes.c_double), ("rtol", ctypes.c_double), ("atol", ctypes.c_double),
        ("y0", ctypes.c_void_p), ("times", ctypes.c_void_p), ("params", ctypes.c_void_p),
        ("weights", ctypes.c_void_p), ("hist", ctypes.c_void_p), ("accepted", ctypes.c_void_p),
        ("rejected", ctypes.c_void_p), ("loop_steps", ctypes.c_void_p), ("status", ctypes.c_void_p),
        ("hook_out", ctypes.c_void_p), ("order", ctypes.c_void_p), ("workspace", ctypes.c_void_p),
        ("workspace_bytes", ctypes.c_size_t), ("ckpt", ctypes.c_void_p),
        ("ckpt_count", ctypes.c_void_p), ("ckpt_capacity", ctypes.c_longlong),
        ("grid_blocks", ctypes.c_int), ("reserved", ctypes.c_int),
        ("hist_host", ctypes.c_void_p),
    ]


class GradDesc(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int), ("n_traj", ctypes.c_int), ("n_save", ctypes.c_int),
        ("count", ctypes.c_int), ("times", ctypes.c_void_p), ("params", ctypes.c_void_p),
        ("ckpt", ctypes.c_void_p), ("ckpt_count", ctypes.c_void_p),
        ("ckpt_capacity", ctypes.c_longlong), ("grad_hist", ctypes.c_void_p),
        ("grad_y0", ctypes.c_void_p), ("grad_params", ctypes.c_void_p), ("status", ctypes.c_void_p),
        ("order", ctypes.c_void_p), ("tasks", ctypes.c_void_p), ("n_tasks", ctypes.c_int),
        ("n_slots", ctypes.c_int), ("task_out", ctypes.c_void_p), ("combine", ctypes.c_void_p),
        ("n_combine", ctypes.c_int),
    ]


def _library_sources():
    return [CSRC / "mdx_runtime.cpp", CSRC / "mdx_peak.cu", CSRC / "mdx_noalloc.cu",
            CSRC / "mdx_internal.h", KERNEL_DIR / "mdx_args.h", INCLUDE_DIR / "menodax.h"]


def build_library(force: bool = False) -> Path:
    """Compile the native runtime into ``menodax_b200/libmenodax_b200.so``."""
    srcs = _library_sources()
    if LIB_PATH.exists() and not force:
        newest = max(s.stat().st_mtime for s in srcs)
        if LIB_PATH.stat().st_mtime >= newest:
            return LIB_PATH
    cmd = [
        str(CUDA_HOME / "bin" / "nvcc"), "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
        "-Xcompiler", "-Wall", f"-I{CUDA_HOME / 'include'}", str(CSRC / "mdx_runtime.cpp"), str(CSRC / "mdx_peak.cu"),
        str(CSRC / "mdx_noalloc.cu"),
        "-o", str(LIB_PATH), f"-L{CUDA_HOME / 'lib64'}", "-lnvrtc", "-ldl",
        f"-Xlinker=-rpath,{CUDA_HOME / 'lib64'}",
    ]
    subprocess.run(cmd, check=True)
    return LIB_PATH


_lib = None
_lib_lock = threading.Lock()


def lib():
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise NativeError(
                f"{LIB_PATH} is missing: build it with menodax_b200._native.build_library() "
                "(the solvers have no other implementation)"
            )
        L = ctypes.CDLL(str(LIB_PATH))
        L.mdx_compile.argtypes = [
            ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
            ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t), ctypes.c_char_p,
            ctypes.c_size_t,
        ]
        L.mdx_free.argtypes = [ctypes.c_void_p]
        L.mdx_free.restype = None
        L.mdx_plan_create.argtypes = [ctypes.POINTER(PlanDesc), ctypes.POINTER(ctypes.c_void_p)]
        L.mdx_plan_destroy.argtypes = [ctypes.c_void_p]
        L.mdx_workspace_size.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
        L.mdx_checkpoint_size.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.POINTER(ctypes.c_size_t)]
        L.mdx_occupancy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.mdx_solve.argtypes = [ctypes.c_void_p, ctypes.POINTER(SolveDesc), ctypes.c_void_p]
        L.mdx_grad.argtypes = [ctypes.c_void_p, ctypes.POINTER(GradDesc), ctypes.c_void_p]
        L.mdx_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        L.mdx_version.restype = ctypes.c_char_p
        L.mdx_solve_persistent_noalloc.argtypes = [ctypes.c_void_p, ctypes.POINTER(SolveDesc), ctypes.c_void_p]
        L.mdx_measure_fma_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        _lib = L
        return _lib


def measure_fma_peak(double_precision: bool = True) -> float:
    """FLOP/s of the current device's CUDA-core FMA pipe (an FMA counts two)."""
    out = ctypes.c_double()
    check(lib().mdx_measure_fma_peak(1 if double_precision else 0, ctypes.byref(out)), "mdx_measure_fma_peak")
    return out.value


def last_error() -> str:
    buf = ctypes.create_string_buffer(8192)
    lib().mdx_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int, what: str):
    if rc != MDX_OK:
        raise NativeError(f"{what} failed ({rc}): {last_error()}")


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.MULTILINE)
_header_text: dict[str, bytes] = {}


def _included_headers(source: str) -> list[str]:
    """The kernel headers ``source`` includes, directly or through other headers, sorted."""
    seen: set[str] = set()
    todo = _INCLUDE.findall(source)
    while todo:
        name = todo.pop()
        if name in seen:
            continue
        path = KERNEL_DIR / name
        if not path.is_file():
            continue
        seen.add(name)
        if name not in _header_text:
            _header_text[name] = path.read_bytes()
        todo.extend(_INCLUDE.findall(_header_text[name].decode()))
    return sorted(seen)


def compile_cubin(source: str, options: list[str], name: str = "mdx_problem.cu") -> bytes:
    """NVRTC-compile ``source`` for sm_100a, through an on-disk cache keyed on its
    text, the text of every kernel header it includes, and the options.  The key
    leaves out where the kernel headers sit on disk (their text is in it), so a
    cache built in one checkout serves another."""
    opts = [f"-I{KERNEL_DIR}", "-arch=sm_100a", "-std=c++17", "-default-device", "-lineinfo"] + list(options)
    h = hashlib.sha256()
    for part in (source, "-I<kernels>", *opts[1:]):
        h.update(part.encode())
        h.update(b"\0")
    for header in _included_headers(source):
        h.update(header.encode())
        h.update(_header_text[header])
    key = h.hexdigest()
    cache_dir = Path(os.environ.get("MENODAX_CUBIN_CACHE", CUBIN_CACHE))
    path = cache_dir / f"{key}.cubin"
    if path.exists():
        return path.read_bytes()
    arr = (ctypes.c_char_p * len(opts))(*[o.encode() for o in opts])
    out = ctypes.c_void_p()
    size = ctypes.c_size_t()
    log = ctypes.create_string_buffer(1 << 16)
    rc = lib().mdx_compile(source.encode(), name.encode(), arr, len(opts), ctypes.byref(out),
                           ctypes.byref(size), log, len(log))
    check(rc, "NVRTC compilation")
    data = ctypes.string_at(out, size.value)
    lib().mdx_free(out)
    try:
        cache_dir.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(f".tmp{os.getpid()}")
        tmp.write_bytes(data)
        os.replace(tmp, path)
    except OSError:
        pass
    return data


class Plan:
    """Owns one ``mdx_plan``: a compiled problem, loaded lazily per CUDA context."""

    def __init__(self, solver: int, n_vars: int, n_system: int, n_params: int, tpb: int,
                 flags: int, cubin: bytes, ckpt_stride: int = 1, team_size: int = 1,
                 shared_bytes: int = 0):
        self._cubin = ctypes.create_string_buffer(cubin, len(cubin))
        desc = PlanDesc(
            struct_size=ctypes.sizeof(PlanDesc), solver=solver, n_vars=n_vars, n_system=n_system,
            n_params=n_params, threads_per_block=tpb, flags=flags, ckpt_stride=ckpt_stride,
            team_size=team_size, shared_bytes=shared_bytes,
            cubin=ctypes.cast(self._cubin, ctypes.c_void_p), cubin_size=len(cubin),
        )
        handle = ctypes.c_void_p()
        check(lib().mdx_plan_create(ctypes.byref(desc), ctypes.byref(handle)), "mdx_plan_create")
        self.handle = handle
        self.tpb = tpb
        self.flags = flags
        self.team_size = team_size
        self.shared_bytes = shared_bytes
        self._lib = lib()

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.mdx_plan_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None

    def occupancy(self, mode: int) -> tuple[int, int]:
        b, s = ctypes.c_int(), ctypes.c_int()
        check(lib().mdx_occupancy(self.handle, mode, ctypes.byref(b), ctypes.byref(s)), "mdx_occupancy")
        return b.value, s.value

    def checkpoint_size(self, n_traj: int, capacity: int) -> int:
        out = ctypes.c_size_t()
        check(lib().mdx_checkpoint_size(self.handle, n_traj, capacity, ctypes.byref(out)), "mdx_checkpoint_size")
        return out.value

    def workspace_size(self, mode: int, n_traj: int) -> int:
        out = ctypes.c_size_t()
        check(lib().mdx_workspace_size(self.handle, mode, n_traj, ctypes.byref(out)), "mdx_workspace_size")
        return out.value

    def solve(self, desc: SolveDesc, stream: int):
        desc.struct_size = ctypes.sizeof(SolveDesc)
        check(lib().mdx_solve(self.handle, ctypes.byref(desc), ctypes.c_void_p(stream)), "mdx_solve")

    def grad(self, desc: GradDesc, stream: int):
        desc.struct_size = ctypes.sizeof(GradDesc)
        check(lib().mdx_grad(self.handle, ctypes.byref(desc), ctypes.c_void_p(stream)), "mdx_grad")
