"""Build the NVRTC source of one problem, compile it, and cache the plan.

This is the host-side planning layer of the reference (``KernelOptions`` and
``_make_kernel``, ``modax/rodas5P.py:137-165, 306-1007``; ``modax/tsit5.py:156-487``):
everything that selects a compiled kernel besides the right-hand side and the
shapes is a field of ``KernelOptions``, which is also the cache key.
"""

from __future__ import annotations

import threading
from dataclasses import dataclass

from menodax_b200 import _native
from menodax_b200._codegen import (
    SensLayout,
    emit_adjoint_pieces,
    emit_neg_jac,
    emit_rhs,
    emit_save_hook,
    emit_sens_coupling,
    lit,
)
from menodax_b200._sparse_direct import MAX_UNROLLED_SUBSTITUTIONS, sparse_lu_for
from menodax_b200._sparse_direct import emit_cuda as emit_sparse_lu
from menodax_b200._team import TEAM_SIZES, dense_lda, emit_team_adjoint_functions, emit_team_functions
from menodax_b200._team import slice_bytes as team_slice_bytes
from menodax_b200._sparsity import dense_jacobian
from menodax_b200._trace import trace, trace_array_rhs, trace_hook

TSIT5_EXPONENT = -1.0 / 5.0   # modax/tsit5.py:90
DENSE_UNROLL_MAX = 12          # mdx_dense_lu.cuh: register-resident dense LU up to this size
RODAS5P_EXPONENT = -1.0 / 6.0  # modax/rodas5P.py:113


@dataclass(frozen=True)
class KernelOptions:
    """Everything besides ``ode_fn`` and the sizes that selects a compiled kernel."""

    solver: str = "rodas5P"
    pcoeff: float = 0.0
    icoeff: float = 1.0
    dcoeff: float = 0.0
    lu_precision: str = "fp32"
    threads_per_block: int = 32
    min_blocks: int = 1
    sparsity: tuple | None = None
    ordering: str = "amd"
    sparse_code: str = "auto"
    tf_index: int = -1
    max_registers: int | None = None
    save_history: bool = True
    runtime_weights: bool = False
    # Forward sensitivities: (n_y0_dirs, param columns, error_control), or None.
    sens: tuple | None = None
    checkpoint: bool = False
    ckpt_stride: int = 1
    adjoint: bool = False
    # Fast arithmetic for the FP32-LU path: LU in the LU type throughout, the
    # reciprocal diagonal multiplied in, a float-precision controller exponent.
    fast: bool = False
    # A save hook hook(save_idx, y, t, p_row, acc) traced into the kernel, and the
    # width of its per-trajectory output row (modax/rodas5P.py:157-164).
    save_hook: object = None
    hook_size: int = 0
    # Lanes per trajectory: 0 for the thread-per-trajectory kernels, else 4, 8,
    # 16 or 32 for the team kernel (Rodas5P, no sensitivities, hooks or adjoint).
    team: int = 0
    # Tsit5: the stage vectors k1..k6 in shared memory, one column per thread
    # (the reference's "shared" backend, modax/tsit5.py:117-139).
    shared_stages: bool = False
    # Rodas5P: an array-form right-hand side array_rhs(y, t, p, out) for the stage
    # evaluations; derivatives still come from ode_fn (modax/rodas5P.py:382-391).
    array_rhs: object = None
    # Fast FP32-LU thread kernels: solve the stages in double against the
    # widened factors (True) or in FP32 (False); None picks by size (wide_solve).
    wide_solve: bool | None = None


def controller_exponents(options: KernelOptions):
    exponent = TSIT5_EXPONENT if options.solver == "tsit5" else RODAS5P_EXPONENT
    e1 = exponent * (options.icoeff + options.pcoeff + options.dcoeff)
    e2 = -exponent * (options.pcoeff + 2.0 * options.dcoeff)
    e3 = exponent * options.dcoeff
    return e1, e2, e3


@dataclass
class Problem:
    """A compiled problem: its plan plus what the host needs to call it."""

    plan: _native.Plan
    source: str
    n_vars: int
    n_system: int
    n_params: int
    n_error: int
    options: KernelOptions
    lu_size: int
    sparse: object = None
    hook_tables: tuple = ()


def _sens_layout(n_vars, n_params, sens):
    if sens is None:
        return None
    n_y0_dirs, cols, _ = sens
    return SensLayout(n_vars, n_params, n_y0_dirs, tuple(cols))


# Fast arithmetic on systems up to this size solves in double against the FP32
# factors by default (kernels/mdx_rodas5p.cuh, MDX_WIDE_SOLVE); larger thread
# kernels keep FP32 solves unless the autotuner measured the wide ones faster.
WIDE_SOLVE_MAX_VARS = 8


def wide_solve_applies(options: KernelOptions) -> bool:
    """Whether the build has the choice at all: a fast FP32-LU Rodas5P thread kernel."""
    return (options.solver == "rodas5P" and not options.team and options.fast
            and options.lu_precision == "fp32")


def wide_solve(options: KernelOptions, n_vars: int) -> bool:
    """Whether a thread-kernel Rodas5P build solves its stages in double against
    FP32 factors: ``options.wide_solve`` when set, else for systems of at most
    ``WIDE_SOLVE_MAX_VARS`` states (a joint sensitivity system follows its base
    system, so its state rows match the plain solve's)."""
    if not wide_solve_applies(options):
        return False
    if options.wide_solve is not None:
        return bool(options.wide_solve)
    return n_vars <= WIDE_SOLVE_MAX_VARS


def team_block_threads(n_vars: int, n_params: int, options: KernelOptions, preferred: int = 128) -> int:
    """Threads per block for a team launch: ``preferred`` or fewer, whole warps, and
    no more trajectories than a block's shared memory holds (a bound that assumes
    the slice carries ``df/dt``)."""
    team = int(options.team)
    lu_bytes = 4 if options.lu_precision == "fp32" else 8
    dense = options.sparsity is None
    if dense:
        lu_size = n_vars * dense_lda(n_vars)
    else:
        lu_size = sparse_lu_for(options.sparsity, options.ordering).slots.size
    per = team_slice_bytes(n_vars, n_params, lu_size, lu_bytes, dense=dense, autonomous=False,
                           fast=options.fast)
    fit = max(1, _native.MDX_MAX_SHARED_BYTES // per)
    threads = min(preferred // team, fit) * team
    threads = threads // 32 * 32
    if threads < 32:
        if 32 // team > fit:
            raise ValueError(f"a warp of {team}-lane teams needs {32 // team} slices of {per} B; "
                             "they exceed a block's shared memory")
        threads = 32
    return threads


def _build_team_source(tr, n_vars: int, n_params: int, options: KernelOptions, stage_tr=None):
    """The team kernel's source: class loops for f, -J and df/dt, the matrix in shared memory."""
    if options.solver != "rodas5P":
        raise ValueError("the team kernel runs Rodas5P")
    if options.team not in TEAM_SIZES:
        raise ValueError(f"team must be one of {TEAM_SIZES}; got {options.team}")
    if options.sens is not None:
        raise ValueError("the team kernel integrates the plain system: no forward sensitivities")
    if (options.checkpoint or options.adjoint) and options.sparsity is None:
        raise ValueError("the team kernel's checkpoints and reverse sweep need a sparse LU (a sparsity pattern)")
    tpb = int(options.threads_per_block)
    if tpb % 32 or tpb % options.team:
        raise ValueError(f"threads_per_block {tpb} is not a whole number of warps")
    lu_t = "float" if options.lu_precision == "fp32" else "double"
    lu_bytes = 4 if lu_t == "float" else 8
    e1, e2, e3 = controller_exponents(options)
    dense = options.sparsity is None
    extra = []
    if dense:
        structure = dense_jacobian(n_vars)
        lda = dense_lda(n_vars)
        lu_size = n_vars * lda
        code = emit_team_functions(tr, structure, lambda row, col: row * lda + col, skip_zero=True,
                                   stage_outputs=stage_tr.outputs if stage_tr is not None else None)
        clear = "-0.0"
        extra.append(f"#define MDX_TEAM_LDA {lda}")
        extra.append("__device__ __forceinline__ int mdx_team_diag_slot(int d) { return d * MDX_TEAM_LDA + d; }")
        sparse = None
        sparse_registers = 0
    else:
        sparse = sparse_lu_for(options.sparsity, options.ordering)
        structure = sparse.slots
        lu_size = structure.size
        store = structure.store_slots()

        def lu_slot(row, colour):
            slot = int(store[row * structure.n_colours + colour])
            return None if slot < 0 else slot

        code = emit_team_functions(tr, structure, lu_slot, skip_zero=False,
                                   stage_outputs=stage_tr.outputs if stage_tr is not None else None)
        clear = "0.0"
        diag = ", ".join(str(int(d)) for d in structure.diagonal)
        extra.append(f"__device__ const int mdx_team_diag[{n_vars}] = {{{diag}}};")
        extra.append("__device__ __forceinline__ int mdx_team_diag_slot(int d) { return mdx_team_diag[d]; }")
        extra.append(emit_sparse_lu(sparse.structure, options.sparse_code, fast=options.fast))
        substitutions = sparse.structure.counts()[2]
        sparse_registers = int(options.sparse_code == "unrolled" or (
            options.sparse_code == "auto" and substitutions <= MAX_UNROLLED_SUBSTITUTIONS))
    slice_size = team_slice_bytes(n_vars, n_params, lu_size, lu_bytes, dense=dense,
                                  autonomous=code.autonomous, fast=options.fast)
    shared = slice_size * (tpb // options.team)
    if shared > _native.MDX_MAX_SHARED_BYTES:
        raise ValueError(
            f"{tpb // options.team} trajectories of {slice_size} B exceed a block's shared memory; "
            "use fewer threads per block or a larger team")
    parts = [
        f"// generated problem source: rodas5P team kernel, n_vars={n_vars}, n_params={n_params}, "
        f"team={options.team}, {'dense' if dense else 'sparse'}",
        f"#define MDX_NV {n_vars}",
        f"#define MDX_NS {n_vars}",
        f"#define MDX_NP {n_params}",
        "#define MDX_NSENS 0",
        f"#define MDX_NERR {lit(float(n_vars))}",
        f"#define MDX_LU_T {lu_t}",
        f"#define MDX_TF_INDEX {int(options.tf_index)}",
        f"#define MDX_E1 {lit(e1)}",
        f"#define MDX_E2 {lit(e2)}",
        f"#define MDX_E3 {lit(e3)}",
        f"#define MDX_USE_E2 {'true' if e2 != 0.0 else 'false'}",
        f"#define MDX_USE_E3 {'true' if e3 != 0.0 else 'false'}",
        f"#define MDX_WEIGHTS_RUNTIME {1 if options.runtime_weights else 0}",
        f"#define MDX_SAVE_HISTORY {1 if options.save_history else 0}",
        f"#define MDX_CHECKPOINT {1 if options.checkpoint else 0}",
        f"#define MDX_CKPT_SEG {int(options.ckpt_stride)}",
        f"#define MDX_HAS_HOOK {1 if options.save_hook is not None else 0}",
        f"#define MDX_HOOK_SIZE {max(1, int(options.hook_size))}",
        f"#define MDX_FAST {1 if options.fast else 0}",
        f"#define MDX_TPB {tpb}",
        f"#define MDX_MIN_BLOCKS {int(options.min_blocks)}",
        f"#define MDX_TEAM {int(options.team)}",
        f"#define MDX_TEAM_DENSE {1 if dense else 0}",
        f"#define MDX_TEAM_LU_SIZE {lu_size}",
        f"#define MDX_TEAM_LU_CLEAR {clear}",
        f"#define MDX_TEAM_SLICE_BYTES {slice_size}",
        f"#define MDX_TEAM_SPARSE_REGISTERS {sparse_registers}",
        '#include "mdx_common.cuh"',
        "__device__ __forceinline__ double mdx_const_weight(int) { return 1.0; }",
        code.source,
        *extra,
    ]
    hook_tables = []
    if options.save_hook is not None:
        hook = trace_hook(options.save_hook, n_vars, n_params, int(options.hook_size))
        parts.append(emit_save_hook(hook))
        hook_tables = hook.bounds()
    parts.append('#include "mdx_team.cuh"')
    grad_bytes = 0
    if options.adjoint:
        grad_bytes = team_grad_slice_bytes(slice_size, n_vars, n_params, int(options.ckpt_stride),
                                           autonomous=code.autonomous)
        if (tpb // options.team) * grad_bytes > STATIC_SHARED_MAX:
            raise ValueError(
                f"{tpb // options.team} reverse-sweep slices of {grad_bytes} B exceed a block's static "
                f"shared memory; use fewer threads per block")
        parts.append(emit_team_adjoint_functions(tr))
        parts.append('#include "mdx_team_adjoint.cuh"')
    meta = dict(n_system=n_vars, n_error=n_vars, lu_size=lu_size, sparse=sparse, hook_tables=hook_tables,
                shared_bytes=shared, slice_bytes=slice_size, rhs_classes=code.n_rhs_classes,
                jac_classes=code.n_jac_classes, grad_slice_bytes=grad_bytes)
    return "\n".join(parts) + "\n", meta


STATIC_SHARED_MAX = 48 * 1024  # a block's static shared memory


def team_grad_slice_bytes(slice_bytes: int, n_vars: int, n_params: int, ckpt_stride: int, *,
                          autonomous: bool) -> int:
    """Bytes of one trajectory's reverse-sweep slice (``mdx::team_adjoint::GradSlice``):
    the forward slice, the eight stage cotangents, six (seven with df/dt) vectors,
    the parameter cotangent and the segment's start states and times."""
    doubles = 8 * n_vars + (6 if autonomous else 7) * n_vars + max(1, n_params)
    doubles += ckpt_stride * n_vars + ckpt_stride
    return slice_bytes + 8 * doubles


def team_grad_block_threads(n_vars: int, n_params: int, options: KernelOptions) -> int:
    """Threads per block of a team gradient module: as many whole-warp teams as let
    the reverse sweep's slices fit a block's static shared memory (and the forward
    slices its dynamic shared memory)."""
    team = int(options.team)
    sparse = sparse_lu_for(options.sparsity, options.ordering)
    lu_bytes = 4 if options.lu_precision == "fp32" else 8
    fwd = team_slice_bytes(n_vars, n_params, sparse.slots.size, lu_bytes, dense=False, autonomous=False,
                           fast=options.fast)
    grad = team_grad_slice_bytes(fwd, n_vars, n_params, int(options.ckpt_stride), autonomous=False)
    teams = max(1, min(STATIC_SHARED_MAX // grad, 128 // team))
    threads = teams * team // 32 * 32
    if threads < 32 or (threads // team) * grad > STATIC_SHARED_MAX:
        raise ValueError(f"a warp of {team}-lane teams needs {32 // team} reverse-sweep slices of {grad} B; "
                         "they exceed a block's static shared memory")
    return threads


def tsit5_stage_bytes(n_system: int, threads_per_block: int) -> int:
    """Shared memory of the Tsit5 kernel's stage arrays k1..k6 for one block."""
    return 6 * n_system * threads_per_block * 8


def build_source(ode_fn, n_vars: int, n_params: int, options: KernelOptions):
    """Generate the full NVRTC source; returns ``(source, meta)``."""
    tr = trace(ode_fn, n_vars, n_params)
    # The stage evaluations' right-hand side: array_rhs when given (the plain
    # solve only, as in the reference: a joint sensitivity system is built from
    # ode_fn), else ode_fn itself.
    stage_tr = tr
    if options.array_rhs is not None and options.sens is None:
        stage_tr = trace_array_rhs(options.array_rhs, tr)
    if options.shared_stages and options.solver != "tsit5":
        raise ValueError("shared_stages places Tsit5's stage vectors; Rodas5P's shared layout is the team kernel")
    if options.team:
        return _build_team_source(tr, n_vars, n_params, options, stage_tr)
    sens = _sens_layout(n_vars, n_params, options.sens)
    n_sens = 0 if sens is None else sens.n_sens
    n_system = n_vars * (1 + n_sens)
    error_control = True if options.sens is None else bool(options.sens[2])
    n_error = n_system if error_control else n_vars
    e1, e2, e3 = controller_exponents(options)
    rodas = options.solver == "rodas5P"
    lu_t = "float" if options.lu_precision == "fp32" else "double"
    wide = wide_solve(options, n_vars)
    parts = [
        f"// generated problem source: {options.solver}, n_vars={n_vars}, n_params={n_params}, n_sens={n_sens}",
        f"#define MDX_NV {n_vars}",
        f"#define MDX_NS {n_system}",
        f"#define MDX_NP {n_params}",
        f"#define MDX_NSENS {n_sens}",
        f"#define MDX_NERR {lit(float(n_error))}",
        f"#define MDX_LU_T {lu_t}",
        f"#define MDX_TF_INDEX {int(options.tf_index)}",
        f"#define MDX_E1 {lit(e1)}",
        f"#define MDX_E2 {lit(e2)}",
        f"#define MDX_E3 {lit(e3)}",
        f"#define MDX_USE_E2 {'true' if e2 != 0.0 else 'false'}",
        f"#define MDX_USE_E3 {'true' if e3 != 0.0 else 'false'}",
        f"#define MDX_WEIGHTS_RUNTIME {1 if options.runtime_weights else 0}",
        f"#define MDX_SAVE_HISTORY {1 if options.save_history else 0}",
        f"#define MDX_CHECKPOINT {1 if options.checkpoint else 0}",
        f"#define MDX_CKPT_SEG {int(options.ckpt_stride)}",
        f"#define MDX_FAST {1 if options.fast else 0}",
        f"#define MDX_HAS_HOOK {1 if options.save_hook is not None else 0}",
        f"#define MDX_HOOK_SIZE {max(1, int(options.hook_size))}",
        f"#define MDX_TPB {int(options.threads_per_block)}",
        f"#define MDX_MIN_BLOCKS {int(options.min_blocks)}",
        f"#define MDX_SOLVE_T {'double' if wide else lu_t}",
        f"#define MDX_WIDE_SOLVE {1 if wide else 0}",
        '#include "mdx_common.cuh"',
    ]
    sens_weight = "1.0" if error_control else "0.0"
    parts.append(
        "__device__ __forceinline__ double mdx_const_weight(int j) "
        f"{{ return j < MDX_NV ? 1.0 : {sens_weight}; }}"
    )
    parts.append(emit_rhs(stage_tr, sens))
    lu_size = 0
    sparse = None
    if rodas:
        if options.sparsity is None and options.fast and n_vars <= DENSE_UNROLL_MAX:
            structure = dense_jacobian(n_vars)
            lu_size = n_vars * n_vars
            parts.append(f"#define MDX_LU_SIZE {lu_size}")
            parts.append(f"#define MDX_IPIV {n_vars}")
            parts.append('#include "mdx_dense_lu.cuh"')
            parts.append(
                "template <class LU, class IP> __device__ __forceinline__ void mdx_factorize(LU& lu, IP& ipiv) "
                "{ mdx::dense_factorize_fast<MDX_NV, MDX_LU_T>(lu, ipiv); }\n"
                "template <class LU, class IP, class R> __device__ __forceinline__ void mdx_solve(const LU& lu, const IP& ipiv, R& rhs) "
                "{ mdx::dense_solve_fast<MDX_NV, MDX_SOLVE_T>(lu, ipiv, rhs); }\n"
                "template <class LU, class IP, class R> __device__ __forceinline__ void mdx_solve_t(const LU& lu, const IP& ipiv, R& rhs) "
                "{ mdx::dense_solve_t_fast<MDX_NV, MDX_SOLVE_T>(lu, ipiv, rhs); }\n"
                "__device__ __forceinline__ int mdx_diag_slot(int d) { return d * MDX_NV + d; }"
            )
        elif options.sparsity is None:
            structure = dense_jacobian(n_vars)
            lu_size = n_vars * n_vars
            parts.append(f"#define MDX_LU_SIZE {lu_size}")
            parts.append(f"#define MDX_IPIV {n_vars}")
            parts.append('#include "mdx_dense_lu.cuh"')
            parts.append(
                "template <class LU, class IP> __device__ __forceinline__ void mdx_factorize(LU& lu, IP& ipiv) "
                "{ mdx::dense_factorize<MDX_NV, MDX_LU_T>(lu, ipiv); }\n"
                "template <class LU, class IP, class R> __device__ __forceinline__ void mdx_solve(const LU& lu, const IP& ipiv, R& rhs) "
                "{ mdx::dense_solve<MDX_NV, MDX_SOLVE_T>(lu, ipiv, rhs); }\n"
                "template <class LU, class IP, class R> __device__ __forceinline__ void mdx_solve_t(const LU& lu, const IP& ipiv, R& rhs) "
                "{ mdx::dense_solve_t<MDX_NV, MDX_SOLVE_T>(lu, ipiv, rhs); }\n"
                "__device__ __forceinline__ int mdx_diag_slot(int d) { return d * MDX_NV + d; }"
            )
        else:
            sparse = sparse_lu_for(options.sparsity, options.ordering)
            structure = sparse.slots
            lu_size = structure.size
            parts.append(f"#define MDX_LU_SIZE {lu_size}")
            parts.append("#define MDX_IPIV 1")
            parts.append(emit_sparse_lu(sparse.structure, options.sparse_code, fast=options.fast))
            diag = structure.diagonal
            cases = " ".join(f"case {d}: return {int(s)};" for d, s in enumerate(diag))
            parts.append(
                "template <class LU, class IP> __device__ __forceinline__ void mdx_factorize(LU& lu, IP&) "
                "{ mdx_sparse_factorize<MDX_LU_T>(lu); }\n"
                "template <class LU, class IP, class R> __device__ __forceinline__ void mdx_solve(const LU& lu, const IP&, R& rhs) "
                "{ mdx_sparse_solve<MDX_SOLVE_T>(lu, rhs); }\n"
                "template <class LU, class IP, class R> __device__ __forceinline__ void mdx_solve_t(const LU& lu, const IP&, R& rhs) "
                "{ mdx_sparse_solve_t<MDX_SOLVE_T>(lu, rhs); }\n"
                f"__device__ __forceinline__ int mdx_diag_slot(int d) {{ switch (d) {{ {cases} default: return 0; }} }}"
            )
        parts.append(emit_neg_jac(tr, structure, lu_size, sens))
        # df/dt structurally zero (and no sensitivity rows): the stages skip its terms.
        autonomous = sens is None and all(
            x is None for x in tr.graph.forward(tr.outputs, {tr.t: tr.graph.const(1.0)}))
        parts.append(f"#define MDX_AUTONOMOUS {1 if autonomous else 0}")
        if options.save_hook is not None:
            hook = trace_hook(options.save_hook, n_system, n_params, int(options.hook_size))
            parts.append(emit_save_hook(hook))
            meta_tables = hook.bounds()
        else:
            meta_tables = []
        if sens is not None:
            parts.append(emit_sens_coupling(tr, sens))
        parts.append('#include "mdx_rodas5p.cuh"')
        parts.append("#define MDX_SOLVER mdx::Rodas5P")
    else:
        meta_tables = []
        parts.append("#define MDX_LU_SIZE 1")
        if options.shared_stages:
            stage_bytes = tsit5_stage_bytes(n_system, int(options.threads_per_block))
            if stage_bytes > STATIC_SHARED_MAX:
                raise ValueError(
                    f"shared Tsit5 stages of {n_system} components x {options.threads_per_block} threads take "
                    f"{stage_bytes} B of shared memory; at most {STATIC_SHARED_MAX} B")
        parts.append(f"#define MDX_TSIT5_SHARED {1 if options.shared_stages else 0}")
        parts.append('#include "mdx_tsit5.cuh"')
        parts.append("#define MDX_SOLVER mdx::Tsit5")
    parts.append('#include "mdx_entry.cuh"')
    if options.adjoint:
        if sens is not None:
            raise ValueError("the discrete adjoint differentiates the plain solve; drop sens")
        parts.append(emit_adjoint_pieces(tr))
        parts.append("#define MDX_ADJOINT_RODAS5P" if rodas else "#define MDX_ADJOINT_TSIT5")
        parts.append('#include "mdx_adjoint.cuh"')
    meta = dict(n_system=n_system, n_error=n_error, lu_size=lu_size, sparse=sparse,
                hook_tables=meta_tables, shared_bytes=0)
    return "\n".join(parts) + "\n", meta


def compile_options(options: KernelOptions) -> list[str]:
    opts = []
    if options.max_registers is not None:
        opts.append(f"--maxrregcount={int(options.max_registers)}")
    return opts


_cache: dict = {}
_cache_lock = threading.Lock()


def get_problem(ode_fn, n_vars: int, n_params: int, options: KernelOptions) -> Problem:
    """The compiled problem for these options, built once per process."""
    key = (ode_fn, n_vars, n_params, options)
    with _cache_lock:
        found = _cache.get(key)
    if found is not None:
        return found
    source, meta = build_source(ode_fn, n_vars, n_params, options)
    cubin = _native.compile_cubin(source, compile_options(options))
    flags = (_native.MDX_PLAN_CHECKPOINT if options.checkpoint else 0) | (
        _native.MDX_PLAN_ADJOINT if options.adjoint else 0
    ) | (_native.MDX_PLAN_SAVE_HOOK if options.save_hook is not None else 0) | (
        0 if options.save_history else _native.MDX_PLAN_NO_HISTORY
    )
    solver = _native.MDX_SOLVER_TSIT5 if options.solver == "tsit5" else _native.MDX_SOLVER_RODAS5P
    plan = _native.Plan(solver, n_vars, meta["n_system"], n_params, options.threads_per_block, flags, cubin,
                        ckpt_stride=int(options.ckpt_stride), team_size=max(1, int(options.team)),
                        shared_bytes=int(meta["shared_bytes"]))
    prob = Problem(
        plan=plan, source=source, n_vars=n_vars, n_system=meta["n_system"], n_params=n_params,
        n_error=meta["n_error"], options=options, lu_size=meta["lu_size"], sparse=meta["sparse"],
        hook_tables=tuple(meta["hook_tables"]),
    )
    with _cache_lock:
        _cache.setdefault(key, prob)
        return _cache[key]


def clear_caches() -> None:
    """Drop every compiled problem (``modax/tsit5.py:142-153``)."""
    with _cache_lock:
        _cache.clear()
    sparse_lu_for.cache_clear()
