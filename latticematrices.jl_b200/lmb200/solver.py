"""CG on D'D behind the reference's solver API (LinearAlgebras/cg.jl,
Operators/DiracOperators.jl).

`cg_(x, DdagDOp(D, temp), b, r, p, Ap; ...)` with a Wilson or Wilson-clover D
runs the whole solve in liblmb200 (lmb_cg_ddagd): stencils, vector updates and
reductions on the GPU, scalars on the GPU, FP64 throughout by default or an
FP32 / int16 inner solve with FP64 reliable updates (precision="single" /
"half").  Any other operator (a user-defined one with `mul_`) runs the
reference's generic loop (cg.jl:73-137) on device tensors.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from ._lib import (ArgumentError, CG_REASONS, CGParams, CGResultC, PREC,
                   OP_DOMAINWALL, OP_HISQ, OP_STAGGERED, OP_WILSON,
                   OP_WILSON_CLOVER)
from .lattice import require_single_rank, LatticeMatrix, mark_halo_dirty_
from .operators import (HISQDiracOperator4D, StaggeredDiracOperator4D,
                        WilsonDiracCloverOperator4D, WilsonDiracOperator4D,
                        _stream, adjoint, mul_)


@dataclass
class CGResult:
    """CGResult (cg.jl:1-13)."""
    converged: bool
    iterations: int
    residual_norm: float
    relative_residual: float
    reason: str
    reliable_updates: int = 0
    true_residual_norm: float = float("nan")
    dslash_ms: float = 0.0
    update_ms: float = 0.0
    dslash_launches: int = 0
    update_launches: int = 0
    kernel_launches: int = 0
    link_reals: int = 18


class DdagDOp:
    """D' D with a caller-owned temporary (DiracOperators.jl:93-121)."""

    def __init__(self, D, temp=None):
        self.D = D
        self.temp = temp

    def adjoint(self):
        return self

    def mul_(self, y, x):
        if self.temp is None:
            raise ArgumentError("DdagDOp needs a temporary field")
        if self.temp is x or self.temp is y:
            raise ArgumentError(
                "DdagDOp temporary field must not alias its input or output")
        mul_(self.temp, self.D, x)
        mul_(y, adjoint(self.D), self.temp)
        return y


def _validate_cg_arguments(x, b, r, p, Ap, rtol, atol, maxiter):
    # cg.jl:33-47
    fields = (x, b, r, p, Ap)
    names = ("x", "b", "r", "p", "Ap")
    for i in range(len(fields)):
        for j in range(i + 1, len(fields)):
            if fields[i] is not None and fields[i] is fields[j]:
                raise ArgumentError(
                    f"CG fields {names[i]} and {names[j]} must not alias")
    if not rtol >= 0:
        raise ArgumentError("rtol must be nonnegative")
    if not atol >= 0:
        raise ArgumentError("atol must be nonnegative")
    if not math.isfinite(rtol):
        raise ArgumentError("rtol must be finite")
    if not math.isfinite(atol):
        raise ArgumentError("atol must be finite")
    if maxiter < 0:
        raise ArgumentError("maxiter must be nonnegative")


def _native_operator(A):
    if not isinstance(A, DdagDOp):
        return None
    D = A.D
    if isinstance(D, WilsonDiracCloverOperator4D):
        return D, OP_WILSON_CLOVER
    if isinstance(D, WilsonDiracOperator4D):
        return D, OP_WILSON
    if isinstance(D, StaggeredDiracOperator4D):
        return D, OP_STAGGERED
    if isinstance(D, HISQDiracOperator4D):
        return D, OP_HISQ
    from .hisq import HISQDiracCache4D
    if isinstance(D, HISQDiracCache4D):
        return D, OP_HISQ
    from .domainwall import _DomainwallBase
    if isinstance(D, _DomainwallBase):
        return D, OP_DOMAINWALL
    return None


def cg_(x, A, b, r=None, p=None, Ap=None, *, rtol=1e-10, atol=0.0,
        maxiter=5000, precision="double", delta=0.1, check_interval=0,
        profile=False):
    """cg!(x, A, b, r, p, Ap; rtol, atol, maxiter) -> CGResult."""
    _validate_cg_arguments(x, b, r, p, Ap, rtol, atol, maxiter)
    if precision not in PREC:
        raise ArgumentError(f"unknown precision {precision!r}")
    native = _native_operator(A)
    if native is not None and b.dims != (1,) * b.dim and not _grid_native(native[0], b):
        # fields split over a process grid: the reference's loop with
        # all-reduced dots, D applied per rank block (Wilson / clover only)
        if op_allows_blocks(native[0]) and precision == "double":
            return _cg_generic(x, A, b, r or b.similar(), p or b.similar(),
                               Ap or b.similar(), rtol, atol, maxiter)
        raise ArgumentError(
            "on a process grid cg! runs the Wilson and Wilson-clover "
            "operators in FP64; other operators and mixed precision take one "
            "rank per lattice")
    if native is not None:
        if not _grid_native(native[0], b):
            require_single_rank(b)
        D, op = native
        binder = D.wilson if op == OP_WILSON_CLOVER else D
        prm = CGParams()
        prm.op = op
        prm.kappa = getattr(D, "kappa", 0.0)
        prm.csw = getattr(D, "cSW", 0.0)
        prm.mass = getattr(D, "mass", 0.0)
        prm.naik_epsilon = getattr(D, "naik_epsilon", 0.0)
        prm.rtol, prm.atol, prm.maxiter = float(rtol), float(atol), int(maxiter)
        prm.precision = PREC[precision]
        prm.delta = float(delta)
        prm.check_interval = int(check_interval)
        prm.profile = int(bool(profile))
        st = _stream()
        if op == OP_DOMAINWALL:
            D._validate(x, b)
        ctx = binder._bind(b, st)
        res = CGResultC()
        ctx.check(ctx.lib.lmb_cg_ddagd(ctx.handle, ctypes.byref(prm),
                                       x.data_ptr(), b.data_ptr(),
                                       ctypes.byref(res), st))
        mark_halo_dirty_(x)
        return CGResult(bool(res.converged), res.iterations, res.residual_norm,
                        res.relative_residual, CG_REASONS[res.reason],
                        res.reliable_updates, res.true_residual_norm,
                        res.dslash_ms, res.update_ms, res.dslash_launches,
                        res.update_launches, res.kernel_launches,
                        res.link_reals)
    if precision != "double":
        raise ArgumentError("mixed precision needs a native DdagDOp operator")
    return _cg_generic(x, A, b, r, p, Ap, rtol, atol, maxiter)


def operator_timing(D, psi, napply=50, *, precision="double", dagger=False):
    """Device milliseconds per application of D (or D^+) on the library's
    resident fields (lmb_operator_timing): psi is packed once, then D is
    applied 2 + napply times with input and output swapped after each
    application, the last napply timed with CUDA events.  The loop of
    benchmark/hisq_dirac_scaling.jl:82-100 without its per-call layout: what
    one Krylov iteration pays for the stencil."""
    if precision not in PREC:
        raise ArgumentError(f"unknown precision {precision!r}")
    native = _native_operator(DdagDOp(D, psi))
    if native is None:
        raise ArgumentError("operator_timing needs a native Dirac operator")
    require_single_rank(psi)
    D, op = native
    binder = D.wilson if op == OP_WILSON_CLOVER else D
    prm = CGParams()
    prm.op = op
    prm.kappa = getattr(D, "kappa", 0.0)
    prm.csw = getattr(D, "cSW", 0.0)
    prm.mass = getattr(D, "mass", 0.0)
    prm.naik_epsilon = getattr(D, "naik_epsilon", 0.0)
    prm.precision = PREC[precision]
    st = _stream()
    ctx = binder._bind(psi, st)
    ms = ctypes.c_double()
    ctx.check(ctx.lib.lmb_operator_timing(ctx.handle, ctypes.byref(prm),
                                          psi.data_ptr(), int(napply),
                                          int(bool(dagger)), ctypes.byref(ms), st))
    return ms.value


def solve_evenodd_(x, D, b, *, rtol=1e-10, atol=0.0, maxiter=5000,
                   precision="double", delta=0.1, check_interval=0,
                   profile=False):
    """Solve D x = b for a Wilson or Wilson-clover D by even/odd (Schur)
    preconditioning (liblmb200 lmb_solve_evenodd): CG on Dh Dh^+ over the even
    sites, Dh = A_ee - kappa^2 H_eo A_oo^-1 H_oe, then the odd sites from
    x_o = A_oo^-1 (b_o + kappa H_oe x_e).  Parity as the reference's even/odd
    kernels (linearalgebra_D.jl:2815-2930).  With the reference API the same
    x comes from cg!(x, DdagDOp(D), D'b); here the solve stops on the FP64
    residual of D x = b itself, |b - D x| <= max(atol, rtol |b|)
    (true_residual_norm of the result).  Zero start; every extent even."""
    _validate_cg_arguments(x, b, None, None, None, rtol, atol, maxiter)
    if precision not in PREC:
        raise ArgumentError(f"unknown precision {precision!r}")
    if isinstance(D, WilsonDiracCloverOperator4D):
        op, binder = OP_WILSON_CLOVER, D.wilson
    elif isinstance(D, WilsonDiracOperator4D):
        op, binder = OP_WILSON, D
    else:
        raise ArgumentError(
            "solve_evenodd_ takes a WilsonDiracOperator4D or WilsonDiracCloverOperator4D")
    from .operators import _validate_application
    _validate_application(x, binder.U, b, 4)
    if any(v % 2 for v in b.gsize):
        raise ArgumentError(
            f"even/odd preconditioning needs even lattice extents, got {b.gsize}")
    prm = CGParams()
    prm.op = op
    prm.kappa = D.kappa
    prm.csw = getattr(D, "cSW", 0.0)
    prm.rtol, prm.atol, prm.maxiter = float(rtol), float(atol), int(maxiter)
    prm.precision = PREC[precision]
    prm.delta = float(delta)
    prm.check_interval = int(check_interval)
    prm.profile = int(bool(profile))
    st = _stream()
    ctx = binder._bind(b, st)
    res = CGResultC()
    ctx.check(ctx.lib.lmb_solve_evenodd(ctx.handle, ctypes.byref(prm),
                                        x.data_ptr(), b.data_ptr(),
                                        ctypes.byref(res), st))
    mark_halo_dirty_(x)
    return CGResult(bool(res.converged), res.iterations, res.residual_norm,
                    res.relative_residual, CG_REASONS[res.reason],
                    res.reliable_updates, res.true_residual_norm,
                    res.dslash_ms, res.update_ms, res.dslash_launches,
                    res.update_launches, res.kernel_launches, res.link_reals)


def _grid_native(D, b):
    """A field split over a process grid whose D'D CG runs natively: CUDA
    fields on an NCCL group, an operator with the sharded stencils (Wilson,
    Wilson-clover, staggered, HISQ on given fat / long links); every
    precision, the reductions summed over the ranks in the library."""
    from .distributed import native_grid
    from .hisq import HISQDiracCache4D
    if isinstance(D, HISQDiracCache4D):
        return False
    return native_grid(b) and isinstance(
        D, (WilsonDiracOperator4D, WilsonDiracCloverOperator4D,
            StaggeredDiracOperator4D, HISQDiracOperator4D))


def op_allows_blocks(D):
    return isinstance(D, (WilsonDiracOperator4D, WilsonDiracCloverOperator4D))


def _rdot(a: LatticeMatrix, b: LatticeMatrix) -> float:
    local = float((a.core_view().conj() * b.core_view()).sum().real)
    if a.dims != (1,) * a.dim:
        from .distributed import allreduce_complex
        return allreduce_complex(local, a.A.device).real
    return local


def _axpby(a, X, b, Y):
    Y.core_view().mul_(b).add_(X.core_view(), alpha=a)
    mark_halo_dirty_(Y)


def _result(conv, it, rn, bn, reason):
    rel = (0.0 if rn == 0 else math.inf) if bn == 0 else rn / bn
    return CGResult(conv, it, rn, rel, reason)


def _cg_generic(x, A, b, r, p, Ap, rtol, atol, maxiter):
    # cg.jl:73-137, line for line, for user-defined operators
    if r is None or p is None or Ap is None:
        raise ArgumentError("the generic CG needs caller-owned r, p, Ap")
    bb = _rdot(b, b)
    if not math.isfinite(bb) or bb < 0:
        return _result(False, 0, math.nan, math.nan, "numerical_breakdown")
    bn = math.sqrt(bb)
    tol = max(atol, rtol * bn)
    mul_(Ap, A, x)
    _axpby(1, b, 0, r)
    _axpby(-1, Ap, 1, r)
    _axpby(1, r, 0, p)
    rr = _rdot(r, r)
    if not math.isfinite(rr) or rr < 0:
        return _result(False, 0, math.nan, bn, "numerical_breakdown")
    rn = math.sqrt(rr)
    if rn <= tol:
        return _result(True, 0, rn, bn, "converged")
    for it in range(1, maxiter + 1):
        mul_(Ap, A, p)
        pAp = _rdot(p, Ap)
        if not math.isfinite(pAp):
            return _result(False, it - 1, rn, bn, "numerical_breakdown")
        if pAp <= 0:
            return _result(False, it - 1, rn, bn, "nonpositive_curvature")
        alpha = rr / pAp
        _axpby(alpha, p, 1, x)
        _axpby(-alpha, Ap, 1, r)
        rr_new = _rdot(r, r)
        if not math.isfinite(rr_new) or rr_new < 0:
            return _result(False, it, math.nan, bn, "numerical_breakdown")
        rn = math.sqrt(rr_new)
        if rn <= tol:
            return _result(True, it, rn, bn, "converged")
        beta = rr_new / rr
        _axpby(1, r, beta, p)
        rr = rr_new
    return _result(False, maxiter, rn, bn, "maximum_iterations")


def solve_(x, A, b, r=None, p=None, Ap=None, **kwargs):
    """solve!(x, A::DdagDOp, b, r, p, Ap; kwargs...) (DiracOperators.jl:130-143)."""
    return cg_(x, A, b, r, p, Ap, **kwargs)


def dot(a: LatticeMatrix, b: LatticeMatrix, ctx=None) -> complex:
    """dot(A, B) = sum conj(A) B over the core (linearalgebra_D.jl:3325-3341),
    reduced on the GPU by lmb_field_dot."""
    from ._lib import Context
    if not a.same_geometry(b) or (a.NC1, a.NC2) != (b.NC1, b.NC2):
        raise ArgumentError("dot requires fields of the same shape")
    if a.elementtype != b.elementtype:
        raise ArgumentError("dot requires fields of the same element type")
    ctx = ctx or _dot_context(a)
    # the local block (the whole lattice on one rank)
    ctx.set_geometry(a.PN, a.nw, a.phases, a.coords, a.dtype_code)
    out = (ctypes.c_double * 2)()
    st = _stream()
    ctx.check(ctx.lib.lmb_field_dot(ctx.handle, a.data_ptr(), b.data_ptr(),
                                    a.NC1 * a.NC2, out, st))
    local = complex(out[0], out[1])
    if a.dims != (1,) * a.dim:
        from .distributed import allreduce_complex
        return allreduce_complex(local, a.A.device)
    return local


_DOT_CTX = {}


def _dot_context(a):
    from ._lib import Context
    dev = a.A.device.index or 0
    if dev not in _DOT_CTX:
        _DOT_CTX[dev] = Context(dev)
    return _DOT_CTX[dev]


def pseudofermion_action(D, phi, eta, Deta, r, p, Ap, **kwargs):
    """real(dot(phi, (D'D)^-1 phi)) (DiracOperators.jl:145-163)."""
    res = solve_(eta, DdagDOp(D, Deta), phi, r, p, Ap, **kwargs)
    if not res.converged:
        raise RuntimeError(
            f"CG failed with reason {res.reason} after {res.iterations} "
            f"iterations; relative residual = {res.relative_residual}")
    return dot(phi, eta).real


def cg_batched_(systems, *, rtol=1e-10, atol=0.0, maxiter=5000, delta=0.1,
                check_interval=0, precision="single"):
    """Solve D'D x = b for every (x, b) of every system in one batched CG
    (lmb_cg_ddagd_batched): systems = [(WilsonDiracOperator4D, [(x, b), ...]),
    ...], lattices of any sizes.  FP32 arithmetic on FP32 (precision="single")
    or int16 (precision="half") iterated fields with FP64 reliable updates;
    each right-hand side stops on its own FP64 true residual.  Returns (list
    of CGResult per right-hand side, tuning dict)."""
    from ._lib import BatchLattice, BatchTuning
    if precision not in ("single", "half"):
        raise ArgumentError("the batched CG runs FP32 arithmetic on FP32 or int16 fields "
                            "(precision 'single' or 'half')")
    if not systems:
        raise ArgumentError("no systems")
    lats = (BatchLattice * len(systems))()
    keep = []
    ctx = None
    st = _stream()
    total = 0
    for i, (D, pairs) in enumerate(systems):
        if not isinstance(D, WilsonDiracOperator4D):
            raise ArgumentError("the batched CG is built for WilsonDiracOperator4D")
        if not pairs:
            raise ArgumentError("a system needs at least one right-hand side")
        for x, b in pairs:
            _validate_cg_arguments(x, b, None, None, None, rtol, atol, maxiter)
            if not x.same_geometry(b) or x.phases != b.phases:
                raise ArgumentError("x and b must share geometry and phases")
            if x.elementtype != np.complex128:
                raise ArgumentError("the batched CG takes ComplexF64 fields")
        b0 = pairs[0][1]
        lat = lats[i]
        lat.L = (ctypes.c_int * 4)(*b0.gsize)
        lat.nw = b0.nw
        lat.phase_re = (ctypes.c_double * 4)(*[complex(p).real for p in b0.phases])
        lat.phase_im = (ctypes.c_double * 4)(*[complex(p).imag for p in b0.phases])
        lat.U = (ctypes.c_void_p * 4)(*[u.data_ptr() for u in D.U])
        lat.epoch = (ctypes.c_uint64 * 4)(*[u.halo_epoch.core for u in D.U])
        lat.kappa = D.kappa
        lat.nrhs = len(pairs)
        xs = (ctypes.c_void_p * len(pairs))(*[x.data_ptr() for x, _ in pairs])
        bs = (ctypes.c_void_p * len(pairs))(*[b.data_ptr() for _, b in pairs])
        keep += [xs, bs]
        lat.x = ctypes.cast(xs, ctypes.POINTER(ctypes.c_void_p))
        lat.b = ctypes.cast(bs, ctypes.POINTER(ctypes.c_void_p))
        total += len(pairs)
        ctx = ctx or D.ctx
    prm = CGParams()
    prm.op = 0
    prm.kappa = 0.0
    prm.rtol, prm.atol, prm.maxiter = float(rtol), float(atol), int(maxiter)
    prm.precision = PREC[precision]
    prm.delta = float(delta)
    prm.check_interval = int(check_interval)
    res = (CGResultC * total)()
    tun = BatchTuning()
    ctx.check(ctx.lib.lmb_cg_ddagd_batched(ctx.handle, ctypes.byref(prm),
                                           len(systems), lats, res,
                                           ctypes.byref(tun), st))
    for _, pairs in systems:
        for x, _ in pairs:
            mark_halo_dirty_(x)
    out = [CGResult(bool(r.converged), r.iterations, r.residual_norm,
                    r.relative_residual, CG_REASONS[r.reason],
                    r.reliable_updates, r.true_residual_norm,
                    link_reals=r.link_reals) for r in res]
    return out, dict(rhs_block=tun.rhs_block, threads=tun.threads,
                     ms_per_iteration=tun.ms_per_iteration,
                     graph_iterations=tun.graph_iterations,
                     kernel_family=tun.kernel_family,
                     ms_stencils=tun.ms_stencils)
