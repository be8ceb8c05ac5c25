"""Wilson-clover link pullback and fermion force (the adjoint of the
operator of operators.WilsonDiracCloverOperator4D)."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import ArgumentError
from .lattice import require_single_rank, mark_halo_dirty_
from .operators import WilsonDiracCloverOperator4D, _stream


def _ptrs(fields):
    return (ctypes.c_void_p * 4)(*[f.data_ptr() for f in fields])


def _validate(dlinks, cache, links, result_cotangent, psi):
    """_validate_wilson_clover_link_pullback (WilsonCloverPullback.jl:295-330)."""
    if not isinstance(cache, WilsonDiracCloverOperator4D):
        raise ArgumentError("Wilson--clover pullback needs a WilsonDiracCloverOperator4D")
    if len(dlinks) != 4:
        raise ArgumentError("Wilson--clover link pullback requires four destination links")
    if len(links) != 4:
        raise ArgumentError("Wilson--clover link pullback requires four primal links")
    if result_cotangent.nw < 1:
        raise ArgumentError("Wilson--clover link pullback requires nw >= 1")
    nc = result_cotangent.NC1
    for d in dlinks:
        if (d.NC1, d.NC2) != (nc, nc) or d.nw != result_cotangent.nw or d.gsize != result_cotangent.gsize:
            raise ArgumentError("Wilson--clover destination links must match the fermion lattice")
    for u in links:
        if (u.NC1, u.NC2) != (nc, nc) or u.nw != result_cotangent.nw or u.gsize != result_cotangent.gsize:
            raise ArgumentError("Wilson--clover primal links must match the fermion lattice")
    if result_cotangent.NC2 != 4 or psi.NC2 != 4:
        raise ArgumentError("Wilson--clover pullback requires four-spinor fields")
    if nc != 3:
        raise ArgumentError("the GPU Wilson--clover pullback is built for three colours")
    if not result_cotangent.same_geometry(psi) or result_cotangent.phases != psi.phases:
        raise ArgumentError("result cotangent and source must share geometry and boundary phases")
    if not all(f.elementtype == psi.elementtype for f in list(links) + list(dlinks) + [result_cotangent]):
        raise ArgumentError("links and fermion fields must share an element type")
    for d in dlinks:
        for u in links:
            if d is u or d.A.data_ptr() == u.A.data_ptr():
                raise ArgumentError("Wilson--clover link cotangents must not alias primal links")


def wilson_clover_link_pullback_(dlinks, cache, links, result_cotangent, psi, coefficient=1):
    """wilson_clover_link_pullback!(dlinks, cache, links, result_cotangent,
    psi; coefficient=1) (WilsonCloverPullback.jl:342-403): accumulate into
    dlinks the link gradient of coefficient * Re<result_cotangent,
    D(links) psi>, hopping and four-leaf clover terms included."""
    if not isinstance(coefficient, (int, float, np.floating, np.integer)) or isinstance(coefficient, bool):
        raise ArgumentError("Wilson--clover pullback coefficient must be real")
    _validate(dlinks, cache, links, result_cotangent, psi)
    st = _stream()
    ctx = cache.ctx
    require_single_rank(psi)
    ctx.set_geometry(psi.gsize, psi.nw, psi.phases, psi.coords, psi.dtype_code)
    ctx.check(ctx.lib.lmb_wilson_clover_link_pullback(
        ctx.handle, _ptrs(links), cache.kappa, cache.cSW, float(coefficient),
        result_cotangent.data_ptr(), psi.data_ptr(), _ptrs(dlinks), st))
    for d in dlinks:
        mark_halo_dirty_(d)
    return dlinks


def wilson_clover_fermion_force_(dlinks, D, phi, *, rtol=1e-12, atol=0.0, maxiter=20000,
                                 precision="double", delta=0.1):
    """dS/dU of S = phi^+ (D^+D)^-1 phi for a WilsonDiracCloverOperator4D:
    eta = (D^+D)^-1 phi by CG, chi = D eta, force = -2 d/dU Re<chi, D(U) eta>
    accumulated into dlinks.  Returns the CGResult of the solve."""
    from ._lib import CG_REASONS, CGParams, CGResultC, PREC
    from .solver import CGResult
    _validate(dlinks, D, D.U, phi, phi)
    prm = CGParams()
    prm.rtol, prm.atol, prm.maxiter = float(rtol), float(atol), int(maxiter)
    prm.precision = PREC[precision]
    prm.delta = float(delta)
    res = CGResultC()
    st = _stream()
    ctx = D.ctx
    require_single_rank(phi)
    ctx.set_geometry(phi.gsize, phi.nw, phi.phases, phi.coords, phi.dtype_code)
    ep = (ctypes.c_uint64 * 4)(*[u.halo_epoch.core for u in D.U])
    ctx.check(ctx.lib.lmb_wilson_clover_fermion_force(
        ctx.handle, _ptrs(D.U), ep, D.kappa, D.cSW, phi.data_ptr(), _ptrs(dlinks),
        ctypes.byref(prm), ctypes.byref(res), st))
    for d in dlinks:
        mark_halo_dirty_(d)
    return CGResult(bool(res.converged), res.iterations, res.residual_norm,
                    res.relative_residual, CG_REASONS[res.reason],
                    res.reliable_updates, res.true_residual_norm)
