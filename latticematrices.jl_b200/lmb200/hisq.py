"""HISQ link smearing and the cached HISQ operator, behind the reference's
names (Operators/HISQSmearing.jl, Operators/HISQFullSmearing.jl).

All smearing arithmetic is FP64 in liblmb200 (lmb_hisq_fat7,
lmb_hisq_project_u3, lmb_hisq_naik, lmb_hisq_links_from_thin)."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import ArgumentError, Context
from .lattice import require_single_rank, mark_halo_dirty_
from .operators import (HISQDiracOperator4D, HISQLinks4D, _AdjointApply,
                        _stream, _validate_staggered_application,
                        _validate_staggered_links)

LEVEL1 = (1 / 8, 1 / 16, 1 / 64, 1 / 384, 0.0)


def level2_coefficients(naik_epsilon):
    return (1 + naik_epsilon / 8, 1 / 16, 1 / 64, 1 / 384, -1 / 8)


_CTX = {}


def _ctx_for(field):
    dev = field.A.device.index or 0
    if dev not in _CTX:
        _CTX[dev] = Context(dev)
    c = _CTX[dev]
    require_single_rank(field)
    c.set_geometry(field.gsize, field.nw, (1, 1, 1, 1), field.coords,
                   field.dtype_code)
    return c


def _ptrs(fields):
    return (ctypes.c_void_p * 4)(*[f.data_ptr() for f in fields])


def _validate_smearing(out, inp):
    """_validate_hisq_smearing_output (HISQSmearing.jl:976-1000)."""
    _validate_staggered_links(inp)
    _validate_staggered_links(out)
    for o in out:
        if o.gsize != inp[0].gsize or o.nw != inp[0].nw or \
                (o.NC1, o.NC2) != (inp[0].NC1, inp[0].NC2) or \
                o.elementtype != inp[0].elementtype:
            raise ArgumentError(
                "HISQ smearing input and output links must share one geometry")
    for o in out:
        for i in inp:
            if o is i or o.A.data_ptr() == i.A.data_ptr():
                raise ArgumentError("HISQ smearing output must not alias its input")
    if inp[0].NC1 != 3:
        raise ArgumentError("HISQ smearing requires three-color links")


def _fat7(out, inp, coefficients):
    _validate_smearing(out, inp)
    c = _ctx_for(inp[0])
    coef = (ctypes.c_double * 5)(*[float(v) for v in coefficients])
    c.check(c.lib.lmb_hisq_fat7(c.handle, _ptrs(inp), coef, _ptrs(out),
                                _stream()))
    for o in out:
        mark_halo_dirty_(o)
    return out


def hisq_fat7_level1_(fat_links, thin_links):
    """hisq_fat7_level1! (HISQSmearing.jl:1112-1148)."""
    return _fat7(fat_links, thin_links, LEVEL1)


def hisq_fat7_level2_(fat_links, reunitarized_links, naik_epsilon=0.0):
    """hisq_fat7_level2! (HISQSmearing.jl:1313-1340)."""
    nw = reunitarized_links[0].nw
    if nw and nw < 2:
        raise ArgumentError("HISQ level-2 Fat7 smearing requires nw >= 2 or nw == 0")
    return _fat7(fat_links, reunitarized_links,
                 level2_coefficients(float(naik_epsilon)))


def hisq_project_u3_(projected_links, fat_links):
    """hisq_project_u3! (HISQFullSmearing.jl:100-128)."""
    _validate_smearing(projected_links, fat_links)
    c = _ctx_for(fat_links[0])
    c.check(c.lib.lmb_hisq_project_u3(c.handle, _ptrs(fat_links),
                                      _ptrs(projected_links), _stream()))
    for o in projected_links:
        mark_halo_dirty_(o)
    return projected_links


def hisq_naik_links_(long_links, reunitarized_links):
    """hisq_naik_links! (HISQFullSmearing.jl:151-195)."""
    nw = reunitarized_links[0].nw
    if nw and nw < 2:
        raise ArgumentError("HISQ Naik link construction requires nw >= 2 or nw == 0")
    _validate_smearing(long_links, reunitarized_links)
    c = _ctx_for(reunitarized_links[0])
    c.check(c.lib.lmb_hisq_naik(c.handle, _ptrs(reunitarized_links),
                                _ptrs(long_links), _stream()))
    for o in long_links:
        mark_halo_dirty_(o)
    return long_links


def hisq_links_from_thin(thin_links, naik_epsilon=0.0):
    """hisq_links_from_thin (HISQFullSmearing.jl:313-338): HISQLinks4D."""
    _validate_staggered_links(thin_links)
    if thin_links[0].NC1 != 3:
        raise ArgumentError("full HISQ smearing requires three-color thin links")
    nw = thin_links[0].nw
    if not (nw == 0 or nw >= 3):
        raise ArgumentError("full HISQ smearing requires nw=0 or nw>=3")
    fat = [u.similar() for u in thin_links]
    lng = [u.similar() for u in thin_links]
    c = _ctx_for(thin_links[0])
    ep = (ctypes.c_uint64 * 4)(*[u.halo_epoch.core for u in thin_links])
    c.check(c.lib.lmb_hisq_links_from_thin(
        c.handle, _ptrs(thin_links), ep, float(naik_epsilon), _ptrs(fat),
        _ptrs(lng), _stream()))
    for o in fat + lng:
        mark_halo_dirty_(o)
    return HISQLinks4D(fat, lng)


class HISQDiracCache4D:
    """Thin links -> cached HISQ links and operator (HISQFullSmearing.jl:
    340-441).  The smeared links live in the cache's lmb_ctx and are rebuilt
    when a thin link's identity or core epoch changes."""

    def __init__(self, thin_links, mass, naik_epsilon=0.0):
        _validate_staggered_links(thin_links)
        nw = thin_links[0].nw
        if not (nw == 0 or nw >= 3):
            raise ArgumentError("full HISQ smearing requires nw=0 or nw>=3")
        mass, eps = float(mass), float(naik_epsilon)
        if not np.isfinite(mass):
            raise ArgumentError("mass must be finite")
        if not np.isfinite(eps):
            raise ArgumentError("naik_epsilon must be finite")
        self.thin_links = list(thin_links)
        self.mass = mass
        self.naik_epsilon = eps
        dev = thin_links[0].A.device
        self.ctx = Context(dev.index or 0)

    def adjoint(self):
        return _AdjointApply(self)

    def update_(self, U):
        _validate_staggered_links(U)
        self.thin_links = list(U)
        return self

    def _bind(self, psi, stream):
        require_single_rank(psi)
        ctx = self.ctx
        ctx.set_geometry(psi.gsize, psi.nw, psi.phases, psi.coords,
                         psi.dtype_code)
        ep = (ctypes.c_uint64 * 4)(*[u.halo_epoch.core for u in self.thin_links])
        ctx.check(ctx.lib.lmb_hisq_links_from_thin(
            ctx.handle, _ptrs(self.thin_links), ep, self.naik_epsilon, None,
            None, stream))
        return ctx

    def _apply(self, out, psi, dagger, precision):
        from ._lib import PREC
        _validate_staggered_application(out, self.thin_links, psi)
        st = _stream()
        ctx = self._bind(psi, st)
        ctx.check(ctx.lib.lmb_hisq_apply(
            ctx.handle, out.data_ptr(), psi.data_ptr(), self.mass,
            self.naik_epsilon, int(dagger), PREC[precision], st))
        mark_halo_dirty_(out)
        return out


def mul_cached_hisq_(result, cache, U1, U2, U3, U4, psi):
    """mul_cached_hisq!(result, cache, U1, U2, U3, U4, psi)
    (HISQFullSmearing.jl:443-466)."""
    from .operators import mul_
    cache.update_([U1, U2, U3, U4])
    return mul_(result, cache, psi)


def mul_cached_hisq_adjoint_(result, cache, U1, U2, U3, U4, psi):
    """mul_cached_hisq_adjoint! (HISQFullSmearing.jl:468-485)."""
    from .operators import adjoint, mul_
    cache.update_([U1, U2, U3, U4])
    return mul_(result, adjoint(cache), psi)


def _validate_pullback(dthin_links, thin_links, result_cotangent, psi):
    """_validate_hisq_link_pullback (HISQPullback.jl:560-618)."""
    if len(dthin_links) != 4:
        raise ArgumentError("HISQ link pullback requires four thin-link cotangents")
    ref = thin_links[0]
    if (ref.NC1, ref.NC2) != (3, 3):
        raise ArgumentError("HISQ link pullback currently requires three-color thin links")
    if ref.nw < 3 and ref.nw != 0:
        raise ArgumentError("HISQ link pullback requires halo width nw >= 3")
    if (result_cotangent.NC1, result_cotangent.NC2, psi.NC1, psi.NC2) != (3, 1, 3, 1):
        raise ArgumentError(
            "HISQ link pullback requires three-color one-column fermion fields")
    if not result_cotangent.same_geometry(psi) or result_cotangent.phases != psi.phases:
        raise ArgumentError(
            "HISQ result cotangent and source must share geometry and boundary phases")
    if ref.gsize != psi.gsize or ref.nw != psi.nw:
        raise ArgumentError(
            "HISQ thin links and fermion fields must share one lattice geometry")
    if not (ref.elementtype == psi.elementtype == result_cotangent.elementtype):
        raise ArgumentError("HISQ links and fermion fields must share an element type")
    for d in dthin_links:
        if d.gsize != ref.gsize or d.nw != ref.nw or (d.NC1, d.NC2) != (3, 3):
            raise ArgumentError("HISQ thin-link cotangents must match the links")
        for u in thin_links:
            if d is u or d.A.data_ptr() == u.A.data_ptr():
                raise ArgumentError("HISQ thin-link cotangents must not alias primal links")


def hisq_link_pullback_(dthin_links, cache, thin_links, result_cotangent, psi,
                        coefficient=1.0):
    """hisq_link_pullback!(dthin_links, cache, thin_links, result_cotangent,
    psi; coefficient) (HISQPullback.jl:620-699): accumulate into dthin_links
    the thin-link gradient of coefficient * Re<result_cotangent, D(U) psi>."""
    _validate_pullback(dthin_links, thin_links, result_cotangent, psi)
    cache.update_(thin_links)
    st = _stream()
    ctx = cache.ctx
    require_single_rank(psi)
    ctx.set_geometry(psi.gsize, psi.nw, psi.phases, psi.coords, psi.dtype_code)
    ctx.check(ctx.lib.lmb_hisq_link_pullback(
        ctx.handle, _ptrs(thin_links), cache.naik_epsilon, float(coefficient),
        result_cotangent.data_ptr(), psi.data_ptr(), _ptrs(dthin_links), st))
    for d in dthin_links:
        mark_halo_dirty_(d)
    return dthin_links


def hisq_fermion_force_(dthin_links, cache, phi, *, rtol=1e-12, atol=0.0,
                        maxiter=20000, precision="double", delta=0.1):
    """dS/dU of S = phi^+ (D^+D)^-1 phi for the cached HISQ operator
    (dSFdU, ext/LatticeMatricesEnzymeExt.jl:387-460): eta = (D^+D)^-1 phi,
    chi = D eta, force accumulated into dthin_links.  Returns the CGResult."""
    from ._lib import CG_REASONS, CGParams, CGResultC, PREC
    from .solver import CGResult
    thin = cache.thin_links
    _validate_pullback(dthin_links, thin, phi, phi)
    prm = CGParams()
    prm.rtol, prm.atol, prm.maxiter = float(rtol), float(atol), int(maxiter)
    prm.precision = PREC[precision]
    prm.delta = float(delta)
    res = CGResultC()
    st = _stream()
    ctx = cache.ctx
    require_single_rank(phi)
    ctx.set_geometry(phi.gsize, phi.nw, phi.phases, phi.coords, phi.dtype_code)
    ep = (ctypes.c_uint64 * 4)(*[u.halo_epoch.core for u in thin])
    ctx.check(ctx.lib.lmb_hisq_fermion_force(
        ctx.handle, _ptrs(thin), ep, cache.mass, cache.naik_epsilon,
        phi.data_ptr(), _ptrs(dthin_links), ctypes.byref(prm),
        ctypes.byref(res), st))
    for d in dthin_links:
        mark_halo_dirty_(d)
    return CGResult(bool(res.converged), res.iterations, res.residual_norm,
                    res.relative_residual, CG_REASONS[res.reason],
                    res.reliable_updates, res.true_residual_norm)
