"""Dirac operators behind the reference's operator API.

`mul_(out, D, psi)` is Julia's `mul!(out, D, psi)`; `adjoint(D)` gives the
adjoint operator as `D'` does.  Every application calls liblmb200 through its
C ABI on the device pointers of the LatticeMatrix storage; the operator keeps
its own lmb_ctx, which caches the repacked links and the clover blocks keyed
by link identity and core epoch (CloverCacheState,
WilsonDiracCloverOperator.jl:418-432).
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import (ArgumentError, Context, LINKS_THIN, PREC)
from .lattice import require_single_rank, LatticeMatrix, mark_halo_dirty_

_NC_SUPPORTED = 3


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _validate_links(U, what="gauge link"):
    if len(U) != 4:
        raise ArgumentError("U must be a vector of length 4")
    ref = U[0]
    if ref.NC1 != ref.NC2:
        raise ArgumentError("gauge links must be square matrices")
    for mu, link in enumerate(U, start=1):
        if (link.NC1, link.NC2) != (ref.NC1, ref.NC2):
            raise ArgumentError("all gauge links must have the same matrix size")
        if link.gsize != ref.gsize:
            raise ArgumentError("all gauge links must have the same global lattice size")
        if link.nw != ref.nw:
            raise ArgumentError("all gauge links must have the same halo width")
        if link.dims != ref.dims:
            raise ArgumentError("all gauge links must use the same process grid")
        if any(p != 1 for p in link.phases):
            raise ArgumentError(f"{what} U[{mu}] must use periodic boundary phases")
        if link.elementtype != ref.elementtype:
            raise ArgumentError("all gauge links must have the same element type")


def _validate_application(result, U, psi, nc2, split_ok=False):
    if not split_ok:
        require_single_rank(psi)
    elif psi.dims != (1,) * psi.dim:
        if psi.nw < 1:
            raise ArgumentError("a field split over a process grid needs nw >= 1 "
                                "for its neighbours' ghosts")
        if any(link.dims != psi.dims for link in U):
            raise ArgumentError("gauge links and fermion field use different process grids")
    if result is psi:
        raise ArgumentError("mul! requires distinct result and input fields")
    if not result.same_geometry(psi):
        raise ArgumentError("result and fermion fields must use the same lattice geometry")
    if result.phases != psi.phases:
        raise ArgumentError("result and fermion fields must use the same boundary phases")
    if psi.NC2 != nc2 or result.NC2 != nc2:
        raise ArgumentError(f"fermion fields must have {nc2} spin components per site")
    for mu, link in enumerate(U, start=1):
        if link.NC1 != psi.NC1:
            raise ArgumentError(
                f"gauge link U[{mu}] and fermion field have different color sizes")
        if link.elementtype != psi.elementtype:
            raise ArgumentError(
                f"gauge link U[{mu}] and fermion field have different element types")
        if link.gsize != psi.gsize or link.nw != psi.nw:
            raise ArgumentError(
                f"gauge link U[{mu}] and fermion field use different lattice geometry")
    if psi.NC1 != _NC_SUPPORTED:
        raise ArgumentError(
            f"the sm_100a kernels implement NC={_NC_SUPPORTED}; got NC={psi.NC1}")


class _Adjoint:
    def __init__(self, parent):
        self.parent = parent


def adjoint(op):
    """`op'`: adjoint wrapper; adjoint(adjoint(op)) is op."""
    if isinstance(op, _Adjoint):
        return op.parent
    if hasattr(op, "adjoint"):
        return op.adjoint()
    return _Adjoint(op)


class _LinkOperator:
    """Shared machinery: context, geometry and link upload."""

    def __init__(self, U):
        _validate_links(U)
        self.U = list(U)
        self._ctx = None

    @property
    def ctx(self) -> Context:
        if self._ctx is None:
            dev = self.U[0].A.device
            self._ctx = Context(dev.index or 0)
        return self._ctx

    def _bind(self, psi, stream):
        if psi.dims != (1,) * psi.dim:
            from .distributed import bind_grid, native_grid
            if native_grid(psi):   # NCCL: faces exchanged under the interior sites
                return bind_grid(self.ctx, psi, [(LINKS_THIN, self.U)], stream)
            return self._bind_block(psi, stream)
        ctx = self.ctx
        ctx.set_geometry(psi.gsize, psi.nw, psi.phases, psi.coords,
                         psi.dtype_code)
        ctx.upload_links(LINKS_THIN, [u.data_ptr() for u in self.U],
                         [u.halo_epoch.core for u in self.U], stream)
        return ctx

    def _bind_block(self, psi, stream):
        """A field split over a process grid: after the halo exchange
        (ensure_halo!, with the boundary phases) a rank's padded block of
        PN + 2 nw sites holds every neighbour of its core sites, the clover
        leaves' diagonal links included.  The kernels run on that block as a
        lattice of its own, with no wrap phase (the ghosts carry them); the
        core of their result is exact and its ghosts are left stale (the
        output is marked dirty)."""
        from .lattice import ensure_halo_
        for u in self.U:
            ensure_halo_(u)
        ensure_halo_(psi)
        ctx = self.ctx
        box = tuple(n + 2 * psi.nw for n in psi.PN)
        ctx.set_geometry(box, 0, (1, 1, 1, 1), (0, 0, 0, 0), psi.dtype_code)
        ctx.upload_links(LINKS_THIN, [u.data_ptr() for u in self.U],
                         [u.halo_epoch.core for u in self.U], stream)
        return ctx


class WilsonDiracOperator4D(_LinkOperator):
    """Wilson operator (WilsonDiracOperator.jl:1-76)."""

    def __init__(self, U, kappa):
        if len(U) != 4:
            raise ArgumentError("U must be a vector of length 4.")
        super().__init__(U)
        self.kappa = float(kappa)

    def adjoint(self):
        return AdjointWilsonDiracOperator4D(self)

    def _apply(self, out, psi, dagger, precision):
        _validate_application(out, self.U, psi, 4, split_ok=True)
        st = _stream()
        ctx = self._bind(psi, st)
        ctx.check(ctx.lib.lmb_wilson_apply(
            ctx.handle, out.data_ptr(), psi.data_ptr(), self.kappa,
            int(dagger), PREC[precision], st))
        mark_halo_dirty_(out)
        return out


class AdjointWilsonDiracOperator4D(_Adjoint):
    def _apply(self, out, psi, dagger, precision):
        return self.parent._apply(out, psi, not dagger, precision)


class CloverFieldStrength4D:
    """The six anti-Hermitian clover components (12,13,14,23,24,34)
    (WilsonDiracCloverOperator.jl:15-35)."""

    def __init__(self, operator):
        self.operator = operator
        self.components = None

    def refresh(self, psi_template):
        op = self.operator
        U = op.wilson.U
        st = _stream()
        ctx = op.wilson._bind(psi_template, st)
        comps = [U[0].similar() for _ in range(6)]
        arr = (ctypes.c_void_p * 6)(*[c.data_ptr() for c in comps])
        ctx.check(ctx.lib.lmb_clover_field_strength(ctx.handle, arr, st))
        for c in comps:
            mark_halo_dirty_(c)
        self.components = comps
        return self

    def __getitem__(self, i):
        return self.components[i]

    def __len__(self):
        return 6


class WilsonDiracCloverOperator4D:
    """D = D_W - kappa cSW sum_{mu<nu} g_mu g_nu F_mu_nu
    (WilsonDiracCloverOperator.jl:401-456)."""

    def __init__(self, U, kappa, cSW):
        self.wilson = WilsonDiracOperator4D(U, kappa)
        self.cSW = float(cSW)
        self.clover = CloverFieldStrength4D(self)

    @property
    def kappa(self):
        return self.wilson.kappa

    @property
    def U(self):
        return self.wilson.U

    @property
    def ctx(self):
        return self.wilson.ctx

    def adjoint(self):
        return AdjointWilsonDiracCloverOperator4D(self)

    def field_strength(self, psi_template=None):
        """Refresh and return the CloverFieldStrength4D components."""
        tmpl = psi_template
        if tmpl is None:
            tmpl = LatticeMatrix(3, 4, 4, self.U[0].gsize, nw=self.U[0].nw,
                                 elementtype=self.U[0].elementtype,
                                 device=self.U[0].A.device)
        return self.clover.refresh(tmpl)

    def _apply(self, out, psi, dagger, precision):
        _validate_application(out, self.U, psi, 4, split_ok=True)
        st = _stream()
        ctx = self.wilson._bind(psi, st)
        ctx.check(ctx.lib.lmb_wilson_clover_apply(
            ctx.handle, out.data_ptr(), psi.data_ptr(), self.kappa, self.cSW,
            int(dagger), PREC[precision], st))
        mark_halo_dirty_(out)
        return out


class AdjointWilsonDiracCloverOperator4D(_Adjoint):
    def _apply(self, out, psi, dagger, precision):
        return self.parent._apply(out, psi, not dagger, precision)


def update_clover_(operator, U=None):
    """update_clover!(operator[, U]) (WilsonDiracCloverOperator.jl:458-479).
    The link cache is keyed by link identity and core epoch, so a refresh
    only needs the new references."""
    if U is not None:
        _validate_links(U)
        operator.wilson.U[:] = list(U)
    return operator


def mul_(out, operator, psi, precision="double"):
    """mul!(out, operator, psi).  precision: "double" (the reference's
    arithmetic), or "single" / "half" storage for the inner solver."""
    if precision not in PREC:
        raise ArgumentError(f"unknown precision {precision!r}")
    if hasattr(operator, "_apply"):
        return operator._apply(out, psi, False, precision)
    if hasattr(operator, "mul_"):
        return operator.mul_(out, psi)
    raise ArgumentError(f"no mul! method for {type(operator).__name__}")


def mul_cached_clover_(result, cache, U1, U2, U3, U4, psi):
    """mul_cached_clover!(result, cache, U1, U2, U3, U4, psi)
    (WilsonDiracCloverOperator.jl:627-651): links given explicitly; the
    cached clover blocks are rebuilt when their identity or epoch changes."""
    update_clover_(cache, [U1, U2, U3, U4])
    return mul_(result, cache, psi)


def mul_cached_clover_adjoint_(result, cache, U1, U2, U3, U4, psi):
    """mul_cached_clover_adjoint! (WilsonDiracCloverOperator.jl:653-668)."""
    update_clover_(cache, [U1, U2, U3, U4])
    return mul_(result, adjoint(cache), psi)


# ---------------------------------------------------------------------------
# staggered and HISQ
# ---------------------------------------------------------------------------
def _validate_staggered_links(U, label="gauge link U"):
    """_validate_staggered_gauge_links (StaggeredDiracOperator.jl:23-45)."""
    if len(U) != 4:
        raise ArgumentError("U must be a vector of length 4")
    ref = U[0]
    if ref.NC1 != ref.NC2:
        raise ArgumentError("staggered gauge links must be square matrices")
    for mu, link in enumerate(U, start=1):
        if (link.NC1, link.NC2) != (ref.NC1, ref.NC2):
            raise ArgumentError("all gauge links must have the same matrix size")
        if link.gsize != ref.gsize:
            raise ArgumentError("all gauge links must have the same global lattice size")
        if link.nw != ref.nw:
            raise ArgumentError("all gauge links must have the same halo width")
        if any(p != 1 for p in link.phases):
            raise ArgumentError(f"{label}[{mu}] must use periodic boundary phases")


def _validate_staggered_application(result, links, psi, what="gauge link U",
                                    depth=1):
    """_validate_staggered_application (StaggeredDiracOperator.jl:66-92).
    A field split over a process grid runs on the native sharded stencils
    (CUDA fields on an NCCL group) with links split the same way and a halo
    of at least the stencil's reach `depth`; any other split field takes one
    rank per lattice."""
    from .distributed import native_grid
    if not native_grid(psi):
        require_single_rank(psi)
    elif psi.nw < depth or any(link.dims != psi.dims for link in links):
        raise ArgumentError(
            f"a field split over a process grid needs links split the same "
            f"way and nw >= {depth}")
    if result is psi:
        raise ArgumentError("staggered mul! requires distinct result and input fields")
    if not result.same_geometry(psi):
        raise ArgumentError("result and fermion fields must use the same lattice geometry")
    if result.phases != psi.phases:
        raise ArgumentError("result and fermion fields must use the same boundary phases")
    tol = np.sqrt(np.finfo(np.float32 if psi.elementtype == np.complex64
                           else np.float64).eps)
    for mu, ph in enumerate(psi.phases, start=1):
        if not np.isclose(abs(complex(ph)), 1.0, atol=tol, rtol=tol):
            raise ArgumentError(f"fermion boundary phase {mu} must have unit magnitude")
    if psi.NC2 != 1 or result.NC2 != 1:
        raise ArgumentError("staggered fields have one spin component per site")
    for mu, link in enumerate(links, start=1):
        if link.NC1 != psi.NC1:
            raise ArgumentError(
                f"{what}[{mu}] and fermion field have different color sizes")
        if link.elementtype != psi.elementtype:
            raise ArgumentError(
                f"{what}[{mu}] and fermion field have different element types")
        if link.gsize != psi.gsize or link.nw != psi.nw:
            raise ArgumentError(
                f"{what}[{mu}] and fermion field use different lattice geometry")
    if psi.NC1 != _NC_SUPPORTED:
        raise ArgumentError(
            f"the sm_100a kernels implement NC={_NC_SUPPORTED}; got NC={psi.NC1}")


class StaggeredDiracOperator4D(_LinkOperator):
    """One-link staggered operator, Bridge++ normalisation
    (StaggeredDiracOperator.jl:1-55)."""

    def __init__(self, U, mass):
        _validate_staggered_links(U)
        super().__init__(U)
        mass = float(mass)
        if not np.isfinite(mass):
            raise ArgumentError("mass must be finite")
        self.mass = mass

    def adjoint(self):
        return _AdjointApply(self)

    def _apply(self, out, psi, dagger, precision):
        _validate_staggered_application(out, self.U, psi)
        st = _stream()
        ctx = self._bind(psi, st)
        ctx.check(ctx.lib.lmb_staggered_apply(
            ctx.handle, out.data_ptr(), psi.data_ptr(), self.mass,
            int(dagger), PREC[precision], st))
        mark_halo_dirty_(out)
        return out


class _AdjointApply(_Adjoint):
    def _apply(self, out, psi, dagger, precision):
        return self.parent._apply(out, psi, not dagger, precision)


class HISQLinks4D:
    """Fat links X_mu and forward-anchored Naik links L_mu
    (HISQDiracOperator.jl:1-53)."""

    def __init__(self, fat_links, long_links):
        _validate_staggered_links(fat_links, "fat link X")
        _validate_staggered_links(long_links, "long link L")
        ref = fat_links[0]
        for mu, link in enumerate(long_links, start=1):
            if (link.NC1, link.NC2) != (ref.NC1, ref.NC2):
                raise ArgumentError(
                    f"long link L[{mu}] and fat links have different matrix sizes")
            if link.gsize != ref.gsize or link.nw != ref.nw:
                raise ArgumentError(
                    f"long link L[{mu}] and fat links use different lattice geometry")
            if link.elementtype != ref.elementtype:
                raise ArgumentError(
                    f"long link L[{mu}] and fat links have different element types")
        nw = ref.nw
        if not (nw == 0 or nw >= 3):
            raise ArgumentError(
                "HISQ links require nw=0 or nw>=3 for the three-hop Naik term")
        if nw and any(extent < nw for extent in ref.gsize):
            raise ArgumentError(
                f"each local lattice extent must be at least the halo width nw={nw}")
        self.fat_links = list(fat_links)
        self.long_links = list(long_links)


class HISQDiracOperator4D:
    """HISQ stencil (HISQDiracOperator.jl:55-110):
    m psi + sum eta {1/2 [X psi(x+mu) - X' psi(x-mu)]
                     - (1+eps)/48 [L psi(x+3mu) - L' psi(x-3mu)]}."""

    def __init__(self, links, mass, naik_epsilon=0.0):
        if not isinstance(links, HISQLinks4D):
            raise ArgumentError("HISQDiracOperator4D needs HISQLinks4D")
        mass, eps = float(mass), float(naik_epsilon)
        if not np.isfinite(mass):
            raise ArgumentError("mass must be finite")
        if not np.isfinite(eps):
            raise ArgumentError("naik_epsilon must be finite")
        self.links = links
        self.mass = mass
        self.naik_epsilon = eps
        self._ctx = None

    @property
    def ctx(self):
        if self._ctx is None:
            dev = self.links.fat_links[0].A.device
            self._ctx = Context(dev.index or 0)
        return self._ctx

    def adjoint(self):
        return _AdjointApply(self)

    def _bind(self, psi, stream):
        from ._lib import LINKS_FAT, LINKS_LONG
        from .distributed import bind_grid, native_grid
        if native_grid(psi):   # NCCL: three-layer faces under the interior sites
            return bind_grid(self.ctx, psi,
                             [(LINKS_FAT, self.links.fat_links),
                              (LINKS_LONG, self.links.long_links)], stream)
        require_single_rank(psi)
        ctx = self.ctx
        ctx.set_geometry(psi.gsize, psi.nw, psi.phases, psi.coords,
                         psi.dtype_code)
        for which, links in ((LINKS_FAT, self.links.fat_links),
                             (LINKS_LONG, self.links.long_links)):
            ctx.upload_links(which, [u.data_ptr() for u in links],
                             [u.halo_epoch.core for u in links], stream)
        return ctx

    def _apply(self, out, psi, dagger, precision):
        _validate_staggered_application(
            out, self.links.fat_links + self.links.long_links, psi,
            "fat link X", depth=3)
        st = _stream()
        ctx = self._bind(psi, st)
        ctx.check(ctx.lib.lmb_hisq_apply(
            ctx.handle, out.data_ptr(), psi.data_ptr(), self.mass,
            self.naik_epsilon, int(dagger), PREC[precision], st))
        mark_halo_dirty_(out)
        return out
