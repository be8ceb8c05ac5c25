"""Five-dimensional domain-wall operators (Operators/DiracOperators_5D.jl).

`D5DW_GeneralizedDomainwallOperator5D(U, L5, mass, M, a, b, c)` is
    D5 = A [1 - F + D_W (B + C F)]
with A, B, C the diagonal fifth-coordinate coefficients a_s, b_s, c_s
(DiracOperators_5D.jl:48-115, kernel :226-256), D_W = (4 + M) - 1/2 H the 4D
Wilson kernel on every s-slice with the shared 4D links, and F the chiral hop
in s (spins 1, 2 from s - 1, spins 3, 4 from s + 1, -mass across the walls;
apply_F_5D!, :862-915).  `D5DW_MobiusDomainwallOperator5D(U, L5, mass, M, b,
c)` (:8-46, kernel :171-202) is the same operator with a = 1,
b_s = (b + c)/2, c_s = (b - c)/2.  `adjoint(D)` gives D5^+ (:117-135,
:1507-1660).

Fields are 5D LatticeMatrix objects (NC, 4, X, Y, Z, T, L5) with nw >= 1
(_require_5d_halo, :155-159); their first four phases twist the 4D wraps and
the fifth is not used (the walls carry -mass).  Every application is one
liblmb200 call (lmb_domainwall_apply); `cg_(x, DdagDOp(D), b)` runs in
lmb_cg_ddagd with op = LMB_OP_DOMAINWALL.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from ._lib import ArgumentError, DimensionMismatch, PREC
from .lattice import require_single_rank, mark_halo_dirty_
from .operators import _Adjoint, _LinkOperator, _stream, _NC_SUPPORTED


class _DomainwallBase(_LinkOperator):
    """Context binding and argument checks shared by both forms."""

    _label = "D5DW operator"

    def _init(self, U, L5, mass, M, a, b, c):
        if len(U) != 4:
            raise ArgumentError(f"{self._label} requires four gauge links")
        if isinstance(L5, bool) or not isinstance(L5, (int, np.integer)):
            raise ArgumentError("L5 must be an integer")
        if L5 <= 0:
            raise ArgumentError("L5 must be positive")
        super().__init__(U)
        self.L5 = int(L5)
        self.mass = float(mass)
        self.M = float(M)
        # Wilson_parameters(kappa = 1/(2 Dim r + 2M), M) (:27-29, :96-98)
        self.kappa_wilson = 1.0 / (8.0 + 2.0 * self.M)
        self._abc = tuple(np.asarray(v, dtype=np.float64).copy() for v in (a, b, c))
        self._dw_key = None

    def abc(self):
        """get_abc: the coefficient vectors a, b, c (length L5 each)."""
        return self._abc

    def _bind(self, psi, stream):
        require_single_rank(psi)
        ctx = self.ctx
        ctx.set_geometry(psi.gsize[:4], psi.nw, psi.phases[:4],
                         psi.coords[:4], psi.dtype_code)
        ctx.upload_links(0, [u.data_ptr() for u in self.U],
                         [u.halo_epoch.core for u in self.U], stream)
        key = (self.L5, self.mass, self.M) + tuple(
            tuple(v.tolist()) for v in self._abc)
        if key != self._dw_key:
            a, b, c = (np.ascontiguousarray(v) for v in self._abc)
            dp = ctypes.POINTER(ctypes.c_double)
            ctx.check(ctx.lib.lmb_domainwall_set(
                ctx.handle, self.L5, self.mass, self.M,
                a.ctypes.data_as(dp), b.ctypes.data_as(dp),
                c.ctypes.data_as(dp), stream))
            self._dw_key = key
        return ctx

    def _validate(self, out, psi):
        require_single_rank(psi)
        if out is psi:
            raise ArgumentError("mul! requires distinct result and input fields")
        for f, what in ((out, "result"), (psi, "fermion")):
            if f.dim != 5:
                raise ArgumentError(
                    f"{self._label} acts on five-dimensional fields; the "
                    f"{what} field has dim={f.dim}")
            if f.NC2 != 4:
                raise ArgumentError("fermion fields must have 4 spin components per site")
        if psi.nw <= 0 or out.nw <= 0:
            raise ArgumentError(
                "5D Dirac operators do not support nw=0 yet; construct the "
                "5D fields with nw >= 1")
        if not out.same_geometry(psi) or out.phases != psi.phases:
            raise ArgumentError(
                "result and fermion fields must use the same lattice geometry")
        if out.NC1 != psi.NC1 or out.elementtype != psi.elementtype:
            raise ArgumentError("result and fermion fields must have the same type")
        if psi.gsize[4] != self.L5:
            raise DimensionMismatch(
                f"fermion field has fifth extent {psi.gsize[4]}, operator L5={self.L5}")
        for mu, link in enumerate(self.U, start=1):
            if link.NC1 != psi.NC1:
                raise ArgumentError(
                    f"gauge link U[{mu}] and fermion field have different color sizes")
            if link.elementtype != psi.elementtype:
                raise ArgumentError(
                    f"gauge link U[{mu}] and fermion field have different element types")
            if link.gsize != psi.gsize[:4] or link.nw != psi.nw:
                raise ArgumentError(
                    f"gauge link U[{mu}] and fermion field use different lattice geometry")
        if psi.NC1 != _NC_SUPPORTED:
            raise ArgumentError(
                f"the sm_100a kernels implement NC={_NC_SUPPORTED}; got NC={psi.NC1}")

    def _apply(self, out, psi, dagger, precision):
        self._validate(out, psi)
        st = _stream()
        ctx = self._bind(psi, st)
        ctx.check(ctx.lib.lmb_domainwall_apply(
            ctx.handle, out.data_ptr(), psi.data_ptr(), int(dagger),
            PREC[precision], st))
        mark_halo_dirty_(out)
        return out


class D5DW_GeneralizedDomainwallOperator5D(_DomainwallBase):
    """D5DW_GeneralizedDomainwallOperator5D(U, L5, mass, M, a, b, c)
    (DiracOperators_5D.jl:48-115)."""

    _label = "D5DW_GeneralizedDomainwallOperator5D"

    def __init__(self, U, L5, mass, M, a, b, c):
        if isinstance(L5, (int, np.integer)) and not isinstance(L5, bool) and L5 > 0:
            for name, coefficients in (("a", a), ("b", b), ("c", c)):
                if len(coefficients) != L5:
                    raise DimensionMismatch(
                        f"{name} must have length L5={L5}, got {len(coefficients)}")
        for name, coefficients in (("a", a), ("b", b), ("c", c)):
            if not all(math.isfinite(float(v)) for v in coefficients):
                raise ArgumentError(f"{name} coefficients must all be finite")
        self._init(U, L5, mass, M, a, b, c)

    def adjoint(self):
        return Adjoint_D5DW_GeneralizedDomainwallOperator5D(self)


class D5DW_MobiusDomainwallOperator5D(_DomainwallBase):
    """D5DW_MobiusDomainwallOperator5D(U, L5, mass, M, b, c)
    (DiracOperators_5D.jl:8-46): the generalised operator with a = 1,
    b_s = (b + c)/2, c_s = (b - c)/2 on every slice."""

    _label = "D5DW_MobiusDomainwallOperator5D"

    def __init__(self, U, L5, mass, M, b, c):
        self.b, self.c = float(b), float(c)
        n = int(L5) if isinstance(L5, (int, np.integer)) and L5 > 0 else 0
        self._init(U, L5, mass, M, [1.0] * n, [(self.b + self.c) / 2] * n,
                   [(self.b - self.c) / 2] * n)
        # the reference names the kernel the parameters select (:31-37)
        if self.b == 1 and self.c == 1:
            print("Shamir kernel (standard DW) is used")
        elif self.b == 2 and self.c == 0:
            print("Borici/Wilson kernel (truncated overlap) is used")
        elif self.b == 2 and self.c == 1:
            print("scaled Shamir kernel (Mobius DW) is used")

    def bc(self):
        """get_bc (DiracOperators_5D.jl:144-146)."""
        return self.b, self.c

    def adjoint(self):
        return Adjoint_D5DW_MobiusDomainwallOperator5D(self)


class Adjoint_D5DW_GeneralizedDomainwallOperator5D(_Adjoint):
    def _apply(self, out, psi, dagger, precision):
        return self.parent._apply(out, psi, not dagger, precision)


class Adjoint_D5DW_MobiusDomainwallOperator5D(_Adjoint):
    def _apply(self, out, psi, dagger, precision):
        return self.parent._apply(out, psi, not dagger, precision)
