"""LatticeMatrix: a halo-padded 4D (or 5D domain-wall) field in device memory.

Mirrors the reference container LatticeMatrix_standard
(LatticeMatrices_core.jl:159-184, constructors :297-461): element (ic, jc) of
site (x, y, z, t) sits at column-major position
(ic, jc, x+nw, y+nw, z+nw, t+nw) of an (NC1, NC2, X+2nw, Y+2nw, Z+2nw, T+2nw)
complex array.  The storage is a torch tensor of the reversed shape, so its
bytes are exactly the bytes of the CuArray behind a Julia LatticeMatrix, and
its data pointer is what the C ABI receives.  A 5D field (domain-wall
fermions, DiracOperators_5D.jl) adds the fifth coordinate s as the slowest
index: (NC1, NC2, X+2nw, .., T+2nw, L5+2nw).

Single-rank only (PEs = (1,1,1,1)): the halo is never filled, because the
kernels wrap periodically with the fermion phase; `halo_epoch` still tracks
core writes so that link caches can be invalidated exactly as
mark_halo_dirty! does (LatticeMatrices_core.jl:196-203).
"""
from __future__ import annotations

import numpy as np

from ._lib import ArgumentError

_DTYPES = {np.dtype(np.complex128): 0, np.dtype(np.complex64): 1}


class HaloEpoch:
    __slots__ = ("core", "halo")

    def __init__(self):
        self.core = 0
        self.halo = 0


class LatticeMatrix:
    """`LatticeMatrix(NC1, NC2, dim, gsize, PEs; nw, elementtype, phases)`."""

    def __init__(self, NC1, NC2, dim, gsize, PEs=None, *, nw=1,
                 elementtype=np.complex128, phases=None, device="cuda"):
        # validation follows LatticeMatrices_core.jl:315-343
        if PEs is None:
            PEs = (1,) * dim
        if nw < 0:
            raise ArgumentError(f"nw must be non-negative, got {nw}")
        if dim not in (4, 5):
            raise ArgumentError(
                "the B200 path handles four-dimensional lattices and "
                "five-dimensional domain-wall fields")
        gsize = tuple(int(v) for v in gsize)
        if len(gsize) != dim:
            raise ArgumentError(
                f"global size must have {dim} entries, got {len(gsize)}")
        if len(PEs) != dim:
            raise ArgumentError(
                f"process grid must have {dim} entries, got {len(PEs)}")
        phases = tuple(phases) if phases is not None else (1,) * dim
        if len(phases) != dim:
            raise ArgumentError(
                f"phases must have {dim} entries, got {len(phases)}")
        if NC1 <= 0 or NC2 <= 0:
            raise ArgumentError("matrix dimensions must be positive")
        if any(v <= 0 for v in gsize):
            raise ArgumentError(
                f"global lattice sizes must be positive, got {gsize}")
        if any(p == 0 for p in phases):
            raise ArgumentError(
                "boundary phases must be nonzero because negative wraps use inv(phase)")
        if tuple(PEs) != (1,) * dim:
            raise ArgumentError(
                "one process per GPU: this build takes a single-rank process grid")
        for d in range(dim):
            if nw > gsize[d]:
                raise ArgumentError(
                    f"halo width nw={nw} exceeds local lattice size {gsize[d]} "
                    f"in dimension {d + 1}; the nearest-neighbor halo exchange "
                    f"requires nw <= local size")
        dt = np.dtype(elementtype)
        if dt not in _DTYPES:
            raise ArgumentError(f"unsupported element type {dt}")
        import torch
        self.NC1, self.NC2, self.dim = int(NC1), int(NC2), dim
        self.gsize = gsize
        self.PN = gsize
        self.nw = int(nw)
        self.phases = tuple(phases)
        self.elementtype = dt
        self.coords = (0,) * dim
        self.dims = (1,) * dim
        self.halo_epoch = HaloEpoch()
        padded = tuple(v + 2 * self.nw for v in gsize)
        tdt = torch.complex128 if dt == np.complex128 else torch.complex64
        self.A = torch.zeros(padded[::-1] + (self.NC2, self.NC1), dtype=tdt,
                             device=device)

    # -- construction from a host array (LatticeMatrices_core.jl:405-461) --
    @classmethod
    def from_array(cls, A, dim=4, PEs=None, *, nw=1, phases=None,
                   device="cuda"):
        A = np.asarray(A)
        NC1, NC2 = A.shape[:2]
        if PEs is None:
            PEs = (1,) * dim
        lm = cls(NC1, NC2, dim, A.shape[2:], PEs, nw=nw,
                 elementtype=A.dtype, phases=phases, device=device)
        lm.set_core(A)
        return lm

    @property
    def dtype_code(self) -> int:
        return _DTYPES[self.elementtype]

    def data_ptr(self) -> int:
        return self.A.data_ptr()

    def core_view(self):
        n = self.nw
        return self.A[tuple(slice(n, n + v) for v in self.gsize[::-1])]

    def set_core(self, A):
        import torch
        A = np.asarray(A, dtype=self.elementtype)
        if A.shape != (self.NC1, self.NC2) + self.gsize:
            raise ArgumentError(
                f"array shape {A.shape} does not match lattice "
                f"{(self.NC1, self.NC2) + self.gsize}")
        host = torch.from_numpy(np.ascontiguousarray(A.T))
        self.core_view().copy_(host.to(self.A.device))
        mark_halo_dirty_(self)

    def gather_matrix(self):
        """Core values as a Fortran-ordered (NC1, NC2, X, Y, Z, T[, L5]) array
        (gather_matrix, LatticeMatrices_core.jl:936-993)."""
        return np.asfortranarray(self.core_view().cpu().numpy().T)

    def similar(self):
        return LatticeMatrix(self.NC1, self.NC2, self.dim, self.gsize,
                             self.dims, nw=self.nw,
                             elementtype=self.elementtype, phases=self.phases,
                             device=self.A.device)

    def same_geometry(self, other) -> bool:
        return (self.dim == other.dim and self.gsize == other.gsize and
                self.nw == other.nw and self.dims == other.dims)


def mark_halo_dirty_(ls: LatticeMatrix):
    """mark_halo_dirty! (LatticeMatrices_core.jl:196-203)."""
    ls.halo_epoch.core += 1
    if ls.nw == 0:
        ls.halo_epoch.halo = ls.halo_epoch.core


def halo_is_dirty(ls: LatticeMatrix) -> bool:
    return ls.halo_epoch.core != ls.halo_epoch.halo


def similar(ls: LatticeMatrix) -> LatticeMatrix:
    return ls.similar()


def clear_matrix_(ls: LatticeMatrix):
    ls.A.zero_()
    mark_halo_dirty_(ls)


def substitute_(dst: LatticeMatrix, src: LatticeMatrix):
    if not dst.same_geometry(src) or (dst.NC1, dst.NC2) != (src.NC1, src.NC2):
        raise ArgumentError("substitute! requires fields of the same shape")
    dst.core_view().copy_(src.core_view())
    mark_halo_dirty_(dst)
