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

One rank per lattice for the stencils (PEs = (1,1,1,1)): they wrap
periodically with the fermion phase and never read the halo; set_halo_ /
ensure_halo_ fill it on request (lmb_set_halo).  A process grid PEs with
prod(PEs) ranks of an initialised torch.distributed group (NCCL, or gloo on
CPU) splits the lattice into blocks of PN = gsize / PEs sites (rank r at the
row-major Cartesian coordinates of r, as MPI_Cart_create numbers them); such
fields support the halo exchange (exchange_dim!, distributed.py), gather and
dot, not the stencils.  `halo_epoch` tracks core writes so that
link caches are invalidated and ensure_halo_ refills exactly as
mark_halo_dirty! / ensure_halo! do (LatticeMatrices_core.jl:196-203, 569-581).
"""
from __future__ import annotations

import numpy as np

from ._lib import ArgumentError, LMBError

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
        PEs = tuple(int(v) for v in PEs)
        coords = (0,) * dim
        if PEs != (1,) * dim:
            from .distributed import cart_coords
            coords = cart_coords(PEs, gsize)
        PN = tuple(g // p for g, p in zip(gsize, PEs))
        for d in range(dim):
            if nw > PN[d]:
                raise ArgumentError(
                    f"halo width nw={nw} exceeds local lattice size {PN[d]} "
                    f"in dimension {d + 1}; the nearest-neighbor halo exchange "
                    f"requires nw <= local size")
        dt = np.dtype(elementtype)
        if dt not in _DTYPES:
            raise ArgumentError(f"unsupported element type {dt}")
        import torch
        self.NC1, self.NC2, self.dim = int(NC1), int(NC2), dim
        self.gsize = gsize
        self.PN = PN
        self.nw = int(nw)
        self.phases = tuple(phases)
        self.elementtype = dt
        self.coords = coords
        self.dims = PEs
        self.halo_epoch = HaloEpoch()
        padded = tuple(v + 2 * self.nw for v in PN)
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
        # every rank keeps its block of the global array
        block = tuple(slice(c * n, (c + 1) * n) for c, n in zip(lm.coords, lm.PN))
        lm.set_core(A[(slice(None), slice(None)) + block])
        return lm

    @property
    def dtype_code(self) -> int:
        return _DTYPES[self.elementtype]

    def data_ptr(self) -> int:
        return self.A.data_ptr()

    def core_view(self):
        n = self.nw
        return self.A[tuple(slice(n, n + v) for v in self.PN[::-1])]

    def set_core(self, A):
        import torch
        A = np.asarray(A, dtype=self.elementtype)
        if A.shape != (self.NC1, self.NC2) + self.PN:
            raise ArgumentError(
                f"array shape {A.shape} does not match the local lattice "
                f"{(self.NC1, self.NC2) + self.PN}")
        host = torch.from_numpy(np.ascontiguousarray(A.T))
        self.core_view().copy_(host.to(self.A.device))
        mark_halo_dirty_(self)

    def gather_matrix(self):
        """Core values of the whole lattice as a Fortran-ordered
        (NC1, NC2, X, Y, Z, T[, L5]) array (gather_matrix,
        LatticeMatrices_core.jl:936-993); every rank of a process grid gets
        the assembled array."""
        local = np.asfortranarray(self.core_view().cpu().numpy().T)
        if self.dims == (1,) * self.dim:
            return local
        from .distributed import gather_blocks
        return gather_blocks(self, local)

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


def set_halo_(ls: LatticeMatrix):
    """set_halo!(ls) (LatticeMatrices_core.jl:550-567) on one process: the
    ghosts take the periodic image of the core times the boundary phase
    (exchange_dim_local!, :707-723), written by liblmb200's lmb_set_halo on
    the field's device; the halo epoch is then clean."""
    if ls.nw > 0 and ls.dims != (1,) * ls.dim:
        from .distributed import exchange_halo
        exchange_halo(ls)
    elif ls.nw > 0:
        import ctypes
        import torch
        from ._lib import load
        if ls.A.device.type != "cuda":
            raise LMBError("set_halo! runs in liblmb200 on the GPU; the field is on "
                           f"{ls.A.device}")
        lib = load()
        D = ls.dim
        L = (ctypes.c_int * D)(*ls.gsize)
        re = (ctypes.c_double * D)(*[complex(p).real for p in ls.phases])
        im = (ctypes.c_double * D)(*[complex(p).imag for p in ls.phases])
        with torch.cuda.device(ls.A.device):
            st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
            rc = lib.lmb_set_halo(ls.A.data_ptr(), ls.dtype_code,
                                  ls.NC1 * ls.NC2, D, L, ls.nw, re, im, st)
        if rc == -1:
            raise ArgumentError("lmb_set_halo rejected the field geometry")
        if rc != 0:
            raise LMBError(f"lmb_set_halo failed ({rc})")
    ls.halo_epoch.halo = ls.halo_epoch.core


def ensure_halo_(ls: LatticeMatrix):
    """ensure_halo!(ls) (LatticeMatrices_core.jl:569-581): set_halo! only
    when the core changed since the last fill."""
    if halo_is_dirty(ls):
        set_halo_(ls)


def require_single_rank(ls: LatticeMatrix):
    """The stencils and solvers take one rank per lattice."""
    if ls.dims != (1,) * ls.dim:
        raise ArgumentError(
            f"the sm_100a stencils run one rank per lattice; this field is split "
            f"over the process grid {ls.dims} (halo exchange, gather and dot "
            f"support that)")


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
