"""Seeded synthetic inputs generated on the GPU by liblmb200
(lmb_random_su3_links, lmb_gaussian_field): SU(3) links exp(i a H)
reunitarized, and unit-variance complex Gaussian fields, from Philox4x32-10
site streams (the same streams as the reference's decomposition-independent
fills, utilities/randomgenerator.jl:247-340)."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import ArgumentError, Context
from .lattice import require_single_rank, LatticeMatrix, mark_halo_dirty_
from .operators import _stream

_CTX = {}


def _ctx(field: LatticeMatrix) -> Context:
    dev = field.A.device.index or 0
    if dev not in _CTX:
        _CTX[dev] = Context(dev)
    c = _CTX[dev]
    require_single_rank(field)
    c.set_geometry(field.gsize, field.nw, field.phases, field.coords,
                   field.dtype_code)
    return c


def random_su3_links(gsize, amplitude, seed, *, nw=1,
                     elementtype=np.complex128, device="cuda"):
    U = [LatticeMatrix(3, 3, 4, gsize, nw=nw, elementtype=elementtype,
                       device=device) for _ in range(4)]
    c = _ctx(U[0])
    arr = (ctypes.c_void_p * 4)(*[u.data_ptr() for u in U])
    c.check(c.lib.lmb_random_su3_links(c.handle, arr, float(amplitude),
                                       int(seed), _stream()))
    for u in U:
        mark_halo_dirty_(u)
    return U


def gaussian_fermion(gsize, nc, nspin, seed, *, nw=1, phases=None,
                     elementtype=np.complex128, device="cuda"):
    if nc <= 0 or nspin <= 0:
        raise ArgumentError("field shape must be positive")
    f = LatticeMatrix(nc, nspin, 4, gsize, nw=nw, elementtype=elementtype,
                      phases=phases, device=device)
    c = _ctx(f)
    c.check(c.lib.lmb_gaussian_field(c.handle, f.data_ptr(), nc * nspin,
                                     int(seed), _stream()))
    mark_halo_dirty_(f)
    return f
