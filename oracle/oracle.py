"""ctypes front-end of the CPU oracle (``liblmb_oracle.so``).

TEST INFRASTRUCTURE ONLY.  Imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``; the product library never calls it.

Fields are numpy complex128 arrays in the reference's logical index order
``(NC1, NC2, X, Y, Z, T)`` stored column-major (Fortran order), i.e. exactly
the core of a ``LatticeMatrix`` with ``nw = 0`` (LatticeMatrices_core.jl:4-9).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblmb_oracle.so")
_lib = None

OP_WILSON, OP_CLOVER, OP_STAGGERED, OP_HISQ = 0, 1, 2, 3
CG_REASONS = ("converged", "maximum_iterations", "nonpositive_curvature",
              "numerical_breakdown")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) <
            os.path.getmtime(os.path.join(_HERE, "lmb_oracle.c"))):
        subprocess.run(["make", "-s", "-C", _HERE] + (["-B"] if force else []),
                       check=True)
    return _LIB_PATH


class _Operator(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int), ("nc", ctypes.c_int),
        ("L", ctypes.c_int * 4), ("phases", ctypes.c_double * 8),
        ("eta_offset", ctypes.c_int * 4),
        ("kappa", ctypes.c_double), ("csw", ctypes.c_double),
        ("mass", ctypes.c_double), ("naik_epsilon", ctypes.c_double),
        ("links", ctypes.c_void_p * 8), ("F", ctypes.c_void_p * 6),
    ]


class _CGResult(ctypes.Structure):
    _fields_ = [
        ("converged", ctypes.c_int), ("iterations", ctypes.c_int),
        ("residual_norm", ctypes.c_double),
        ("relative_residual", ctypes.c_double), ("reason", ctypes.c_int),
    ]


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.orc_cg_ddagd_iterations.restype = ctypes.c_double
        _lib.orc_field_reals.restype = ctypes.c_int64
        _lib.orc_num_threads.restype = ctypes.c_int
    return _lib


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def _ptrs(arrs):
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def _check(a: np.ndarray):
    assert a.dtype == np.complex128 and a.flags.f_contiguous, \
        "oracle fields are Fortran-ordered complex128"
    return a


def _ivec(v):
    return (ctypes.c_int * 4)(*[int(x) for x in v])


def _phases(phases):
    ph = [complex(p) for p in phases]
    return (ctypes.c_double * 8)(*[c for p in ph for c in (p.real, p.imag)])


def lattice_shape(x):
    return tuple(int(v) for v in x.shape[2:])


def zeros(nc1, nc2, L):
    return np.zeros((nc1, nc2) + tuple(L), dtype=np.complex128, order="F")


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


# ----------------------------------------------------------------------------
# operators
# ----------------------------------------------------------------------------
def wilson(U, psi, kappa, phases=(1, 1, 1, -1), dagger=False):
    L = lattice_shape(psi)
    out = zeros(psi.shape[0], 4, L)
    lib().orc_wilson(_ivec(L), _phases(phases), psi.shape[0],
                     ctypes.c_double(kappa), int(dagger),
                     _ptrs([_check(u) for u in U]), _ptr(_check(psi)),
                     _ptr(out))
    return out


def wilson_donly(U, psi, phases=(1, 1, 1, -1), dagger=False):
    L = lattice_shape(psi)
    out = zeros(psi.shape[0], 4, L)
    lib().orc_wilson_donly(_ivec(L), _phases(phases), psi.shape[0],
                           int(dagger), _ptrs([_check(u) for u in U]),
                           _ptr(_check(psi)), _ptr(out))
    return out


def clover_field_strength(U):
    nc = U[0].shape[0]
    L = lattice_shape(U[0])
    F = [zeros(nc, nc, L) for _ in range(6)]
    lib().orc_clover_field_strength(_ivec(L), nc,
                                    _ptrs([_check(u) for u in U]), _ptrs(F))
    return F


def wilson_clover(U, psi, kappa, csw, phases=(1, 1, 1, -1), dagger=False,
                  F=None):
    if F is None:
        F = clover_field_strength(U)
    L = lattice_shape(psi)
    out = zeros(psi.shape[0], 4, L)
    lib().orc_wilson_clover(_ivec(L), _phases(phases), psi.shape[0],
                            ctypes.c_double(kappa), ctypes.c_double(csw),
                            int(dagger), _ptrs([_check(u) for u in U]),
                            _ptrs(F), _ptr(_check(psi)), _ptr(out))
    return out


def staggered(U, psi, mass, phases=(1, 1, 1, -1), dagger=False,
              eta_offset=(0, 0, 0, 0)):
    L = lattice_shape(psi)
    out = zeros(psi.shape[0], 1, L)
    lib().orc_staggered(_ivec(L), _phases(phases), _ivec(eta_offset),
                        psi.shape[0], ctypes.c_double(mass), int(dagger),
                        _ptrs([_check(u) for u in U]), _ptr(_check(psi)),
                        _ptr(out))
    return out


def domainwall(U, psi, mass, M, a, b, c, phases=(1, 1, 1, -1), dagger=False):
    """Generalised domain-wall D5 (or D5^+) on a (nc, 4, X, Y, Z, T, L5)
    field; a, b, c: L5 coefficients (Mobius: ones, (b+c)/2, (b-c)/2)."""
    L = tuple(int(v) for v in psi.shape[2:6])
    L5 = int(psi.shape[6])
    dvec = lambda v: (ctypes.c_double * L5)(*[float(x) for x in v])
    out = np.zeros(psi.shape, dtype=np.complex128, order="F")
    lib().orc_domainwall(_ivec(L), L5, _phases(phases), psi.shape[0],
                         ctypes.c_double(mass), ctypes.c_double(M), dvec(a),
                         dvec(b), dvec(c), int(dagger),
                         _ptrs([_check(u) for u in U]), _ptr(_check(psi)),
                         _ptr(out))
    return out


def mobius_coefficients(L5, b, c):
    """D5DW_MobiusDomainwallOperator5D(b, c) as the generalised operator."""
    return [1.0] * L5, [(b + c) / 2] * L5, [(b - c) / 2] * L5


def hisq(X, Lng, psi, mass, naik_epsilon=0.0, phases=(1, 1, 1, -1),
         dagger=False, eta_offset=(0, 0, 0, 0)):
    L = lattice_shape(psi)
    out = zeros(psi.shape[0], 1, L)
    lib().orc_hisq(_ivec(L), _phases(phases), _ivec(eta_offset),
                   psi.shape[0], ctypes.c_double(mass),
                   ctypes.c_double(naik_epsilon), int(dagger),
                   _ptrs([_check(u) for u in X]),
                   _ptrs([_check(u) for u in Lng]), _ptr(_check(psi)),
                   _ptr(out))
    return out


# ----------------------------------------------------------------------------
# HISQ smearing
# ----------------------------------------------------------------------------
LEVEL1 = (1 / 8, 1 / 16, 1 / 64, 1 / 384, 0.0)


def level2_coefficients(naik_epsilon):
    return (1 + naik_epsilon / 8, 1 / 16, 1 / 64, 1 / 384, -1 / 8)


def hisq_fat7(U, coefficients):
    nc = U[0].shape[0]
    L = lattice_shape(U[0])
    V = [zeros(nc, nc, L) for _ in range(4)]
    lib().orc_hisq_fat7(_ivec(L), nc,
                        (ctypes.c_double * 5)(*coefficients),
                        _ptrs([_check(u) for u in U]), _ptrs(V))
    return V


def hisq_project_u3(V):
    L = lattice_shape(V[0])
    W = [zeros(3, 3, L) for _ in range(4)]
    lib().orc_hisq_project_u3(_ivec(L), _ptrs([_check(v) for v in V]),
                              _ptrs(W))
    return W


def hisq_naik(W):
    nc = W[0].shape[0]
    L = lattice_shape(W[0])
    Lng = [zeros(nc, nc, L) for _ in range(4)]
    lib().orc_hisq_naik(_ivec(L), nc, _ptrs([_check(w) for w in W]),
                        _ptrs(Lng))
    return Lng


def hisq_links_from_thin(U, naik_epsilon=0.0):
    L = lattice_shape(U[0])
    X = [zeros(3, 3, L) for _ in range(4)]
    Lng = [zeros(3, 3, L) for _ in range(4)]
    lib().orc_hisq_links_from_thin(_ivec(L), ctypes.c_double(naik_epsilon),
                                   _ptrs([_check(u) for u in U]), _ptrs(X),
                                   _ptrs(Lng))
    return X, Lng


# ----------------------------------------------------------------------------
# CG
# ----------------------------------------------------------------------------
class Operator:
    """A Dirac operator description for the oracle's D'D CG."""

    def __init__(self, kind, links, L, nc=3, phases=(1, 1, 1, -1), kappa=0.0,
                 csw=0.0, mass=0.0, naik_epsilon=0.0, F=None,
                 eta_offset=(0, 0, 0, 0)):
        self._keep = list(links) + list(F or [])
        s = _Operator()
        s.kind = kind
        s.nc = nc
        s.L = _ivec(L)
        s.phases = _phases(phases)
        s.eta_offset = _ivec(eta_offset)
        s.kappa, s.csw, s.mass, s.naik_epsilon = kappa, csw, mass, naik_epsilon
        for i, a in enumerate(links):
            s.links[i] = _check(a).ctypes.data
        for i, a in enumerate(F or []):
            s.F[i] = _check(a).ctypes.data
        self.s = s
        self.L = tuple(L)
        self.nc = nc
        self.spins = 4 if kind in (OP_WILSON, OP_CLOVER) else 1

    def field(self):
        return zeros(self.nc, self.spins, self.L)

    def apply(self, psi, dagger=False):
        out = self.field()
        lib().orc_apply(ctypes.byref(self.s), int(dagger), _ptr(_check(psi)),
                        _ptr(out))
        return out

    def ddagd(self, psi):
        return self.apply(self.apply(psi), dagger=True)


def cg_ddagd(op: Operator, b, x0=None, rtol=1e-10, atol=0.0, maxiter=5000):
    x = op.field() if x0 is None else np.array(x0, order="F", copy=True)
    res = _CGResult()
    lib().orc_cg_ddagd(ctypes.byref(op.s), _ptr(x), _ptr(_check(b)),
                       ctypes.c_double(rtol), ctypes.c_double(atol),
                       int(maxiter), ctypes.byref(res))
    return x, dict(converged=bool(res.converged), iterations=res.iterations,
                   residual_norm=res.residual_norm,
                   relative_residual=res.relative_residual,
                   reason=CG_REASONS[res.reason])


def cg_iterations_seconds(op: Operator, b, iterations: int) -> float:
    x = op.field()
    return lib().orc_cg_ddagd_iterations(ctypes.byref(op.s), _ptr(x),
                                         _ptr(_check(b)), int(iterations))


# ----------------------------------------------------------------------------
# seeded inputs
# ----------------------------------------------------------------------------
def random_su3_links(L, amplitude, seed):
    U = [zeros(3, 3, L) for _ in range(4)]
    lib().orc_random_su3_links(_ivec(L), ctypes.c_double(amplitude),
                               ctypes.c_uint64(seed), _ptrs(U))
    return U


def gaussian_field(L, nc, spins, seed):
    out = zeros(nc, spins, L)
    lib().orc_gaussian_field(_ivec(L), nc * spins, ctypes.c_uint64(seed),
                             _ptr(out))
    return out


def philox4x32(counter, key):
    c = (ctypes.c_uint32 * 4)(*counter)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib().orc_philox4x32(c, k, o)
    return tuple(o)


def dot(a, b):
    out = (ctypes.c_double * 2)()
    lib().orc_dot(ctypes.c_int64(a.size), _ptr(_check(a)), _ptr(_check(b)),
                  out)
    return complex(out[0], out[1])
