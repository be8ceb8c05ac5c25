"""ctypes binding of liblmb200.so (the C ABI declared in include/lmb200.h).

The library is the only compute path: nothing here falls back to another
implementation.  Loading fails loudly when the shared object is missing or no
CUDA device is present.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
# LMB200_LIB selects another build of the library (e.g. a tuning variant)
LIB_PATH = os.environ.get("LMB200_LIB", os.path.join(_HERE, "liblmb200.so"))

LMB_OK = 0
LMB_ERR_ARG = -1
LMB_ERR_CUDA = -2
LMB_ERR_STATE = -3
LMB_ERR_UNSUPPORTED = -4

DTYPE_C128, DTYPE_C64 = 0, 1
PREC = {"double": 0, "single": 1, "half": 2}
OP_WILSON, OP_WILSON_CLOVER, OP_STAGGERED, OP_HISQ, OP_DOMAINWALL = 0, 1, 2, 3, 4
LINKS_THIN, LINKS_FAT, LINKS_LONG = 0, 1, 2
CG_REASONS = ("converged", "maximum_iterations", "nonpositive_curvature",
              "numerical_breakdown")

# every symbol include/lmb200.h declares
EXPORTED = (
    "lmb_create", "lmb_destroy", "lmb_last_error", "lmb_version",
    "lmb_set_geometry", "lmb_links_upload", "lmb_wilson_apply",
    "lmb_wilson_clover_apply", "lmb_clover_field_strength", "lmb_cg_ddagd",
    "lmb_field_dot", "lmb_random_su3_links", "lmb_gaussian_field",
    "lmb_field_dot_noalloc", "lmb_staggered_apply", "lmb_hisq_apply",
    "lmb_hisq_fat7", "lmb_hisq_project_u3", "lmb_hisq_naik",
    "lmb_hisq_links_from_thin", "lmb_cg_ddagd_batched",
    "lmb_hisq_link_pullback", "lmb_hisq_fermion_force",
    "lmb_wilson_clover_link_pullback", "lmb_wilson_clover_fermion_force",
    "lmb_domainwall_set", "lmb_domainwall_apply", "lmb_solve_evenodd",
    "lmb_set_halo", "lmb_operator_timing", "lmb_nccl_unique_id",
    "lmb_set_process_grid",
)


class ArgumentError(ValueError):
    """Validation failure; the reference raises Julia's ArgumentError."""


class DimensionMismatch(ArgumentError):
    """Length mismatch; the reference raises Julia's DimensionMismatch."""


class LMBError(RuntimeError):
    """CUDA or state failure reported by liblmb200."""


class CGParams(ctypes.Structure):
    _fields_ = [
        ("op", ctypes.c_int), ("kappa", ctypes.c_double),
        ("csw", ctypes.c_double), ("mass", ctypes.c_double),
        ("naik_epsilon", ctypes.c_double), ("rtol", ctypes.c_double),
        ("atol", ctypes.c_double), ("maxiter", ctypes.c_int),
        ("precision", ctypes.c_int), ("delta", ctypes.c_double),
        ("check_interval", ctypes.c_int), ("profile", ctypes.c_int),
    ]


class CGResultC(ctypes.Structure):
    _fields_ = [
        ("converged", ctypes.c_int), ("iterations", ctypes.c_int),
        ("residual_norm", ctypes.c_double),
        ("relative_residual", ctypes.c_double), ("reason", ctypes.c_int),
        ("reliable_updates", ctypes.c_int),
        ("true_residual_norm", ctypes.c_double),
        ("dslash_ms", ctypes.c_double), ("update_ms", ctypes.c_double),
        ("dslash_launches", ctypes.c_int), ("update_launches", ctypes.c_int),
        ("kernel_launches", ctypes.c_longlong), ("link_reals", ctypes.c_int),
    ]


class BatchLattice(ctypes.Structure):
    _fields_ = [
        ("L", ctypes.c_int * 4), ("nw", ctypes.c_int),
        ("phase_re", ctypes.c_double * 4), ("phase_im", ctypes.c_double * 4),
        ("U", ctypes.c_void_p * 4), ("epoch", ctypes.c_uint64 * 4),
        ("kappa", ctypes.c_double), ("nrhs", ctypes.c_int),
        ("x", ctypes.POINTER(ctypes.c_void_p)),
        ("b", ctypes.POINTER(ctypes.c_void_p)),
    ]


class BatchTuning(ctypes.Structure):
    _fields_ = [
        ("rhs_block", ctypes.c_int), ("threads", ctypes.c_int),
        ("ms_per_iteration", ctypes.c_double),
        ("graph_iterations", ctypes.c_int),
        ("kernel_family", ctypes.c_int),
        ("ms_stencils", ctypes.c_double),
    ]


_lock = threading.Lock()
_lib = None


def load(path: str = LIB_PATH):
    """Load liblmb200.so and declare its signatures (no CUDA call)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise LMBError(
                f"{path} is missing: build it with `make -C "
                f"latticematrices.jl_b200/csrc` (or __graft_entry__.build())")
        lib = ctypes.CDLL(path)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), \
            ctypes.POINTER(ctypes.c_double)
        lib.lmb_create.restype = vp
        lib.lmb_create.argtypes = [ctypes.c_int]
        lib.lmb_destroy.restype = None
        lib.lmb_destroy.argtypes = [vp]
        lib.lmb_last_error.restype = ctypes.c_char_p
        lib.lmb_last_error.argtypes = [vp]
        lib.lmb_version.restype = ctypes.c_int
        lib.lmb_set_geometry.argtypes = [vp, ip, ctypes.c_int, dp, dp, ip,
                                         ctypes.c_int]
        lib.lmb_links_upload.argtypes = [
            vp, ctypes.c_int, ctypes.POINTER(vp),
            ctypes.POINTER(ctypes.c_uint64), vp]
        lib.lmb_wilson_apply.argtypes = [vp, vp, vp, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_int, vp]
        lib.lmb_wilson_clover_apply.argtypes = [
            vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
            ctypes.c_int, vp]
        lib.lmb_clover_field_strength.argtypes = [vp, ctypes.POINTER(vp), vp]
        lib.lmb_staggered_apply.argtypes = [vp, vp, vp, ctypes.c_double,
                                            ctypes.c_int, ctypes.c_int, vp]
        lib.lmb_hisq_apply.argtypes = [vp, vp, vp, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int,
                                       ctypes.c_int, vp]
        pvp = ctypes.POINTER(vp)
        lib.lmb_hisq_fat7.argtypes = [vp, pvp, dp, pvp, vp]
        lib.lmb_hisq_project_u3.argtypes = [vp, pvp, pvp, vp]
        lib.lmb_hisq_naik.argtypes = [vp, pvp, pvp, vp]
        lib.lmb_cg_ddagd_batched.argtypes = [
            vp, ctypes.POINTER(CGParams), ctypes.c_int,
            ctypes.POINTER(BatchLattice), ctypes.POINTER(CGResultC),
            ctypes.POINTER(BatchTuning), vp]
        lib.lmb_hisq_link_pullback.argtypes = [
            vp, ctypes.POINTER(vp), ctypes.c_double, ctypes.c_double, vp, vp,
            ctypes.POINTER(vp), vp]
        lib.lmb_hisq_fermion_force.argtypes = [
            vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_uint64),
            ctypes.c_double, ctypes.c_double, vp, ctypes.POINTER(vp),
            ctypes.POINTER(CGParams), ctypes.POINTER(CGResultC), vp]
        lib.lmb_wilson_clover_link_pullback.argtypes = [
            vp, ctypes.POINTER(vp), ctypes.c_double, ctypes.c_double,
            ctypes.c_double, vp, vp, ctypes.POINTER(vp), vp]
        lib.lmb_wilson_clover_fermion_force.argtypes = [
            vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_uint64),
            ctypes.c_double, ctypes.c_double, vp, ctypes.POINTER(vp),
            ctypes.POINTER(CGParams), ctypes.POINTER(CGResultC), vp]
        lib.lmb_domainwall_set.argtypes = [
            vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, dp, dp, dp,
            vp]
        lib.lmb_domainwall_apply.argtypes = [vp, vp, vp, ctypes.c_int,
                                             ctypes.c_int, vp]
        lib.lmb_hisq_links_from_thin.argtypes = [
            vp, pvp, ctypes.POINTER(ctypes.c_uint64), ctypes.c_double, pvp,
            pvp, vp]
        lib.lmb_cg_ddagd.argtypes = [vp, ctypes.POINTER(CGParams), vp, vp,
                                     ctypes.POINTER(CGResultC), vp]
        lib.lmb_set_halo.argtypes = [vp, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ip, ctypes.c_int, dp, dp,
                                     vp]
        lib.lmb_solve_evenodd.argtypes = [vp, ctypes.POINTER(CGParams), vp,
                                          vp, ctypes.POINTER(CGResultC), vp]
        lib.lmb_field_dot.argtypes = [vp, vp, vp, ctypes.c_int, dp, vp]
        lib.lmb_operator_timing.argtypes = [vp, ctypes.POINTER(CGParams), vp,
                                            ctypes.c_int, ctypes.c_int, dp, vp]
        lib.lmb_nccl_unique_id.argtypes = [vp]
        lib.lmb_set_process_grid.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int,
                                             ip, ip, ctypes.c_uint, ip, ip]
        lib.lmb_random_su3_links.argtypes = [vp, ctypes.POINTER(vp),
                                             ctypes.c_double, ctypes.c_uint64,
                                             vp]
        lib.lmb_gaussian_field.argtypes = [vp, vp, ctypes.c_int,
                                           ctypes.c_uint64, vp]
        lib.lmb_field_dot_noalloc.argtypes = [vp, vp, ip, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int,
                                              vp, vp]
        for name in EXPORTED:
            if name not in ("lmb_create", "lmb_destroy", "lmb_last_error",
                            "lmb_version"):
                getattr(lib, name).restype = ctypes.c_int
        _lib = lib
        return lib


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise LMBError("liblmb200 needs a CUDA device; none is visible")


def nccl_unique_id() -> bytes:
    """128 bytes naming a new NCCL communicator (ncclGetUniqueId, through
    liblmb200's run-time NCCL)."""
    lib = load()
    buf = ctypes.create_string_buffer(128)
    rc = lib.lmb_nccl_unique_id(buf)
    if rc != LMB_OK:
        raise LMBError(f"lmb_nccl_unique_id failed ({rc}): NCCL unavailable")
    return buf.raw


class Context:
    """One lmb_ctx: geometry, link/clover caches and solver workspaces."""

    def __init__(self, device: int = 0):
        require_cuda()
        self.lib = load()
        self.device = device
        self.handle = self.lib.lmb_create(device)
        if not self.handle:
            raise LMBError(f"lmb_create({device}) failed")
        self._geom = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                self.lib.lmb_destroy(h)
            except Exception:
                pass
            self.handle = None

    def check(self, rc: int):
        if rc == LMB_OK:
            return
        msg = self.lib.lmb_last_error(self.handle).decode(errors="replace")
        if rc == LMB_ERR_ARG:
            raise ArgumentError(msg)
        raise LMBError(f"liblmb200 error {rc}: {msg}")

    def set_geometry(self, L, nw, phases, coords=(0, 0, 0, 0),
                     dtype=DTYPE_C128):
        key = (tuple(L), nw, tuple(complex(p) for p in phases), tuple(coords),
               dtype)
        if key == self._geom:
            return
        Lc = (ctypes.c_int * 4)(*[int(v) for v in L])
        re = (ctypes.c_double * 4)(*[complex(p).real for p in phases])
        im = (ctypes.c_double * 4)(*[complex(p).imag for p in phases])
        cc = (ctypes.c_int * 4)(*[int(v) for v in coords])
        self.check(self.lib.lmb_set_geometry(self.handle, Lc, int(nw), re, im,
                                             cc, int(dtype)))
        self._geom = key

    def set_process_grid(self, nccl_id, nranks, rank, dims, coords, split,
                         nb_minus, nb_plus):
        """lmb_set_process_grid: this context's fields become the block of
        `rank` in a process grid `dims` (NCCL communicator from the 128-byte
        `nccl_id`); `split` lists the exchanged dimensions.  nccl_id None:
        back to one lattice per context."""
        iv = lambda v: (ctypes.c_int * 4)(*[int(x) for x in v])
        mask = sum(1 << mu for mu in range(4) if split[mu])
        idbuf = None if nccl_id is None else ctypes.create_string_buffer(bytes(nccl_id), 128)
        self.check(self.lib.lmb_set_process_grid(
            self.handle, idbuf, int(nranks), int(rank), iv(dims), iv(coords),
            mask, iv(nb_minus), iv(nb_plus)))
        self._geom = None

    def upload_links(self, which, ptrs, epochs, stream=None):
        arr = (ctypes.c_void_p * 4)(*ptrs)
        ep = (ctypes.c_uint64 * 4)(*[int(e) for e in epochs])
        self.check(self.lib.lmb_links_upload(self.handle, int(which), arr, ep,
                                             stream))
