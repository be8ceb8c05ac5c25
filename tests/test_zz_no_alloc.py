"""lmb_field_dot_noalloc: the inner product for callers that cannot allocate
device memory (pool-managed memory near its limit, host applications that
forbid allocations outside their own allocator, loops where an allocation
would synchronise the device).  Its result
must equal lmb_field_dot's, call after call, although its scratch is a static
device array shared by every call.  Collected last so that a failure here
comes after every other test has run."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_dot(lib, a, b, out, stream):
    L = (ctypes.c_int * 4)(*a.gsize)
    rc = lib.lmb_field_dot_noalloc(a.data_ptr(), b.data_ptr(), L, a.nw,
                                   a.dtype_code, a.NC1 * a.NC2,
                                   out.data_ptr(), stream)
    return rc


def _setup():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lmb200 as lmb
    lib = lmb.load()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return torch, lmb, lib, out, stream


def _field(lmb, L, nc1, nc2, nw, dtype, seed):
    rng = np.random.default_rng(seed)
    shape = (nc1, nc2) + tuple(L)
    A = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)
    return lmb.LatticeMatrix.from_array(A.astype(dtype), nw=nw), A.astype(dtype)


def test_dot_noalloc_matches_dot_on_consecutive_calls():
    torch, lmb, lib, out, stream = _setup()
    L = (8, 8, 4, 6)
    a = lmb.gaussian_fermion(L, 3, 4, 21, nw=1)
    b = lmb.gaussian_fermion(L, 3, 4, 22, nw=1)
    for x, y in ((a, b), (b, a)):           # two calls in a row, same scratch
        out.fill_(np.nan)
        assert _noalloc_dot(lib, x, y, out, stream) == 0
        torch.cuda.synchronize()
        got = complex(*out.cpu().tolist())
        ref = lmb.dot(x, y)                   # existing entry point
        assert abs(got - ref) <= 1e-12 * abs(ref), (got, ref)
    # a volume beyond the static scratch is rejected before any launch
    big = (ctypes.c_int * 4)(256, 256, 256, 2)
    assert lib.lmb_field_dot_noalloc(a.data_ptr(), b.data_ptr(), big, 0, 0,
                                     12, out.data_ptr(), stream) == -1
    # an unsupported component count is refused
    small = (ctypes.c_int * 4)(*L)
    assert lib.lmb_field_dot_noalloc(a.data_ptr(), b.data_ptr(), small, 1, 0,
                                     5, out.data_ptr(), stream) != 0


# (lattice, NC1, NC2, nw, element type): an odd volume whose last block is
# partly empty (5*3*3*7 = 315 sites), ComplexF32 fields, 1 / 3 / 9 / 12
# components, no halo
CASES = [
    ((5, 3, 3, 7), 3, 4, 1, np.complex128),
    ((5, 3, 3, 7), 3, 1, 0, np.complex64),
    ((4, 6, 2, 8), 3, 3, 2, np.complex64),
    ((6, 4, 4, 4), 1, 1, 0, np.complex64),
    ((6, 4, 4, 4), 3, 1, 1, np.complex128),
]


@pytest.mark.parametrize("L,nc1,nc2,nw,dtype", CASES)
def test_dot_noalloc_shapes_and_types(L, nc1, nc2, nw, dtype):
    torch, lmb, lib, out, stream = _setup()
    a, ha = _field(lmb, L, nc1, nc2, nw, dtype, 31)
    b, hb = _field(lmb, L, nc1, nc2, nw, dtype, 32)
    out.fill_(np.nan)
    assert _noalloc_dot(lib, a, b, out, stream) == 0
    torch.cuda.synchronize()
    got = complex(*out.cpu().tolist())
    ref = lmb.dot(a, b)
    host = np.vdot(ha.astype(np.complex128).ravel(), hb.astype(np.complex128).ravel())
    assert abs(got - ref) <= 1e-12 * abs(ref), (got, ref)
    assert abs(got - host) <= 1e-12 * abs(host), (got, host)


def test_dot_noalloc_small_call_after_large_call():
    """A large lattice leaves partials in the shared scratch for many blocks;
    a following small call on the same stream must read only its own."""
    torch, lmb, lib, out, stream = _setup()
    big_a, hba = _field(lmb, (16, 16, 16, 16), 3, 1, 1, np.complex128, 41)
    big_b, hbb = _field(lmb, (16, 16, 16, 16), 3, 1, 1, np.complex128, 42)
    sm_a, hsa = _field(lmb, (3, 5, 3, 3), 3, 1, 1, np.complex128, 43)
    sm_b, hsb = _field(lmb, (3, 5, 3, 3), 3, 1, 1, np.complex128, 44)
    out_big = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert _noalloc_dot(lib, big_a, big_b, out_big, stream) == 0
    assert _noalloc_dot(lib, sm_a, sm_b, out, stream) == 0
    torch.cuda.synchronize()
    for o, ha, hb in ((out_big, hba, hbb), (out, hsa, hsb)):
        got = complex(*o.cpu().tolist())
        ref = np.vdot(ha.ravel(), hb.ravel())
        assert abs(got - ref) <= 1e-12 * abs(ref), (got, ref)
