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


def test_dot_noalloc_matches_dot_on_consecutive_calls():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lmb200 as lmb
    lib = lmb.load()
    L = (8, 8, 4, 6)
    a = lmb.gaussian_fermion(L, 3, 4, 21, nw=1)
    b = lmb.gaussian_fermion(L, 3, 4, 22, nw=1)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
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
