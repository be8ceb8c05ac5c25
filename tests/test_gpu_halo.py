"""GPU: set_halo! / ensure_halo! of single-rank fields (lmb_set_halo) against
the reference's dimension-by-dimension exchange restated densely."""
import numpy as np
import pytest

import refdata as rd

pytestmark = pytest.mark.gpu

TWISTED = tuple(np.exp(1j * a) for a in (0.13, -0.21, 0.34, np.pi - 0.17))


@pytest.fixture(scope="module")
def lmb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lmb200
    lmb200.load()
    return lmb200


def _padded(ls):
    """Whole padded storage in the reference's (NC1, NC2, X+2nw, ...) order."""
    return ls.A.cpu().numpy().T


@pytest.mark.parametrize("nc,dim,L,nw,phases,dtype", [
    ((3, 4), 4, (4, 4, 4, 6), 1, TWISTED, np.complex128),
    ((3, 4), 4, (4, 3, 2, 6), 2, (1, 1, 1, -1), np.complex128),
    ((3, 3), 4, (3, 4, 5, 3), 3, (1, 1, 1, 1), np.complex64),
    ((3, 1), 4, (6, 6, 6, 6), 3, TWISTED, np.complex128),
    ((3, 4), 5, (4, 2, 2, 4, 3), 1, TWISTED + (1,), np.complex128),
])
def test_set_halo_matches_reference_exchange(lmb, nc, dim, L, nw, phases, dtype):
    import torch
    ls = lmb.LatticeMatrix(nc[0], nc[1], dim, L, nw=nw, elementtype=dtype, phases=phases)
    rng = np.random.default_rng(7)
    full = rng.normal(size=ls.A.shape) + 1j * rng.normal(size=ls.A.shape)
    ls.A.copy_(torch.from_numpy(full.astype(dtype)).to(ls.A.device))
    lmb.mark_halo_dirty_(ls)
    before = _padded(ls)
    assert lmb.halo_is_dirty(ls)
    lmb.set_halo_(ls)
    torch.cuda.synchronize()
    assert not lmb.halo_is_dirty(ls)
    ref = rd.set_halo_dense(before, nw, phases)
    got = _padded(ls)
    tol = 1e-15 if dtype == np.complex128 else 1e-6
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
    # the core is read only
    core = tuple([slice(None)] * 2 + [slice(nw, nw + v) for v in L])
    assert np.array_equal(got[core], before[core])


def test_ensure_halo_follows_the_epoch(lmb):
    import torch
    ls = lmb.LatticeMatrix(3, 4, 4, (4, 4, 4, 4), nw=1, phases=TWISTED)
    arr = np.asfortranarray(np.random.default_rng(3).normal(size=(3, 4, 4, 4, 4, 4)) + 0j)
    ls.set_core(arr)
    lmb.ensure_halo_(ls)
    ref = rd.set_halo_dense(_padded(ls), 1, TWISTED)
    assert np.allclose(_padded(ls), ref, rtol=0, atol=1e-14)
    # clean: a second ensure_halo! writes nothing (halo edits survive)
    ls.A[0, 0, 0, 0] = 5.0
    lmb.ensure_halo_(ls)
    torch.cuda.synchronize()
    assert complex(ls.A[0, 0, 0, 0, 0, 0]) == 5.0
    # a core write makes it dirty again and the next ensure_halo! refills
    ls.set_core(arr * 2)
    lmb.ensure_halo_(ls)
    assert np.allclose(_padded(ls), rd.set_halo_dense(_padded(ls), 1, TWISTED), rtol=0, atol=1e-14)
