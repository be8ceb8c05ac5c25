"""CPU checks of the boundary: the C-ABI library loads, exports every symbol
include/lmb200.h declares, and the host mirror validates arguments the way the
reference does before any CUDA call."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    src = open(os.path.join(ROOT, "include", "lmb200.h")).read()
    return sorted(set(re.findall(r"\b(lmb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import lmb200
    lib = lmb200.load()
    declared = _declared_symbols()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(lmb200.EXPORTED) == declared
    assert lib.lmb_version() >= 100


def _cpu_field(lmb, nc1, nc2, L=(4, 4, 4, 4), **kw):
    return lmb.LatticeMatrix(nc1, nc2, 4, L, device="cpu", **kw)


def test_lattice_validation():
    import lmb200 as lmb
    with pytest.raises(lmb.ArgumentError):
        lmb.LatticeMatrix(3, 4, 4, (4, 4, 4, 4), nw=-1, device="cpu")
    with pytest.raises(lmb.ArgumentError):
        lmb.LatticeMatrix(3, 4, 4, (4, 4, 0, 4), device="cpu")
    with pytest.raises(lmb.ArgumentError):
        lmb.LatticeMatrix(3, 4, 4, (4, 4, 4, 4), phases=(1, 1, 0, -1),
                          device="cpu")
    with pytest.raises(lmb.ArgumentError):
        lmb.LatticeMatrix(3, 4, 4, (4, 4, 2, 4), nw=3, device="cpu")
    f = _cpu_field(lmb, 3, 4, phases=(1, 1, 1, -1))
    arr = np.asfortranarray(np.random.default_rng(0).normal(size=(3, 4, 4, 4, 4, 4))
                            + 0j)
    f.set_core(arr)
    assert np.array_equal(f.gather_matrix(), arr)
    assert f.halo_epoch.core == 1
    # padded storage is the Julia column-major layout
    j = f.A.numpy()
    assert j[1 + 2, 1 + 1, 1 + 0, 1 + 3, 2, 1] == arr[1, 2, 3, 0, 1, 2]


def test_operator_validation_before_cuda():
    import lmb200 as lmb
    U = [_cpu_field(lmb, 3, 3) for _ in range(4)]
    psi = _cpu_field(lmb, 3, 4, phases=(1, 1, 1, -1))
    D = lmb.WilsonDiracCloverOperator4D(U, 0.12, 1.0)
    with pytest.raises(lmb.ArgumentError, match="distinct"):
        lmb.mul_(psi, D, psi)
    other = _cpu_field(lmb, 3, 4, phases=(1, 1, 1, 1))
    with pytest.raises(lmb.ArgumentError, match="boundary phases"):
        lmb.mul_(other, D, psi)
    bad = _cpu_field(lmb, 3, 4, L=(4, 4, 4, 8))
    with pytest.raises(lmb.ArgumentError, match="geometry"):
        lmb.mul_(bad, D, psi)
    with pytest.raises(lmb.ArgumentError, match="periodic"):
        lmb.WilsonDiracOperator4D(
            [_cpu_field(lmb, 3, 3, phases=(1, 1, 1, -1)) for _ in range(4)], 0.1)
    with pytest.raises(lmb.ArgumentError):
        lmb.WilsonDiracOperator4D(U[:3], 0.1)
    U2 = [_cpu_field(lmb, 2, 2) for _ in range(4)]
    psi2 = _cpu_field(lmb, 2, 4)
    with pytest.raises(lmb.ArgumentError, match="NC=3"):
        lmb.mul_(psi2.similar(), lmb.WilsonDiracOperator4D(U2, 0.1), psi2)
    with pytest.raises(lmb.ArgumentError):
        lmb.mul_(psi.similar(), D, psi, precision="quad")
    assert lmb.adjoint(lmb.adjoint(D)) is D


def test_cg_validation_before_cuda():
    import lmb200 as lmb
    x = _cpu_field(lmb, 3, 4)
    b = _cpu_field(lmb, 3, 4)
    with pytest.raises(lmb.ArgumentError, match="alias"):
        lmb.cg_(x, None, b, x, None, None)
    with pytest.raises(lmb.ArgumentError, match="rtol"):
        lmb.cg_(x, None, b, rtol=-1)
    with pytest.raises(lmb.ArgumentError, match="maxiter"):
        lmb.cg_(x, None, b, maxiter=-1)
    with pytest.raises(lmb.ArgumentError, match="finite"):
        lmb.cg_(x, None, b, atol=float("inf"))
    D = lmb.DdagDOp(None, b)
    with pytest.raises(lmb.ArgumentError, match="alias"):
        D.mul_(x, b)


def test_domainwall_validation_before_cuda():
    """Constructor and application checks of DiracOperators_5D.jl:15-21,
    66-91 and _require_5d_halo (:155-159), raised before any CUDA call."""
    import lmb200 as lmb
    U = [_cpu_field(lmb, 3, 3) for _ in range(4)]
    L5 = 3
    psi = lmb.LatticeMatrix(3, 4, 5, (4, 4, 4, 4, L5), device="cpu")
    out = psi.similar()
    assert out.dim == 5 and out.gsize == (4, 4, 4, 4, L5)
    # 5D storage: the fifth coordinate is the slowest padded index
    arr = np.asfortranarray(np.random.default_rng(1).normal(size=(3, 4, 4, 4, 4, 4, L5)) + 0j)
    psi.set_core(arr)
    assert np.array_equal(psi.gather_matrix(), arr)
    assert psi.A.numpy()[1 + 2, 1 + 0, 1 + 3, 1 + 1, 1 + 2, 3, 2] == arr[2, 3, 2, 1, 3, 0, 2]
    with pytest.raises(lmb.ArgumentError, match="four gauge links"):
        lmb.D5DW_MobiusDomainwallOperator5D(U[:3], L5, 0.1, -1.8, 2.0, 1.0)
    with pytest.raises(lmb.ArgumentError, match="integer"):
        lmb.D5DW_MobiusDomainwallOperator5D(U, 3.0, 0.1, -1.8, 2.0, 1.0)
    with pytest.raises(lmb.ArgumentError, match="positive"):
        lmb.D5DW_MobiusDomainwallOperator5D(U, 0, 0.1, -1.8, 2.0, 1.0)
    with pytest.raises(lmb.DimensionMismatch, match="length L5"):
        lmb.D5DW_GeneralizedDomainwallOperator5D(U, L5, 0.1, -1.8, [1] * 3, [1] * 2, [0] * 3)
    with pytest.raises(lmb.ArgumentError, match="finite"):
        lmb.D5DW_GeneralizedDomainwallOperator5D(U, L5, 0.1, -1.8, [1] * 3, [1, np.nan, 1], [0] * 3)
    D = lmb.D5DW_GeneralizedDomainwallOperator5D(U, L5, 0.1, -1.8, [1] * 3, [1.5] * 3, [0.5] * 3)
    assert D.kappa_wilson == pytest.approx(1 / (8 - 3.6))
    M = lmb.D5DW_MobiusDomainwallOperator5D(U, L5, 0.1, -1.8, 2.0, 1.0)
    a, b, c = M.abc()
    assert list(a) == [1.0] * L5 and list(b) == [1.5] * L5 and list(c) == [0.5] * L5
    assert lmb.adjoint(lmb.adjoint(D)) is D
    with pytest.raises(lmb.ArgumentError, match="distinct"):
        lmb.mul_(psi, D, psi)
    with pytest.raises(lmb.ArgumentError, match="five-dimensional"):
        lmb.mul_(_cpu_field(lmb, 3, 4), D, _cpu_field(lmb, 3, 4))
    with pytest.raises(lmb.DimensionMismatch, match="fifth extent"):
        wrong = lmb.LatticeMatrix(3, 4, 5, (4, 4, 4, 4, 2), device="cpu")
        lmb.mul_(wrong.similar(), D, wrong)
    flat = lmb.LatticeMatrix(3, 4, 5, (4, 4, 4, 4, L5), nw=0, device="cpu")
    with pytest.raises(lmb.ArgumentError, match="nw=0"):
        lmb.mul_(flat.similar(), D, flat)
    other = lmb.LatticeMatrix(3, 4, 5, (4, 4, 2, 4, L5), device="cpu")
    with pytest.raises(lmb.ArgumentError, match="geometry"):
        lmb.mul_(other.similar(), D, other)
    with pytest.raises(lmb.ArgumentError, match="distinct|alias"):
        lmb.cg_(psi, lmb.DdagDOp(D, out), psi)


def test_halo_fill_host_rules():
    """nw = 0 has no ghosts (set_halo! only marks the epoch clean); a field
    off the GPU cannot be filled (the fill is the library's kernel)."""
    import lmb200 as lmb
    flat = _cpu_field(lmb, 3, 4, nw=0)
    lmb.mark_halo_dirty_(flat)
    lmb.set_halo_(flat)
    assert not lmb.halo_is_dirty(flat)
    f = _cpu_field(lmb, 3, 4)
    lmb.mark_halo_dirty_(f)
    with pytest.raises(lmb.LMBError, match="GPU"):
        lmb.ensure_halo_(f)
