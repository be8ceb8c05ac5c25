"""GPU parity of the D'D CG (cg.jl:73-137) against the oracle, and the
mixed-precision solves' FP64 true residual."""
import numpy as np
import pytest

import refdata as rd

pytestmark = pytest.mark.gpu
PHASES = (1, 1, 1, -1)


@pytest.fixture(scope="module")
def lmb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lmb200
    lmb200.load()
    return lmb200


def _setup(lmb, orc, L, kappa, csw, amplitude=0.3, nw=1):
    U = orc.random_su3_links(L, amplitude, 1)
    b = orc.gaussian_field(L, 3, 4, 2)
    Ud = [lmb.LatticeMatrix.from_array(u, nw=nw) for u in U]
    bd = lmb.LatticeMatrix.from_array(b, nw=nw, phases=PHASES)
    if csw:
        D = lmb.WilsonDiracCloverOperator4D(Ud, kappa, csw)
        F = orc.clover_field_strength(U)
        op = orc.Operator(orc.OP_CLOVER, U, L, kappa=kappa, csw=csw, F=F)
    else:
        D = lmb.WilsonDiracOperator4D(Ud, kappa)
        op = orc.Operator(orc.OP_WILSON, U, L, kappa=kappa)
    return U, b, Ud, bd, D, op


def _true_rel(op, x, b):
    return np.linalg.norm(b - op.ddagd(x)) / np.linalg.norm(b)


@pytest.mark.parametrize("csw", [0.0, 1.0])
def test_cg_fp64_matches_oracle(lmb, orc, csw):
    L = (8, 8, 8, 8)
    U, b, Ud, bd, D, op = _setup(lmb, orc, L, 0.125, csw)
    x_ref, res_ref = orc.cg_ddagd(op, b, rtol=1e-10)
    x = bd.similar()
    res = lmb.cg_(x, lmb.DdagDOp(D, bd.similar()), bd, rtol=1e-10)
    assert res.converged and res.reason == "converged"
    # same algorithm, same inputs: iteration counts agree up to reduction order
    assert abs(res.iterations - res_ref["iterations"]) <= 1
    xs = x.gather_matrix()
    assert rd.rel_err(xs, x_ref) <= 1e-8
    assert _true_rel(op, xs, b) <= 1e-9


@pytest.mark.parametrize("precision", ["single", "half"])
@pytest.mark.parametrize("csw", [0.0, 1.0])
def test_cg_mixed_true_residual(lmb, orc, precision, csw):
    L = (8, 8, 8, 16)
    U, b, Ud, bd, D, op = _setup(lmb, orc, L, 0.1355 if csw else 0.125, csw,
                                 amplitude=0.2)
    x = bd.similar()
    res = lmb.cg_(x, lmb.DdagDOp(D, bd.similar()), bd, rtol=1e-10,
                  precision=precision, delta=0.1)
    assert res.converged, res
    assert res.reliable_updates >= 1
    xs = x.gather_matrix()
    # the solve stops on the FP64 true residual; the oracle confirms it
    assert _true_rel(op, xs, b) <= 1.05e-10
    x_ref, _ = orc.cg_ddagd(op, b, rtol=1e-12)
    assert rd.rel_err(xs, x_ref) <= 1e-6


def test_cg_edge_cases(lmb, orc):
    L = (4, 4, 4, 4)
    U, b, Ud, bd, D, op = _setup(lmb, orc, L, 0.125, 1.0)
    A = lmb.DdagDOp(D, bd.similar())
    x = bd.similar()
    stopped = lmb.cg_(x, A, bd, maxiter=0)
    assert not stopped.converged and stopped.reason == "maximum_iterations"
    zero = bd.similar()
    zr = lmb.cg_(x, A, zero, rtol=1e-13)
    assert zr.converged and zr.iterations == 0
    assert zr.residual_norm == 0 and zr.relative_residual == 0
    few = lmb.cg_(bd.similar(), A, bd, maxiter=3)
    assert few.reason == "maximum_iterations" and few.iterations == 3
    few_m = lmb.cg_(bd.similar(), A, bd, maxiter=3, precision="half")
    assert few_m.reason == "maximum_iterations" and not few_m.converged
    with pytest.raises(lmb.ArgumentError):
        lmb.cg_(x, A, bd, rtol=-1)
    with pytest.raises(lmb.ArgumentError):
        lmb.cg_(x, A, bd, maxiter=-1)
    with pytest.raises(lmb.ArgumentError):
        lmb.cg_(x, A, bd, x, None, None)


def test_cg_initial_guess(lmb, orc):
    L = (4, 4, 4, 8)
    U, b, Ud, bd, D, op = _setup(lmb, orc, L, 0.125, 1.0)
    x_ref, _ = orc.cg_ddagd(op, b, rtol=1e-12)
    x = lmb.LatticeMatrix.from_array(x_ref, nw=1, phases=PHASES)
    res = lmb.cg_(x, lmb.DdagDOp(D, bd.similar()), bd, rtol=1e-10)
    assert res.converged and res.iterations == 0


def test_generic_cg_scaled_operator(lmb):
    """The reference's mock-operator CG test (test/cg.jl:1-64)."""
    class Scaled:
        def __init__(self, s):
            self.s = s

        def mul_(self, y, x):
            y.core_view().copy_(x.core_view() * self.s)
            lmb.mark_halo_dirty_(y)
            return y

    arr = np.asfortranarray(np.arange(1, 5, dtype=np.complex128).reshape(1, 1, 4, 1, 1, 1))
    b = lmb.LatticeMatrix.from_array(arr, nw=1)
    x, r, p, Ap = b.similar(), b.similar(), b.similar(), b.similar()
    res = lmb.cg_(x, Scaled(4.0), b, r, p, Ap, rtol=1e-13, maxiter=10)
    assert res.converged and res.iterations == 1
    assert np.allclose(x.gather_matrix(), arr / 4, atol=2e-13)
    ind = lmb.cg_(b.similar(), Scaled(-1.0), b, r, p, Ap, maxiter=10)
    assert ind.reason == "nonpositive_curvature" and not ind.converged
