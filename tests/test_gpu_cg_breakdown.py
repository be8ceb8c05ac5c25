"""The native D^+D CG's failure paths against the reference's cg! contract
(src/LinearAlgebras/cg.jl:79-121), with the oracle (its restatement) run on
the same inputs:

* a non-finite |b|^2 returns at iteration 0 with a NaN residual norm and a
  NaN relative residual, reason numerical_breakdown (cg.jl:79-84);
* a non-finite gauge link makes the initial residual b - D'D x non-finite
  (NaN * 0 is NaN, so a zero start does not hide it): iteration 0, NaN
  residual, numerical_breakdown (cg.jl:93-98), in FP64 and with FP32 or int16
  inner iterations alike, whose low-precision copies are never used then.

The NaN is an ordinary value written into a host array before upload; no
kernel is made to fault."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
PHASES = (1, 1, 1, -1)
L = (4, 4, 4, 8)


@pytest.fixture(scope="module")
def lmb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lmb200
    lmb200.load()
    return lmb200


def _clover_case(lmb, orc, poison):
    U = orc.random_su3_links(L, 0.2, 1)
    b = orc.gaussian_field(L, 3, 4, 2)
    if poison == "link":
        U[2][1, 0, 1, 2, 3, 4] = np.nan
    else:
        b[0, 3, 2, 1, 0, 5] = np.nan
    Ud = [lmb.LatticeMatrix.from_array(u, nw=1) for u in U]
    bd = lmb.LatticeMatrix.from_array(b, nw=1, phases=PHASES)
    D = lmb.WilsonDiracCloverOperator4D(Ud, 0.1355, 1.0)
    op = orc.Operator(orc.OP_CLOVER, U, L, kappa=0.1355, csw=1.0,
                      F=orc.clover_field_strength(U))
    return D, bd, op, b


def _staggered_case(lmb, orc, poison):
    U = orc.random_su3_links(L, 0.2, 3)
    b = orc.gaussian_field(L, 3, 1, 4)
    if poison == "link":
        U[0][2, 2, 0, 1, 2, 3] = complex(np.inf, 0.0)
    else:
        b[1, 0, 3, 3, 3, 7] = np.nan
    Ud = [lmb.LatticeMatrix.from_array(u, nw=1) for u in U]
    bd = lmb.LatticeMatrix.from_array(b, nw=1, phases=PHASES)
    D = lmb.StaggeredDiracOperator4D(Ud, 0.05)
    op = orc.Operator(orc.OP_STAGGERED, U, L, mass=0.05)
    return D, bd, op, b


@pytest.mark.parametrize("poison", ["link", "source"])
@pytest.mark.parametrize("case,precisions", [
    ("clover", ("double", "single", "half")),
    ("staggered", ("double", "single", "half"))])
def test_nonfinite_input_breaks_down_like_the_reference(lmb, orc, case, precisions, poison):
    build = _clover_case if case == "clover" else _staggered_case
    D, bd, op, b = build(lmb, orc, poison)
    _, ref = orc.cg_ddagd(op, b, rtol=1e-10)
    assert ref["reason"] == "numerical_breakdown" and ref["iterations"] == 0
    assert math.isnan(ref["residual_norm"])
    for precision in precisions:
        x = bd.similar()
        res = lmb.cg_(x, lmb.DdagDOp(D, bd.similar()), bd, rtol=1e-10,
                      precision=precision)
        assert not res.converged, (precision, res)
        assert res.reason == ref["reason"], (precision, res)
        assert res.iterations == ref["iterations"], (precision, res)
        assert math.isnan(res.residual_norm), (precision, res)
        assert math.isnan(res.relative_residual) == math.isnan(ref["relative_residual"])


def test_lowprecision_apply_refuses_nonfinite_links(lmb, orc):
    D, bd, _, _ = _clover_case(lmb, orc, "link")
    out = bd.similar()
    lmb.mul_(out, D, bd)                         # FP64: NaN propagates
    assert np.isnan(out.gather_matrix()).any()
    for precision in ("single", "half"):
        with pytest.raises(lmb.ArgumentError, match="non-finite"):
            lmb.mul_(out, D, bd, precision=precision)
