"""GPU: even/odd (Schur) preconditioned solve of D x = b (Wilson and
Wilson-clover) against the oracle: the FP64 residual |b - D x| / |b| of the
oracle's operator, and the solution of the reference's route to the same x,
cg!(x, DdagDOp(D), D'b), solved by the oracle."""
import numpy as np
import pytest

import refdata as rd

pytestmark = pytest.mark.gpu

TWISTED = tuple(np.exp(1j * a) for a in (0.13, -0.21, 0.34, np.pi - 0.17))
PHASES = (1, 1, 1, -1)


@pytest.fixture(scope="module")
def lmb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lmb200
    lmb200.load()
    return lmb200


def _setup(lmb, orc, L, csw, kappa, phases, nw=1, amplitude=0.3, dtype=np.complex128):
    U = orc.random_su3_links(L, amplitude, 1)
    b = orc.gaussian_field(L, 3, 4, 2)
    Ud = [lmb.LatticeMatrix.from_array(u.astype(dtype), nw=nw) for u in U]
    bd = lmb.LatticeMatrix.from_array(b.astype(dtype), nw=nw, phases=phases)
    if csw:
        D = lmb.WilsonDiracCloverOperator4D(Ud, kappa, csw)
        apply = lambda v, dagger=False: orc.wilson_clover(U, v, kappa, csw, phases, dagger=dagger)
        op = orc.Operator(orc.OP_CLOVER, U, L, kappa=kappa, csw=csw, phases=phases,
                          F=orc.clover_field_strength(U))
    else:
        D = lmb.WilsonDiracOperator4D(Ud, kappa)
        apply = lambda v, dagger=False: orc.wilson(U, v, kappa, phases, dagger=dagger)
        op = orc.Operator(orc.OP_WILSON, U, L, kappa=kappa, phases=phases)
    return U, b, bd, D, apply, op


def _rel_residual(apply, x, b):
    return np.linalg.norm((b - apply(np.asfortranarray(x))).ravel()) / np.linalg.norm(b.ravel())


@pytest.mark.parametrize("csw,kappa", [(0.0, 0.125), (1.0, 0.1355)])
@pytest.mark.parametrize("L,nw,phases", [((4, 4, 4, 8), 1, PHASES), ((6, 4, 2, 4), 0, TWISTED),
                                         ((8, 8, 8, 8), 2, TWISTED)])
def test_evenodd_fp64_solves_D(lmb, orc, csw, kappa, L, nw, phases):
    U, b, bd, D, apply, op = _setup(lmb, orc, L, csw, kappa, phases, nw=nw)
    x = bd.similar()
    res = lmb.solve_evenodd_(x, D, bd, rtol=1e-10)
    assert res.converged and res.reason == "converged", res
    xs = x.gather_matrix()
    rel = _rel_residual(apply, xs, b)
    assert rel <= 1.05e-10
    assert abs(res.true_residual_norm / np.linalg.norm(b) - rel) <= 1e-3 * rel + 1e-14
    # the reference's route: cg!(x, DdagDOp(D), D'b)
    Db = apply(b, dagger=True)
    x_ref, _ = orc.cg_ddagd(op, Db, rtol=1e-13)
    assert rd.rel_err(xs, x_ref) <= 1e-7
    # preconditioning: fewer iterations than the unpreconditioned normal
    # equations at the same tolerance
    _, info = orc.cg_ddagd(op, Db, rtol=1e-10)
    assert res.iterations < info["iterations"]


@pytest.mark.parametrize("precision", ["single", "half"])
@pytest.mark.parametrize("csw,kappa", [(0.0, 0.125), (1.0, 0.1355)])
def test_evenodd_mixed_true_residual(lmb, orc, precision, csw, kappa):
    L = (8, 8, 8, 16)
    U, b, bd, D, apply, op = _setup(lmb, orc, L, csw, kappa, PHASES, amplitude=0.2)
    x = bd.similar()
    res = lmb.solve_evenodd_(x, D, bd, rtol=1e-10, precision=precision, delta=0.1)
    assert res.converged, res
    assert res.reliable_updates >= 1
    assert _rel_residual(apply, x.gather_matrix(), b) <= 1.05e-10


def test_evenodd_edge_cases(lmb, orc):
    L = (4, 4, 4, 4)
    U, b, bd, D, apply, op = _setup(lmb, orc, L, 1.0, 0.13, PHASES)
    x = bd.similar()
    zero = bd.similar()
    zr = lmb.solve_evenodd_(x, D, zero)
    assert zr.converged and zr.iterations == 0 and zr.true_residual_norm == 0
    assert not np.any(x.gather_matrix())
    few = lmb.solve_evenodd_(x, D, bd, maxiter=2)
    assert not few.converged and few.reason == "maximum_iterations"
    with pytest.raises(lmb.ArgumentError):
        lmb.solve_evenodd_(x, D, x)
    odd = lmb.LatticeMatrix.from_array(orc.gaussian_field((4, 4, 4, 5), 3, 4, 3), phases=PHASES)
    Uo = [lmb.LatticeMatrix.from_array(u) for u in orc.random_su3_links((4, 4, 4, 5), 0.3, 1)]
    with pytest.raises(lmb.ArgumentError, match="even"):
        lmb.solve_evenodd_(odd.similar(), lmb.WilsonDiracOperator4D(Uo, 0.12), odd)


def test_evenodd_complex64_fields(lmb, orc):
    L = (4, 4, 4, 8)
    U, b, bd, D, apply, op = _setup(lmb, orc, L, 1.0, 0.13, PHASES, dtype=np.complex64)
    x = bd.similar()
    res = lmb.solve_evenodd_(x, D, bd, rtol=1e-6)
    assert res.converged
    Uc = [np.asfortranarray(u.astype(np.complex64).astype(np.complex128)) for u in U]
    bc = np.asfortranarray(b.astype(np.complex64).astype(np.complex128))
    r = bc - orc.wilson_clover(Uc, np.asfortranarray(x.gather_matrix().astype(np.complex128)), 0.13, 1.0, PHASES)
    assert np.linalg.norm(r) / np.linalg.norm(bc) <= 2e-6
