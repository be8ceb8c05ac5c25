"""GPU parity: generalised / Mobius domain-wall D5 (DiracOperators_5D.jl)
through the C ABI against the oracle (pinned to the reference's dense
domain-wall test, test/domainwall.jl), and the D5^+ D5 CG.

Bars: FP64 relative norm error <= 1e-13; FP32 storage <= 5e-6; int16
storage <= 2e-3; CG true residual from the oracle.
"""
import numpy as np
import pytest

import refdata as rd

pytestmark = pytest.mark.gpu

TWISTED = tuple(np.exp(1j * a) for a in (0.13, -0.21, 0.34, np.pi - 0.17))
PHASES = (1, 1, 1, -1)
MOBIUS = [(1.0, 1.0), (2.0, 0.0), (2.0, 1.0)]


@pytest.fixture(scope="module")
def lmb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lmb200
    lmb200.load()
    return lmb200


def _gauss5(orc, L, L5, seed):
    # Fortran (3, 4, X, Y, Z, T, L5) has the bytes of (3, 4, X, Y, Z, T*L5)
    X, Y, Z, T = L
    g = orc.gaussian_field((X, Y, Z, T * L5), 3, 4, seed)
    return np.asfortranarray(g.reshape((3, 4, X, Y, Z, T, L5), order="F"))


def _fields(lmb, orc, L, L5, nw=1, phases=PHASES, dtype=np.complex128, seed=1,
            amplitude=0.3):
    U = orc.random_su3_links(L, amplitude, seed)
    psi = _gauss5(orc, L, L5, seed + 1)
    Ud = [lmb.LatticeMatrix.from_array(u.astype(dtype), nw=nw) for u in U]
    pd = lmb.LatticeMatrix.from_array(psi.astype(dtype), dim=5, nw=nw,
                                      phases=tuple(phases) + (1,))
    return U, psi, Ud, pd


def _general(L5, seed):
    rng = np.random.default_rng(seed)
    return (list(0.8 + 0.4 * rng.random(L5)), list(0.9 + 0.6 * rng.random(L5)),
            list(-0.3 + 0.6 * rng.random(L5)))


@pytest.mark.parametrize("L,L5,nw,phases", [
    ((4, 4, 4, 4), 4, 1, PHASES), ((3, 2, 2, 4), 3, 1, TWISTED),
    ((6, 4, 2, 8), 5, 2, TWISTED)])
@pytest.mark.parametrize("bc", MOBIUS)
@pytest.mark.parametrize("dagger", [False, True])
def test_mobius_fp64_matches_oracle(lmb, orc, L, L5, nw, phases, bc, dagger):
    U, psi, Ud, pd = _fields(lmb, orc, L, L5, nw=nw, phases=phases)
    mass, M = 0.13, -1.0
    D = lmb.D5DW_MobiusDomainwallOperator5D(Ud, L5, mass, M, *bc)
    out = pd.similar()
    lmb.mul_(out, lmb.adjoint(D) if dagger else D, pd)
    a, b, c = orc.mobius_coefficients(L5, *bc)
    ref = orc.domainwall(U, psi, mass, M, a, b, c, phases, dagger=dagger)
    assert rd.rel_err(out.gather_matrix(), ref) <= 1e-13


@pytest.mark.parametrize("L,L5", [((4, 4, 4, 8), 6), ((4, 2, 2, 4), 1),
                                  ((2, 2, 2, 2), 2)])
@pytest.mark.parametrize("dagger", [False, True])
def test_generalized_fp64_matches_oracle(lmb, orc, L, L5, dagger):
    U, psi, Ud, pd = _fields(lmb, orc, L, L5, phases=TWISTED, seed=5)
    a, b, c = _general(L5, 7)
    D = lmb.D5DW_GeneralizedDomainwallOperator5D(Ud, L5, 0.07, -1.8, a, b, c)
    out = pd.similar()
    lmb.mul_(out, lmb.adjoint(D) if dagger else D, pd)
    ref = orc.domainwall(U, psi, 0.07, -1.8, a, b, c, TWISTED, dagger=dagger)
    assert rd.rel_err(out.gather_matrix(), ref) <= 1e-13


def test_adjoint_identity(lmb, orc):
    L, L5 = (4, 4, 2, 6), 5
    U, psi, Ud, pd = _fields(lmb, orc, L, L5, phases=TWISTED, seed=9)
    left = _gauss5(orc, L, L5, 31)
    ld = lmb.LatticeMatrix.from_array(left, dim=5, phases=TWISTED + (1,))
    D = lmb.D5DW_GeneralizedDomainwallOperator5D(Ud, L5, 0.2, -1.4, *_general(L5, 3))
    Dpsi, Dl = pd.similar(), pd.similar()
    lmb.mul_(Dpsi, D, pd)
    lmb.mul_(Dl, lmb.adjoint(D), ld)
    lhs = np.vdot(left, Dpsi.gather_matrix())
    rhs = np.vdot(Dl.gather_matrix(), psi)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("precision,bar", [("single", 5e-6), ("half", 2e-3)])
@pytest.mark.parametrize("dagger", [False, True])
def test_reduced_precision_storage(lmb, orc, precision, bar, dagger):
    L, L5 = (4, 4, 4, 8), 8
    U, psi, Ud, pd = _fields(lmb, orc, L, L5)
    D = lmb.D5DW_MobiusDomainwallOperator5D(Ud, L5, 0.1, -1.8, 2.0, 1.0)
    out = pd.similar()
    lmb.mul_(out, lmb.adjoint(D) if dagger else D, pd, precision=precision)
    a, b, c = orc.mobius_coefficients(L5, 2.0, 1.0)
    ref = orc.domainwall(U, psi, 0.1, -1.8, a, b, c, PHASES, dagger=dagger)
    assert rd.rel_err(out.gather_matrix(), ref) <= bar


def test_complex64_fields(lmb, orc):
    L, L5 = (4, 4, 4, 4), 4
    U, psi, Ud, pd = _fields(lmb, orc, L, L5, dtype=np.complex64)
    D = lmb.D5DW_MobiusDomainwallOperator5D(Ud, L5, 0.1, -1.8, 2.0, 1.0)
    out = pd.similar()
    lmb.mul_(out, D, pd)
    Uc = [np.asfortranarray(u.astype(np.complex64).astype(np.complex128)) for u in U]
    pc = np.asfortranarray(psi.astype(np.complex64).astype(np.complex128))
    a, b, c = orc.mobius_coefficients(L5, 2.0, 1.0)
    ref = orc.domainwall(Uc, pc, 0.1, -1.8, a, b, c, PHASES)
    assert rd.rel_err(out.gather_matrix().astype(np.complex128), ref) <= 1e-6


def _ddagd(orc, U, x, mass, M, a, b, c):
    y = orc.domainwall(U, x, mass, M, a, b, c, PHASES)
    return orc.domainwall(U, np.asfortranarray(y), mass, M, a, b, c, PHASES, dagger=True)


@pytest.mark.parametrize("precision,rtol,bar", [
    ("double", 1e-10, 1e-9), ("single", 1e-10, 1.05e-10), ("half", 1e-10, 1.05e-10)])
def test_cg_true_residual(lmb, orc, precision, rtol, bar):
    L, L5 = (4, 4, 4, 8), 8
    U, b, Ud, bd, = _fields(lmb, orc, L, L5, amplitude=0.2, seed=3)
    mass, M = 0.1, -1.8
    D = lmb.D5DW_MobiusDomainwallOperator5D(Ud, L5, mass, M, 2.0, 1.0)
    x = bd.similar()
    res = lmb.cg_(x, lmb.DdagDOp(D, bd.similar()), bd, rtol=rtol,
                  precision=precision, maxiter=5000)
    assert res.converged and res.reason == "converged", res
    if precision != "double":
        assert res.reliable_updates >= 1
    a, bb, c = orc.mobius_coefficients(L5, 2.0, 1.0)
    xs = x.gather_matrix()
    true_rel = np.linalg.norm(b - _ddagd(orc, U, xs, mass, M, a, bb, c)) / np.linalg.norm(b)
    assert true_rel <= bar


def test_cg_generalized_edge_cases(lmb, orc):
    L, L5 = (4, 4, 2, 4), 3
    U, b, Ud, bd = _fields(lmb, orc, L, L5, seed=11)
    D = lmb.D5DW_GeneralizedDomainwallOperator5D(Ud, L5, 0.3, -1.5, *_general(L5, 13))
    A = lmb.DdagDOp(D, bd.similar())
    x = bd.similar()
    zr = lmb.cg_(x, A, bd.similar(), rtol=1e-13)
    assert zr.converged and zr.iterations == 0 and zr.residual_norm == 0
    few = lmb.cg_(x, A, bd, maxiter=2)
    assert few.reason == "maximum_iterations" and few.iterations == 2
    res = lmb.cg_(bd.similar(), A, bd, rtol=1e-11)
    assert res.converged


@pytest.mark.parametrize("dagger", [False, True])
def test_two_pass_kernels_match_oracle(lmb, orc, monkeypatch, dagger):
    """LMB_DW_TWO_PASS=1 (read when the context is created) selects the
    two-pass kernels; L5 > 128 takes them in any case."""
    monkeypatch.setenv("LMB_DW_TWO_PASS", "1")
    for L, L5 in (((4, 4, 2, 4), 5), ((2, 2, 2, 2), 130)):
        U, psi, Ud, pd = _fields(lmb, orc, L, L5, phases=TWISTED, seed=17)
        a, b, c = _general(L5, 19)
        D = lmb.D5DW_GeneralizedDomainwallOperator5D(Ud, L5, 0.05, -1.2, a, b, c)
        for prec, bar in (("double", 1e-13), ("single", 5e-6)):
            out = pd.similar()
            lmb.mul_(out, lmb.adjoint(D) if dagger else D, pd, precision=prec)
            ref = orc.domainwall(U, psi, 0.05, -1.2, a, b, c, TWISTED, dagger=dagger)
            assert rd.rel_err(out.gather_matrix(), ref) <= bar


def test_long_fifth_dimension_cg(lmb, orc):
    """L5 = 130 > 128: two-pass kernels inside the CG driver."""
    L, L5 = (2, 2, 2, 4), 130
    U, b, Ud, bd = _fields(lmb, orc, L, L5, seed=23)
    D = lmb.D5DW_MobiusDomainwallOperator5D(Ud, L5, 0.2, -1.5, 1.5, 0.5)
    x = bd.similar()
    res = lmb.cg_(x, lmb.DdagDOp(D, bd.similar()), bd, rtol=1e-10, precision="half")
    assert res.converged
    a, bb, c = orc.mobius_coefficients(L5, 1.5, 0.5)
    xs = x.gather_matrix()
    true_rel = np.linalg.norm(b - _ddagd(orc, U, xs, 0.2, -1.5, a, bb, c)) / np.linalg.norm(b)
    assert true_rel <= 1.05e-10
