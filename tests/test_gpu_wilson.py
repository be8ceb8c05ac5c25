"""GPU parity: Wilson and Wilson-clover through the C ABI against the oracle.

Bar: FP64 relative norm error <= 1e-13 (the reference's operator-parity bar);
FP32 storage <= 5e-6; int16 storage <= 2e-3.
"""
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


def _fields(lmb, orc, L, amplitude=0.3, nw=1, phases=PHASES, dtype=np.complex128,
            seed=1):
    U = orc.random_su3_links(L, amplitude, seed)
    psi = orc.gaussian_field(L, 3, 4, seed + 1)
    Ud = [lmb.LatticeMatrix.from_array(u.astype(dtype), nw=nw) for u in U]
    pd = lmb.LatticeMatrix.from_array(psi.astype(dtype), nw=nw, phases=phases)
    return U, psi, Ud, pd


@pytest.mark.parametrize("L,nw,phases", [
    ((4, 4, 4, 4), 1, PHASES), ((3, 2, 2, 4), 0, TWISTED),
    ((6, 4, 4, 8), 3, TWISTED), ((8, 8, 8, 8), 1, PHASES)])
@pytest.mark.parametrize("dagger", [False, True])
def test_wilson_fp64_matches_oracle(lmb, orc, L, nw, phases, dagger):
    U, psi, Ud, pd = _fields(lmb, orc, L, nw=nw, phases=phases)
    D = lmb.WilsonDiracOperator4D(Ud, 0.125)
    out = pd.similar()
    lmb.mul_(out, lmb.adjoint(D) if dagger else D, pd)
    ref = orc.wilson(U, psi, 0.125, phases, dagger=dagger)
    assert rd.rel_err(out.gather_matrix(), ref) <= 1e-13


@pytest.mark.parametrize("L,nw,phases", [
    ((4, 4, 4, 4), 1, PHASES), ((3, 2, 2, 4), 0, TWISTED),
    ((6, 4, 2, 8), 2, TWISTED), ((8, 8, 8, 16), 1, PHASES)])
@pytest.mark.parametrize("dagger", [False, True])
def test_wilson_clover_fp64_matches_oracle(lmb, orc, L, nw, phases, dagger):
    U, psi, Ud, pd = _fields(lmb, orc, L, nw=nw, phases=phases)
    D = lmb.WilsonDiracCloverOperator4D(Ud, 0.1355, 1.0)
    out = pd.similar()
    lmb.mul_(out, lmb.adjoint(D) if dagger else D, pd)
    ref = orc.wilson_clover(U, psi, 0.1355, 1.0, phases, dagger=dagger)
    assert rd.rel_err(out.gather_matrix(), ref) <= 1e-13


def test_clover_field_strength_matches_oracle(lmb, orc):
    L = (4, 2, 6, 4)
    U, psi, Ud, pd = _fields(lmb, orc, L)
    D = lmb.WilsonDiracCloverOperator4D(Ud, 0.12, 1.17)
    F = D.field_strength(pd)
    ref = orc.clover_field_strength(U)
    for plane in range(6):
        assert rd.rel_err(F[plane].gather_matrix(), ref[plane]) <= 1e-13


def test_complex64_fields(lmb, orc):
    L = (4, 4, 4, 8)
    U, psi, Ud, pd = _fields(lmb, orc, L, dtype=np.complex64)
    D = lmb.WilsonDiracCloverOperator4D(Ud, 0.13, 1.0)
    out = pd.similar()
    lmb.mul_(out, D, pd)
    Uc = [np.asfortranarray(u.astype(np.complex64).astype(np.complex128)) for u in U]
    pc = np.asfortranarray(psi.astype(np.complex64).astype(np.complex128))
    ref = orc.wilson_clover(Uc, pc, 0.13, 1.0, PHASES)
    assert rd.rel_err(out.gather_matrix(), ref) <= 1e-6


@pytest.mark.parametrize("precision,tol", [("single", 5e-6), ("half", 2e-3)])
@pytest.mark.parametrize("clover", [False, True])
@pytest.mark.parametrize("L,pair,adj", [((8, 4, 4, 8), "1", "1"), ((8, 4, 4, 8), "1", "0"),
                                        ((8, 4, 4, 8), "0", "1"), ((6, 4, 4, 2), "1", "1"),
                                        ((6, 4, 4, 2), "1", "0"), ((4, 6, 4, 5), "1", "1"),
                                        ((5, 4, 4, 6), "1", "1"), ((5, 3, 4, 5), "1", "1")])
def test_low_precision_storage(lmb, orc, precision, tol, clover, L, pair, adj, monkeypatch):
    """Two sites per thread in packed FP32 unless LMB_PAIR_SITES=0: int16
    storage with an even x extent pairs x-neighbours (256-bit loads) unless
    LMB_ADJ_SITES=0; otherwise an even T pairs s and s + V/2 (T = 2 puts every
    t-hop of one lane across the boundary); odd x and T run one site per
    thread."""
    monkeypatch.setenv("LMB_PAIR_SITES", pair)
    monkeypatch.setenv("LMB_ADJ_SITES", adj)
    U, psi, Ud, pd = _fields(lmb, orc, L, phases=TWISTED)
    D = lmb.WilsonDiracCloverOperator4D(Ud, 0.1355, 1.0) if clover \
        else lmb.WilsonDiracOperator4D(Ud, 0.1355)
    out = pd.similar()
    for dag in (False, True):
        lmb.mul_(out, lmb.adjoint(D) if dag else D, pd, precision=precision)
        ref = orc.wilson_clover(U, psi, 0.1355, 1.0, TWISTED, dagger=dag) if clover \
            else orc.wilson(U, psi, 0.1355, TWISTED, dagger=dag)
        assert rd.rel_err(out.gather_matrix(), ref) <= tol


def test_link_cache_follows_epoch(lmb, orc):
    L = (4, 4, 4, 4)
    U, psi, Ud, pd = _fields(lmb, orc, L)
    D = lmb.WilsonDiracCloverOperator4D(Ud, 0.12, 1.0)
    out = pd.similar()
    lmb.mul_(out, D, pd)
    U2 = [u.copy(order="F") for u in U]
    U2[0][0, 0, 1, 2, 3, 0] += 0.07 + 0.02j
    Ud[0].set_core(U2[0])          # bumps halo_epoch.core
    lmb.mul_(out, D, pd)
    ref = orc.wilson_clover(U2, psi, 0.12, 1.0, PHASES)
    assert rd.rel_err(out.gather_matrix(), ref) <= 1e-13
    # mul_cached_clover! with explicit links
    lmb.mul_cached_clover_(out, D, *Ud, pd)
    assert rd.rel_err(out.gather_matrix(), ref) <= 1e-13
    lmb.mul_cached_clover_adjoint_(out, D, *Ud, pd)
    refd = orc.wilson_clover(U2, psi, 0.12, 1.0, PHASES, dagger=True)
    assert rd.rel_err(out.gather_matrix(), refd) <= 1e-13


def test_reference_test_links_nc3(lmb, orc):
    """Non-unitary deterministic links of the reference tests
    (staggered_dirac.jl:19-35) exercise the half-precision link scale."""
    L = (4, 2, 2, 2)
    U = rd.staggered_test_links(L, 3)
    psi = rd.clover_test_spinor(L, NC=3)
    Ud = [lmb.LatticeMatrix.from_array(u, nw=1) for u in U]
    pd = lmb.LatticeMatrix.from_array(psi, nw=1, phases=TWISTED)
    D = lmb.WilsonDiracCloverOperator4D(Ud, 0.12, 1.17)
    out = pd.similar()
    lmb.mul_(out, D, pd)
    ref = orc.wilson_clover(U, psi, 0.12, 1.17, TWISTED)
    assert rd.rel_err(out.gather_matrix(), ref) <= 1e-13
    lmb.mul_(out, D, pd, precision="half")
    assert rd.rel_err(out.gather_matrix(), ref) <= 5e-3


def test_dot(lmb, orc):
    L = (4, 4, 2, 6)
    a = orc.gaussian_field(L, 3, 4, 5)
    b = orc.gaussian_field(L, 3, 4, 6)
    A = lmb.LatticeMatrix.from_array(a, nw=2)
    B = lmb.LatticeMatrix.from_array(b, nw=2)
    got = lmb.dot(A, B)
    assert abs(got - np.vdot(a, b)) <= 1e-12 * abs(np.vdot(a, b))


def test_seeded_inputs_match_oracle_generator(lmb, orc):
    L = (4, 2, 6, 4)
    U = lmb.random_su3_links(L, 0.25, 11, nw=2)
    ref = orc.random_su3_links(L, 0.25, 11)
    for mu in range(4):
        assert rd.rel_err(U[mu].gather_matrix(), ref[mu]) <= 1e-13
    f = lmb.gaussian_fermion(L, 3, 4, 12, nw=1)
    assert rd.rel_err(f.gather_matrix(), orc.gaussian_field(L, 3, 4, 12)) <= 1e-13
