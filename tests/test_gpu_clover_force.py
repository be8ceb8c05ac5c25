"""Wilson-clover force adjoint (wilson_clover_link_pullback!, the clover
fermion force) against central finite differences of the oracle: the
reference pins its pullbacks with finite-difference identities
(test/hisq_end_to_end_ad.jl:97-251 for HISQ; the clover pullback follows
WilsonCloverPullback.jl:342-403)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
PHASES = (1, 1, 1, -1)
TWISTED = tuple(np.exp(1j * a) for a in (0.13, -0.21, 0.34, np.pi - 0.17))


@pytest.fixture(scope="module")
def lmb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lmb200
    lmb200.load()
    return lmb200


def _rand_dir(L, seed):
    rng = np.random.default_rng(seed)
    return [np.asfortranarray(rng.normal(size=(3, 3) + L) + 1j * rng.normal(size=(3, 3) + L))
            for _ in range(4)]


@pytest.mark.parametrize("L,phases,csw", [((4, 4, 4, 4), PHASES, 1.0), ((4, 6, 4, 6), TWISTED, 1.3),
                                          ((3, 4, 5, 4), PHASES, 0.0)])
def test_link_pullback_matches_oracle_finite_differences(lmb, orc, L, phases, csw):
    kappa, coef = 0.13, 1.7
    U = orc.random_su3_links(L, 0.2, 41)
    psi = orc.gaussian_field(L, 3, 4, 42)
    dr = orc.gaussian_field(L, 3, 4, 43)
    Ud = [lmb.LatticeMatrix.from_array(u, nw=1) for u in U]
    D = lmb.WilsonDiracCloverOperator4D(Ud, kappa, csw)
    psid = lmb.LatticeMatrix.from_array(psi, nw=1, phases=phases)
    drd = lmb.LatticeMatrix.from_array(dr, nw=1, phases=phases)
    dU = [u.similar() for u in Ud]
    lmb.wilson_clover_link_pullback_(dU, D, Ud, drd, psid, coefficient=coef)
    G = [d.gather_matrix() for d in dU]

    def loss(Uh):
        out = orc.wilson_clover([np.asfortranarray(u) for u in Uh], psi, kappa, csw, phases)
        return coef * np.vdot(dr, out).real

    for seed in range(3):
        V = _rand_dir(L, 200 + seed)
        h = 1e-5
        fd = (loss([u + h * v for u, v in zip(U, V)]) - loss([u - h * v for u, v in zip(U, V)])) / (2 * h)
        an = sum(np.vdot(g, v).real for g, v in zip(G, V))
        assert abs(an - fd) <= 1e-8 * max(abs(fd), 1.0), (seed, an, fd)
    # accumulation: a second call adds the same gradient
    lmb.wilson_clover_link_pullback_(dU, D, Ud, drd, psid, coefficient=coef)
    assert np.allclose(dU[2].gather_matrix(), 2 * G[2], rtol=1e-13, atol=1e-13)


def test_fermion_force_matches_action_finite_differences(lmb, orc):
    L = (4, 4, 4, 4)
    kappa, csw = 0.12, 1.0
    U = orc.random_su3_links(L, 0.2, 51)
    phi = orc.gaussian_field(L, 3, 4, 52)
    Ud = [lmb.LatticeMatrix.from_array(u, nw=1) for u in U]
    phid = lmb.LatticeMatrix.from_array(phi, nw=1, phases=PHASES)
    D = lmb.WilsonDiracCloverOperator4D(Ud, kappa, csw)
    dU = [u.similar() for u in Ud]
    res = lmb.wilson_clover_fermion_force_(dU, D, phid, rtol=1e-13)
    assert res.converged
    G = [d.gather_matrix() for d in dU]

    def action(Uh):
        Uh = [np.asfortranarray(u) for u in Uh]
        op = orc.Operator(orc.OP_CLOVER, Uh, L, kappa=kappa, csw=csw, F=orc.clover_field_strength(Uh))
        x, r = orc.cg_ddagd(op, phi, rtol=1e-14, maxiter=20000)
        return np.vdot(phi, x).real

    V = _rand_dir(L, 9)
    h = 1e-5
    fd = (action([u + h * v for u, v in zip(U, V)]) - action([u - h * v for u, v in zip(U, V)])) / (2 * h)
    an = sum(np.vdot(g, v).real for g, v in zip(G, V))
    assert abs(an - fd) <= 1e-7 * abs(fd), (an, fd)


def test_pullback_rejects_bad_arguments(lmb, orc):
    L = (4, 4, 4, 4)
    U = orc.random_su3_links(L, 0.2, 1)
    Ud = [lmb.LatticeMatrix.from_array(u, nw=1) for u in U]
    psi = lmb.LatticeMatrix.from_array(orc.gaussian_field(L, 3, 4, 2), nw=1, phases=PHASES)
    D = lmb.WilsonDiracCloverOperator4D(Ud, 0.12, 1.0)
    with pytest.raises(lmb.ArgumentError, match="must not alias"):
        lmb.wilson_clover_link_pullback_(Ud, D, Ud, psi, psi)
    with pytest.raises(lmb.ArgumentError, match="coefficient must be real"):
        lmb.wilson_clover_link_pullback_([u.similar() for u in Ud], D, Ud, psi, psi, coefficient=1j)
    with pytest.raises(lmb.ArgumentError, match="four destination links"):
        lmb.wilson_clover_link_pullback_([Ud[0].similar()], D, Ud, psi, psi)
