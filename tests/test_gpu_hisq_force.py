"""HISQ force adjoint (hisq_link_pullback!, dSFdU) against central finite
differences: the reference pins this path with FD identities
(test/hisq_end_to_end_ad.jl:97-251); its Enzyme gradient needs Julia, which
this environment lacks."""
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


def _rand_dir(L, seed):
    rng = np.random.default_rng(seed)
    return [np.asfortranarray(rng.normal(size=(3, 3) + L) + 1j * rng.normal(size=(3, 3) + L))
            for _ in range(4)]


def _loss(orc, U, dr, psi, eps, coef):
    X, Ln = orc.hisq_links_from_thin(U, eps)
    out = orc.hisq(X, Ln, psi, 0.07, eps, PHASES)
    return coef * np.vdot(dr, out).real


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (4, 6, 4, 6)])
def test_link_pullback_matches_oracle_finite_differences(lmb, orc, L):
    eps, coef = -0.083, 1.7
    U = orc.random_su3_links(L, 0.2, 21)
    psi = orc.gaussian_field(L, 3, 1, 22)
    dr = orc.gaussian_field(L, 3, 1, 23)
    Ud = [lmb.LatticeMatrix.from_array(u, nw=3) for u in U]
    cache = lmb.HISQDiracCache4D(Ud, 0.07, eps)
    psid = lmb.LatticeMatrix.from_array(psi, nw=3, phases=PHASES)
    drd = lmb.LatticeMatrix.from_array(dr, nw=3, phases=PHASES)
    dU = [u.similar() for u in Ud]
    lmb.hisq_link_pullback_(dU, cache, Ud, drd, psid, coefficient=coef)
    G = [d.gather_matrix() for d in dU]
    for seed in range(3):
        V = _rand_dir(L, 100 + seed)
        h = 1e-5
        Up = [u + h * v for u, v in zip(U, V)]
        Um = [u - h * v for u, v in zip(U, V)]
        fd = (_loss(orc, [np.asfortranarray(a) for a in Up], dr, psi, eps, coef) -
              _loss(orc, [np.asfortranarray(a) for a in Um], dr, psi, eps, coef)) / (2 * h)
        an = sum(np.vdot(g, v).real for g, v in zip(G, V))
        assert abs(an - fd) <= 1e-8 * max(abs(fd), 1.0), (seed, an, fd)


def test_fermion_force_matches_action_finite_differences(lmb, orc):
    L = (4, 4, 4, 4)
    mass, eps = 0.2, 0.0
    U = orc.random_su3_links(L, 0.2, 31)
    phi = orc.gaussian_field(L, 3, 1, 32)
    Ud = [lmb.LatticeMatrix.from_array(u, nw=3) for u in U]
    phid = lmb.LatticeMatrix.from_array(phi, nw=3, phases=PHASES)
    cache = lmb.HISQDiracCache4D(Ud, mass, eps)
    dU = [u.similar() for u in Ud]
    res = lmb.hisq_fermion_force_(dU, cache, phid, rtol=1e-13)
    assert res.converged
    G = [d.gather_matrix() for d in dU]

    def action(Uh):
        X, Ln = orc.hisq_links_from_thin(Uh, eps)
        op = orc.Operator(orc.OP_HISQ, list(X) + list(Ln), L, mass=mass,
                          naik_epsilon=eps)
        x, r = orc.cg_ddagd(op, phi, rtol=1e-14, maxiter=20000)
        return np.vdot(phi, x).real

    V = _rand_dir(L, 7)
    h = 1e-5
    fd = (action([np.asfortranarray(u + h * v) for u, v in zip(U, V)]) -
          action([np.asfortranarray(u - h * v) for u, v in zip(U, V)])) / (2 * h)
    an = sum(np.vdot(g, v).real for g, v in zip(G, V))
    assert abs(an - fd) <= 1e-7 * abs(fd), (an, fd)
