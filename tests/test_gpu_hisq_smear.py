"""GPU parity of the HISQ smearing chain: SIMULATeQCD golden fingerprints
(the reference's own pins, tests/golden) and the oracle on random links."""
import json
import os

import numpy as np
import pytest

import refdata as rd

pytestmark = pytest.mark.gpu
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                     "reference_fingerprints.json")))
PHASES = (1, 1, 1, -1)


@pytest.fixture(scope="module")
def lmb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lmb200
    lmb200.load()
    return lmb200


def _dev(lmb, arrs, nw):
    return [lmb.LatticeMatrix.from_array(a, nw=nw) for a in arrs]


def _approx(a, b, atol, rtol):
    d = np.linalg.norm(np.ravel(a) - np.ravel(b))
    return d <= max(atol, rtol * max(np.linalg.norm(np.ravel(a)), np.linalg.norm(np.ravel(b))))


def test_level1_fat7_simulateqcd_fingerprints_gpu(lmb):
    g = GOLDEN["simulateqcd_level1_fat7"]
    U = _dev(lmb, rd.staggered_test_links(tuple(g["lattice"])), 1)
    V = [u.similar() for u in U]
    lmb.hisq_fat7_level1_(V, U)
    for mu in range(4):
        fp = rd.fingerprint(V[mu].gather_matrix())
        assert _approx(fp, np.array(g["expected"][mu]), g["atol"], g["rtol"]), (mu, fp)


def test_full_hisq_simulateqcd_fingerprints_gpu(lmb):
    g = GOLDEN["simulateqcd_full_hisq"]
    U = _dev(lmb, rd.near_identity_links(tuple(g["lattice"])), 3)
    links = lmb.hisq_links_from_thin(U, g["naik_epsilon"])
    for mu in range(4):
        assert _approx(rd.fingerprint(links.fat_links[mu].gather_matrix()),
                       np.array(g["fat"][mu]), g["atol"], g["rtol"]), mu
        assert _approx(rd.fingerprint(links.long_links[mu].gather_matrix()),
                       np.array(g["long"][mu]), g["atol"], g["rtol"]), mu


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (6, 4, 8, 4)])
def test_smearing_stages_match_oracle(lmb, orc, L):
    U = orc.random_su3_links(L, 0.25, 9)
    Ud = _dev(lmb, U, 3)
    V = [u.similar() for u in Ud]
    lmb.hisq_fat7_level1_(V, Ud)
    ref1 = orc.hisq_fat7(U, orc.LEVEL1)
    for mu in range(4):
        assert rd.rel_err(V[mu].gather_matrix(), ref1[mu]) <= 1e-13
    W = [u.similar() for u in Ud]
    lmb.hisq_project_u3_(W, V)
    refW = orc.hisq_project_u3(ref1)
    for mu in range(4):
        assert rd.rel_err(W[mu].gather_matrix(), refW[mu]) <= 1e-12
    X = [u.similar() for u in Ud]
    lmb.hisq_fat7_level2_(X, W, -0.083)
    refX = orc.hisq_fat7(refW, orc.level2_coefficients(-0.083))
    Ln = [u.similar() for u in Ud]
    lmb.hisq_naik_links_(Ln, W)
    refL = orc.hisq_naik(refW)
    for mu in range(4):
        assert rd.rel_err(X[mu].gather_matrix(), refX[mu]) <= 1e-12
        assert rd.rel_err(Ln[mu].gather_matrix(), refL[mu]) <= 1e-12


def test_cached_hisq_operator_follows_links(lmb, orc):
    L = (6, 4, 4, 6)
    U = orc.random_su3_links(L, 0.25, 10)
    psi = orc.gaussian_field(L, 3, 1, 11)
    Ud = _dev(lmb, U, 3)
    pd = lmb.LatticeMatrix.from_array(psi, nw=3, phases=PHASES)
    cache = lmb.HISQDiracCache4D(Ud, 0.05, -0.083)
    out = pd.similar()
    lmb.mul_cached_hisq_(out, cache, *Ud, pd)
    X, Ln = orc.hisq_links_from_thin(U, -0.083)
    ref = orc.hisq(X, Ln, psi, 0.05, -0.083, PHASES)
    assert rd.rel_err(out.gather_matrix(), ref) <= 1e-12
    # change one link: the cache must re-smear
    U2 = [u.copy(order="F") for u in U]
    U2[2][:, :, 1, 2, 3, 0] = orc.random_su3_links((1, 1, 1, 1), 0.3, 77)[0][:, :, 0, 0, 0, 0]
    Ud[2].set_core(U2[2])
    lmb.mul_cached_hisq_adjoint_(out, cache, *Ud, pd)
    X2, L2 = orc.hisq_links_from_thin(U2, -0.083)
    ref2 = orc.hisq(X2, L2, psi, 0.05, -0.083, PHASES, dagger=True)
    assert rd.rel_err(out.gather_matrix(), ref2) <= 1e-12


def test_shared_context_follows_a_growing_lattice(lmb, orc):
    """The smearing context is shared by every field of a device; its link
    and clover caches are sized by the volume, so a larger lattice after a
    smaller one must rebuild them (regression: a 16^4 smearing after 8^4
    copied into the 8^4-sized link set)."""
    for L in ((4, 4, 4, 4), (6, 4, 6, 8), (4, 4, 4, 4)):
        U = orc.random_su3_links(L, 0.25, 5)
        Ud = [lmb.LatticeMatrix.from_array(u, nw=3) for u in U]
        links = lmb.hisq_links_from_thin(Ud, -0.083)
        X, Ln = orc.hisq_links_from_thin(U, -0.083)
        for mu in range(4):
            assert rd.rel_err(links.fat_links[mu].gather_matrix(), X[mu]) <= 1e-12
            assert rd.rel_err(links.long_links[mu].gather_matrix(), Ln[mu]) <= 1e-12
