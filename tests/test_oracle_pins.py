"""Pin the CPU oracle to the reference's own known answers.

Each test replays one of LatticeMatrices.jl's tests: the dense in-test oracles
(restated in tests/refdata.py) at the reference's tolerances, and the golden
fingerprints the reference copied from Bridge++ 2.1.3 and SIMULATeQCD 767a1b1
(tests/golden/reference_fingerprints.json, extracted by
tests/golden/extract_fingerprints.py).
"""
import json
import os

import numpy as np
import pytest

import refdata as rd

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                     "reference_fingerprints.json")))
PHASES = (1, 1, 1, -1)
TWISTED = tuple(np.exp(1j * a) for a in (0.13, -0.21, 0.34, np.pi - 0.17))


def _close(a, b, atol, rtol):
    return np.allclose(a, b, atol=atol, rtol=rtol)


def _approx(a, b, atol, rtol):
    # Julia isapprox on arrays: norm(a-b) <= max(atol, rtol*max(norm(a),norm(b)))
    d = np.linalg.norm(np.ravel(a) - np.ravel(b))
    return d <= max(atol, rtol * max(np.linalg.norm(np.ravel(a)),
                                     np.linalg.norm(np.ravel(b))))


# --------------------------------------------------------------------------
# Wilson-clover: test/wilson_clover.jl:153-190 (NC=2, 2^4, kappa .12, csw 1.17)
# --------------------------------------------------------------------------
def test_clover_field_strength_dense(orc):
    L = (2, 2, 2, 2)
    links = rd.clover_test_links(L)
    F = orc.clover_field_strength(links)
    ref = rd.clover_field_strength_dense(links)
    for plane in range(6):
        assert _approx(F[plane], ref[plane], 2e-12, 2e-12)
        for x in rd.sites(L):
            m = rd.mat(F[plane], x)
            assert np.allclose(m.conj().T, -m, atol=2e-12)


@pytest.mark.parametrize("L", [(2, 2, 2, 2), (3, 2, 2, 2)])
def test_wilson_clover_dense(orc, L):
    links = rd.clover_test_links(L)
    psi = rd.clover_test_spinor(L)
    out = orc.wilson_clover(links, psi, 0.12, 1.17, PHASES)
    ref = rd.wilson_clover_dense(links, psi, 0.12, 1.17, PHASES)
    assert _approx(out, ref, 3e-12, 3e-12)


def test_wilson_clover_adjoint_gamma5_and_limits(orc):
    L = (2, 2, 2, 2)
    links = rd.clover_test_links(L)
    psi = rd.clover_test_spinor(L)
    chi = rd.clover_test_spinor(L, offset=0.19)
    Dpsi = orc.wilson_clover(links, psi, 0.12, 1.17, PHASES)
    Ddchi = orc.wilson_clover(links, chi, 0.12, 1.17, PHASES, dagger=True)
    assert np.isclose(np.vdot(chi, Dpsi), np.vdot(Ddchi, psi),
                      atol=5e-11, rtol=5e-12)
    Ddpsi = orc.wilson_clover(links, psi, 0.12, 1.17, PHASES, dagger=True)
    g5 = rd.apply_gamma5(orc.wilson_clover(links, rd.apply_gamma5(psi), 0.12,
                                           1.17, PHASES))
    assert _approx(Ddpsi, g5, 5e-12, 5e-12)
    # csw = 0 reduces to Wilson (wilson_clover.jl:225-240)
    assert _approx(orc.wilson_clover(links, psi, 0.12, 0.0, PHASES),
                   orc.wilson(links, psi, 0.12, PHASES), 2e-12, 2e-12)
    # unit gauge -> F = 0
    unit = [rd.unit_links(L, 2) for _ in range(4)]
    assert all(np.max(np.abs(f)) == 0 for f in orc.clover_field_strength(unit))


def test_wilson_clover_gauge_covariance(orc):
    # wilson_clover.jl:279-303 with the SU(2) transformation recipe :125-150
    L = (2, 2, 2, 2)
    links = rd.clover_test_links(L)
    psi = rd.clover_test_spinor(L)
    G = rd.zeros(2, 2, L)
    for x in rd.sites(L):
        coordinate = x[0] + 3 * x[1] + 4 * x[2] + 7 * x[3]
        G[(slice(None), slice(None)) + rd.idx(x)] = rd.clover_test_su2(
            0.053 * coordinate, 0.097 * (coordinate + 1))
    tl = rd.gauge_transform(links, G)
    tpsi = rd.transform_field(G, psi)
    out = orc.wilson_clover(tl, tpsi, 0.12, 1.17, PHASES)
    expected = rd.transform_field(G, orc.wilson_clover(links, psi, 0.12, 1.17,
                                                       PHASES))
    assert _approx(out, expected, 8e-12, 8e-12)


def test_wilson_nc3_dense_and_donly(orc):
    L = (3, 2, 2, 4)
    links = rd.staggered_test_links(L, 3)
    psi = rd.clover_test_spinor(L, NC=3)
    for dag in (False, True):
        out = orc.wilson(links, psi, 0.125, TWISTED, dagger=dag)
        ref = rd.wilson_clover_dense(links, psi, 0.125, 0.0, TWISTED, dagger=dag) \
            if not dag else None
        if ref is not None:
            assert _approx(out, ref, 3e-12, 3e-12)
    # Donly = (psi - D psi)/(2 kappa) with the hopping only, scaled by 1/2
    d = orc.wilson(links, psi, 0.125, PHASES)
    donly = orc.wilson_donly(links, psi, PHASES)
    assert _approx(donly, (psi - d) / (2 * 0.125), 1e-12, 1e-12)


# --------------------------------------------------------------------------
# staggered: test/staggered_dirac.jl
# --------------------------------------------------------------------------
def test_staggered_dense_and_twisted(orc):
    L = (4, 2, 2, 2)
    links = rd.staggered_test_links(L)
    psi = rd.staggered_test_fermion(L)
    for ph in (PHASES, TWISTED):
        for dag in (False, True):
            out = orc.staggered(links, psi, 0.17, ph, dagger=dag)
            ref = rd.staggered_dense(links, psi, 0.17, ph, dagger=dag)
            assert _approx(out, ref, 4e-12, 4e-12)


def test_staggered_bridgepp_fingerprints(orc):
    g = GOLDEN["bridgepp_staggered"]
    L = tuple(g["lattice"])
    links = rd.staggered_test_links(L)
    psi = rd.staggered_test_fermion(L)
    for mode, dag in (("D", False), ("Ddag", True)):
        fp = rd.fingerprint(orc.staggered(links, psi, g["mass"], PHASES,
                                          dagger=dag))
        assert _approx(fp, np.array(g[mode]), g["atol"], g["rtol"]), (mode, fp)


def test_staggered_epsilon_hermiticity_and_free_spectrum(orc):
    L = (4, 2, 2, 2)
    links = rd.staggered_test_links(L)
    psi = rd.staggered_test_fermion(L)
    chi = rd.staggered_test_fermion(L, offset=0.29)
    Dpsi = orc.staggered(links, psi, 0.17, PHASES)
    Ddchi = orc.staggered(links, chi, 0.17, PHASES, dagger=True)
    assert np.isclose(np.vdot(chi, Dpsi), np.vdot(Ddchi, psi), atol=2e-11,
                      rtol=5e-12)
    eps = rd.zeros(1, 1, L)[0, 0]
    for x in rd.sites(L):
        eps[rd.idx(x)] = 1 if sum(v - 1 for v in x) % 2 == 0 else -1
    Ddpsi = orc.staggered(links, psi, 0.17, PHASES, dagger=True)
    e_D_e = eps * orc.staggered(links, eps * psi, 0.17, PHASES)
    assert _approx(Ddpsi, e_D_e, 4e-12, 4e-12)
    # free D'D plane wave (staggered_dirac.jl:358-382), NC = 1
    E = (4, 4, 4, 4)
    unit = [rd.unit_links(E, 1) for _ in range(4)]
    p = (2 * np.pi / E[0], 0.0, 0.0, np.pi / E[3])
    w = rd.plane_wave(E, p)
    out = orc.staggered(unit, orc.staggered(unit, w, 0.17, PHASES), 0.17,
                        PHASES, dagger=True)
    ev = 0.17 ** 2 + sum(np.sin(q) ** 2 for q in p)
    assert _approx(out, ev * w, 8e-12, 8e-12)


def test_staggered_gauge_covariance_and_eta_offset(orc):
    L = (3, 2, 2, 2)
    links = rd.staggered_test_links(L)
    psi = rd.staggered_test_fermion(L)
    G = rd.gauge_transformations(L)
    out = orc.staggered(rd.gauge_transform(links, G), rd.transform_field(G, psi),
                        0.17, PHASES)
    exp = rd.transform_field(G, orc.staggered(links, psi, 0.17, PHASES))
    assert _approx(out, exp, 6e-12, 6e-12)
    # eta uses global coordinates: a rank offset of 3 in x flips eta_2..4
    a = orc.staggered(links, psi, 0.17, PHASES, eta_offset=(3, 0, 0, 0))
    b = orc.staggered(links, psi, 0.17, PHASES, eta_offset=(0, 0, 0, 0))
    assert not np.allclose(a, b)


# --------------------------------------------------------------------------
# HISQ stencil: test/hisq_dirac.jl
# --------------------------------------------------------------------------
def test_hisq_dense_twisted(orc):
    L = (4, 4, 4, 4)
    fat, lng = rd.hisq_test_links(L)
    psi = rd.staggered_test_fermion(L)
    for dag in (False, True):
        out = orc.hisq(fat, lng, psi, 0.17, -0.083, TWISTED, dagger=dag)
        ref = rd.hisq_dense(fat, lng, psi, 0.17, -0.083, TWISTED, dagger=dag)
        assert _approx(out, ref, 8e-12, 8e-12)


def test_hisq_free_spectrum(orc):
    E = (4, 4, 4, 4)
    eps = -0.083
    fs = (9 + eps) / 8
    X = [rd.unit_links(E, 1, fs) for _ in range(4)]
    Ln = [rd.unit_links(E, 1) for _ in range(4)]
    p = (2 * np.pi / E[0], 0.0, 0.0, np.pi / E[3])
    w = rd.plane_wave(E, p)
    out = orc.hisq(X, Ln, orc.hisq(X, Ln, w, 0.17, eps, PHASES), 0.17, eps,
                   PHASES, dagger=True)
    f = lambda q: fs * np.sin(q) - (1 + eps) * np.sin(3 * q) / 24
    ev = 0.17 ** 2 + sum(f(q) ** 2 for q in p)
    assert _approx(out, ev * w, 2e-11, 2e-11)


# --------------------------------------------------------------------------
# HISQ smearing: test/hisq_smearing.jl, test/hisq_full_smearing.jl
# --------------------------------------------------------------------------
def test_fat7_level1_dense(orc):
    L = (4, 3, 3, 3)
    U = rd.staggered_test_links(L)
    V = orc.hisq_fat7(U, orc.LEVEL1)
    ref = rd.fat7_dense(U, orc.LEVEL1)
    for mu in range(4):
        assert _approx(V[mu], ref[mu], 2e-11, 2e-11)


def test_fat7_level1_simulateqcd_fingerprints(orc):
    g = GOLDEN["simulateqcd_level1_fat7"]
    U = rd.staggered_test_links(tuple(g["lattice"]))
    V = orc.hisq_fat7(U, orc.LEVEL1)
    for mu in range(4):
        fp = rd.fingerprint(V[mu])
        assert _approx(fp, np.array(g["expected"][mu]), g["atol"], g["rtol"]), \
            (mu, fp, g["expected"][mu])


def test_fat7_free_field_normalisation(orc):
    # level-1 on unit links: 1/8 + 6/16 + 24/64 + 48/384 = 1
    L = (3, 3, 3, 3)
    unit = [rd.unit_links(L, 3) for _ in range(4)]
    V = orc.hisq_fat7(unit, orc.LEVEL1)
    for mu in range(4):
        assert _approx(V[mu], unit[0], 1e-13, 1e-13)
    V2 = orc.hisq_fat7(unit, orc.level2_coefficients(-0.083))
    assert _approx(V2[0], (9 - 0.083) / 8 * unit[0], 1e-13, 1e-13)


def test_u3_projection_and_level2_naik_dense(orc):
    L = (3, 3, 3, 3)
    U = rd.near_identity_links(L)
    lvl1 = orc.hisq_fat7(U, orc.LEVEL1)
    W = orc.hisq_project_u3(lvl1)
    Wref = rd.project_u3_dense(lvl1)
    for mu in range(4):
        assert _approx(W[mu], Wref[mu], 2e-11, 2e-11)
    X = orc.hisq_fat7(W, orc.level2_coefficients(-0.083))
    Xref = rd.fat7_dense(W, orc.level2_coefficients(-0.083))
    Ln = orc.hisq_naik(W)
    Lref = rd.naik_dense(W)
    for mu in range(4):
        assert _approx(X[mu], Xref[mu], 2e-11, 2e-11)
        assert _approx(Ln[mu], Lref[mu], 2e-11, 2e-11)


def test_full_hisq_simulateqcd_fingerprints(orc):
    g = GOLDEN["simulateqcd_full_hisq"]
    U = rd.near_identity_links(tuple(g["lattice"]))
    X, Ln = orc.hisq_links_from_thin(U, g["naik_epsilon"])
    for mu in range(4):
        assert _approx(rd.fingerprint(X[mu]), np.array(g["fat"][mu]),
                       g["atol"], g["rtol"]), mu
        assert _approx(rd.fingerprint(Ln[mu]), np.array(g["long"][mu]),
                       g["atol"], g["rtol"]), mu


# --------------------------------------------------------------------------
# CG (cg.jl:73-137) on a real Dirac operator, and seeded inputs
# --------------------------------------------------------------------------
def test_cg_ddagd_true_residual(orc):
    L = (4, 4, 4, 4)
    U = orc.random_su3_links(L, 0.3, 1)
    b = orc.gaussian_field(L, 3, 4, 2)
    op = orc.Operator(orc.OP_WILSON, U, L, kappa=0.125)
    x, res = orc.cg_ddagd(op, b, rtol=1e-10)
    assert res["converged"] and res["reason"] == "converged"
    r = b - op.ddagd(x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-10
    # maxiter = 0 -> maximum_iterations; zero rhs -> converged at 0
    _, res0 = orc.cg_ddagd(op, b, maxiter=0)
    assert res0["reason"] == "maximum_iterations" and not res0["converged"]
    _, resz = orc.cg_ddagd(op, orc.Operator.field(op))
    assert resz["converged"] and resz["iterations"] == 0
    assert resz["relative_residual"] == 0.0


def test_random_links_are_su3_and_seeded(orc):
    L = (2, 2, 2, 2)
    U = orc.random_su3_links(L, 0.2, 1)
    U2 = orc.random_su3_links(L, 0.2, 1)
    U3 = orc.random_su3_links(L, 0.2, 7)
    assert all(np.array_equal(a, b) for a, b in zip(U, U2))
    assert not np.allclose(U[0], U3[0])
    for mu in range(4):
        for x in rd.sites(L):
            m = rd.mat(U[mu], x)
            assert np.allclose(m @ m.conj().T, np.eye(3), atol=1e-14)
            assert np.isclose(np.linalg.det(m), 1.0, atol=1e-14)
    b = orc.gaussian_field((8, 8, 8, 8), 3, 4, 2)
    v = b.ravel()
    assert abs(np.mean(np.abs(v) ** 2) - 1.0) < 0.02
    assert abs(np.mean(v.real)) < 0.02


def test_philox_known_answer(orc):
    # Random123 Philox4x32-10 known-answer vectors (kat_vectors):
    # counter 0, key 0 and counter all-ones, key all-ones.
    assert orc.philox4x32((0, 0, 0, 0), (0, 0)) == (
        0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)
    assert orc.philox4x32((0xffffffff,) * 4, (0xffffffff,) * 2) == (
        0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)


DW_PHASES = (np.exp(0.13j), np.exp(-0.21j), np.exp(0.34j), np.exp(1j * (np.pi - 0.17)))


@pytest.mark.parametrize("nc", [2, 3])
def test_domainwall_matches_reference_dense_oracle(orc, nc):
    """test/domainwall.jl:205-299: Mobius (b, c) in {(1,1), (2,0), (2,1)} and a
    generalised operator on the reference's deterministic inputs (lattice
    2^4, L5 = 3, mass 0.13, M = -1, twisted phases), at its 8e-12 bars."""
    L, L5, mass, M = (2, 2, 2, 2), 3, 0.13, -1.0
    links = [np.asfortranarray(rd.domainwall_test_values(nc, nc, L, 7 * (mu + 1))) for mu in range(4)]
    psi = np.asfortranarray(rd.domainwall_test_values(nc, 4, L + (L5,), 11))
    left = np.asfortranarray(rd.domainwall_test_values(nc, 4, L + (L5,), 23))
    cases = [orc.mobius_coefficients(L5, b, c) for b, c in ((1.0, 1.0), (2.0, 0.0), (2.0, 1.0))]
    cases.append(([0.83, 1.17, 1.31], [1.2, 0.91, 1.47], [-0.18, 0.37, 0.22]))
    for a, b, c in cases:
        got = orc.domainwall(links, psi, mass, M, a, b, c, DW_PHASES)
        ref = rd.domainwall_dense(links, psi, mass, M, a, b, c, DW_PHASES)
        assert np.allclose(got, ref, atol=8e-12, rtol=8e-12)
        gotd = orc.domainwall(links, left, mass, M, a, b, c, DW_PHASES, dagger=True)
        refd = rd.domainwall_dense(links, left, mass, M, a, b, c, DW_PHASES, adjoint=True)
        assert np.allclose(gotd, refd, atol=8e-12, rtol=8e-12)
        # <left, D psi> = <D^+ left, psi>
        assert np.isclose(np.vdot(left, got), np.vdot(gotd, psi), atol=2e-10, rtol=2e-11)
