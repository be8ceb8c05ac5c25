"""GPU parity of the staggered and HISQ stencils and their D'D CG against the
oracle (FP64 <= 1e-13 relative norm; FP32 storage <= 5e-6; int16 <= 2e-3)."""
import numpy as np
import pytest

import refdata as rd

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


def _dev(lmb, arrs, nw, phases=None):
    return [lmb.LatticeMatrix.from_array(a, nw=nw, phases=phases) for a in arrs]


@pytest.mark.parametrize("L,nw,phases", [((4, 2, 2, 2), 1, PHASES),
                                         ((3, 4, 2, 6), 0, TWISTED),
                                         ((8, 8, 8, 8), 2, TWISTED)])
@pytest.mark.parametrize("links", ["reference", "su3"])
def test_staggered_fp64(lmb, orc, L, nw, phases, links):
    U = rd.staggered_test_links(L) if links == "reference" else \
        orc.random_su3_links(L, 0.3, 3)
    psi = orc.gaussian_field(L, 3, 1, 4)
    Ud = _dev(lmb, U, nw)
    (pd,) = _dev(lmb, [psi], nw, phases)
    D = lmb.StaggeredDiracOperator4D(Ud, 0.17)
    out = pd.similar()
    for dag in (False, True):
        lmb.mul_(out, lmb.adjoint(D) if dag else D, pd)
        ref = orc.staggered(U, psi, 0.17, phases, dagger=dag)
        assert rd.rel_err(out.gather_matrix(), ref) <= 1e-13


def test_staggered_bridgepp_fingerprint_on_gpu(lmb, orc):
    import json, os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                    "reference_fingerprints.json")))["bridgepp_staggered"]
    L = tuple(g["lattice"])
    Ud = _dev(lmb, rd.staggered_test_links(L), 1)
    (pd,) = _dev(lmb, [rd.staggered_test_fermion(L)], 1, PHASES)
    D = lmb.StaggeredDiracOperator4D(Ud, g["mass"])
    out = pd.similar()
    for mode, op in (("D", D), ("Ddag", lmb.adjoint(D))):
        lmb.mul_(out, op, pd)
        fp = rd.fingerprint(out.gather_matrix())
        assert np.allclose(fp, g[mode], atol=g["atol"], rtol=g["rtol"]), (mode, fp)


@pytest.mark.parametrize("L,nw,phases", [((4, 4, 4, 4), 3, TWISTED),
                                         ((4, 4, 4, 6), 0, PHASES),
                                         ((2, 3, 4, 5), 0, TWISTED),
                                         ((8, 6, 4, 12), 3, PHASES)])
def test_hisq_fp64(lmb, orc, L, nw, phases):
    fat, lng = rd.hisq_test_links(L)
    psi = orc.gaussian_field(L, 3, 1, 5)
    X, Ln = _dev(lmb, fat, nw), _dev(lmb, lng, nw)
    (pd,) = _dev(lmb, [psi], nw, phases)
    D = lmb.HISQDiracOperator4D(lmb.HISQLinks4D(X, Ln), 0.17, -0.083)
    out = pd.similar()
    for dag in (False, True):
        lmb.mul_(out, lmb.adjoint(D) if dag else D, pd)
        ref = orc.hisq(fat, lng, psi, 0.17, -0.083, phases, dagger=dag)
        assert rd.rel_err(out.gather_matrix(), ref) <= 1e-13


@pytest.mark.parametrize("precision,tol", [("single", 5e-6), ("half", 2e-3)])
def test_hisq_low_precision(lmb, orc, precision, tol):
    L = (8, 8, 4, 8)
    U = orc.random_su3_links(L, 0.25, 7)
    fat, lng = orc.hisq_links_from_thin(U, -0.083)
    psi = orc.gaussian_field(L, 3, 1, 8)
    D = lmb.HISQDiracOperator4D(lmb.HISQLinks4D(_dev(lmb, fat, 3), _dev(lmb, lng, 3)),
                                0.05, -0.083)
    (pd,) = _dev(lmb, [psi], 3, TWISTED)
    out = pd.similar()
    lmb.mul_(out, D, pd, precision=precision)
    ref = orc.hisq(fat, lng, psi, 0.05, -0.083, TWISTED)
    assert rd.rel_err(out.gather_matrix(), ref) <= tol


@pytest.mark.parametrize("precision,tol", [("single", 5e-6), ("half", 2e-3)])
@pytest.mark.parametrize("L,adj", [((8, 8, 4, 8), "1"), ((8, 8, 4, 8), "0"), ((6, 4, 4, 3), "1"),
                                   ((5, 4, 4, 6), "1"), ((4, 6, 8, 4), "1")])
def test_fp32_two_site_paths(lmb, orc, L, adj, monkeypatch, precision, tol):
    """FP32- and int16-storage HISQ and staggered (18-real links) with
    antiperiodic t: an even x extent runs two x-adjacent sites per thread
    (packed FP32, 256-bit loads) unless LMB_ADJ_SITES=0; an odd x extent runs
    one site per thread."""
    monkeypatch.setenv("LMB_ADJ_SITES", adj)
    U = orc.random_su3_links(L, 0.25, 7)
    fat, lng = orc.hisq_links_from_thin(U, -0.083)
    psi = orc.gaussian_field(L, 3, 1, 8)
    D = lmb.HISQDiracOperator4D(lmb.HISQLinks4D(_dev(lmb, fat, 3), _dev(lmb, lng, 3)),
                                0.05, -0.083)
    (pd,) = _dev(lmb, [psi], 3, PHASES)
    out = pd.similar()
    for dag in (False, True):
        lmb.mul_(out, lmb.adjoint(D) if dag else D, pd, precision=precision)
        ref = orc.hisq(fat, lng, psi, 0.05, -0.083, PHASES, dagger=dag)
        assert rd.rel_err(out.gather_matrix(), ref) <= tol
    # plain staggered on non-unitary links (no reconstruction: 18 reals)
    Un = rd.staggered_test_links(L, 3)
    S = lmb.StaggeredDiracOperator4D(_dev(lmb, Un, 1), 0.07)
    (p1,) = _dev(lmb, [psi], 1, PHASES)
    o1 = p1.similar()
    for dag in (False, True):
        lmb.mul_(o1, lmb.adjoint(S) if dag else S, p1, precision=precision)
        ref = orc.staggered(Un, psi, 0.07, PHASES, dagger=dag)
        assert rd.rel_err(o1.gather_matrix(), ref) <= tol


@pytest.mark.parametrize("precision", ["double", "single", "half"])
def test_hisq_cg(lmb, orc, precision):
    L = (8, 8, 8, 8)
    U = orc.random_su3_links(L, 0.25, 1)
    fat, lng = orc.hisq_links_from_thin(U, 0.0)
    b = orc.gaussian_field(L, 3, 1, 2)
    D = lmb.HISQDiracOperator4D(lmb.HISQLinks4D(_dev(lmb, fat, 3), _dev(lmb, lng, 3)),
                                0.05, 0.0)
    (bd,) = _dev(lmb, [b], 3, PHASES)
    x = bd.similar()
    res = lmb.cg_(x, lmb.DdagDOp(D, bd.similar()), bd, rtol=1e-10,
                  precision=precision)
    assert res.converged, res
    op = orc.Operator(orc.OP_HISQ, list(fat) + list(lng), L, mass=0.05,
                      naik_epsilon=0.0)
    xs = x.gather_matrix()
    assert np.linalg.norm(b - op.ddagd(xs)) / np.linalg.norm(b) <= 1.05e-10
    if precision == "double":
        _, ref = orc.cg_ddagd(op, b, rtol=1e-10)
        assert abs(res.iterations - ref["iterations"]) <= 1


def test_staggered_cg_mixed(lmb, orc):
    L = (8, 8, 8, 16)
    U = orc.random_su3_links(L, 0.3, 1)
    b = orc.gaussian_field(L, 3, 1, 2)
    D = lmb.StaggeredDiracOperator4D(_dev(lmb, U, 1), 0.05)
    (bd,) = _dev(lmb, [b], 1, PHASES)
    x = bd.similar()
    res = lmb.cg_(x, lmb.DdagDOp(D, bd.similar()), bd, rtol=1e-10,
                  precision="half")
    assert res.converged and res.reliable_updates >= 1
    op = orc.Operator(orc.OP_STAGGERED, U, L, mass=0.05)
    xs = x.gather_matrix()
    assert np.linalg.norm(b - op.ddagd(xs)) / np.linalg.norm(b) <= 1.05e-10


def test_staggered_validation(lmb, orc):
    L = (4, 4, 4, 4)
    Ud = _dev(lmb, orc.random_su3_links(L, 0.3, 1), 1)
    (pd,) = _dev(lmb, [orc.gaussian_field(L, 3, 1, 2)], 1, PHASES)
    D = lmb.StaggeredDiracOperator4D(Ud, 0.1)
    with pytest.raises(lmb.ArgumentError, match="distinct"):
        lmb.mul_(pd, D, pd)
    bad = lmb.LatticeMatrix(3, 1, 4, L, nw=1, phases=(1, 1, 1, 2))
    with pytest.raises(lmb.ArgumentError, match="unit magnitude"):
        lmb.mul_(bad.similar(), D, bad)
    with pytest.raises(lmb.ArgumentError, match="finite"):
        lmb.StaggeredDiracOperator4D(Ud, float("nan"))


def test_operator_timing_on_resident_fields(lmb, orc):
    """lmb_operator_timing: device time per application of the bound
    operator on the library's internal fields (the bench's Dslash rate)."""
    L = (8, 8, 8, 8)
    U = lmb.random_su3_links(L, 0.25, 1, nw=3)
    links = lmb.hisq_links_from_thin(U, -0.083)
    D = lmb.HISQDiracOperator4D(links, 0.0, -0.083)
    psi = lmb.gaussian_fermion(L, 3, 1, 2, nw=3, phases=PHASES)
    for prec in ("double", "single", "half"):
        ms = lmb.operator_timing(D, psi, 5, precision=prec)
        assert 0.0 < ms < 100.0, (prec, ms)
    assert lmb.operator_timing(D, psi, 3, dagger=True) > 0.0
    with pytest.raises(lmb.ArgumentError):
        lmb.operator_timing(D, psi, 0)
