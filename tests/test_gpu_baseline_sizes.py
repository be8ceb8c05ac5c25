"""GPU parity at the benchmark configurations' own lattice sizes.

The other parity files test every kernel path on small lattices; these tests
repeat the headline checks at full size, where an indexing bug that only
large extents reach (32-bit offsets, the two-site lane pairing, the number of
blocks of a grid reduction, the int16 scales of a large field) would show:

* Wilson-clover D and D^+ on 32^3x64 (kappa 0.1355, cSW 1.0, links
  exp(0.2 i H) seed 1, Gaussian source seed 2) against the oracle: FP64 to
  1e-13 relative norm (the reference's operator bar,
  test/wilson_clover.jl:177-188), FP32 storage 5e-6, int16 storage 2e-3;
* HISQ D and D^+ after the full smearing chain (links exp(0.25 i H),
  m 0.01) on 48^3x96 when the host has the memory for the oracle's copy of
  the fat and Naik links (about 20 GB), else on 32^3x64;
* the batched solve of the uneven lattice set 8^4 x4, 12^4 x4, 16^4 x2,
  24^4 x1 plus two right-hand sides on 32^4, against the oracle's solutions;
* the HISQ fermion force on 24^4 (m 0.02, links exp(0.2 i H)) against
  central finite differences of the oracle's action along two random link
  directions.
"""
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


# ---------------------------------------------------------------------------
# Wilson-clover, 32^3 x 64
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def clover32(lmb, orc):
    L = (32, 32, 32, 64)
    U = orc.random_su3_links(L, 0.2, 1)
    psi = orc.gaussian_field(L, 3, 4, 2)
    Ud = [lmb.LatticeMatrix.from_array(u, nw=1) for u in U]
    pd = lmb.LatticeMatrix.from_array(psi, nw=1, phases=PHASES)
    D = lmb.WilsonDiracCloverOperator4D(Ud, 0.1355, 1.0)
    refs = {dag: orc.wilson_clover(U, psi, 0.1355, 1.0, PHASES, dagger=dag)
            for dag in (False, True)}
    del U, psi
    return D, pd, refs


@pytest.mark.parametrize("precision,tol", [("double", 1e-13), ("single", 5e-6),
                                           ("half", 2e-3)])
def test_wilson_clover_32x64_matches_oracle(lmb, clover32, precision, tol):
    D, pd, refs = clover32
    out = pd.similar()
    for dag in (False, True):
        lmb.mul_(out, lmb.adjoint(D) if dag else D, pd, precision=precision)
        err = rd.rel_err(out.gather_matrix(), refs[dag])
        assert err <= tol, (precision, dag, err)


# ---------------------------------------------------------------------------
# HISQ after the full smearing chain
# ---------------------------------------------------------------------------
def _hisq_lattice():
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:          # pragma: no cover - psutil is in the image
        avail = 0
    return (48, 48, 48, 96) if avail >= 48 * 2**30 else (32, 32, 32, 64)


def test_hisq_full_size_matches_oracle(lmb, orc):
    L = _hisq_lattice()
    mass, eps = 0.01, 0.0
    U = lmb.random_su3_links(L, 0.25, 1, nw=0)
    links = lmb.hisq_links_from_thin(U, eps)
    del U
    psi = orc.gaussian_field(L, 3, 1, 2)
    pd = lmb.LatticeMatrix.from_array(psi, nw=0, phases=PHASES)
    D = lmb.HISQDiracOperator4D(links, mass, eps)
    out = pd.similar()
    X = [x.gather_matrix() for x in links.fat_links]
    Ln = [x.gather_matrix() for x in links.long_links]
    for dag in (False, True):
        ref = orc.hisq(X, Ln, psi, mass, eps, PHASES, dagger=dag)
        for precision, tol in (("double", 1e-13), ("single", 5e-6), ("half", 2e-3)):
            lmb.mul_(out, lmb.adjoint(D) if dag else D, pd, precision=precision)
            err = rd.rel_err(out.gather_matrix(), ref)
            assert err <= tol, (L, precision, dag, err)


# ---------------------------------------------------------------------------
# batched solve of the uneven lattice set
# ---------------------------------------------------------------------------
def test_batched_benchmark_lattice_set(lmb, orc):
    shapes = [((8, 8, 8, 8), 4), ((12, 12, 12, 12), 4), ((16, 16, 16, 16), 2),
              ((24, 24, 24, 24), 1), ((32, 32, 32, 32), 2)]
    kappa = 0.12
    systems, host = [], []
    for i, (L, n) in enumerate(shapes):
        U = orc.random_su3_links(L, 0.2, 10 + i)
        Ud = [lmb.LatticeMatrix.from_array(u, nw=1) for u in U]
        D = lmb.WilsonDiracOperator4D(Ud, kappa)
        pairs, bs = [], []
        for r in range(n):
            b = orc.gaussian_field(L, 3, 4, 100 * i + r)
            bd = lmb.LatticeMatrix.from_array(b, nw=1, phases=PHASES)
            pairs.append((bd.similar(), bd))
            bs.append(b)
        systems.append((D, pairs))
        host.append((U, L, bs))
    results, _ = lmb.cg_batched_(systems, rtol=1e-10)
    k = 0
    for (D, pairs), (U, L, bs) in zip(systems, host):
        op = orc.Operator(orc.OP_WILSON, U, L, kappa=kappa)
        for j, ((x, _), b) in enumerate(zip(pairs, bs)):
            res = results[k]
            k += 1
            assert res.converged, (L, j, res)
            xs = x.gather_matrix()
            true_rel = np.linalg.norm(b - op.ddagd(xs)) / np.linalg.norm(b)
            assert true_rel <= 1.05e-10, (L, j, true_rel)
            if j == 0:              # one oracle solve per lattice
                x_ref, _ = orc.cg_ddagd(op, b, rtol=1e-12)
                assert rd.rel_err(xs, x_ref) <= 1e-6, L


# ---------------------------------------------------------------------------
# HISQ fermion force, 24^4
# ---------------------------------------------------------------------------
def test_hisq_force_24_matches_oracle_finite_differences(lmb, orc):
    """dS/dU of S = phi^+ (D^+D)^-1 phi against central differences of the
    oracle's action.  S(U') - S(U) = phi^+ d with A' d = phi - A' x0,
    x0 = A^-1 phi, so the difference of two nearly equal actions is formed
    without cancellation."""
    L = (24, 24, 24, 24)
    mass, eps = 0.02, 0.0
    U = orc.random_su3_links(L, 0.2, 1)
    phi = orc.gaussian_field(L, 3, 1, 2)
    Ud = [lmb.LatticeMatrix.from_array(u, nw=3) for u in U]
    phid = lmb.LatticeMatrix.from_array(phi, nw=3, phases=PHASES)
    cache = lmb.HISQDiracCache4D(Ud, mass, eps)
    dU = [u.similar() for u in Ud]
    res = lmb.hisq_fermion_force_(dU, cache, phid, rtol=1e-12)
    assert res.converged
    G = [d.gather_matrix() for d in dU]
    del dU, Ud

    def operator(Uh):
        X, Ln = orc.hisq_links_from_thin(Uh, eps)
        return orc.Operator(orc.OP_HISQ, list(X) + list(Ln), L, mass=mass,
                            naik_epsilon=eps)

    x0, r0 = orc.cg_ddagd(operator(U), phi, rtol=1e-12, maxiter=20000)
    assert r0["converged"]

    def delta_action(Uh):
        op = operator(Uh)
        rhs = phi - op.ddagd(x0)
        d, r = orc.cg_ddagd(op, rhs, rtol=1e-10, maxiter=20000)
        assert r["converged"]
        return np.vdot(phi, d).real

    h = 1e-5
    rng = np.random.default_rng(64)
    for _ in range(2):
        V = [np.asfortranarray(rng.normal(size=(3, 3) + L) + 1j * rng.normal(size=(3, 3) + L))
             for _ in range(4)]
        fd = (delta_action([np.asfortranarray(u + h * v) for u, v in zip(U, V)]) -
              delta_action([np.asfortranarray(u - h * v) for u, v in zip(U, V)])) / (2 * h)
        an = sum(np.vdot(g, v).real for g, v in zip(G, V))
        assert abs(an - fd) <= 1e-7 * abs(fd), (an, fd)
