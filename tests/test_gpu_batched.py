"""Batched multi-RHS / multi-lattice D'D CG (lmb_cg_ddagd_batched): every
right-hand side reaches its FP64 true residual, confirmed by the oracle, and
matches a single-system solve -- with FP32 or int16 iterated fields, and with
each kernel family (0: links in registers for groups of 1-4 right-hand sides;
1: links staged in shared memory for groups of 4-16; 2: int16 only, the
single-lattice x-adjacent pair stencil on (tile, member) tasks;
LMB_BATCH_FAMILY restricts the autotuner to one)."""
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


@pytest.mark.parametrize("family", [-1, 0, 1, 2])
@pytest.mark.parametrize("precision", ["single", "half"])
def test_batched_uneven_lattices(lmb, orc, monkeypatch, precision, family):
    monkeypatch.setenv("LMB_BATCH_FAMILY", str(family))   # read when the context is made
    shapes = [((4, 4, 4, 4), 3), ((6, 6, 6, 6), 2), ((8, 8, 8, 8), 1), ((4, 6, 8, 4), 17)]
    systems, host = [], []
    for li, (L, n) in enumerate(shapes):
        U = orc.random_su3_links(L, 0.3, 10 + li)
        Ud = [lmb.LatticeMatrix.from_array(u, nw=1) for u in U]
        D = lmb.WilsonDiracOperator4D(Ud, 0.12)
        pairs, bs = [], []
        for r in range(n):
            b = orc.gaussian_field(L, 3, 4, 100 * li + r)
            bd = lmb.LatticeMatrix.from_array(b, nw=1, phases=PHASES)
            pairs.append((bd.similar(), bd))
            bs.append(b)
        systems.append((D, pairs))
        host.append((U, L, bs))
    if family == 2 and precision == "single":          # the pair family is int16 only
        with pytest.raises(lmb.LMBError, match="family"):
            lmb.cg_batched_(systems, rtol=1e-10, precision=precision)
        return
    results, tuning = lmb.cg_batched_(systems, rtol=1e-10, precision=precision)
    assert tuning["rhs_block"] in (1, 2, 4, 8, 16) and tuning["threads"] in (64, 128, 256)
    if family >= 0:
        assert tuning["kernel_family"] == family, tuning
    k = 0
    for (D, pairs), (U, L, bs) in zip(systems, host):
        op = orc.Operator(orc.OP_WILSON, U, L, kappa=0.12)
        for (x, _), b in zip(pairs, bs):
            res = results[k]
            k += 1
            assert res.converged, (precision, family, res)
            xs = x.gather_matrix()
            assert np.linalg.norm(b - op.ddagd(xs)) / np.linalg.norm(b) <= 1.05e-10
            x_ref, _ = orc.cg_ddagd(op, b, rtol=1e-12)
            assert rd.rel_err(xs, x_ref) <= 1e-6


@pytest.mark.parametrize("precision", ["single", "half"])
def test_batched_matches_single_and_second_call(lmb, orc, precision):
    L = (8, 8, 8, 8)
    U = orc.random_su3_links(L, 0.3, 3)
    Ud = [lmb.LatticeMatrix.from_array(u, nw=1) for u in U]
    D = lmb.WilsonDiracOperator4D(Ud, 0.125)
    bs = [lmb.LatticeMatrix.from_array(orc.gaussian_field(L, 3, 4, s), nw=1,
                                       phases=PHASES) for s in (5, 6, 7, 8)]
    pairs = [(b.similar(), b) for b in bs]
    r1, t1 = lmb.cg_batched_([(D, pairs)], rtol=1e-10, precision=precision)
    r2, t2 = lmb.cg_batched_([(D, pairs)], rtol=1e-10, precision=precision)     # cached tuning
    assert (t1["rhs_block"], t1["threads"]) == (t2["rhs_block"], t2["threads"])
    assert all(r.converged for r in r1 + r2)
    x1 = bs[0].similar()
    single = lmb.cg_(x1, lmb.DdagDOp(D, bs[0].similar()), bs[0], rtol=1e-10,
                     precision=precision)
    assert single.converged
    assert rd.rel_err(pairs[0][0].gather_matrix(), x1.gather_matrix()) <= 1e-6


def test_batched_rejects_bad_input(lmb, orc):
    L = (4, 4, 4, 4)
    U = rd.staggered_test_links(L)          # not SU(3)
    Ud = [lmb.LatticeMatrix.from_array(u, nw=1) for u in U]
    D = lmb.WilsonDiracOperator4D(Ud, 0.1)
    b = lmb.LatticeMatrix.from_array(orc.gaussian_field(L, 3, 4, 1), nw=1, phases=PHASES)
    with pytest.raises(lmb.LMBError, match="SU\\(3\\)"):
        lmb.cg_batched_([(D, [(b.similar(), b)])])
    with pytest.raises(lmb.ArgumentError):
        lmb.cg_batched_([(D, [])])
    with pytest.raises(lmb.ArgumentError):
        lmb.cg_batched_([(D, [(b.similar(), b)])], precision="double")
