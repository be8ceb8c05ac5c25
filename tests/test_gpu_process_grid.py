"""The sharded path (lmb_set_process_grid) on one GPU: a one-rank NCCL
communicator whose split dimensions exchange their faces with the rank itself.
Every piece of the multi-rank path runs -- face packing with the boundary
phases of the global edge, NCCL send / receive into ghost buffers on the
communication stream, the interior kernel, the ghost-aware boundary kernel,
link ghosts from the caller's halo, the all-reduce of every CG reduction --
and the result must equal the whole-lattice operator and the oracle
(FP64 <= 1e-13, FP32 storage 5e-6, int16 storage 2e-3).  A block split
along t only runs its interior slab on the single-lattice kernels (int16
x-adjacent pairs, persistent reductions); other splits of an int16 block
with an even x extent run the pairs with both sites interior on the pair
stencil, and the rest on the one-site interior kernel."""
import ctypes

import numpy as np
import pytest

import refdata as rd

pytestmark = pytest.mark.gpu
TWISTED = tuple(np.exp(1j * a) for a in (0.13, -0.21, 0.34, np.pi - 0.17))
PHASES = (1, 1, 1, -1)
PREC = {"double": 0, "single": 1, "half": 2}


@pytest.fixture(scope="module")
def lmb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lmb200
    lmb200.load()
    return lmb200


def _grid_ctx(lmb, L, nw, phases, split):
    from lmb200._lib import Context, nccl_unique_id
    ctx = Context(0)
    ctx.set_geometry(L, nw, phases, (0, 0, 0, 0), 0)
    ctx.set_process_grid(nccl_unique_id(), 1, 0, (1, 1, 1, 1), (0, 0, 0, 0), split,
                         (0, 0, 0, 0), (0, 0, 0, 0))
    ctx.set_geometry(L, nw, phases, (0, 0, 0, 0), 0)
    return ctx


def _links(lmb, arrs, nw):
    Ud = [lmb.LatticeMatrix.from_array(u, nw=nw) for u in arrs]
    for u in Ud:
        lmb.set_halo_(u)          # the caller's exchange fills the link halo
    return Ud


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


# (1, 0, 0, 0): x alone, whose int16 boundary is the two face pairs of every
# row on the pair stencil (here every site: x extent 4)
@pytest.mark.parametrize("split", [(1, 0, 0, 1), (1, 1, 1, 1), (0, 1, 0, 0), (0, 0, 0, 1), (1, 0, 0, 0)])
@pytest.mark.parametrize("clover", [False, True])
def test_wilson_on_a_split_block_matches_oracle(lmb, orc, split, clover):
    L, kappa, csw = (4, 6, 4, 8), 0.1355, 1.0
    U = orc.random_su3_links(L, 0.3, 1)
    psi = orc.gaussian_field(L, 3, 4, 2)
    Ud = _links(lmb, U, 1)
    pd = lmb.LatticeMatrix.from_array(psi, nw=1, phases=TWISTED)
    ctx = _grid_ctx(lmb, L, 1, TWISTED, split)
    st = _stream()
    ctx.upload_links(0, [u.data_ptr() for u in Ud], [u.halo_epoch.core for u in Ud], st)
    out = pd.similar()
    for dag in (0, 1):
        ref = orc.wilson_clover(U, psi, kappa, csw, TWISTED, dagger=bool(dag)) if clover \
            else orc.wilson(U, psi, kappa, TWISTED, dagger=bool(dag))
        for prec, tol in (("double", 1e-13), ("single", 5e-6), ("half", 2e-3)):
            if clover:
                rc = ctx.lib.lmb_wilson_clover_apply(ctx.handle, out.data_ptr(), pd.data_ptr(), kappa, csw, dag,
                                                     PREC[prec], st)
            else:
                rc = ctx.lib.lmb_wilson_apply(ctx.handle, out.data_ptr(), pd.data_ptr(), kappa, dag, PREC[prec], st)
            ctx.check(rc)
            err = rd.rel_err(out.gather_matrix(), ref)
            assert err <= tol, (split, clover, dag, prec, err)


def _cg(lmb, ctx, op, x, b, prec, **kw):
    from lmb200._lib import CGParams, CGResultC
    prm = CGParams()
    prm.op = op
    prm.kappa = kw.get("kappa", 0.0)
    prm.csw = kw.get("csw", 0.0)
    prm.mass = kw.get("mass", 0.0)
    prm.naik_epsilon = kw.get("eps", 0.0)
    prm.rtol, prm.atol, prm.maxiter = 1e-10, 0.0, 5000
    prm.precision = PREC[prec]
    prm.delta = 0.1
    res = CGResultC()
    ctx.check(ctx.lib.lmb_cg_ddagd(ctx.handle, ctypes.byref(prm), x.data_ptr(), b.data_ptr(),
                                   ctypes.byref(res), _stream()))
    return res


# (8, 4, 4, 6) split along x: the int16 interior runs on x-adjacent pairs
# with both sites interior (x = 2..5), the x partners of the face sites go to
# the boundary kernel
@pytest.mark.parametrize("split,L", [((1, 0, 1, 1), (4, 4, 6, 8)), ((0, 0, 0, 1), (4, 4, 6, 8)),
                                     ((1, 0, 0, 1), (8, 4, 4, 6)), ((1, 0, 0, 0), (8, 4, 4, 6))])
@pytest.mark.parametrize("prec", ["double", "single", "half"])
def test_clover_cg_on_a_split_block(lmb, orc, prec, split, L):
    kappa, csw = 0.1355, 1.0
    U = orc.random_su3_links(L, 0.2, 3)
    b = orc.gaussian_field(L, 3, 4, 4)
    Ud = _links(lmb, U, 1)
    bd = lmb.LatticeMatrix.from_array(b, nw=1, phases=PHASES)
    ctx = _grid_ctx(lmb, L, 1, PHASES, split)
    st = _stream()
    ctx.upload_links(0, [u.data_ptr() for u in Ud], [u.halo_epoch.core for u in Ud], st)
    x = bd.similar()
    res = _cg(lmb, ctx, 1, x, bd, prec, kappa=kappa, csw=csw)
    assert res.converged and res.reason == 0, (prec, split, res.iterations)
    op = orc.Operator(orc.OP_CLOVER, U, L, kappa=kappa, csw=csw, F=orc.clover_field_strength(U))
    xs = x.gather_matrix()
    true_rel = np.linalg.norm(b - op.ddagd(xs)) / np.linalg.norm(b)
    assert true_rel <= 1.05e-10, (prec, true_rel)
    if prec == "double":
        _, ref = orc.cg_ddagd(op, b, rtol=1e-10)
        assert abs(res.iterations - ref["iterations"]) <= 1, (res.iterations, ref["iterations"])


@pytest.mark.parametrize("split,L,phases", [((1, 1, 1, 1), (6, 4, 6, 6), TWISTED),
                                            ((0, 0, 1, 1), (6, 4, 6, 6), TWISTED),
                                            ((0, 0, 0, 1), (4, 4, 4, 8), TWISTED),
                                            ((0, 0, 0, 1), (4, 4, 4, 8), PHASES),
                                            # t phase only, x extent 10: the interior on x-adjacent
                                            # pairs (x = 4, 5 with both sites interior at depth 3)
                                            ((1, 0, 0, 0), (10, 4, 4, 6), PHASES),
                                            ((1, 0, 1, 1), (10, 4, 8, 8), PHASES)])
def test_hisq_on_a_split_block_matches_oracle(lmb, orc, split, L, phases):
    mass, eps = 0.05, -0.083
    U = orc.random_su3_links(L, 0.25, 5)
    X, Ln = orc.hisq_links_from_thin(U, eps)
    psi = orc.gaussian_field(L, 3, 1, 6)
    Xd, Ld = _links(lmb, X, 3), _links(lmb, Ln, 3)
    pd = lmb.LatticeMatrix.from_array(psi, nw=3, phases=phases)
    ctx = _grid_ctx(lmb, L, 3, phases, split)
    st = _stream()
    ctx.upload_links(1, [u.data_ptr() for u in Xd], [u.halo_epoch.core for u in Xd], st)
    ctx.upload_links(2, [u.data_ptr() for u in Ld], [u.halo_epoch.core for u in Ld], st)
    out = pd.similar()
    for dag in (0, 1):
        ref = orc.hisq(X, Ln, psi, mass, eps, phases, dagger=bool(dag))
        for prec, tol in (("double", 1e-13), ("single", 5e-6), ("half", 2e-3)):
            ctx.check(ctx.lib.lmb_hisq_apply(ctx.handle, out.data_ptr(), pd.data_ptr(), mass, eps, dag,
                                             PREC[prec], st))
            err = rd.rel_err(out.gather_matrix(), ref)
            assert err <= tol, (split, dag, prec, err)
    # and the CG on the block, FP64 and FP32 / int16 inner iterations
    bd = lmb.LatticeMatrix.from_array(psi, nw=3, phases=phases)
    op = orc.Operator(orc.OP_HISQ, list(X) + list(Ln), L, phases=phases, mass=mass, naik_epsilon=eps)
    for prec in ("double", "single", "half"):
        x = bd.similar()
        res = _cg(lmb, ctx, 3, x, bd, prec, mass=mass, eps=eps)
        assert res.converged, (prec, res.iterations)
        xs = x.gather_matrix()
        true_rel = np.linalg.norm(psi - op.ddagd(xs)) / np.linalg.norm(psi)
        assert true_rel <= 1.05e-10, (prec, true_rel)


@pytest.mark.parametrize("split", [(0, 1, 1, 0), (0, 0, 0, 1)])
def test_staggered_on_a_split_block_matches_oracle(lmb, orc, split):
    L, mass = (4, 6, 4, 4), 0.07
    U = orc.random_su3_links(L, 0.3, 7)
    psi = orc.gaussian_field(L, 3, 1, 8)
    Ud = _links(lmb, U, 1)
    pd = lmb.LatticeMatrix.from_array(psi, nw=1, phases=TWISTED)
    ctx = _grid_ctx(lmb, L, 1, TWISTED, split)
    st = _stream()
    ctx.upload_links(0, [u.data_ptr() for u in Ud], [u.halo_epoch.core for u in Ud], st)
    out = pd.similar()
    for dag in (0, 1):
        ref = orc.staggered(U, psi, mass, TWISTED, dagger=bool(dag))
        for prec, tol in (("double", 1e-13), ("single", 5e-6), ("half", 2e-3)):
            ctx.check(ctx.lib.lmb_staggered_apply(ctx.handle, out.data_ptr(), pd.data_ptr(), mass, dag,
                                                  PREC[prec], st))
            err = rd.rel_err(out.gather_matrix(), ref)
            assert err <= tol, (dag, prec, err)


def test_process_grid_arguments(lmb):
    from lmb200._lib import Context, nccl_unique_id
    ctx = Context(0)
    ctx.set_geometry((4, 4, 4, 4), 1, PHASES, (0, 0, 0, 0), 0)
    nid = nccl_unique_id()
    with pytest.raises(lmb.ArgumentError):   # 2 ranks along x must be split
        ctx.set_process_grid(nid, 2, 0, (2, 1, 1, 1), (0, 0, 0, 0), (0, 0, 0, 0), (1, 0, 0, 0), (1, 0, 0, 0))
    with pytest.raises(lmb.ArgumentError):   # grid and communicator sizes differ
        ctx.set_process_grid(nid, 1, 0, (2, 1, 1, 1), (0, 0, 0, 0), (1, 0, 0, 0), (0, 0, 0, 0), (0, 0, 0, 0))
    ctx.set_process_grid(None, 1, 0, (1, 1, 1, 1), (0, 0, 0, 0), (0, 0, 0, 0), (0, 0, 0, 0), (0, 0, 0, 0))


@pytest.mark.parametrize("split,L", [((0, 0, 0, 1), (4, 4, 6, 8)), ((1, 1, 0, 1), (4, 4, 6, 8)),
                                     ((1, 0, 0, 0), (8, 4, 6, 4)), ((1, 1, 0, 1), (8, 4, 6, 4)),
                                     ((0, 1, 1, 0), (8, 4, 6, 4))])
def test_split_block_matches_the_single_lattice_kernels(lmb, orc, split, L):
    """The interior / boundary split against the unsplit operator on the same
    links and field: FP64 to rounding (the same arithmetic in another order
    at the boundary sites), int16 storage within a tenth of a per-mille
    (its quantisation step is 2^-15 of a site's largest entry).  With an
    x extent of 8 the int16 interior of any split but t alone runs on
    x-adjacent pairs, the x split's face partners on the boundary kernel."""
    from lmb200._lib import Context
    kappa, csw = 0.1355, 1.0
    U = orc.random_su3_links(L, 0.25, 11)
    psi = orc.gaussian_field(L, 3, 4, 12)
    Ud = _links(lmb, U, 1)
    pd = lmb.LatticeMatrix.from_array(psi, nw=1, phases=PHASES)
    st = _stream()
    whole = Context(0)
    whole.set_geometry(L, 1, PHASES, (0, 0, 0, 0), 0)
    whole.upload_links(0, [u.data_ptr() for u in Ud], [u.halo_epoch.core for u in Ud], st)
    grid = _grid_ctx(lmb, L, 1, PHASES, split)
    grid.upload_links(0, [u.data_ptr() for u in Ud], [u.halo_epoch.core for u in Ud], st)
    for dag in (0, 1):
        for prec, tol in (("double", 1e-14), ("half", 1e-4)):
            a, b = pd.similar(), pd.similar()
            for ctx, out in ((whole, a), (grid, b)):
                ctx.check(ctx.lib.lmb_wilson_clover_apply(ctx.handle, out.data_ptr(), pd.data_ptr(), kappa, csw,
                                                          dag, PREC[prec], st))
            err = rd.rel_err(b.gather_matrix(), a.gather_matrix())
            assert err <= tol, (split, dag, prec, err)
