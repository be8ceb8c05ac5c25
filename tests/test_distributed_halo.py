"""Process grids on CPU (gloo, 2 and 4 ranks): the halo exchange of fields
split over PEs (exchange_dim!, LatticeMatrices_core.jl:742-921), the gather
of the global core, the all-reduce of dot's partial sums, and the staggered
stencils refusing a split field.  Every rank's padded storage after set_halo! must
equal the periodic image of the global array with the boundary phase per
global wrap -- the single-rank ghost rule applied to the whole lattice."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TWISTED = tuple(complex(np.exp(1j * a)) for a in (0.13, -0.21, 0.34, np.pi - 0.17))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _expected_local(G, coords, PN, nw, phases):
    """Local padded block: global coordinate g = c PN + i - nw of every
    padded index i, read at g mod L, times phase^floor(g / L) per dimension."""
    idx, fac = [], []
    for d, (c, n, L) in enumerate(zip(coords, PN, G.shape[2:])):
        g = c * n + np.arange(n + 2 * nw) - nw
        idx.append(np.mod(g, L))
        fac.append(np.asarray(phases[d], dtype=complex) ** np.floor_divide(g, L))
    out = G[np.ix_(range(G.shape[0]), range(G.shape[1]), *idx)].astype(complex)
    for d, f in enumerate(fac):
        shape = [1] * out.ndim
        shape[d + 2] = f.size
        out = out * f.reshape(shape)
    return out


def _rank_main(rank, ws, port, dim, PEs, gsize, nw, phases, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, os.path.join(ROOT, "latticematrices.jl_b200"))
    from datetime import timedelta
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    try:
        import lmb200 as lmb
        rng = np.random.default_rng(5)
        G = np.asfortranarray(rng.normal(size=(3, 4) + gsize) + 1j * rng.normal(size=(3, 4) + gsize))
        ls = lmb.LatticeMatrix.from_array(G, dim, PEs, nw=nw, phases=phases, device="cpu")
        assert ls.PN == tuple(g // p for g, p in zip(gsize, PEs))
        assert lmb.halo_is_dirty(ls)
        lmb.set_halo_(ls)
        clean = not lmb.halo_is_dirty(ls)
        got = ls.A.numpy().T
        err = float(np.max(np.abs(got - _expected_local(G, ls.coords, ls.PN, nw, phases))))
        gathered = bool(np.array_equal(ls.gather_matrix(), G))
        from lmb200.distributed import allreduce_complex
        red = allreduce_complex(complex(rank + 1, -rank), "cpu")
        refused = False
        if dim == 4:
            U = [lmb.LatticeMatrix.from_array(np.asfortranarray(np.zeros((3, 3) + gsize, complex)),
                                              4, PEs, nw=nw, device="cpu") for _ in range(4)]
            # staggered stencils take one rank per lattice (Wilson and
            # clover run on rank blocks: tests/test_gpu_distributed.py)
            D = lmb.StaggeredDiracOperator4D(U, 0.1)
            try:
                lmb.mul_(ls.similar(), D, ls)
            except lmb.ArgumentError as e:
                refused = "one rank per lattice" in str(e)
        else:
            refused = True
        q.put((rank, ls.coords, err, clean, gathered, red, refused))
    finally:
        dist.destroy_process_group()


def _run(ws, dim, PEs, gsize, nw, phases):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, dim, PEs, gsize, nw, phases, q))
             for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return sorted(q.get(timeout=10) for _ in range(ws))


@pytest.mark.parametrize("ws,dim,PEs,gsize,nw,phases", [
    (2, 4, (2, 1, 1, 1), (4, 4, 2, 4), 1, TWISTED),
    (2, 4, (1, 1, 1, 2), (2, 2, 2, 8), 2, (1, 1, 1, -1)),
    (4, 4, (2, 1, 1, 2), (4, 2, 2, 4), 1, TWISTED),
    (2, 5, (2, 1, 1, 1, 1), (4, 2, 2, 2, 3), 1, TWISTED + (1,)),
])
def test_halo_exchange_over_a_process_grid(ws, dim, PEs, gsize, nw, phases):
    got = _run(ws, dim, PEs, gsize, nw, phases)
    assert [g[0] for g in got] == list(range(ws))
    # rank r sits at the row-major Cartesian coordinates of r
    assert [g[1] for g in got] == [tuple(int(c) for c in np.unravel_index(r, PEs)) for r in range(ws)]
    for rank, coords, err, clean, gathered, red, refused in got:
        assert err <= 1e-14, (rank, err)
        assert clean and gathered and refused
        assert red == pytest.approx(complex(ws * (ws + 1) / 2, -ws * (ws - 1) / 2))


def test_process_grid_validation():
    sys.path.insert(0, os.path.join(ROOT, "latticematrices.jl_b200"))
    import lmb200 as lmb
    with pytest.raises(lmb.ArgumentError, match="process group"):
        lmb.LatticeMatrix(3, 4, 4, (4, 4, 4, 4), (2, 1, 1, 1), device="cpu")
