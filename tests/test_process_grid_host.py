"""Host side of the native sharded operators on CPU (gloo, 2 and 4 ranks):
the arguments every rank passes to lmb_set_process_grid -- its Cartesian
coordinates (MPI_Cart_create's row-major numbering,
LatticeMatrices_core.jl:350-358), the split dimensions and the neighbour
ranks of exchange_dim! (:742-921) -- must describe one consistent periodic
grid, and the NCCL unique id made on rank 0 must reach every rank unchanged.
The device path itself (NCCL faces, interior / boundary kernels) is checked
against the oracle in test_gpu_process_grid.py."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, ws, port, PEs, gsize, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, os.path.join(ROOT, "latticematrices.jl_b200"))
    from datetime import timedelta
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    try:
        import lmb200 as lmb
        from lmb200.distributed import grid_arguments, native_grid, shared_unique_id
        ls = lmb.LatticeMatrix.from_array(np.zeros((3, 1) + gsize, complex, order="F"), 4, PEs,
                                          nw=1, device="cpu")
        args = grid_arguments(ls)
        try:
            nid = shared_unique_id()
        except lmb.LMBError:
            nid = None   # NCCL absent: the id cannot be made
        q.put((rank, args, nid, native_grid(ls)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("PEs,gsize", [((1, 1, 1, 2), (4, 4, 4, 8)),
                                       ((2, 1, 1, 2), (4, 4, 4, 8)),
                                       ((1, 2, 2, 1), (4, 4, 4, 4))])
def test_process_grid_arguments_are_consistent(PEs, gsize):
    ws = int(np.prod(PEs))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, PEs, gsize, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = {}
    try:
        for _ in range(ws):
            rank, args, nid, native = q.get(timeout=240)
            res[rank] = (args, nid, native)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert sorted(res) == list(range(ws))
    for r, ((dims, coords, split, nbm, nbp), nid, native) in res.items():
        assert dims == PEs
        assert coords == tuple(int(c) for c in np.unravel_index(r, PEs))
        assert split == tuple(int(p > 1) for p in PEs)
        assert not native               # gloo keeps the exchange-then-compute path
        for d in range(4):
            cm, cp = list(coords), list(coords)
            cm[d] = (cm[d] - 1) % PEs[d]
            cp[d] = (cp[d] + 1) % PEs[d]
            assert nbm[d] == int(np.ravel_multi_index(cm, PEs))
            assert nbp[d] == int(np.ravel_multi_index(cp, PEs))
            # my plus neighbour's minus neighbour is me, and the other way round
            assert res[nbp[d]][0][3][d] == r and res[nbm[d]][0][4][d] == r
            if PEs[d] == 1:
                assert nbm[d] == nbp[d] == r
    ids = {nid for _, nid, _ in res.values()}
    assert len(ids) == 1
    nid = ids.pop()
    assert nid is None or len(nid) == 128
