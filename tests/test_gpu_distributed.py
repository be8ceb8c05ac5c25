"""GPU: Wilson and Wilson-clover D on fields split over a process grid, and
the D'D CG with all-reduced dots, against the oracle on the whole lattice.

Two ranks share the one GPU and exchange halos through gloo (host copies);
their kernels never wait on each other.  Each rank applies D to its padded
block after the exchange (ghosts with boundary phases), so the gathered
result must match the single-lattice operator to FP64 rounding."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TWISTED = tuple(complex(np.exp(1j * a)) for a in (0.13, -0.21, 0.34, np.pi - 0.17))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _rank_main(rank, ws, port, PEs, L, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(ws))
    for p in (ROOT, os.path.join(ROOT, "latticematrices.jl_b200")):
        sys.path.insert(0, p)
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=120))
    try:
        import lmb200 as lmb
        from oracle import oracle as orc
        orc.lib()
        U = orc.random_su3_links(L, 0.3, 1)
        psi = orc.gaussian_field(L, 3, 4, 2)
        Ud = [lmb.LatticeMatrix.from_array(u, 4, PEs, nw=1) for u in U]
        pd = lmb.LatticeMatrix.from_array(psi, 4, PEs, nw=1, phases=TWISTED)
        out = {}
        for name, D, ref in (
                ("wilson", lmb.WilsonDiracOperator4D(Ud, 0.125),
                 lambda v, dag=False: orc.wilson(U, v, 0.125, TWISTED, dagger=dag)),
                ("clover", lmb.WilsonDiracCloverOperator4D(Ud, 0.13, 1.0),
                 lambda v, dag=False: orc.wilson_clover(U, v, 0.13, 1.0, TWISTED, dagger=dag))):
            o = pd.similar()
            lmb.mul_(o, D, pd)
            out[name] = _rel(o.gather_matrix(), ref(psi))
            lmb.mul_(o, lmb.adjoint(D), pd)
            out[name + "_dag"] = _rel(o.gather_matrix(), ref(psi, True))
            x = pd.similar()
            res = lmb.cg_(x, lmb.DdagDOp(D, pd.similar()), pd, rtol=1e-10)
            xs = np.asfortranarray(x.gather_matrix())
            r = psi - ref(np.asfortranarray(ref(xs)), True)
            out[name + "_cg"] = (res.converged, res.iterations,
                                 float(np.linalg.norm(r) / np.linalg.norm(psi)))
        out["dot"] = abs(lmb.dot(pd, pd) - np.vdot(psi, psi)) / abs(np.vdot(psi, psi))
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("PEs,L", [((1, 1, 1, 2), (4, 4, 4, 8)), ((2, 1, 1, 1), (8, 4, 4, 4))])
def test_split_wilson_clover_and_cg(PEs, L):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, PEs, L, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(600)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict(q.get(timeout=10) for _ in range(ws))
    for rank, out in got.items():
        for name in ("wilson", "clover"):
            assert out[name] <= 1e-13 and out[name + "_dag"] <= 1e-13, (rank, name, out)
            conv, it, rel = out[name + "_cg"]
            assert conv and rel <= 2e-10, (rank, name, out)
        assert out["dot"] <= 1e-13
    # both ranks ran the same iterations (same all-reduced scalars)
    assert got[0]["clover_cg"][1] == got[1]["clover_cg"][1]
