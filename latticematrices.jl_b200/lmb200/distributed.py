"""Lattices split over a process grid, one rank per GPU, on torch.distributed.

The reference builds a periodic Cartesian communicator from PEs
(MPI.Cart_create, LatticeMatrices_core.jl:350-358; local size PN = gsize ./
PEs, :338) and exchanges halos one dimension after another (exchange_dim!,
:742-921).  Here the ranks of the initialised torch.distributed group (NCCL
for CUDA tensors, gloo on CPU) take the same row-major Cartesian coordinates,
and each dimension's exchange is one batch of point-to-point transfers:

* the minus face goes to the minus neighbour (its plus ghost) and the plus
  face to the plus neighbour (its minus ghost); a face that crosses the
  global boundary carries phase_d (minus face of coordinate 0) or 1/phase_d
  (plus face of coordinate dims_d - 1), as exchange_dim! multiplies them;
* a dimension with one rank is exchanged in place (exchange_dim_local!);
* slabs span the full padded extent of the other dimensions, so corners
  pick up every dimension's wrap, as the reference's sequential exchange
  leaves them.

gather_matrix assembles the global core on every rank, and dot all-reduces
the ranks' partial sums (linearalgebra_D.jl:3325-3341, MPI.Allreduce).
"""
from __future__ import annotations

import numpy as np

from ._lib import ArgumentError


def _dist():
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        raise ArgumentError(
            "a process grid other than all ones needs an initialised "
            "torch.distributed process group (one rank per GPU)")
    return dist


def cart_coords(PEs, gsize):
    """Cartesian coordinates of this rank in the grid PEs (row-major, as
    MPI_Cart_create numbers ranks); checks the grid against the group."""
    dist = _dist()
    n = int(np.prod(PEs))
    ws = dist.get_world_size()
    if ws != n:
        raise ArgumentError(f"process grid {tuple(PEs)} needs {n} ranks; the "
                            f"process group has {ws}")
    for d, (g, p) in enumerate(zip(gsize, PEs)):
        if p <= 0 or g % p:
            raise ArgumentError(
                f"global size {g} in dimension {d + 1} is not divisible by the "
                f"process grid extent {p}")
    return tuple(int(c) for c in np.unravel_index(dist.get_rank(), tuple(PEs)))


def cart_rank(PEs, coords):
    return int(np.ravel_multi_index(tuple(coords), tuple(PEs)))


def neighbours(ls, d):
    """Ranks of the minus and plus neighbours in dimension d (periodic)."""
    cm, cp = list(ls.coords), list(ls.coords)
    cm[d] = (cm[d] - 1) % ls.dims[d]
    cp[d] = (cp[d] + 1) % ls.dims[d]
    return cart_rank(ls.dims, cm), cart_rank(ls.dims, cp)


def _slab(ls, d, rng):
    # the torch storage holds the reversed shape: dimension d is axis dim-1-d
    idx = [slice(None)] * ls.A.ndim
    idx[ls.dim - 1 - d] = rng
    return ls.A[tuple(idx)]


def exchange_halo(ls):
    """set_halo! of a field split over a process grid (exchange_dim! for
    every dimension, in order)."""
    import torch
    dist = _dist()
    nw, D = ls.nw, ls.dim
    for d in range(D):
        n = ls.PN[d] + 2 * nw
        fminus = _slab(ls, d, slice(nw, 2 * nw))
        fplus = _slab(ls, d, slice(n - 2 * nw, n - nw))
        gminus = _slab(ls, d, slice(0, nw))
        gplus = _slab(ls, d, slice(n - nw, n))
        ph = complex(ls.phases[d])
        if ls.dims[d] == 1:
            gminus.copy_(fplus)
            gplus.copy_(fminus)
            if ph != 1:
                gminus.mul_(1 / ph)
                gplus.mul_(ph)
            continue
        rm, rp = neighbours(ls, d)
        send_m = fminus.contiguous().clone()
        send_p = fplus.contiguous().clone()
        if ls.coords[d] == 0 and ph != 1:
            send_m.mul_(ph)
        if ls.coords[d] == ls.dims[d] - 1 and ph != 1:
            send_p.mul_(1 / ph)
        if _host_staged(dist, ls.A):
            send_m, send_p = send_m.cpu(), send_p.cpu()
        recv_m = torch.empty_like(send_p)
        recv_p = torch.empty_like(send_m)
        # tags as exchange_dim!: a minus face arrives as a plus ghost (tag d),
        # a plus face as a minus ghost (tag d + D); sends precede receives in
        # the same order on every rank, which is how NCCL pairs them
        ops = [dist.P2POp(dist.isend, torch.view_as_real(send_m), rm, tag=d),
               dist.P2POp(dist.isend, torch.view_as_real(send_p), rp, tag=d + D),
               dist.P2POp(dist.irecv, torch.view_as_real(recv_p), rp, tag=d),
               dist.P2POp(dist.irecv, torch.view_as_real(recv_m), rm, tag=d + D)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        gminus.copy_(recv_m.to(ls.A.device))
        gplus.copy_(recv_p.to(ls.A.device))


def _host_staged(dist, t):
    """gloo moves CPU tensors: CUDA data goes through host copies."""
    return t.is_cuda and dist.get_backend() == "gloo"


def gather_blocks(ls, local):
    """The global core assembled from every rank's block (Fortran order)."""
    import torch
    dist = _dist()
    dev = "cpu" if _host_staged(dist, ls.A) else ls.A.device
    t = torch.view_as_real(torch.from_numpy(np.ascontiguousarray(local.T)).to(dev))
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, t)
    out = np.zeros((ls.NC1, ls.NC2) + ls.gsize, dtype=ls.elementtype, order="F")
    for r, part in enumerate(parts):
        c = np.unravel_index(r, ls.dims)
        block = tuple(slice(ci * n, (ci + 1) * n) for ci, n in zip(c, ls.PN))
        out[(slice(None), slice(None)) + block] = torch.view_as_complex(part).cpu().numpy().T
    return out


def allreduce_complex(z, device):
    """Sum of a complex partial result over the ranks (FP64)."""
    import torch
    dist = _dist()
    if str(device).startswith("cuda") and dist.get_backend() == "gloo":
        device = "cpu"
    t = torch.tensor([complex(z).real, complex(z).imag], dtype=torch.float64, device=device)
    dist.all_reduce(t)
    return complex(float(t[0]), float(t[1]))


# ---------------------------------------------------------------------------
# the native sharded operators (lmb_set_process_grid)
# ---------------------------------------------------------------------------
def native_grid(ls) -> bool:
    """True when the blocks of `ls` run the native sharded stencils: CUDA
    fields of a 4-dimensional lattice on an NCCL process group.  (gloo
    groups keep the exchange-then-compute path of the operators.)"""
    if ls.dims == (1,) * ls.dim or ls.dim != 4 or not ls.A.is_cuda:
        return False
    return _dist().get_backend() == "nccl"


def grid_arguments(ls):
    """(dims, coords, split, nb_minus, nb_plus) of lmb_set_process_grid for
    this rank's block of `ls`: the dimensions held by more than one rank are
    split (faces exchanged with the Cartesian neighbours, exchange_dim!);
    the others wrap inside the block with the boundary phase
    (exchange_dim_local!)."""
    split = tuple(int(p > 1) for p in ls.dims)
    nbm, nbp = [], []
    for d in range(4):
        m, p = neighbours(ls, d)
        nbm.append(m)
        nbp.append(p)
    return tuple(ls.dims), tuple(ls.coords), split, tuple(nbm), tuple(nbp)


def shared_unique_id() -> bytes:
    """An NCCL unique id made on rank 0 and broadcast to every rank of the
    default group (a collective call)."""
    from ._lib import nccl_unique_id
    dist = _dist()
    box = [nccl_unique_id() if dist.get_rank() == 0 else None]
    dist.broadcast_object_list(box, src=0)
    return box[0]


def attach_process_grid(ctx, ls):
    """Give context `ctx` the process grid of `ls` (collective on the first
    call and whenever the grid changes; a no-op afterwards)."""
    dist = _dist()
    args = grid_arguments(ls)
    key = (dist.get_world_size(), dist.get_rank()) + args
    if getattr(ctx, "_grid_key", None) == key:
        return
    nid = shared_unique_id()
    dims, coords, split, nbm, nbp = args
    ctx.set_process_grid(nid, dist.get_world_size(), dist.get_rank(), dims,
                         coords, split, nbm, nbp)
    ctx._grid_key = key


def bind_grid(ctx, psi, link_sets, stream):
    """Bind the block of `psi` and the link sets [(which, links), ...] to a
    context with the native process grid: the links' halos are filled first
    (ensure_halo!, the ghost links of the backward hops come from them)."""
    from .lattice import ensure_halo_
    for _, links in link_sets:
        for u in links:
            ensure_halo_(u)
    attach_process_grid(ctx, psi)
    ctx.set_geometry(psi.PN, psi.nw, psi.phases, psi.coords, psi.dtype_code)
    for which, links in link_sets:
        ctx.upload_links(which, [u.data_ptr() for u in links],
                         [u.halo_epoch.core for u in links], stream)
    return ctx
