// lmb_dist_host.cuh -- host side of the sharded operators: the process grid
// of a context, its NCCL communicator and the ghost-link and boundary-site
// caches (kernels in lmb_dist.cuh, drivers in lmb_dist_ops.cu).
//
// NCCL is opened at run time (dlopen of libnccl.so.2, the library a PyTorch
// process has already loaded), so liblmb200.so loads without it and only
// lmb_set_process_grid needs it.
#pragma once
#include <nccl.h>

#include <map>
#include <string>

#include "lmb_dist.cuh"
#include "lmb_internal.cuh"

namespace lmb {

struct NcclApi {
  ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  const char *(*GetErrorString)(ncclResult_t) = nullptr;
  bool loaded = false;
  std::string error;
};
// loads NCCL on first use; api.loaded false (api.error says why) if absent
const NcclApi &nccl_api();

}  // namespace lmb

struct lmb_dist {
  int nranks = 1, rank = 0;
  int dims[4] = {1, 1, 1, 1}, coords[4] = {0, 0, 0, 0};
  int nb_minus[4] = {0, 0, 0, 0}, nb_plus[4] = {0, 0, 0, 0};  // neighbour ranks
  unsigned split = 0;  // dimensions exchanged with the neighbours
  ncclComm_t comm = nullptr;
  cudaStream_t comm_stream = nullptr;
  // the boundary kernels run here (higher priority), beside the interior
  // kernel, with reduction scratch of their own
  cudaStream_t bnd_stream = nullptr;
  cudaEvent_t ev_packed = nullptr, ev_comm = nullptr, ev_bnd = nullptr;
  unsigned *bcounter = nullptr;
  double *sums = nullptr;  // two device doubles: interior and boundary totals
  // boundary sites of the block for each halo depth (device lists; key
  // 2 depth + 1: with the x partners of boundary sites, for the x-adjacent
  // pair interior)
  std::map<int, std::pair<int *, int>> boundary;
  // link ghosts per link set and dimension, and what they were built from
  lmb::LinkSet ghost[3][4];
  uint64_t ghost_of_version[3] = {~0ull, ~0ull, ~0ull};
  int ghost_depth[3] = {0, 0, 0};
};

namespace lmb {

// view of the process grid for a stencil of halo depth `depth`
DistView dist_view(const lmb_ctx *ctx, int depth);
// boundary site list of the block for `depth` (built on first use); pairs:
// also every site whose x partner (x xor 1) is a boundary site, the sites the
// x-adjacent pair interior leaves out
int dist_boundary(lmb_ctx *ctx, int depth, bool pairs, const int **list, int *n);
// ghost links of link set `which` at `depth` layers, in precision prec
int dist_link_ghosts(lmb_ctx *ctx, int which, int depth, int prec, bool allow_recon, cudaStream_t st);
// exchange of one field's faces: pack on `st`, NCCL on the communication
// stream; ev_comm marks the arrival of every ghost layer
template <int P, int NC>
int dist_exchange(lmb_ctx *ctx, const Field<P, NC> &in, const DistView &dv, GhostSpinors<P, NC> &gh,
                  cudaStream_t st);
// sum of the two partial totals over the ranks, on `st`
int dist_allreduce_sums(lmb_ctx *ctx, cudaStream_t st);
void dist_release(lmb_ctx *ctx);

}  // namespace lmb
